// gs_k_x.cu -- x pass: picks the field-count class of the per-point op.
#include "gs_launch.h"
#include "gs_passes.cuh"

namespace gs {

template <typename T, int FM, int GM, class Op> cudaError_t launch_x_class(XArgs<T>& a, cudaStream_t s);

// the launch-range check of an x pass: F input and G output fields per
// simulation, the B table, the K tables, the per-simulation scales
template <typename T> static cudaError_t x_ranges(const XArgs<T>& a, bool ktab) {
  if (!bounds_check_on()) return cudaSuccess;
  const long long ns = a.nsim > 1 ? a.nsim : 1, fstride = (long long)a.n0 * a.n1 * a.h;
  GS_RANGE(a.in, ns * a.F * fstride, cplx<T>, sizeof(cplx<T>), "x pass", "input spectra");
  GS_RANGE(a.out, ns * a.G * fstride, cplx<T>, sizeof(cplx<T>), "x pass", "output spectra");
  if (a.btab)
    GS_RANGE(a.btab, (long long)(a.n0 / 2 + 1) * a.bt_d1 * a.bt_d2 * a.bt_stride, T, 2 * sizeof(T), "x pass",
             "B table");
  if (a.simscale) GS_RANGE(a.simscale, ns, T, sizeof(T), "x pass", "simulation scales");
  if (ktab) {
    GS_RANGE(a.pu.ktab[0], a.n0, T, sizeof(T), "x pass", "K table (axis 0)");
    GS_RANGE(a.pu.ktab[1], a.n1, T, sizeof(T), "x pass", "K table (axis 1)");
    GS_RANGE(a.pu.ktab[2], a.n2, T, sizeof(T), "x pass", "K table (axis 2)");
  }
  return cudaSuccess;
}

template <typename T> cudaError_t launch_xcontract(XArgs<T>& a, cudaStream_t s) {
  if (const cudaError_t e = x_ranges(a, false)) return e;
  if (a.btab) {  // B from the octant table (square contraction, F = G)
    if (a.F != a.G) return cudaErrorInvalidValue;
    if constexpr (sizeof(T) == 4) {
      const cudaError_t e = launch_xtma(a, s);
      if (e != cudaErrorNotSupported) return e;
    }
    if (a.F <= 3) return launch_x_class<T, 3, 3, TableOp>(a, s);
    if (a.F <= 5) return launch_x_class<T, 5, 5, TableOp>(a, s);
    return launch_x_class<T, 9, 9, TableOp>(a, s);
  }
  if (a.F <= 3 && a.G <= 3) return launch_x_class<T, 3, 3, ContractOp>(a, s);
  if (a.F <= 5 && a.G <= 5) return launch_x_class<T, 5, 5, ContractOp>(a, s);
  if (a.F <= 8 && a.G <= 6) return launch_x_class<T, 8, 6, ContractOp>(a, s);
  return launch_x_class<T, 9, 9, ContractOp>(a, s);
}

template <typename T> cudaError_t launch_xprecip_adjoint(XArgs<T>& a, cudaStream_t s) {
  if (a.F != 2 || a.G != 3) return cudaErrorInvalidValue;
  if (const cudaError_t e = x_ranges(a, true)) return e;
  return launch_x_class<T, 2, 3, PrecipAdjOp>(a, s);
}
template cudaError_t launch_xprecip_adjoint<float>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_xprecip_adjoint<double>(XArgs<double>&, cudaStream_t);

template <typename T> cudaError_t launch_xprecip_eta(XArgs<T>& a, cudaStream_t s) {
  if (a.F != 1 || a.G != 1) return cudaErrorInvalidValue;
  if (const cudaError_t e = x_ranges(a, true)) return e;
  return launch_x_class<T, 1, 1, PrecipEtaOp>(a, s);
}
template cudaError_t launch_xprecip_eta<float>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_xprecip_eta<double>(XArgs<double>&, cudaStream_t);

template <typename T> cudaError_t launch_xprecip(XArgs<T>& a, cudaStream_t s) {
  if (const cudaError_t e = x_ranges(a, true)) return e;
  if (a.F == 2 && a.G == 1 && a.nsim >= 1) return launch_x_class<T, 2, 1, PrecipPairOp>(a, s);  // pair slices
  if (a.F <= 10 && a.G <= 5) return launch_x_class<T, 10, 5, PrecipOp>(a, s);
  return launch_x_class<T, 18, 9, PrecipOp>(a, s);
}

template cudaError_t launch_xcontract<float>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_xcontract<double>(XArgs<double>&, cudaStream_t);
template cudaError_t launch_xprecip<float>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_xprecip<double>(XArgs<double>&, cudaStream_t);

}  // namespace gs
