// gs_k_mart_impl.cuh -- launcher template of the fused martensite update
// (instantiated per dtype in its own translation unit).
#pragma once
#include "gs_launch.h"
#include "gs_mart.cuh"

namespace gs {

template <typename T, int H, int VM, bool ST, bool BA, bool FU = false, bool HA = false>
cudaError_t mu_n(MartArgs<T>& a, cudaStream_t s, int* nblocks, int nsim) {
  using L = Line<T, H>;
  const int per = L::P * a.mc.V;
  // default: blocks of about 192 threads (8 rows of 3 variants of length-128
  // lines measured 0.300 ms against 0.322 ms for 10 rows at 256^3 x 3); the
  // kernel's launch bounds allow 256 threads
  long long lr = 192 / per;
  if (a.lr_req > 0 && (long long)a.lr_req * per <= 256) lr = a.lr_req;
  if (lr < 1) lr = 1;
  if (lr > a.nrows) lr = a.nrows;
  a.lr = (int)lr;
  const size_t smem = (size_t)lr * a.mc.V * L::PAD * sizeof(cplx<T>);
  allow_max_smem<k_mart_update<T, H, VM, ST, BA, FU, true, HA>>();
  const long long grid = (a.nrows + lr - 1) / lr;
  if (bounds_check_on()) {
    const char* k = "martensite update";
    const long long ns = BA ? nsim : 1, N = a.nrows * a.n2, VN = (long long)a.mc.V * N;
    constexpr size_t va = ((2 * H) % 4 == 0 ? 4 : 2) * sizeof(T) < 16 ? ((2 * H) % 4 == 0 ? 4 : 2) * sizeof(T) : 16;
    GS_RANGE(a.spec, ns * VN / 2, cplx<T>, sizeof(cplx<T>), k, "R spectra");
    GS_RANGE(a.eta_in, ns * VN, T, va, k, "eta");
    if (!ST) GS_RANGE(a.eta_out, ns * VN, T, va, k, "eta out");
    if (a.mc.has_defect) GS_RANGE(a.defect, N, T, va, k, "defect mask");
    if (a.mc.has_K) GS_RANGE(a.K, VN, T, va, k, "dislocation field");
    if (!BA && a.r_out) GS_RANGE(a.r_out, VN, T, va, k, "R out");
    if (FU) GS_RANGE(a.spec_next, ns * VN / 2, cplx<T>, sizeof(cplx<T>), k, "next spectra");
    if (HA) GS_RANGE(a.halo, 2 * (long long)a.mc.V * a.n1 * a.n2, T, va, k, "halo planes");
    if (ST) GS_RANGE(a.partials, grid * ACC_N, double, sizeof(double), k, "statistics partials");
  }
  if (nblocks) *nblocks = (int)grid;
  k_mart_update<T, H, VM, ST, BA, FU, true, HA>
      <<<dim3((unsigned)grid, (unsigned)nsim), (unsigned)(per * lr), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T, int H> cudaError_t mu_h(MartArgs<T>& a, bool stats, cudaStream_t s, int* nb, int nsim) {
  const bool fu = a.spec_next != nullptr && !stats;
  if (a.halo) {  // a slab of a split grid: one simulation, fused z forward, no statistics
    if (!fu || nsim > 0) return cudaErrorInvalidValue;
    if constexpr (sizeof(T) == 4) {
      if (a.mc.V == 3) return mu_n<T, H, 3, false, false, true, true>(a, s, nb, 1);
    }
    if (a.mc.V <= 4) return mu_n<T, H, 4, false, false, true, true>(a, s, nb, 1);
    return mu_n<T, H, 8, false, false, true, true>(a, s, nb, 1);
  }
  if (nsim > 0) {  // batched simulations (device-resident constants)
    if constexpr (sizeof(T) == 4) {
      if (a.mc.V == 3 && fu) return mu_n<T, H, 3, false, true, true>(a, s, nb, nsim);
      if (a.mc.V == 2 && fu) return mu_n<T, H, 2, false, true, true>(a, s, nb, nsim);
    }
    if (a.mc.V <= 4)
      return fu ? mu_n<T, H, 4, false, true, true>(a, s, nb, nsim) : mu_n<T, H, 4, false, true>(a, s, nb, nsim);
    return fu ? mu_n<T, H, 8, false, true, true>(a, s, nb, nsim) : mu_n<T, H, 8, false, true>(a, s, nb, nsim);
  }
  // two or three variants exactly: no runtime bound in the variant loops
  if constexpr (sizeof(T) == 4) {
    if (a.mc.V == 3 && fu) return mu_n<T, H, 3, false, false, true>(a, s, nb, 1);
  }
  if (a.mc.V == 2 && fu) return mu_n<T, H, 2, false, false, true>(a, s, nb, 1);
  if (a.mc.V <= 4) {
    if (stats) return mu_n<T, H, 4, true, false>(a, s, nb, 1);
    return fu ? mu_n<T, H, 4, false, false, true>(a, s, nb, 1) : mu_n<T, H, 4, false, false>(a, s, nb, 1);
  }
  if (stats) return mu_n<T, H, 8, true, false>(a, s, nb, 1);
  return fu ? mu_n<T, H, 8, false, false, true>(a, s, nb, 1) : mu_n<T, H, 8, false, false>(a, s, nb, 1);
}

template <typename T>
cudaError_t launch_mart_update(MartArgs<T>& a, int H, bool stats, cudaStream_t s, int* nblocks, int nsim) {
  switch (H) {
#define GS_C(N_) \
  case N_:       \
    return mu_h<T, N_>(a, stats, s, nblocks, nsim);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace gs
