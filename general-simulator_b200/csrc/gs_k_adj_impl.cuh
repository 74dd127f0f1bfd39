// gs_k_adj_impl.cuh -- launchers of the adjoint martensite sweep
// (instantiated per dtype in its own translation unit).
#pragma once
#include "gs_adjoint.cuh"
#include "gs_launch.h"

namespace gs {

template <typename T, int H, int VM> cudaError_t adj_n(AdjArgs<T>& a, cudaStream_t s, int* nblocks) {
  using L = Line<T, H>;
  const int per = L::P * a.mc.V;
  long long lr = 256 / per;
  if (lr < 1) lr = 1;
  if (lr > a.nrows) lr = a.nrows;
  a.lr = (int)lr;
  const size_t smem = (size_t)lr * a.mc.V * L::PAD * sizeof(cplx<T>);
  allow_max_smem<k_adj_update<T, H, VM>>();
  const long long grid = (a.nrows + lr - 1) / lr;
  if (bounds_check_on()) {
    const char* k = "adjoint update";
    const long long VN = (long long)a.mc.V * a.nrows * a.n2;
    constexpr size_t va = ((2 * H) % 4 == 0 ? 4 : 2) * sizeof(T) < 16 ? ((2 * H) % 4 == 0 ? 4 : 2) * sizeof(T) : 16;
    GS_RANGE(a.spec, VN / 2, cplx<T>, sizeof(cplx<T>), k, "Q spectra");
    GS_RANGE(a.eta, VN, T, va, k, "eta");
    GS_RANGE(a.lam_in, VN, T, va, k, "lambda in");
    GS_RANGE(a.lam_out, VN, T, va, k, "lambda out");
    GS_RANGE(a.R, VN, T, va, k, "R");
    GS_RANGE(a.partials, grid * ADJ_N, double, sizeof(double), k, "partials");
  }
  if (nblocks) *nblocks = (int)grid;
  k_adj_update<T, H, VM><<<(unsigned)grid, (unsigned)(per * lr), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_adj_update(AdjArgs<T>& a, int H, cudaStream_t s, int* nblocks) {
  switch (H) {
#define GS_C(N_)                                                                    \
  case N_:                                                                          \
    return a.mc.V == 3 ? adj_n<T, N_, 3>(a, s, nblocks)                              \
           : a.mc.V <= 4 ? adj_n<T, N_, 4>(a, s, nblocks) : adj_n<T, N_, 8>(a, s, nblocks);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T> cudaError_t launch_adj_seed(AdjSeedArgs<T>& a, cudaStream_t s, int* nblocks) {
  long long nb = (a.n + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  if (nb < 1) nb = 1;
  *nblocks = (int)nb;
  k_adj_seed<T><<<(unsigned)nb, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace gs
