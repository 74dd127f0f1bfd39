// gs_k_x_impl.cuh -- launcher template of the x pass for one field-count
// class (FM inputs, GM outputs at most); instantiated per class in its own
// translation unit so the classes compile in parallel.
#pragma once
#include "gs_launch.h"
#include "gs_passes.cuh"

namespace gs {

template <typename T, int N0, int FM, int GM, class Op> static cudaError_t xc_n(XArgs<T>& a, cudaStream_t s) {
  using L = Line<T, N0>;
  const int groups = a.F > a.G ? a.F : a.G;
  // 8-column tiles for the FP32 hot sizes: a 3-field block then needs 384
  // threads x 80 registers, so two blocks share an SM and one block's
  // contraction overlaps the other's loads and stores
  int tz = pick_tz(a.h);
  if (sizeof(T) == 4 && N0 >= 64 && tz > 8) tz = 8;
  if (a.tz_req > 0 && (a.tz_req & (a.tz_req - 1)) == 0 && a.h % a.tz_req == 0) tz = a.tz_req;
  auto smem_of = [&](int tzv) {  // line regions, packed-column results, twiddles
    return (size_t)groups * tzv * L::PAD * sizeof(cplx<T>) + (size_t)(GM + 1) * N0 * sizeof(cplx<T>);
  };
  constexpr int maxthr = XBounds<FM, GM>::v;
  while (tz > 1 && (smem_of(tz) > 200 * 1024 || tz * L::P * groups > maxthr)) tz >>= 1;
  if (tz * L::P * groups > maxthr) return cudaErrorInvalidConfiguration;
  a.tz = tz;
  a.groups = groups;
  const size_t smem = smem_of(tz);
  dim3 grid(a.h / tz, a.n1, a.nsim > 1 ? a.nsim : 1);
  if constexpr (sizeof(T) == 4 && N0 >= 64) {
    if (tz == 8) {
      // exact field counts known at compile time: the three- and five-field
      // table contractions, the precipitate's (state, force) -> state slices
      if constexpr ((FM == GM && (FM == 3 || FM == 5) && KxPair<Op>::v) || (FM == 2 && GM == 1) ||
                    (FM == 1 && GM == 1)) {
        if (a.F == FM && a.G == GM) {
          allow_max_smem<k_xpass<T, N0, FM, GM, 8, Op, true>>();
          k_xpass<T, N0, FM, GM, 8, Op, true><<<grid, tz * L::P * groups, smem, s>>>(a);
          return cudaGetLastError();
        }
      }
      allow_max_smem<k_xpass<T, N0, FM, GM, 8, Op>>();
      k_xpass<T, N0, FM, GM, 8, Op><<<grid, tz * L::P * groups, smem, s>>>(a);
      return cudaGetLastError();
    }
  }
  allow_max_smem<k_xpass<T, N0, FM, GM, 0, Op>>();
  k_xpass<T, N0, FM, GM, 0, Op><<<grid, tz * L::P * groups, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T, int FM, int GM, class Op> cudaError_t launch_x_class(XArgs<T>& a, cudaStream_t s) {
  switch (a.n0) {
#define GS_C(N_) \
  case N_:       \
    return xc_n<T, N_, FM, GM, Op>(a, s);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace gs
