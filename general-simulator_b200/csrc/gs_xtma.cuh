// gs_xtma.cuh -- the x pass fed by the Tensor Memory Accelerator.
//
// The plain x pass (k_xpass) loads a column tile, transforms it and stores it,
// one tile per block: its loads and its arithmetic do not overlap (at 256^3
// the loads and shuffles alone take about as long as the arithmetic).  This
// kernel is persistent: each block walks a strided list of (ky, kz tile)
// tiles and keeps two shared-memory stages.  While it transforms the tile in
// one stage, one thread has already asked the TMA unit for the next tile
// (cp.async.bulk.tensor, one 4D box per field: TZ columns x 1 ky x N0 kx,
// completion counted on an mbarrier), so HBM streams the next tile during the
// arithmetic.  After a tile's inputs are in registers its stage is reused as
// the working region of the FFTs, so a stage costs no more shared memory
// than the plain kernel's working region.  The arithmetic is xpass_tile, the
// same code as the plain kernel's, so both give the same bits.
//
// Every wait on an mbarrier gives up after about a second (clock64), counts
// the event in gs_x_wait_timeouts and ends the block, after waiting (again
// bounded) for the copies it still has in flight.
#pragma once
#include <cuda.h>

#include "gs_bulk.cuh"
#include "gs_passes.cuh"

namespace gs {

// waits that gave up (device counter; this header belongs to one translation unit)
static __device__ unsigned int g_x_wait_timeouts = 0;

// One 4D tiled box (coordinates innermost first) into shared memory; the
// bytes are counted on bar.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

// Threads per block of the TMA-fed pass: FM fields x TZ columns x P threads
// per line.
template <int N0, int FM, int TZ> struct XTmaShape {
  using L = Line<float, N0>;
  static constexpr int threads = FM * TZ * L::P;
  static constexpr int min_blocks = threads <= 384 ? 2 : 1;  // resident blocks per SM the registers allow
  static constexpr int region = L::PAD * TZ;                  // values per field stage
  static constexpr size_t region_bytes = region * sizeof(cplx<float>);
  static_assert(region_bytes % 128 == 0, "TMA destinations must be 128-byte aligned");
};

// tin: 4D map of the input spectra, dims (h, n1, n0, F) of 8-byte values,
// box (TZ, 1, N0, 1).  a.F fields in, a.G = a.F out (square table
// contraction), one simulation.  ntiles = (h / TZ) * n1.
template <int N0, int FM, int TZ, class Op>
__global__ void __launch_bounds__(XTmaShape<N0, FM, TZ>::threads, XTmaShape<N0, FM, TZ>::min_blocks)
    k_xpass_tma(XArgs<float> a, const __grid_constant__ CUtensorMap tin, int ntiles) {
  using T = float;
  using L = Line<T, N0>;
  using V = cplx<T>;
  using S = XTmaShape<N0, FM, TZ>;
  extern __shared__ __align__(1024) unsigned char smtma[];
  // two stages of F fields, the packed-column results, the twiddles, two mbarriers (one value each)
  GS_BC_SMEM_GUARD(2LL * a.F * S::region + (FM + 1) * N0 + 2, V, BC_X_SMEM)
  const int F = a.F;
  V* const stage0 = reinterpret_cast<V*>(smtma);  // stage s at stage0 + s * F * region
  V* part = stage0 + 2 * F * S::region;           // GM x N0 values of the packed columns
  V* tws = part + FM * N0;                          // the x twiddles, as in the plain pass
  uint64_t* bar = reinterpret_cast<uint64_t*>(tws + N0);
  const int gsz = TZ * L::P;
  const int grp = threadIdx.x / gsz, l = threadIdx.x - grp * gsz;
  const int c = l % TZ, t = l / TZ;
  const int nkz = a.h / TZ;
  const uint32_t tile_bytes = (uint32_t)(F * TZ * N0 * sizeof(V));
  auto issue = [&](int tile, int s) {
    const int ky = tile / nkz, kz0 = (tile - ky * nkz) * TZ;
    mbar_arrive_expect_tx(&bar[s], tile_bytes);
    for (int f = 0; f < F; ++f) tma_load_4d(stage0 + (s * F + f) * S::region, &tin, kz0, ky, 0, f, &bar[s]);
  };
  for (int i = threadIdx.x; i < N0; i += blockDim.x) tws[i] = a.tw[i];
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
    fence_proxy_async();
  }
  __syncthreads();
  if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
  int it = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int s = it & 1;
    const int next = tile + gridDim.x;
    // the other stage was last used by the previous tile, which every thread
    // has finished (the loop ends with a barrier)
    if (threadIdx.x == 0 && next < ntiles) {
      fence_proxy_async();
      issue(next, s ^ 1);
    }
    const bool ok = mbar_wait_bounded(&bar[s], (uint32_t)(it >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicAdd(&g_x_wait_timeouts, 1u);
        // let the copies still in flight land before the block's shared memory goes
        mbar_wait_bounded(&bar[s], (uint32_t)(it >> 1) & 1u);
        if (next < ntiles) mbar_wait_bounded(&bar[s ^ 1], (uint32_t)((it + 1) >> 1) & 1u);
      }
      __syncthreads();
      return;
    }
    const int ky = tile / nkz, kz0 = (tile - ky * nkz) * TZ;
    V v[L::R1];
    const bool fw = grp < F;
    {
      // dense box layout: value (kx, column c) of field f at f * region + kx * TZ + c
      const V* src = stage0 + (s * F + (fw ? grp : 0)) * S::region + t * TZ + c;
#pragma unroll
      for (int r = 0; r < L::R1; ++r) v[r] = fw ? src[r * L::P * TZ] : mk2((T)0, (T)0);
    }
    __syncthreads();  // the stage becomes the padded working region of the FFTs
    xpass_tile<T, N0, FM, FM, Op, true>(a, stage0 + s * F * S::region, part, TZ, grp, c, t, kz0, ky, a.out, v, tws);
    __syncthreads();
  }
}

}  // namespace gs
