// gs_k_mart.cu -- instances and launchers of the fused martensite update and
// of the FP64 partial-sum reduction.
#include "gs_launch.h"
#include "gs_mart.cuh"

namespace gs {

__global__ void k_reduce_partials(const double* __restrict__ partials, int nb, int n, double* __restrict__ out) {
  // one warp per accumulator; lanes stride over blocks, then a compensated
  // combine of the 32 lane sums
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int i = warp; i < n; i += nwarps) {
    Neu s;
    for (int b = lane; b < nb; b += 32) s.add(partials[(long long)b * n + i]);
    double hi = s.s, lo = s.c;
    for (int o = 16; o > 0; o >>= 1) {
      const double h2 = __shfl_xor_sync(0xffffffffu, hi, o);
      const double l2 = __shfl_xor_sync(0xffffffffu, lo, o);
      const double t = hi + h2;
      const double e = fabs(hi) >= fabs(h2) ? (hi - t) + h2 : (h2 - t) + hi;
      hi = t;
      lo = lo + l2 + e;
    }
    if (lane == 0) out[i] = hi + lo;
  }
}

cudaError_t launch_reduce(const double* partials, int nb, int n, double* out, cudaStream_t s) {
  k_reduce_partials<<<1, 256, 0, s>>>(partials, nb, n, out);
  return cudaGetLastError();
}

}  // namespace gs
