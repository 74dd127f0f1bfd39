// gs_k_mart_f32.cu -- float instances of the fused martensite update.
#include "gs_k_mart_impl.cuh"
namespace gs {
template cudaError_t launch_mart_update<float>(MartArgs<float>&, int, bool, cudaStream_t, int*, int);
template <> cudaError_t launch_bump_step<float>(MartConst<float>* mcs, int n, cudaStream_t s) {
  k_bump_step<float><<<(n + 127) / 128, 128, 0, s>>>(mcs, n);
  return cudaGetLastError();
}
}  // namespace gs
