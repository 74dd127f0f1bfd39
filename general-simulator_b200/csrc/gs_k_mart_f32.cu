// gs_k_mart_f32.cu -- float instances of the fused martensite update.
#include "gs_k_mart_impl.cuh"
namespace gs {
template cudaError_t launch_mart_update<float>(MartArgs<float>&, int, bool, cudaStream_t, int*);
}  // namespace gs
