// gs_k_zy_f32.cu -- float instances of the z-forward and y passes.
#include "gs_k_zy_impl.cuh"
namespace gs {
template cudaError_t launch_zfwd<float>(ZfwdArgs<float>&, int, cudaStream_t, int);
template cudaError_t launch_ypass<float>(YArgs<float>&, int, int, int, cudaStream_t, int, int);
}  // namespace gs
