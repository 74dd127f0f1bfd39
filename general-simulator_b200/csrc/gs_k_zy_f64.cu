// gs_k_zy_f64.cu -- double instances of the z-forward and y passes.
#include "gs_k_zy_impl.cuh"
namespace gs {
template cudaError_t launch_zfwd<double>(ZfwdArgs<double>&, int, cudaStream_t, int);
template cudaError_t launch_ypass<double>(YArgs<double>&, int, int, int, cudaStream_t, int, int);
}  // namespace gs
