// gs_k_mart_f64.cu -- double instances of the fused martensite update.
#include "gs_k_mart_impl.cuh"
namespace gs {
template cudaError_t launch_mart_update<double>(MartArgs<double>&, int, bool, cudaStream_t, int*);
}  // namespace gs
