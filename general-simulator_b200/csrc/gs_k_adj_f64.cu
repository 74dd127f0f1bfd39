// gs_k_adj_f64.cu -- double instances of the adjoint martensite sweep.
#include "gs_k_adj_impl.cuh"
namespace gs {
template cudaError_t launch_adj_update<double>(AdjArgs<double>&, int, cudaStream_t, int*);
template cudaError_t launch_adj_seed<double>(AdjSeedArgs<double>&, cudaStream_t, int*);
}  // namespace gs
