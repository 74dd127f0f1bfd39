// gs_k_adj_f32.cu -- float instances of the adjoint martensite sweep.
#include "gs_k_adj_impl.cuh"
namespace gs {
template cudaError_t launch_adj_update<float>(AdjArgs<float>&, int, cudaStream_t, int*);
template cudaError_t launch_adj_seed<float>(AdjSeedArgs<float>&, cudaStream_t, int*);
}  // namespace gs
