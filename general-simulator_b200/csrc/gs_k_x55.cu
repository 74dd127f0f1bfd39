// gs_k_x55.cu -- x pass instances for 5 fields (concentration + 4 variants).
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 5, 5>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 5, 5>(XArgs<double>&, cudaStream_t);
}  // namespace gs
