// gs_k_x33.cu -- x pass instances (B(n) contraction) for up to 3 input and 3 output fields.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 3, 3, ContractOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 3, 3, ContractOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
