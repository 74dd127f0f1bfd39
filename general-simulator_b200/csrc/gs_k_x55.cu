// gs_k_x55.cu -- x pass instances (B(n) contraction) for up to 5 input and 5 output fields.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 5, 5, ContractOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 5, 5, ContractOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
