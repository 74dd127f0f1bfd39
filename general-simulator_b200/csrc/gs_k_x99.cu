// gs_k_x99.cu -- x pass instances (B(n) contraction) for up to 9 input and 9 output fields.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 9, 9, ContractOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 9, 9, ContractOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
