// gs_k_x86.cu -- x pass instances (B(n) contraction) for up to 8 input and 6 output fields.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 8, 6, ContractOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 8, 6, ContractOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
