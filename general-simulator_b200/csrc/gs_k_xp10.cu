// gs_k_xp10.cu -- x pass instances (precipitate k-space update) for up to 10 input and 5 output fields.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 10, 5, PrecipOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 10, 5, PrecipOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
