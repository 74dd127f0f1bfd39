// gs_k_xp18.cu -- x pass instances (precipitate k-space update) for up to 18 input and 9 output fields.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 18, 9, PrecipOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 18, 9, PrecipOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
