// gs_k_xp2.cu -- x pass instances (precipitate k-space update: the (c, mu) pair, then one u_p per grid-z slice).
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 2, 1, PrecipPairOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 2, 1, PrecipPairOp>(XArgs<double>&, cudaStream_t);
template cudaError_t launch_x_class<float, 1, 1, PrecipEtaOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 1, 1, PrecipEtaOp>(XArgs<double>&, cudaStream_t);
template cudaError_t launch_x_class<float, 2, 3, PrecipAdjOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 2, 3, PrecipAdjOp>(XArgs<double>&, cudaStream_t);
}  // namespace gs
