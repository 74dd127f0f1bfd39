// gs_k_padj.cu -- launchers of the precipitate adjoint's pointwise sweeps.
#include "gs_launch.h"
#include "gs_padj.cuh"

namespace gs {

template <typename T> cudaError_t launch_padj(PadjArgs<T>& a, bool second, cudaStream_t s, int* nblocks) {
  long long nb = (a.N + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  if (nb < 1) nb = 1;
  *nblocks = (int)nb;
  if (!second)
    k_padj_a<T><<<(unsigned)nb, 256, 0, s>>>(a);
  else if (a.V <= 4)
    k_padj_b<T, 4><<<(unsigned)nb, 256, 0, s>>>(a);
  else
    k_padj_b<T, 8><<<(unsigned)nb, 256, 0, s>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_padj<float>(PadjArgs<float>&, bool, cudaStream_t, int*);
template cudaError_t launch_padj<double>(PadjArgs<double>&, bool, cudaStream_t, int*);

}  // namespace gs
