// gs_k_xt.cu -- x pass instances that read B(k) from the octant table, and
// the table fill.
#include "gs_k_x_impl.cuh"
namespace gs {
template cudaError_t launch_x_class<float, 3, 3, TableOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 3, 3, TableOp>(XArgs<double>&, cudaStream_t);
template cudaError_t launch_x_class<float, 5, 5, TableOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 5, 5, TableOp>(XArgs<double>&, cudaStream_t);
template cudaError_t launch_x_class<float, 9, 9, TableOp>(XArgs<float>&, cudaStream_t);
template cudaError_t launch_x_class<double, 9, 9, TableOp>(XArgs<double>&, cudaStream_t);

template <typename T>
cudaError_t launch_btab_fill(const ElasticConst<T>& ec, int n0, int n1, int n2, T* tab, cudaStream_t s) {
  const int d0 = n0 / 2 + 1, d1 = n1 / 2 + 1, d2 = n2 / 2 + 1;
  const long long npt = (long long)d0 * d1 * d2;
  long long nb = (npt + 127) / 128;
  if (nb > 148 * 32) nb = 148 * 32;
  const int c = btab_class(ec.nb);
  if (c == 3)
    k_btab_fill<T, 3><<<(unsigned)nb, 128, 0, s>>>(ec, n0, n1, n2, d0, d1, d2, tab);
  else if (c == 5)
    k_btab_fill<T, 5><<<(unsigned)nb, 128, 0, s>>>(ec, n0, n1, n2, d0, d1, d2, tab);
  else
    k_btab_fill<T, 9><<<(unsigned)nb, 128, 0, s>>>(ec, n0, n1, n2, d0, d1, d2, tab);
  return cudaGetLastError();
}
template cudaError_t launch_btab_fill<float>(const ElasticConst<float>&, int, int, int, float*, cudaStream_t);
template cudaError_t launch_btab_fill<double>(const ElasticConst<double>&, int, int, int, double*, cudaStream_t);
}  // namespace gs
