// gs_k_precip.cu -- launchers of the z-inverse-to-real pass and of the
// precipitate / stress real-space sweeps.
#include "gs_launch.h"
#include "gs_precip.cuh"

namespace gs {

template <typename T, int H> static cudaError_t zinv_n(ZinvArgs<T>& a, cudaStream_t s) {
  using L = Line<T, H>;
  GS_RANGE(a.spec, a.nrows * H, cplx<T>, sizeof(cplx<T>), "z inverse", "spectrum");
  for (long long f = 0; bounds_check_on() && f < a.nrows / a.rows_per_field; ++f)
    GS_RANGE(a.dst[f], a.rows_per_field * 2 * H, T, sizeof(cplx<T>), "z inverse", "field");
  long long lpc = 256 / L::P;
  if (lpc < 1) lpc = 1;
  if (lpc > a.nrows) lpc = a.nrows;
  a.lpc = (int)lpc;
  const size_t smem = (size_t)lpc * L::PAD * sizeof(cplx<T>);
  allow_max_smem<k_zinv<T, H>>();
  const long long grid = (a.nrows + lpc - 1) / lpc;
  k_zinv<T, H><<<(unsigned)grid, (unsigned)(L::P * lpc), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_zinv(ZinvArgs<T>& a, int H, cudaStream_t s) {
  switch (H) {
#define GS_C(N_) \
  case N_:       \
    return zinv_n<T, N_>(a, s);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

static unsigned grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (unsigned)g;
}

template <typename T, int H, int VM> static cudaError_t pmid_n(PrecipMidArgs<T>& a, cudaStream_t s) {
  using L = Line<T, H>;
  const int per = L::P * (a.loc.V + 2);  // threads of one row
  if (per > 256) return cudaErrorInvalidConfiguration;
  const long long N = a.nrows * 2 * H;
  GS_RANGE(a.rspec, (long long)a.F1 * a.nrows * H, cplx<T>, sizeof(cplx<T>), "precipitate middle sweep", "R spectra");
  constexpr size_t va = (2 * H) % 4 == 0 ? 4 * sizeof(T) : 2 * sizeof(T);  // the sweep's vector loads
  GS_RANGE(a.c, N, T, sizeof(cplx<T>), "precipitate middle sweep", "concentration");
  GS_RANGE(a.eta, (long long)a.loc.V * N, T, va < 16 ? va : 16, "precipitate middle sweep", "order parameters");
  GS_RANGE(a.dst, (long long)(a.loc.V + 2) * a.nrows * H, cplx<T>, sizeof(cplx<T>), "precipitate middle sweep",
           "update spectra");
  long long lr = 256 / per;
  if (a.lr_req > 0 && (long long)a.lr_req * per <= 256) lr = a.lr_req;
  if (lr > a.nrows) lr = a.nrows;
  a.lr = (int)lr;
  const int CW = (2 * H) % 4 == 0 ? 4 : 2;
  a.fd_upr = FastDiv((uint32_t)(a.n2 / CW));
  const size_t smem = (size_t)lr * (a.loc.V + 2) * L::PAD * sizeof(cplx<T>);
  allow_max_smem<k_precip_mid<T, H, VM>>();
  const long long grid = (a.nrows + lr - 1) / lr;
  k_precip_mid<T, H, VM><<<(unsigned)grid, (unsigned)(per * lr), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_precip_mid(PrecipMidArgs<T>& a, int H, cudaStream_t s) {
  switch (H) {
#define GS_C(N_) \
  case N_:       \
    return a.loc.V <= 4 ? pmid_n<T, N_, 4>(a, s) : pmid_n<T, N_, 8>(a, s);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T, int H> static cudaError_t pzf_n(PrecipZArgs<T>& a, cudaStream_t s) {
  using L = Line<T, H>;
  const int per = L::P * (a.V + 1);  // threads of one row
  if (per > 256) return cudaErrorInvalidConfiguration;
  GS_RANGE(a.spec, (long long)(a.F1 > a.V + 1 ? a.F1 : a.V + 1) * a.nrows * H, cplx<T>, sizeof(cplx<T>),
           "precipitate last sweep", "spectra");
  GS_RANGE(a.c, a.N, T, sizeof(cplx<T>), "precipitate last sweep", "concentration");
  GS_RANGE(a.eta, (long long)a.V * a.N, T, sizeof(cplx<T>), "precipitate last sweep", "order parameters");
  long long lr = 256 / per;
  if (lr > a.nrows) lr = a.nrows;
  a.lr = (int)lr;
  const size_t smem = (size_t)lr * (a.V + 1) * L::PAD * sizeof(cplx<T>);
  allow_max_smem<k_precip_zinv_fwd<T, H>>();
  const long long grid = (a.nrows + lr - 1) / lr;
  k_precip_zinv_fwd<T, H><<<(unsigned)grid, (unsigned)(per * lr), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_precip_zinv_fwd(PrecipZArgs<T>& a, int H, cudaStream_t s) {
  switch (H) {
#define GS_C(N_) \
  case N_:       \
    return pzf_n<T, N_>(a, s);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T> cudaError_t launch_precip_local(PrecipLocalArgs<T>& a, cudaStream_t s) {
  k_precip_local<T><<<grid_for((a.N + 3) / 4, 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_defect(const T* eta, T* defect, long long N, int V, cudaStream_t s) {
  k_defect<T><<<grid_for(N, 256), 256, 0, s>>>(eta, defect, N, V, (T)0.9);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_precip_stats(PrecipStatsArgs<T>& a, cudaStream_t s, int* nblocks) {
  const unsigned g = grid_for(a.N, 256);
  *nblocks = (int)g;
  k_precip_stats<T><<<g, 256, 0, s>>>(a);
  return cudaGetLastError();
}

#define GS_INST(T)                                                                         \
  template cudaError_t launch_zinv<T>(ZinvArgs<T>&, int, cudaStream_t);                    \
  template cudaError_t launch_precip_local<T>(PrecipLocalArgs<T>&, cudaStream_t);          \
  template cudaError_t launch_precip_mid<T>(PrecipMidArgs<T>&, int, cudaStream_t);          \
  template cudaError_t launch_precip_zinv_fwd<T>(PrecipZArgs<T>&, int, cudaStream_t);       \
  template cudaError_t launch_defect<T>(const T*, T*, long long, int, cudaStream_t);       \
  template cudaError_t launch_precip_stats<T>(PrecipStatsArgs<T>&, cudaStream_t, int*);
GS_INST(float)
GS_INST(double)
#undef GS_INST

}  // namespace gs
