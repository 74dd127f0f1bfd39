// gs_cufft.cu -- the cuFFT comparator step, kept only as a timed comparison.
//
// The martensite step with the library FFT in place of the hand-written
// passes and everything else as in the product step:
//   cufftExecR2C of eta^2, batched over the V variants (planned once),
//   one contraction sweep over the half spectrum [V][n0][n1][n2/2+1] (the
//     octant B table of the product step, or B formed per k when B is not
//     even in every axis),
//   cufftExecC2R of R, batched over V,
//   the product's fused update kernel (k_mart_update) without its z
//     transforms: R read in real space, eta' written, and eta'^2 written as
//     the next step's R2C input.
// The reference performs the same convolution with cufftPlanMany C2C on
// complex copies (src/dynamics_mart.cu:113-117,281-303) and B streamed from
// a [V][V][N] array (src/gtensorb.cu:55-108); gs_plain.cu keeps that
// structure.  Never called by gs_sim_step.
#include <cufft.h>

#include <cstring>

#include "gs_launch.h"
#include "gs_mart.cuh"
#include "gs_sim.h"

using namespace gs;

struct gs_cufft_state {
  cufftHandle r2c = 0, c2r = 0;
  void* spec = nullptr;  // [V][n0][n1][n2/2+1] complex
  void* R = nullptr;     // [V][N] real: the elastic potentials
  void* sq = nullptr;    // [V][N] real: eta^2 of the current field
  long long M = 0;       // points of one half spectrum
  bool sq_valid = false;  // sq holds eta[sq_cur]^2 of step sq_step
  int sq_cur = -1;
  int64_t sq_step = -1;
};

template <typename T> void build_elastic(const gs_sim* s, int which, double scale, ElasticConst<T>& ec);
template <typename T> void build_mart(const gs_sim* s, MartConst<T>& mc);

namespace {

// one thread per half-spectrum point: the V spectra in, R-hat out (in place)
template <typename T, int FM, class Op>
__global__ void k_cufft_contract(XArgs<T> a, cplx<T>* spec, long long M, int hz) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= M) return;
  const int iz = (int)(idx % hz);
  const long long r = idx / hz;
  const int iy = (int)(r % a.n1), ix = (int)(r / a.n1);
  const int nn[3] = {a.n0, a.n1, a.n2};
  cplx<T> in[FM], out[FM];
#pragma unroll
  for (int f = 0; f < FM; ++f) in[f] = f < a.F ? spec[f * M + idx] : mk2((T)0, (T)0);
  Op::template apply<T, FM, FM>(a, nn, ix, iy, iz, in, out);
#pragma unroll
  for (int g = 0; g < FM; ++g)
    if (g < a.G) spec[g * M + idx] = out[g];
}

template <typename T> __global__ void k_cufft_square(const T* eta, T* sq, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sq[i] = eta[i] * eta[i];
}

template <typename T, int FM, class Op> cudaError_t contract_n(XArgs<T>& a, cplx<T>* spec, long long M, int hz,
                                                               cudaStream_t st) {
  const unsigned blocks = (unsigned)((M + 127) / 128);
  k_cufft_contract<T, FM, Op><<<blocks, 128, 0, st>>>(a, spec, M, hz);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_contract(XArgs<T>& a, cplx<T>* spec, long long M, int hz, cudaStream_t st) {
  if (a.btab) {
    switch (btab_class(a.F)) {
      case 3: return contract_n<T, 3, TableOp>(a, spec, M, hz, st);
      case 5: return contract_n<T, 5, TableOp>(a, spec, M, hz, st);
      default: return contract_n<T, 9, TableOp>(a, spec, M, hz, st);
    }
  }
  if (a.F <= 4) return contract_n<T, 4, ContractOp>(a, spec, M, hz, st);
  return contract_n<T, GS_MAXF, ContractOp>(a, spec, M, hz, st);
}

// the update kernel without its z transforms: rows of n2 cells, a block of
// about 256 threads (one run of CW cells each), no shared memory
template <typename T, int H, int VM> cudaError_t upd_n(MartArgs<T>& a, cudaStream_t st) {
  constexpr int CW = (2 * H) % 4 == 0 ? 4 : 2;
  const int upr = a.n2 / CW;
  long long lr = upr >= 256 ? 1 : 256 / upr;
  if (lr > a.nrows) lr = a.nrows;
  a.lr = (int)lr;
  const int threads = (int)(lr * upr < 256 ? lr * upr : 256);
  const long long grid = (a.nrows + lr - 1) / lr;
  k_mart_update<T, H, VM, false, false, true, false><<<dim3((unsigned)grid, 1), (unsigned)threads, 0, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int H> cudaError_t upd_h(MartArgs<T>& a, cudaStream_t st) {
  if constexpr (sizeof(T) == 4) {
    if (a.mc.V == 3) return upd_n<T, H, 3>(a, st);
  }
  if (a.mc.V == 2) return upd_n<T, H, 2>(a, st);
  if (a.mc.V <= 4) return upd_n<T, H, 4>(a, st);
  return upd_n<T, H, 8>(a, st);
}

template <typename T> cudaError_t launch_update_rg(MartArgs<T>& a, int H, cudaStream_t st) {
  switch (H) {
#define GS_C(N_) \
  case N_:       \
    return upd_h<T, N_>(a, st);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T> int cufft_init(gs_sim* s) {
  gs_cufft_state* cs = s->cufft;
  const int V = s->p.nvariants;
  const long long N = s->N;
  const int hz = s->n2 / 2 + 1;
  cs->M = (long long)s->n0 * s->n1 * hz;
  if (gs_cuda_check(cudaMalloc(&cs->spec, sizeof(cplx<T>) * cs->M * V), "cufft spectra") != GS_OK) return GS_ENOMEM;
  if (gs_cuda_check(cudaMalloc(&cs->R, sizeof(T) * N * V), "cufft potentials") != GS_OK) return GS_ENOMEM;
  if (gs_cuda_check(cudaMalloc(&cs->sq, sizeof(T) * N * V), "cufft squares") != GS_OK) return GS_ENOMEM;
  int n[3] = {s->n0, s->n1, s->n2};
  // unit axes lead the canonical grid: plan over the remaining ones
  const int rank = s->n0 > 1 ? 3 : (s->n1 > 1 ? 2 : 1);
  const bool f64 = sizeof(T) == 8;
  if (cufftPlanMany(&cs->r2c, rank, n + (3 - rank), nullptr, 1, (int)N, nullptr, 1, (int)cs->M,
                    f64 ? CUFFT_D2Z : CUFFT_R2C, V) != CUFFT_SUCCESS ||
      cufftPlanMany(&cs->c2r, rank, n + (3 - rank), nullptr, 1, (int)cs->M, nullptr, 1, (int)N,
                    f64 ? CUFFT_Z2D : CUFFT_C2R, V) != CUFFT_SUCCESS)
    return gs_set_error(GS_ECUDA, "cufftPlanMany (R2C / C2R) failed");
  return GS_OK;
}

template <typename T> int cufft_step(gs_sim* s, cudaStream_t st) {
  gs_cufft_state* cs = s->cufft;
  const int V = s->p.nvariants;
  const long long N = s->N, NV = N * V;
  const int hz = s->n2 / 2 + 1;
  const T* in = reinterpret_cast<const T*>(s->eta[s->cur]);
  T* out = reinterpret_cast<T*>(s->eta[s->cur ^ 1]);
  T* sq = reinterpret_cast<T*>(cs->sq);
  T* R = reinterpret_cast<T*>(cs->R);
  cplx<T>* spec = reinterpret_cast<cplx<T>*>(cs->spec);
  int launches = 0;
  if (!(cs->sq_valid && cs->sq_cur == s->cur && cs->sq_step == s->step)) {  // first step, or a field was set
    k_cufft_square<T><<<(unsigned)((NV + 255) / 256), 256, 0, st>>>(in, sq, NV);
    ++launches;
  }
  cufftSetStream(cs->r2c, st);
  cufftSetStream(cs->c2r, st);
  cufftResult r1, r2;
  if constexpr (sizeof(T) == 8)
    r1 = cufftExecD2Z(cs->r2c, reinterpret_cast<cufftDoubleReal*>(sq), reinterpret_cast<cufftDoubleComplex*>(spec));
  else
    r1 = cufftExecR2C(cs->r2c, reinterpret_cast<cufftReal*>(sq), reinterpret_cast<cufftComplex*>(spec));
  XArgs<T> xa;
  memset(&xa, 0, sizeof(xa));
  xa.n0 = s->n0;
  xa.n1 = s->n1;
  xa.n2 = s->n2;
  xa.h = s->h;
  xa.F = V;
  xa.G = V;
  build_elastic<T>(s, 0, 1.0 / (double)N, xa.ec);
  if (s->btab_state == 1 && s->btab_fields == V) {  // the product step's octant table
    xa.btab = reinterpret_cast<const T*>(s->btab);
    xa.bt_d1 = s->n1 / 2 + 1;
    xa.bt_d2 = s->n2 / 2 + 1;
    xa.bt_stride = btab_stride(V);
  }
  if (gs_cuda_check(launch_contract<T>(xa, spec, cs->M, hz, st), "cufft contraction") != GS_OK) return GS_ECUDA;
  if constexpr (sizeof(T) == 8)
    r2 = cufftExecZ2D(cs->c2r, reinterpret_cast<cufftDoubleComplex*>(spec), reinterpret_cast<cufftDoubleReal*>(R));
  else
    r2 = cufftExecC2R(cs->c2r, reinterpret_cast<cufftComplex*>(spec), reinterpret_cast<cufftReal*>(R));
  if (r1 != CUFFT_SUCCESS || r2 != CUFFT_SUCCESS) return gs_set_error(GS_ECUDA, "cufftExec failed");
  MartArgs<T> ma;
  memset(&ma, 0, sizeof(ma));
  ma.eta_in = in;
  ma.eta_out = out;
  ma.defect = reinterpret_cast<const T*>(s->defect);
  ma.K = reinterpret_cast<const T*>(s->K);
  ma.n0 = s->n0;
  ma.n1 = s->n1;
  ma.n2 = s->n2;
  ma.nrows = (long long)s->n0 * s->n1;
  build_mart<T>(s, ma.mc);
  ma.fd_n1 = FastDiv((uint32_t)s->n1);
  ma.fd_upr = FastDiv((uint32_t)(s->n2 % 4 == 0 ? s->n2 / 4 : s->n2 / 2));
  ma.fd_v = FastDiv((uint32_t)V);
  ma.r_in = R;
  ma.sq_out = sq;
  if (gs_cuda_check(launch_update_rg<T>(ma, s->h, st), "cufft update") != GS_OK) return GS_ECUDA;
  launches += 2;  // contraction, update (the cuFFT kernels are the library's)
  s->launches += launches;
  s->cur ^= 1;
  s->step += 1;
  cs->sq_valid = true;
  cs->sq_cur = s->cur;
  cs->sq_step = s->step;
  return GS_OK;
}

}  // namespace

void gs_cufft_free(gs_sim* s) {
  if (!s || !s->cufft) return;
  gs_cufft_state* cs = s->cufft;
  if (cs->r2c) cufftDestroy(cs->r2c);
  if (cs->c2r) cufftDestroy(cs->c2r);
  void* p[] = {cs->spec, cs->R, cs->sq};
  for (void* q : p)
    if (q) cudaFree(q);
  delete cs;
  s->cufft = nullptr;
}

// a field upload makes the kept eta^2 stale
void gs_cufft_invalidate(gs_sim* s) {
  if (s && s->cufft) s->cufft->sq_valid = false;
}

extern "C" int gs_cufft_create(const gs_params* p, gs_sim** out) {
  if (!p || !out) return gs_set_error(GS_EINVAL, "gs_cufft_create: null argument");
  if (p->model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "gs_cufft_create: martensite only");
  int rc = gs_sim_create(p, out);
  if (rc != GS_OK) return rc;
  gs_sim* s = *out;
  s->cufft = new gs_cufft_state();
  rc = p->dtype == GS_DTYPE_F64 ? cufft_init<double>(s) : cufft_init<float>(s);
  if (rc != GS_OK) {
    gs_sim_destroy(s);
    *out = nullptr;
  }
  return rc;
}

extern "C" int gs_cufft_step(gs_sim* s, int nsteps, void* stream) {
  if (!s || !s->cufft) return gs_set_error(GS_EINVAL, "gs_cufft_step: not a cuFFT comparator handle");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
  s->launches = 0;
  for (int i = 0; i < nsteps; ++i) {
    int rc = s->p.dtype == GS_DTYPE_F64 ? cufft_step<double>(s, st) : cufft_step<float>(s, st);
    if (rc != GS_OK) return rc;
  }
  return GS_OK;
}
