// gs_plain.cu -- the plain cuFFT GPU step, kept only as a timed comparator.
//
// It has the reference's structure (src/dynamics_mart.cu:281-303,348-387):
// complex copies of eta^2, cufftPlanMany C2C batched over the variants, a
// precomputed B array [V][V][N] streamed every step (src/gtensorb.cu), and
// one full-field sweep per term.  Same discretisation as the product step,
// so it is checked against the same oracle.  Never called by gs_sim_step.
#include <cufft.h>

#include <cstring>

#include "gs_launch.h"
#include "gs_mart.cuh"
#include "gs_sim.h"

using namespace gs;

struct gs_plain_state {
  cufftHandle plan = 0;
  void* ct = nullptr;    // complex eta^2, [V][N]
  void* B = nullptr;     // [V][V][N]
  void* grad = nullptr;  // [V][N]
  void* chem = nullptr;
  void* elf = nullptr;
};

template <typename T> void build_elastic(const gs_sim* s, int which, double scale, ElasticConst<T>& ec);
template <typename T> void build_mart(const gs_sim* s, MartConst<T>& mc);

namespace {

struct PGeo {
  int n0, n1, n2, V;
  long long N;
  int perm[3];
};

template <typename T> __global__ void k_plain_bfill(T* B, ElasticConst<T> ec, PGeo g) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.N) return;
  const int z = (int)(idx % g.n2), y = (int)((idx / g.n2) % g.n1), x = (int)(idx / ((long long)g.n1 * g.n2));
  const int id[3] = {x, y, z}, nn[3] = {g.n0, g.n1, g.n2};
  T k[3];
  for (int c = 0; c < 3; ++c) k[c] = ec.kscale[c] * (T)fold_idx(id[c], nn[c], ec.refcompat);
  // column b of B: contract a unit input vector e_b
  for (int b = 0; b < g.V; ++b) {
    cplx<T> in[GS_MAXF], out[GS_MAXF];
    for (int f = 0; f < GS_MAXF; ++f) in[f] = mk2(f == b ? (T)1 : (T)0, (T)0);
    for (int a = 0; a < GS_MAXF; ++a) out[a] = mk2((T)0, (T)0);
    contract_k<T, GS_MAXF, GS_MAXF>(ec, k, in, out, ec.scale);
    for (int a = 0; a < g.V; ++a) B[((long long)a * g.V + b) * g.N + idx] = out[a].x;
  }
}

__device__ __forceinline__ long long wrapi(long long i, long long n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

template <typename T> __global__ void k_plain_grad(const T* eta, T* grad, PGeo g, MartConst<T> mc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N * g.V) return;
  const long long v = i / g.N, idx = i % g.N;
  const int z = (int)(idx % g.n2), y = (int)((idx / g.n2) % g.n1), x = (int)(idx / ((long long)g.n1 * g.n2));
  const T* e = eta + v * g.N;
  const T c = e[idx];
  auto at = [&](long long xx, long long yy, long long zz) {
    return e[(wrapi(xx, g.n0) * g.n1 + wrapi(yy, g.n1)) * g.n2 + wrapi(zz, g.n2)];
  };
  grad[i] = mc.lapc[0] * (at(x + 1, y, z) + at(x - 1, y, z) - 2 * c) +
            mc.lapc[1] * (at(x, y + 1, z) + at(x, y - 1, z) - 2 * c) +
            mc.lapc[2] * (at(x, y, z + 1) + at(x, y, z - 1) - 2 * c);
}

template <typename T> __global__ void k_plain_chem(const T* eta, T* chem, PGeo g, MartConst<T> mc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N * g.V) return;
  const long long v = i / g.N, idx = i % g.N;
  const T et = eta[i];
  T s2 = 0;
  for (int q = 0; q < g.V; ++q) {
    const T eq = eta[q * g.N + idx];
    s2 += eq * eq;
  }
  T out;
  if (mc.refcompat) {
    const T se = mc.s * et;
    out = et >= (T)0 ? -mc.wC * se * (mc.a1 - mc.a2 * se * se + mc.a3 * mc.s * mc.s * s2)
                     : (T)1000 * mc.wC * mc.a2 * et * et;
  } else {
    const T e2 = et * et;
    out = -mc.L * (mc.A2 * et - mc.A4 * e2 * et + mc.A6 * s2 * s2 * et + (T)2 * mc.Ac * et * (s2 - e2));
  }
  (void)v;
  chem[i] = out;
}

template <typename T> __global__ void k_plain_square(const T* eta, cplx<T>* ct, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T e = eta[i];
  ct[i] = mk2(e * e, (T)0);
}

template <typename T> __global__ void k_plain_contract(const cplx<T>* ct, cplx<T>* rt, const T* B, PGeo g) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N * g.V) return;
  const long long v = i / g.N, idx = i % g.N;
  cplx<T> s = mk2((T)0, (T)0);
  for (int q = 0; q < g.V; ++q) s = s + ct[q * g.N + idx] * B[(v * g.V + q) * g.N + idx];
  rt[i] = s;
}

template <typename T> __global__ void k_plain_elastic(const cplx<T>* rt, const T* eta, T* elf, long long n, T el) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  elf[i] = el * rt[i].x * eta[i];
}

template <typename T>
__global__ void k_plain_update(const T* eta, T* out, const T* grad, const T* chem, const T* elf, const T* K,
                               const T* defect, PGeo g, MartConst<T> mc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N * g.V) return;
  const int v = (int)(i / g.N);
  const long long idx = i % g.N;
  const T et = eta[i];
  const T Kv = K ? K[i] : (T)0;
  T rhs = grad[i] + chem[i] + elf[i] + (mc.lin[v] + mc.kc * Kv) * et;
  T xi = 0;
  if (mc.noise != (T)0) {
    T z[4];
    normal_quad<T>((uint32_t)(idx >> 2), mc.step, mc.sim, (uint32_t)v, mc.k0, mc.k1, z);
    xi = z[idx & 3];
  }
  T en = et + mc.dt * rhs + mc.noise * xi;
  if (defect) en *= (T)1 - defect[idx];
  out[i] = en;
}

inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }

template <typename T> int plain_init(gs_sim* s) {
  gs_plain_state* ps = s->plain;
  const int V = s->p.nvariants;
  const long long N = s->N;
  const size_t rb = (size_t)N * V * sizeof(T);
  // two complex arrays of V*N elements: eta^2 spectrum and the contraction
  if (gs_cuda_check(cudaMalloc(&ps->ct, 2 * 2 * rb), "plain ct") != GS_OK) return GS_ENOMEM;
  if (gs_cuda_check(cudaMalloc(&ps->B, rb * V), "plain B") != GS_OK) return GS_ENOMEM;
  if (gs_cuda_check(cudaMalloc(&ps->grad, rb), "plain grad") != GS_OK) return GS_ENOMEM;
  if (gs_cuda_check(cudaMalloc(&ps->chem, rb), "plain chem") != GS_OK) return GS_ENOMEM;
  if (gs_cuda_check(cudaMalloc(&ps->elf, rb), "plain elastic") != GS_OK) return GS_ENOMEM;
  int n[3] = {s->n0, s->n1, s->n2};
  // unit axes lead the canonical grid: plan over the remaining ones
  const int rank = s->n0 > 1 ? 3 : (s->n1 > 1 ? 2 : 1);
  const cufftType ty = sizeof(T) == 8 ? CUFFT_Z2Z : CUFFT_C2C;
  if (cufftPlanMany(&ps->plan, rank, n + (3 - rank), nullptr, 1, (int)N, nullptr, 1, (int)N, ty, V) != CUFFT_SUCCESS)
    return gs_set_error(GS_ECUDA, "cufftPlanMany failed");
  PGeo g{s->n0, s->n1, s->n2, V, N, {s->perm[0], s->perm[1], s->perm[2]}};
  ElasticConst<T> ec;
  build_elastic<T>(s, 0, 1.0 / (double)N, ec);
  k_plain_bfill<T><<<nblk(N), 256, 0, s->own_stream>>>(reinterpret_cast<T*>(ps->B), ec, g);
  if (gs_cuda_check(cudaStreamSynchronize(s->own_stream), "plain B fill") != GS_OK) return GS_ECUDA;
  return GS_OK;
}

template <typename T> int plain_step(gs_sim* s, cudaStream_t st) {
  gs_plain_state* ps = s->plain;
  const int V = s->p.nvariants;
  const long long N = s->N, NV = N * V;
  PGeo g{s->n0, s->n1, s->n2, V, N, {s->perm[0], s->perm[1], s->perm[2]}};
  MartConst<T> mc;
  build_mart<T>(s, mc);
  const T* in = reinterpret_cast<const T*>(s->eta[s->cur]);
  T* out = reinterpret_cast<T*>(s->eta[s->cur ^ 1]);
  cplx<T>* ct = reinterpret_cast<cplx<T>*>(ps->ct);
  cplx<T>* rt = ct + NV;
  k_plain_grad<T><<<nblk(NV), 256, 0, st>>>(in, reinterpret_cast<T*>(ps->grad), g, mc);
  k_plain_chem<T><<<nblk(NV), 256, 0, st>>>(in, reinterpret_cast<T*>(ps->chem), g, mc);
  k_plain_square<T><<<nblk(NV), 256, 0, st>>>(in, ct, NV);
  cufftSetStream(ps->plan, st);
  cufftResult r1, r2;
  if (sizeof(T) == 8) {
    r1 = cufftExecZ2Z(ps->plan, (cufftDoubleComplex*)ct, (cufftDoubleComplex*)ct, CUFFT_FORWARD);
  } else {
    r1 = cufftExecC2C(ps->plan, (cufftComplex*)ct, (cufftComplex*)ct, CUFFT_FORWARD);
  }
  k_plain_contract<T><<<nblk(NV), 256, 0, st>>>(ct, rt, reinterpret_cast<const T*>(ps->B), g);
  if (sizeof(T) == 8) {
    r2 = cufftExecZ2Z(ps->plan, (cufftDoubleComplex*)rt, (cufftDoubleComplex*)rt, CUFFT_INVERSE);
  } else {
    r2 = cufftExecC2C(ps->plan, (cufftComplex*)rt, (cufftComplex*)rt, CUFFT_INVERSE);
  }
  if (r1 != CUFFT_SUCCESS || r2 != CUFFT_SUCCESS) return gs_set_error(GS_ECUDA, "cufftExec failed");
  k_plain_elastic<T><<<nblk(NV), 256, 0, st>>>(rt, in, reinterpret_cast<T*>(ps->elf), NV, mc.el);
  k_plain_update<T><<<nblk(NV), 256, 0, st>>>(in, out, reinterpret_cast<const T*>(ps->grad),
                                             reinterpret_cast<const T*>(ps->chem),
                                             reinterpret_cast<const T*>(ps->elf), reinterpret_cast<const T*>(s->K),
                                             reinterpret_cast<const T*>(s->defect), g, mc);
  if (gs_cuda_check(cudaGetLastError(), "plain step") != GS_OK) return GS_ECUDA;
  s->launches += 6;
  s->cur ^= 1;
  s->step += 1;
  return GS_OK;
}

}  // namespace

void gs_plain_free(gs_sim* s) {
  if (!s || !s->plain) return;
  gs_plain_state* ps = s->plain;
  if (ps->plan) cufftDestroy(ps->plan);
  void* p[] = {ps->ct, ps->B, ps->grad, ps->chem, ps->elf};
  for (void* q : p)
    if (q) cudaFree(q);
  delete ps;
  s->plain = nullptr;
}

extern "C" int gs_plain_create(const gs_params* p, gs_sim** out) {
  int rc = gs_sim_create(p, out);
  if (rc != GS_OK) return rc;
  gs_sim* s = *out;
  s->plain = new gs_plain_state();
  rc = p->dtype == GS_DTYPE_F64 ? plain_init<double>(s) : plain_init<float>(s);
  if (rc != GS_OK) {
    gs_sim_destroy(s);
    *out = nullptr;
  }
  return rc;
}

extern "C" int gs_plain_step(gs_sim* s, int nsteps, void* stream) {
  if (!s || !s->plain) return gs_set_error(GS_EINVAL, "gs_plain_step: not a comparator handle");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
  s->launches = 0;
  for (int i = 0; i < nsteps; ++i) {
    int rc = s->p.dtype == GS_DTYPE_F64 ? plain_step<double>(s, st) : plain_step<float>(s, st);
    if (rc != GS_OK) return rc;
  }
  return GS_OK;
}
