// gs_precip.cuh -- real-space sweeps of the precipitate and stress models.
//
// Precipitate (src/dynamics_precipitate.cu:118-195): from c, eta_p and the
// elastic potentials R_a build mu_c (LocalConFreeEnergy, :118-127) and
// g_p = dF/deta_p + Xi 2 eta_p R_p (LocalEtaFreeEnergy :136-162 and the
// elastic term :193,257), with the Philox noise terms; they are the inputs
// of the semi-implicit update in k space.  Stress (src/dynamics_stress.cu:
// 184-191): the defect mask |eta_v| > 0.9, on the device.
#pragma once
#include <type_traits>

#include "gs_mart.cuh"

namespace gs {

template <typename T> struct PrecipLocalArgs {
  const T* c;
  const T* eta;  // [V][N]
  const T* R;    // [F1][N]: R of eta_p^2 (p < V), then of c when c couples
  T* mu;         // [N]
  T* g;          // [V][N]
  long long N;
  int V, c_elastic;
  T A[8], c1, c2, Es, an;  // coefficients, Xi * w_el, noise amplitude
  uint32_t k0, k1, sim, step;
  // fold = 1: g holds u_p = eta_p - dt L g_p (the only combination of eta_p
  // and g_p the semi-implicit update transforms: FFT is linear)
  int fold;
  T dtL;
};

// Lane-wise arithmetic with one rounding per operation, on a scalar or on a
// packed FP32 pair (two cells per instruction): the local terms below are
// written once in these operations, so the packed and the scalar sweeps give
// the same bits lane by lane.
__device__ __forceinline__ float lfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double lfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float2 lfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float lmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double lmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float2 lmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float ladd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double ladd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float2 ladd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float lsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double lsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float2 lsub(float2 a, float2 b) { return psub(a, b); }
template <typename X, typename T> __device__ __forceinline__ X lbc(T s) {
  if constexpr (sizeof(X) == 2 * sizeof(T))
    return X{s, s};
  else
    return s;
}

// mu_c at one cell (s1 = sum_p eta_p^2; rc = R of c when c couples)
//   mu = A1 (c - c1) + A2/2 s1 [+ Xi w_el R_c] + noise z
template <typename X, typename T>
__device__ __forceinline__ X precip_mu(const PrecipLocalArgs<T>& a, X c, X s1, X rc, X z) {
  X mu = lfma(lbc<X>(a.A[1]), lsub(c, lbc<X>(a.c1)), lmul(lbc<X>(a.A[2] / (T)2), s1));
  if (a.c_elastic) mu = lfma(lbc<X>(a.Es), rc, mu);
  return lfma(lbc<X>(a.an), z, mu);
}

// g_p at one cell (t2, t4: sums of eta_r^2, eta_r^4 over r != p)
//   g = (2 A5 x + 4 A6 x^3) t2 + 2 A6 x t4 + 2 A7 x (t2^2 - t4) + A2 x (c - c2)
//       - A3 x^3 + A4 x^5 + 2 Xi w_el x R_p + noise z
template <typename X, typename T>
__device__ __forceinline__ X precip_g(const PrecipLocalArgs<T>& a, X c, X x, X t2, X t4, X rp, X z) {
  const X t22 = lsub(lmul(t2, t2), t4);  // sum over ordered pairs i != j, both != p
  const X x2 = lmul(x, x);
  const X x3 = lmul(x2, x);
  X gv = lfma(lbc<X>((T)4 * a.A[6]), x3, lmul(lbc<X>((T)2 * a.A[5]), x));
  gv = lmul(gv, t2);
  gv = lfma(lmul(lbc<X>((T)2 * a.A[6]), x), t4, gv);
  gv = lfma(lmul(lbc<X>((T)2 * a.A[7]), x), t22, gv);
  gv = lfma(lmul(lbc<X>(a.A[2]), x), lsub(c, lbc<X>(a.c2)), gv);
  gv = lfma(lbc<X>(-a.A[3]), x3, gv);
  gv = lfma(lmul(lbc<X>(a.A[4]), lmul(x2, x2)), x, gv);
  gv = lfma(lmul(lbc<X>((T)2 * a.Es), x), rp, gv);
  return lfma(lbc<X>(a.an), z, gv);
}

template <typename T>
__global__ void k_precip_local(PrecipLocalArgs<T> a) {
  const long long nq = (a.N + 3) >> 2;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x) {
    T zc[4] = {0, 0, 0, 0};
    if (a.an != (T)0) normal_quad<T>((uint32_t)q, a.step, a.sim, (uint32_t)a.V, a.k0, a.k1, zc);
    for (int j = 0; j < 4; ++j) {
      const long long i = 4 * q + j;
      if (i >= a.N) break;
      const T c = a.c[i];
      T s1 = 0, s2 = 0;
      for (int p = 0; p < a.V; ++p) {
        const T e = a.eta[p * a.N + i];
        s1 += e * e;
        s2 += e * e * e * e;
      }
      a.mu[i] = precip_mu(a, c, s1, a.c_elastic ? a.R[(long long)a.V * a.N + i] : (T)0, zc[j]);
    }
    for (int p = 0; p < a.V; ++p) {
      T zp[4] = {0, 0, 0, 0};
      if (a.an != (T)0) normal_quad<T>((uint32_t)q, a.step, a.sim, (uint32_t)p, a.k0, a.k1, zp);
      for (int j = 0; j < 4; ++j) {
        const long long i = 4 * q + j;
        if (i >= a.N) break;
        const T c = a.c[i];
        T t2 = 0, t4 = 0;
        for (int r = 0; r < a.V; ++r)
          if (r != p) {
            const T e = a.eta[r * a.N + i];
            t2 += e * e;
            t4 += e * e * e * e;
          }
        const T x = a.eta[p * a.N + i];
        const T gv = precip_g(a, c, x, t2, t4, a.R[p * a.N + i], zp[j]);
        a.g[p * a.N + i] = a.fold ? x - a.dtL * gv : gv;
      }
    }
  }
}

// The middle of the precipitate step in one sweep over rows: the z C2R of
// the elastic potentials R (chain 1 after its y inverse), the local terms
// mu_c and g_p, and the z R2C of the update fields [c, mu, u_0, .., u_V-1]
// (chain 2), u_p = eta_p - dt L g_p: the Allen-Cahn update
// eta_p' = D (FFT(eta_p) - dt L FFT(g_p)) needs only that combination, which
// FFT linearity lets the sweep form in real space (V + 2 transformed fields
// instead of 2V + 2).  Shared memory holds, per row, one line per update
// field in chain-2 order: c is loaded into its line, R_c and R_p are
// transformed into the lines of mu and u_p, each thread overwrites the R of
// its own cells with mu and u_p, and every line is transformed to the
// chain-2 spectrum rows.  R, mu, g and u never go to HBM.
template <typename T> struct PrecipMidArgs {
  const cplx<T>* rspec;  // [F1][rows][H]: R_eta_p^2 (p < V), then R_c
  const T* c;            // [N]
  const T* eta;          // [V][N]
  cplx<T>* dst;          // [V+2][rows][H]
  int lr_req;            // rows per block asked by the schedule (0: the launcher's choice)
  long long nrows;
  int n2, lr, F1;
  const cplx<T>* tw_h;
  const cplx<T>* tw_n2;
  FastDiv fd_upr;
  PrecipLocalArgs<T> loc;  // coefficients, noise, V, c_elastic (pointers unused)
};

// three resident blocks of 240 threads (the 256^3 tile): at 101 registers
// only two fitted, and the sweep waited on its loads and barriers with 24 %
// of the warp slots occupied
template <typename T, int H, int VM>
__global__ void __launch_bounds__(256, 3) k_precip_mid(PrecipMidArgs<T> a) {
  using L = Line<T, H>;
  using V = cplx<T>;
  constexpr int CW = (2 * H) % 4 == 0 ? 4 : 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int Vn = a.loc.V;
  const int NL = Vn + 2;  // lines per row
  const int n2 = a.n2;
  const long long N = a.nrows * n2;
  const int line = threadIdx.x / L::P, t = threadIdx.x % L::P;
  const int rr = line / NL, f2 = line - rr * NL;
  const long long row = (long long)blockIdx.x * a.lr + rr;
  const bool rok = rr < a.lr && row < a.nrows;
  GS_BC_SMEM_GUARD((long long)(blockDim.x / L::P) * L::PAD, V, BC_PMID_SMEM)
  V* sl = smb + line * L::PAD;
  // R field feeding this line: u_p lines take R_p, the mu line R_c
  int rf = -1;
  if (f2 >= 2) rf = f2 - 2;
  if (f2 == 1 && a.loc.c_elastic && a.F1 > Vn) rf = Vn;
  {
    const bool act = rok && rf >= 0;
    V r[L::R1];
    zinv_row<T, H>(a.rspec + ((long long)(rf >= 0 ? rf : 0) * a.nrows + (rok ? row : 0)) * H, act, t, sl, a.tw_h,
                   a.tw_n2, r, GS_BCX(((long long)(rf >= 0 ? rf : 0) * a.nrows + (rok ? row : 0)) * H),
                   GS_BCX((long long)a.F1 * a.nrows * H));
    __syncthreads();
    if (rf >= 0) {
#pragma unroll
      for (int i = 0; i < L::R1; ++i) sl[L::out_pos(t, i)] = r[i];
    } else if (rok && f2 == 0) {  // c: the row itself
      const V* srow = reinterpret_cast<const V*>(a.c + row * n2);
#pragma unroll
      for (int i = 0; i < L::R1; ++i) sl[L::in_pos(t, i)] = srow[GS_BCO(row * H, L::in_pos(t, i), N / 2, BC_PMID_SRC)];
    } else {
#pragma unroll
      for (int i = 0; i < L::R1; ++i) sl[L::in_pos(t, i)] = mk2((T)0, (T)0);
    }
    __syncthreads();
  }
  // local terms, one thread per run of CW cells, all fields
  const int upr = n2 / CW;
  const int nunits = a.lr * upr;
  const PrecipLocalArgs<T>& lc = a.loc;
#pragma unroll 1
  for (int w = threadIdx.x; w < nunits; w += blockDim.x) {
    const int ur = (int)a.fd_upr.div((uint32_t)w), u = w - ur * upr;
    const long long urow = (long long)blockIdx.x * a.lr + ur;
    if (urow >= a.nrows) continue;
    const int z0 = u * CW;
    const long long cell = urow * n2 + z0;
    T* const lbase = reinterpret_cast<T*>(smb + ur * NL * L::PAD) + z0;
    auto ln = [lbase](int q) { return lbase + q * (2 * L::PAD); };  // line q of this row (reals)
    T e[VM][CW];
#pragma unroll
    for (int p = 0; p < VM; ++p)
      if (p < Vn) ldv<CW>(a.eta + GS_BCR(0, (long long)p * N + cell, CW, Vn * N, BC_PMID_SRC), e[p]);
    const bool hi_pair = CW == 2 && (cell & 2);
    // the run's cells in lanes of X: FP32 runs of four as two packed pairs
    constexpr bool PK = sizeof(T) == 4 && CW == 4;
    using X = typename std::conditional<PK, float2, T>::type;
    constexpr int NX = PK ? CW / 2 : CW;
    auto lx = [](const T* q, int k) -> X {  // lane group k of a shared-memory line
      if constexpr (PK)
        return *reinterpret_cast<const float2*>(q + 2 * k);
      else
        return q[k];
    };
    auto sx = [](T* q, int k, X v) {
      if constexpr (PK)
        *reinterpret_cast<float2*>(q + 2 * k) = v;
      else
        q[k] = v;
    };
    auto rx = [](const T (&r)[CW], int k) -> X {
      if constexpr (PK)
        return X{r[2 * k], r[2 * k + 1]};
      else
        return r[k];
    };
    auto zx = [hi_pair](const T (&z)[4], int k) -> X {  // the noise of lane group k
      if constexpr (PK)
        return X{z[2 * k], z[2 * k + 1]};
      else
        return CW == 2 ? (hi_pair ? z[k + 2 < 4 ? k + 2 : 3] : z[k]) : z[k];
    };
    {
      T zc[4] = {0, 0, 0, 0};
      if (lc.an != (T)0) normal_quad<T>((uint32_t)(cell >> 2), lc.step, lc.sim, (uint32_t)Vn, lc.k0, lc.k1, zc);
#pragma unroll
      for (int k = 0; k < NX; ++k) {
        X s1 = lbc<X>((T)0);
#pragma unroll
        for (int p = 0; p < VM; ++p)
          if (p < Vn) s1 = lfma(rx(e[p], k), rx(e[p], k), s1);
        const X rc = (lc.c_elastic && a.F1 > Vn) ? lx(ln(1), k) : lbc<X>((T)0);
        sx(ln(1), k, precip_mu(lc, lx(ln(0), k), s1, rc, zx(zc, k)));
      }
    }
#pragma unroll
    for (int p = 0; p < VM; ++p) {
      if (p >= Vn) break;
      T zp[4] = {0, 0, 0, 0};
      if (lc.an != (T)0) normal_quad<T>((uint32_t)(cell >> 2), lc.step, lc.sim, (uint32_t)p, lc.k0, lc.k1, zp);
#pragma unroll
      for (int k = 0; k < NX; ++k) {
        X t2 = lbc<X>((T)0), t4 = lbc<X>((T)0);
#pragma unroll
        for (int r = 0; r < VM; ++r)
          if (r < Vn && r != p) {
            const X x2 = lmul(rx(e[r], k), rx(e[r], k));
            t2 = ladd(t2, x2);
            t4 = lfma(x2, x2, t4);
          }
        const X x = rx(e[p], k);
        const X gv = precip_g(lc, lx(ln(0), k), x, t2, t4, lx(ln(2 + p), k), zx(zp, k));
        sx(ln(2 + p), k, lfma(lbc<X>(-lc.dtL), gv, x));  // u_p = eta_p - dt L g_p
      }
    }
  }
  __syncthreads();
  V x[L::R1];
#pragma unroll
  for (int r = 0; r < L::R1; ++r) x[r] = sl[L::in_pos(t, r)];
  __syncthreads();
  zfwd_line<T, H>(x, t, sl, rok ? a.dst + ((long long)f2 * a.nrows + row) * H : nullptr, a.tw_h, a.tw_n2,
                  GS_BCX(((long long)f2 * a.nrows + row) * H), GS_BCX((long long)NL * a.nrows * H));
}

// The end of the precipitate step fused with the start of the next one: the
// z inverse of the updated spectra [c', eta'_0 .. eta'_V-1] into the fields
// (the concentration with its FP64 mass offset added before rounding, as
// k_zinv does), then the z forward of the next step's chain-1 inputs
// [eta'_p^2 (p < V), c'] from the rounded values just stored, written over
// the spectrum rows the block read.  Every field of a row lives in one block,
// so no other block reads those rows; the next step starts at its y forward.
template <typename T> struct PrecipZArgs {
  cplx<T>* spec;  // in: [V+1][rows][H] spectra of c', eta'; out: [F1][rows][H] chain-1 z spectra
  T* c;           // [N]
  T* eta;         // [V][N]
  long long nrows, N;
  int lr, V, F1;  // F1 = V + 1 when c couples elastically (its row is transformed too)
  int mass;       // add `offset` to c' in FP64
  double offset;
  const cplx<T>* tw_h;
  const cplx<T>* tw_n2;
};

template <typename T, int H>
__global__ void __launch_bounds__(256, 3) k_precip_zinv_fwd(PrecipZArgs<T> a) {
  using L = Line<T, H>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int NL = a.V + 1;  // lines per row: c', then eta'_p
  const int line = threadIdx.x / L::P, t = threadIdx.x % L::P;
  const int rr = line / NL, f = line - rr * NL;
  const long long row = (long long)blockIdx.x * a.lr + rr;
  const bool act = rr < a.lr && row < a.nrows;
  GS_BC_SMEM_GUARD((long long)(blockDim.x / L::P) * L::PAD, V, BC_PZF_SMEM)
  // the spectrum holds max(V + 1, F1) fields
  GS_BC_DECL(const long long sext = (long long)(a.F1 > NL ? a.F1 : NL) * a.nrows * H)
  V* sl = smb + line * L::PAD;
  V r[L::R1];
  // its reads of the block's spectrum rows finish before its first barrier
  zinv_row<T, H>(a.spec + ((long long)f * a.nrows + (act ? row : 0)) * H, act, t, sl, a.tw_h, a.tw_n2, r,
                 GS_BCX(((long long)f * a.nrows + (act ? row : 0)) * H), GS_BCX(sext));
  T* const dst = f == 0 ? a.c : a.eta + (long long)(f - 1) * a.N;
  const bool off = f == 0 && a.mass;
#pragma unroll
  for (int i = 0; i < L::R1; ++i) {
    V v = r[i];
    if (off) v = mk2((T)((double)v.x + a.offset), (T)((double)v.y + a.offset));
    if (act)
      reinterpret_cast<V*>(dst + row * (2 * H))[GS_BCO(((f == 0 ? 0 : (long long)(f - 1) * a.N) / 2) + row * H,
                                                       L::out_pos(t, i), (f == 0 ? a.N : (long long)a.V * a.N) / 2,
                                                       BC_PZF_FIELD)] = v;
    r[i] = f == 0 ? v : mk2(v.x * v.x, v.y * v.y);  // the chain-1 input: c' itself, eta'_p^2
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < L::R1; ++i) sl[L::out_pos(t, i)] = r[i];
  __syncthreads();
  V x[L::R1];
#pragma unroll
  for (int q = 0; q < L::R1; ++q) x[q] = sl[L::in_pos(t, q)];
  __syncthreads();
  const int f1 = f == 0 ? a.V : f - 1;  // chain-1 order: eta_p^2, then c
  const bool out = act && f1 < a.F1;
  zfwd_line<T, H>(x, t, sl, out ? a.spec + ((long long)f1 * a.nrows + row) * H : nullptr, a.tw_h, a.tw_n2,
                  GS_BCX(((long long)f1 * a.nrows + row) * H), GS_BCX(sext));
}

template <typename T>
__global__ void k_defect(const T* __restrict__ eta, T* __restrict__ defect, long long N, int V, T cut) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    T d = 0;
    for (int v = 0; v < V; ++v)
      if (fabs(eta[v * N + i]) > cut) d = 1;
    defect[i] = d;
  }
}

template <typename T> struct PrecipStatsArgs {
  const T* c;
  const T* eta;
  const T* R;
  long long N;
  int n0, n1, n2, V, c_elastic;
  T A[8], c1, c2, Es, kc, ke;
  T gcoef[3];  // 1/d^2 per canonical axis (0 on unit axes)
  double* partials;
};

template <typename T>
__device__ __forceinline__ T lap7c(const T* f, int n0, int n1, int n2, int x, int y, int z, const T (&g)[3]) {
  const long long i = ((long long)x * n1 + y) * n2 + z;
  const T c = f[i];
  const int xp = x + 1 == n0 ? 0 : x + 1, xm = x == 0 ? n0 - 1 : x - 1;
  const int yp = y + 1 == n1 ? 0 : y + 1, ym = y == 0 ? n1 - 1 : y - 1;
  const int zp = z + 1 == n2 ? 0 : z + 1, zm = z == 0 ? n2 - 1 : z - 1;
  return g[0] * (f[((long long)xp * n1 + y) * n2 + z] + f[((long long)xm * n1 + y) * n2 + z] - 2 * c) +
         g[1] * (f[((long long)x * n1 + yp) * n2 + z] + f[((long long)x * n1 + ym) * n2 + z] - 2 * c) +
         g[2] * (f[((long long)x * n1 + y) * n2 + zp] + f[((long long)x * n1 + y) * n2 + zm] - 2 * c);
}

template <typename T>
__global__ void k_precip_stats(PrecipStatsArgs<T> a) {
  Neu acc[ACC_N];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(i % a.n2), y = (int)((i / a.n2) % a.n1), x = (int)(i / ((long long)a.n1 * a.n2));
    const T c = a.c[i];
    acc[ACC_MASS].add((double)c);
    double s1 = 0, s2 = 0, s3 = 0;
    for (int p = 0; p < a.V; ++p) {
      const double e = a.eta[p * a.N + i];
      const double e2 = e * e;
      s1 += e2;
      s2 += e2 * e2;
      s3 += e2 * e2 * e2;
      acc[ACC_C].add(e);
      acc[ACC_ETA2 + p].add(e2);
      acc[ACC_VF + p].add(fabs(e) > 0.5 ? 1.0 : 0.0);
      acc[ACC_EEL].add(0.5 * (double)a.Es * e2 * (double)a.R[p * a.N + i]);
      acc[ACC_EGRAD].add(-0.5 * (double)a.ke * e * (double)lap7c(a.eta + p * a.N, a.n0, a.n1, a.n2, x, y, z, a.gcoef));
    }
    if (a.c_elastic) acc[ACC_EEL].add(0.5 * (double)a.Es * (double)c * (double)a.R[(long long)a.V * a.N + i]);
    acc[ACC_EGRAD].add(-0.5 * (double)a.kc * (double)c * (double)lap7c(a.c, a.n0, a.n1, a.n2, x, y, z, a.gcoef));
    const double dc = (double)c - (double)a.c1;
    const double f = (double)a.A[1] / 2 * dc * dc + (double)a.A[2] / 2 * ((double)c - (double)a.c2) * s1 -
                     (double)a.A[3] / 4 * s2 + (double)a.A[4] / 6 * s3 + (double)a.A[5] * (s1 * s1 - s2) / 2 +
                     (double)a.A[6] * (s2 * s1 - s3) + 2.0 * (double)a.A[7] * (s1 * s1 * s1 - 3 * s1 * s2 + 2 * s3) / 6;
    acc[ACC_ECHEM].add(f);
  }
  block_reduce_store(acc, ACC_N, a.partials);
}

}  // namespace gs
