// gs_padj.cuh -- pointwise sweeps of the adjoint of the precipitate step.
//
// Forward (src/dynamics_precipitate.cu:118-289, baseline mode): mu = A1 (c -
// c1) + A2/2 sum eta^2 + Es R_c, g_p = dh/deta_p + 2 Es eta_p R_p, then the
// semi-implicit update in k space.  Given lambda' = dJ/d(c', eta') and the
// spectral pass's real outputs (D lambda', K D lambda', K^a D state' per
// field), the first sweep forms the adjoints of the local terms, dmu =
// -dt M K Dc lambda_c', dg_p = -dt L De lambda_p', the elastic sources dR
// (transposed through the same B convolution by the caller) and the kappa
// sums; the second forms lambda = dJ/d(c, eta) and the coefficient sums.
#pragma once
#include "gs_mart.cuh"

namespace gs {

enum { PADJ_KC = 0, PADJ_KE, PADJ_A1, PADJ_A2, PADJ_A3, PADJ_A4, PADJ_A5, PADJ_A6, PADJ_A7, PADJ_N };

template <typename T> struct PadjArgs {
  long long N;
  int V, F, ce;  // fields of R, c couples elastically
  T A[8], c1, c2, Es, dtM, dtL;
  const T* lc;   // lambda_c' [N]
  const T* le;   // lambda_eta' [V][N]
  const T* zr;   // [3 (V + 1)][N]: per field (c, eta_0, ...): D lambda', K D lambda', K^a D state'
  const T* c;    // state n
  const T* eta;  // [V][N]
  const T* R;    // R of state n [F][N]
  const T* dP;   // B * dR [F][N] (second sweep)
  T* dR;         // [F][N] (first sweep)
  T* lc_out;
  T* le_out;
  double* partials;
};

template <typename T> __global__ void k_padj_a(PadjArgs<T> a) {
  Neu acc[2];
  const long long N = a.N;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    acc[0].add(-(double)a.dtM * (double)a.lc[i] * (double)a.zr[2 * N + i]);
    double ke = 0;
    for (int p = 0; p < a.V; ++p) {
      const long long s = 3LL * (p + 1) * N;
      ke += (double)a.le[p * N + i] * (double)a.zr[s + 2 * N + i];
      const T dg = -a.dtL * a.zr[s + i];
      a.dR[p * N + i] = (T)2 * a.Es * a.eta[p * N + i] * dg;
    }
    acc[1].add(-(double)a.dtL * ke);
    if (a.F > a.V) a.dR[(long long)a.V * N + i] = a.ce ? a.Es * (-a.dtM * a.zr[N + i]) : (T)0;
  }
  block_reduce_store(acc, 2, a.partials);
}

template <typename T, int VM> __global__ void k_padj_b(PadjArgs<T> a) {
  Neu acc[7];
  const long long N = a.N;
  const int V = a.V;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    T e[VM], dg[VM];
    T s2 = 0;
#pragma unroll
    for (int p = 0; p < VM; ++p)
      if (p < V) {
        e[p] = a.eta[p * N + i];
        dg[p] = -a.dtL * a.zr[3LL * (p + 1) * N + i];
        s2 += e[p] * e[p];
      }
    const T c = a.c[i];
    const T dmu = -a.dtM * a.zr[N + i];
    T nlc = a.zr[i] + a.A[1] * dmu + (a.F > V ? a.dP[(long long)V * N + i] : (T)0);
    acc[0].add((double)dmu * ((double)c - (double)a.c1));
    double g2 = (double)dmu * (double)s2 / 2.0, g3 = 0, g4 = 0, g5 = 0, g6 = 0, g7 = 0;
#pragma unroll
    for (int p = 0; p < VM; ++p)
      if (p < V) {
        const T x = e[p];
        T t2 = 0, t4 = 0;
#pragma unroll
        for (int j = 0; j < VM; ++j)
          if (j < V && j != p) {
            t2 += e[j] * e[j];
            t4 += e[j] * e[j] * e[j] * e[j];
          }
        const T t22 = t2 * t2 - t4;
        const double d = (double)dg[p], xd = (double)x;
        nlc += a.A[2] * x * dg[p];
        g2 += d * xd * ((double)c - (double)a.c2);
        g3 += -d * xd * xd * xd;
        g4 += d * xd * xd * xd * xd * xd;
        g5 += d * 2.0 * xd * (double)t2;
        g6 += d * (4.0 * xd * xd * xd * (double)t2 + 2.0 * xd * (double)t4);
        g7 += d * 2.0 * xd * (double)t22;
        // dJ/deta_p
        T v = a.zr[3LL * (p + 1) * N + i] + a.A[2] * x * dmu;
        v += ((2 * a.A[5] + 12 * a.A[6] * x * x) * t2 + 2 * a.A[6] * t4 + 2 * a.A[7] * t22 + a.A[2] * (c - a.c2) -
              3 * a.A[3] * x * x + 5 * a.A[4] * x * x * x * x) *
             dg[p];
#pragma unroll
        for (int q = 0; q < VM; ++q)
          if (q < V && q != p) {  // dh_q/deta_p
            const T y = e[q];
            T u2 = 0;
#pragma unroll
            for (int j = 0; j < VM; ++j)
              if (j < V && j != q) u2 += e[j] * e[j];
            v += ((2 * a.A[5] * y + 4 * a.A[6] * y * y * y) * 2 * x + 2 * a.A[6] * y * 4 * x * x * x +
                  2 * a.A[7] * y * 4 * x * (u2 - x * x)) *
                 dg[q];
          }
        v += (T)2 * a.Es * a.R[p * N + i] * dg[p] + (T)2 * x * a.dP[p * N + i];
        a.le_out[p * N + i] = v;
      }
    a.lc_out[i] = nlc;
    acc[1].add(g2);
    acc[2].add(g3);
    acc[3].add(g4);
    acc[4].add(g5);
    acc[5].add(g6);
    acc[6].add(g7);
  }
  block_reduce_store(acc, 7, a.partials);
}

template <typename T> cudaError_t launch_padj(PadjArgs<T>& a, bool second, cudaStream_t s, int* nblocks);

}  // namespace gs
