// gs_precip.cuh -- real-space sweeps of the precipitate and stress models.
//
// Precipitate (src/dynamics_precipitate.cu:118-195): from c, eta_p and the
// elastic potentials R_a build mu_c (LocalConFreeEnergy, :118-127) and
// g_p = dF/deta_p + Xi 2 eta_p R_p (LocalEtaFreeEnergy :136-162 and the
// elastic term :193,257), with the Philox noise terms; they are the inputs
// of the semi-implicit update in k space.  Stress (src/dynamics_stress.cu:
// 184-191): the defect mask |eta_v| > 0.9, on the device.
#pragma once
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
};

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
      T mu = a.A[1] * (c - a.c1) + a.A[2] / (T)2 * s1;
      if (a.c_elastic) mu += a.Es * a.R[(long long)a.V * a.N + i];
      mu += a.an * zc[j];
      a.mu[i] = mu;
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
        const T t22 = t2 * t2 - t4;  // sum over ordered pairs i != j, both != p
        const T x = a.eta[p * a.N + i];
        const T x2 = x * x;
        T gv = (2 * a.A[5] * x + 4 * a.A[6] * x2 * x) * t2 + (2 * a.A[6] * x) * t4 + (2 * a.A[7] * x) * t22 +
               a.A[2] * x * (c - a.c2) - a.A[3] * x2 * x + a.A[4] * x2 * x2 * x;
        gv += a.Es * (T)2 * x * a.R[p * a.N + i];
        gv += a.an * zp[j];
        a.g[p * a.N + i] = gv;
      }
    }
  }
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
