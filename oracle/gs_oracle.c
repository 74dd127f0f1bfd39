/*
 * gs_oracle.c -- FP64 CPU restatement of General-Simulator's phase-field step.
 *
 * TEST INFRASTRUCTURE ONLY (see gs_oracle.h): the checker for the CUDA path
 * and the timed CPU baseline.  Nothing on the product path calls it.
 *
 * Reference anchors (paths inside the FIST-CMS/General-Simulator tree):
 *   k vector fold and 2*3.14*d*m/n           src/gtensorb.cu:9-12
 *   unit vector, n = 0 for |k| <= 5e-7       src/gtensorb.cu:14-34
 *   sigma = C:eps (host), Omega^-1 = C_iklj n_k n_l, cofactor inverse with
 *   |det| < 1e-8 -> 0, B_pq = C eps_p eps_q - n sigma_p Omega sigma_q n
 *                                            src/gtensorb.cu:75-83,121-181
 *   mart gradient (eta+ + eta- - 2 eta)/(2d)/3 src/dynamics_mart.cu:181-188
 *   mart chemical force (HEAD side)          src/dynamics_mart.cu:222-250
 *   elastic force -wE Re(IFFT(B FFT(eta^2)/N)) eta
 *                                            src/dynamics_mart.cu:270-291
 *   dislocation force -wD 25 sigma:eps eta   src/dynamics_mart.cu:305-331
 *   Euler update + defect mask               src/dynamics_mart.cu:365-387
 *   precipitate local terms                  src/dynamics_precipitate.cu:118-162
 *   precipitate elastic force 2 R eta        src/dynamics_precipitate.cu:180-195
 *   CH / AC semi-implicit spectral updates   src/dynamics_precipitate.cu:197-275
 *   stress field and |eta| > 0.9 defect      src/dynamics_stress.cu:83-92,122-194
 */
#include "gs_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

static int g_threads = 0;
void or_set_threads(int n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10                                                      */
/* ------------------------------------------------------------------ */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* 24-bit uniform in (0,1), exact in FP32 and FP64. */
static double u24(uint32_t x) { return ((double)(x >> 8) + 0.5) * (1.0 / 16777216.0); }

/* Box-Muller (Box & Muller 1958) on two 24-bit uniforms. */
void or_normals4(uint64_t seed, uint32_t cell, uint32_t step, uint32_t sim, uint32_t block, double z[4]) {
  uint32_t ctr[4] = {cell, step, sim, block};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  or_philox4x32_10(ctr, key, o);
  for (int h = 0; h < 2; ++h) {
    double u1 = u24(o[2 * h]), u2 = u24(o[2 * h + 1]);
    double r = sqrt(-2.0 * log(u1));
    z[2 * h] = r * cos(2.0 * M_PI * u2);
    z[2 * h + 1] = r * sin(2.0 * M_PI * u2);
  }
}

/* Noise of one cell: one Philox block per quad of consecutive cells,
 * counter (cell >> 2, step, sim, slot); cell & 3 selects cos / sin of the
 * first Box-Muller pair (words 0, 1) or of the second (words 2, 3). */
static double noise_at(const gs_params* p, int64_t step, uint32_t cell, int slot) {
  double z[4];
  or_normals4(p->seed, cell >> 2, (uint32_t)step, p->sim_id, (uint32_t)slot, z);
  return z[cell & 3u];
}

/* ------------------------------------------------------------------ */
/* FFT: recursive mixed-radix decimation in time, double complex       */
/* ------------------------------------------------------------------ */
#define OR_MAXP 64
typedef struct {
  int n;
  int nf;
  int fac[40];
  cplx* w; /* w[j] = exp(sign 2 pi i j / n) */
} fftplan;

static void plan_make(fftplan* pl, int n, int sign) {
  pl->n = n;
  pl->nf = 0;
  int m = n;
  while (m > 1) {
    int f = 0;
    if (m % 4 == 0)
      f = 4;
    else if (m % 2 == 0)
      f = 2;
    else
      for (int d = 3; d <= m; d += 2)
        if (m % d == 0) {
          f = d;
          break;
        }
    pl->fac[pl->nf++] = f;
    m /= f;
  }
  pl->w = (cplx*)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
  for (int j = 0; j < n; ++j) {
    double a = 2.0 * M_PI * (double)j / (double)n;
    pl->w[j] = cos(a) + (double)sign * sin(a) * I;
  }
}
static void plan_free(fftplan* pl) { free(pl->w); }

static void fft_rec(const cplx* in, long istride, cplx* out, int n, const int* fac, const fftplan* pl,
                    long wstep) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = fac[0], m = n / p;
  for (int q = 0; q < p; ++q) fft_rec(in + q * istride, istride * p, out + (long)q * m, m, fac + 1, pl, wstep * p);
  const long N = pl->n;
  cplx t[OR_MAXP];
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) t[q] = out[(long)q * m + k] * pl->w[((long)q * k * wstep) % N];
    for (int s = 0; s < p; ++s) {
      cplx acc = 0;
      for (int q = 0; q < p; ++q) acc += t[q] * pl->w[((long)q * s * wstep * m) % N];
      out[k + (long)m * s] = acc;
    }
  }
}

static void fft_axis(cplx* a, int n0, int n1, int n2, int axis, int sign) {
  int n = axis == 0 ? n0 : axis == 1 ? n1 : n2;
  if (n == 1) return;
  long stride = axis == 0 ? (long)n1 * n2 : axis == 1 ? n2 : 1;
  long nlines = (long)n0 * n1 * n2 / n;
  fftplan pl;
  plan_make(&pl, n, sign);
#pragma omp parallel
  {
    cplx* tin = (cplx*)malloc(sizeof(cplx) * n);
    cplx* tout = (cplx*)malloc(sizeof(cplx) * n);
#pragma omp for schedule(static)
    for (long L = 0; L < nlines; ++L) {
      long base;
      if (axis == 2)
        base = L * n2;
      else if (axis == 1)
        base = (L / n2) * (long)n1 * n2 + (L % n2);
      else
        base = L;
      for (int j = 0; j < n; ++j) tin[j] = a[base + j * stride];
      fft_rec(tin, 1, tout, n, pl.fac, &pl, 1);
      for (int j = 0; j < n; ++j) a[base + j * stride] = tout[j];
    }
    free(tin);
    free(tout);
  }
  plan_free(&pl);
}

void or_fft3(double* data, int n0, int n1, int n2, int sign) {
  cplx* a = (cplx*)data;
  fft_axis(a, n0, n1, n2, 2, sign);
  fft_axis(a, n0, n1, n2, 1, sign);
  fft_axis(a, n0, n1, n2, 0, sign);
}

/* ------------------------------------------------------------------ */
/* wave vectors and B(n)                                               */
/* ------------------------------------------------------------------ */
static int fold_ref(int i, int n) { return i < n / 2 ? i : i - n; } /* GTensorB_VF */
static int fold_base(int i, int n) { return 2 * i < n ? i : i - n; }

static void kvec(const gs_params* p, int mx, int my, int mz, double k[3]) {
  const int ns[3] = {p->nx, p->ny, p->nz};
  const double ds[3] = {p->dx, p->dy, p->dz};
  const int ms[3] = {mx, my, mz};
  for (int a = 0; a < 3; ++a) {
    if (p->mode == GS_MODE_REFCOMPAT)
      k[a] = 2.0 * 3.14 * ds[a] / ns[a] * ms[a];
    else
      k[a] = 2.0 * M_PI * ms[a] / (ns[a] * ds[a]);
  }
}

/* K(k) of the semi-implicit CH/AC updates: refcompat uses |k|^2 of the
 * 3.14 vector (_gSquare); baseline uses the seven-point Laplacian symbol. */
static double ksym(const gs_params* p, int mx, int my, int mz) {
  if (p->mode == GS_MODE_REFCOMPAT) {
    double k[3];
    kvec(p, mx, my, mz, k);
    return k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  }
  const int ns[3] = {p->nx, p->ny, p->nz};
  const double ds[3] = {p->dx, p->dy, p->dz};
  const int ms[3] = {mx, my, mz};
  double s = 0;
  for (int a = 0; a < 3; ++a) {
    if (ns[a] == 1) continue;
    double sn = sin(M_PI * ms[a] / ns[a]);
    s += 4.0 / (ds[a] * ds[a]) * sn * sn;
  }
  return s;
}

typedef double mat3[3][3];

static void strain_sets(const gs_params* p, int which, mat3* ea, int* na, mat3* eb, int* nb) {
  int V = p->nvariants;
  if (which == 0) {
    for (int v = 0; v < V; ++v) {
      memcpy(ea[v], p->eigenstrain[v], sizeof(mat3));
      memcpy(eb[v], p->eigenstrain[v], sizeof(mat3));
    }
    *na = *nb = V;
  } else if (which == 1) {
    /* unit base strains xx xy xz yy yz zz (src/dynamics_stress.cu:83-89) */
    const int bi[6] = {0, 0, 0, 1, 1, 2}, bj[6] = {0, 1, 2, 1, 2, 2};
    for (int b = 0; b < 6; ++b) {
      memset(ea[b], 0, sizeof(mat3));
      if (p->mode == GS_MODE_REFCOMPAT || bi[b] == bj[b])
        ea[b][bi[b]][bj[b]] = 1.0;
      else {
        ea[b][bi[b]][bj[b]] = 0.5;
        ea[b][bj[b]][bi[b]] = 0.5;
      }
    }
    *na = 6;
    for (int v = 0; v < V; ++v) memcpy(eb[v], p->eigenstrain[v], sizeof(mat3));
    *nb = V;
  } else {
    int F = V;
    for (int v = 0; v < V; ++v) {
      memcpy(ea[v], p->eigenstrain[v], sizeof(mat3));
      memcpy(eb[v], p->eigenstrain[v], sizeof(mat3));
    }
    if (p->c_elastic) {
      memset(ea[V], 0, sizeof(mat3));
      for (int i = 0; i < 3; ++i) ea[V][i][i] = p->misfit_c;
      memcpy(eb[V], ea[V], sizeof(mat3));
      F = V + 1;
    }
    *na = *nb = F;
  }
}

/* B between strain sets at wave vector k (src/gtensorb.cu:110-182).
 * kzero: the k = 0 point: refcompat keeps C:ea:eb, baseline sets 0. */
static void bmat_k(const gs_params* p, const mat3* ea, int na, const mat3* eb, int nb, const double k[3], double* B) {
  const int ref = p->mode == GS_MODE_REFCOMPAT;
  double kk = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  double mo = sqrt(kk);
  double n[3] = {0, 0, 0};
  int zero = ref ? (mo <= 0.0000005) : (kk == 0.0);
  if (zero && !ref) {
    for (int i = 0; i < na * nb; ++i) B[i] = 0;
    return;
  }
  if (!zero)
    for (int a = 0; a < 3; ++a) n[a] = k[a] / mo;
  const double(*C)[3][3][3] = p->cijkl;
  double m[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s += C[i][a][b][j] * n[a] * n[b];
      m[i][j] = s;
    }
  double det = -m[0][2] * m[1][1] * m[2][0] + m[0][1] * m[1][2] * m[2][0] + m[0][2] * m[1][0] * m[2][1] -
               m[0][0] * m[1][2] * m[2][1] - m[0][1] * m[1][0] * m[2][2] + m[0][0] * m[1][1] * m[2][2];
  double om[3][3];
  int ok = ref ? (det >= 1e-8 || det <= -1e-8) : (det != 0.0);
  if (ok) {
    om[0][0] = (-m[1][2] * m[2][1] + m[1][1] * m[2][2]) / det;
    om[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
    om[0][2] = (-m[0][2] * m[1][1] + m[0][1] * m[1][2]) / det;
    om[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det;
    om[1][1] = (-m[0][2] * m[2][0] + m[0][0] * m[2][2]) / det;
    om[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
    om[2][0] = (-m[1][1] * m[2][0] + m[1][0] * m[2][1]) / det;
    om[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
    om[2][2] = (-m[0][1] * m[1][0] + m[0][0] * m[1][1]) / det;
  } else {
    memset(om, 0, sizeof(om));
  }
  for (int a = 0; a < na; ++a) {
    double sa[3][3], sb[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double s = 0;
        for (int q = 0; q < 3; ++q)
          for (int r = 0; r < 3; ++r) s += C[i][j][q][r] * ea[a][q][r];
        sa[i][j] = s;
      }
    for (int b = 0; b < nb; ++b) {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double s = 0;
          for (int q = 0; q < 3; ++q)
            for (int r = 0; r < 3; ++r) s += C[i][j][q][r] * eb[b][q][r];
          sb[i][j] = s;
        }
      double ceps = 0, t = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int q = 0; q < 3; ++q)
            for (int r = 0; r < 3; ++r) {
              ceps += C[i][j][q][r] * ea[a][i][j] * eb[b][q][r];
              t += n[i] * sa[i][j] * om[j][q] * sb[q][r] * n[r];
            }
      B[a * nb + b] = ceps - t;
    }
  }
}

int or_bmat_at(const gs_params* p, int which, int mx, int my, int mz, double* B, int* na, int* nb) {
  mat3 ea[GS_MAX_V + 1], eb[GS_MAX_V + 1];
  strain_sets(p, which, ea, na, eb, nb);
  double k[3];
  kvec(p, mx, my, mz, k);
  bmat_k(p, ea, *na, eb, *nb, k, B);
  return 0;
}

/* ------------------------------------------------------------------ */
/* elastic potential: R_a = Re IFFT((1/N) sum_b B_ab FFT(phi_b))        */
/* ------------------------------------------------------------------ */
static void elastic_potential(const gs_params* p, int which, const double* phi, int nphi, double* R, int nout) {
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz;
  const long N = (long)n0 * n1 * n2;
  cplx* sp = (cplx*)malloc(sizeof(cplx) * N * nphi);
  cplx* ro = (cplx*)malloc(sizeof(cplx) * N * nout);
  for (long i = 0; i < N * nphi; ++i) sp[i] = phi[i];
  for (int f = 0; f < nphi; ++f) or_fft3((double*)(sp + f * N), n0, n1, n2, -1);
  mat3 ea[GS_MAX_V + 1], eb[GS_MAX_V + 1];
  int na, nb;
  strain_sets(p, which, ea, &na, eb, &nb);
  const int ref = p->mode == GS_MODE_REFCOMPAT;
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < N; ++idx) {
    int x = (int)(idx / ((long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
    int mx = ref ? fold_ref(x, n0) : fold_base(x, n0);
    int my = ref ? fold_ref(y, n1) : fold_base(y, n1);
    int mz = ref ? fold_ref(z, n2) : fold_base(z, n2);
    double k[3], B[(GS_MAX_V + 1) * (GS_MAX_V + 1)];
    kvec(p, mx, my, mz, k);
    bmat_k(p, ea, na, eb, nb, k, B);
    for (int a = 0; a < nout; ++a) {
      cplx s = 0;
      for (int b = 0; b < nphi; ++b) s += B[a * nb + b] * sp[b * N + idx];
      ro[a * N + idx] = s / (double)N;
    }
  }
  for (int f = 0; f < nout; ++f) or_fft3((double*)(ro + f * N), n0, n1, n2, +1);
  for (long i = 0; i < N * nout; ++i) R[i] = creal(ro[i]);
  free(sp);
  free(ro);
}

/* ------------------------------------------------------------------ */
/* stencils                                                            */
/* ------------------------------------------------------------------ */
static inline long wrap(long i, long n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

/* sum_a ca[a] (f(+a) + f(-a) - 2 f), periodic. */
static double lap7(const double* f, int n0, int n1, int n2, int x, int y, int z, const double ca[3]) {
  long i = ((long)x * n1 + y) * n2 + z;
  double c = f[i];
  double s = 0;
  if (n0 > 1)
    s += ca[0] * (f[((long)wrap(x + 1, n0) * n1 + y) * n2 + z] + f[((long)wrap(x - 1, n0) * n1 + y) * n2 + z] - 2 * c);
  if (n1 > 1)
    s += ca[1] * (f[((long)x * n1 + wrap(y + 1, n1)) * n2 + z] + f[((long)x * n1 + wrap(y - 1, n1)) * n2 + z] - 2 * c);
  if (n2 > 1) s += ca[2] * (f[((long)x * n1 + y) * n2 + wrap(z + 1, n2)] + f[((long)x * n1 + y) * n2 + wrap(z - 1, n2)] - 2 * c);
  return s;
}

static void lap_coef(const gs_params* p, double ca[3]) {
  const double ds[3] = {p->dx, p->dy, p->dz};
  for (int a = 0; a < 3; ++a) ca[a] = p->mode == GS_MODE_REFCOMPAT ? 1.0 / (2.0 * ds[a]) / 3.0 : 1.0 / (ds[a] * ds[a]);
}

static double contract33(const double a[3][3], const double b[3][3]) {
  double s = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s += a[i][j] * b[i][j];
  return s;
}

/* dislocation stress 6 x N (xx xy xz yy yz zz) -> K_p(x) = sigma(x):eps_p */
static double kdisl(const gs_params* p, const double* ds6, long N, long idx, int v) {
  if (!ds6) return 0;
  double s[3][3];
  s[0][0] = ds6[0 * N + idx];
  s[0][1] = s[1][0] = ds6[1 * N + idx];
  s[0][2] = s[2][0] = ds6[2 * N + idx];
  s[1][1] = ds6[3 * N + idx];
  s[1][2] = s[2][1] = ds6[4 * N + idx];
  s[2][2] = ds6[5 * N + idx];
  return contract33(s, p->eigenstrain[v]);
}

/* ------------------------------------------------------------------ */
/* martensite                                                          */
/* ------------------------------------------------------------------ */
static float ref_a1(const gs_params* p) { return 0.02f * ((float)p->temperature - (float)p->transition_temperature); }

/* local force terms of one cell, variant v; returns the RHS (per unit time,
 * without noise) and the individual terms for the info keys. */
static double mart_rhs(const gs_params* p, const double* eta, long N, long idx, int v, double lapv, double Rv,
                       double Kv, double* tg, double* tc, double* te, double* td) {
  const int V = p->nvariants;
  double e = eta[v * N + idx];
  if (p->mode == GS_MODE_REFCOMPAT) {
    double a1 = ref_a1(p), a2 = p->lpc[2], a3 = p->lpc[3];
    double s = sqrt(fabs(a1 / (a2 - a3)));
    double sum = 0;
    for (int q = 0; q < V; ++q) {
      double t = s * eta[q * N + idx];
      sum += t * t;
    }
    double fc;
    if (e >= 0)
      fc = -p->weight_chemical * (s * e) * (a1 - a2 * (s * e) * (s * e) + a3 * sum);
    else
      fc = 1000.0 * p->weight_chemical * a2 * e * e;
    *tg = p->weight_gradient * lapv;
    *tc = fc;
    *te = -p->weight_elastic * Rv * e;
    *td = -p->weight_dislocation * 25.0 * Kv * e;
    return *tg + *tc + *te + *td;
  }
  double A2 = p->landau[0], A4 = p->landau[1], A6 = p->landau[2], Ac = p->landau[3];
  double s2 = 0;
  for (int q = 0; q < V; ++q) s2 += eta[q * N + idx] * eta[q * N + idx];
  double fp = A2 * e - A4 * e * e * e + A6 * s2 * s2 * e + 2.0 * Ac * e * (s2 - e * e);
  double L = p->mobility;
  double lin = 2.0 * (contract33(p->applied_stress, p->eigenstrain[v]) + p->weight_dislocation * Kv);
  *tg = L * p->kappa * lapv;
  *tc = -L * fp;
  *te = -L * p->weight_elastic * 2.0 * e * Rv;
  *td = L * lin * e;
  return *tg + *tc + *te + *td;
}

int or_mart_potential(const gs_params* p, const double* eta, double* R) {
  const long N = (long)p->nx * p->ny * p->nz;
  const int V = p->nvariants;
  double* S = (double*)malloc(sizeof(double) * N * V);
  for (long i = 0; i < N * V; ++i) S[i] = eta[i] * eta[i];
  elastic_potential(p, 0, S, V, R, V);
  free(S);
  return 0;
}

int or_mart_run(const gs_params* p, double* eta, const double* defect, const double* dstress, int nsteps,
                int64_t step0) {
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz, V = p->nvariants;
  const long N = (long)n0 * n1 * n2;
  double* R = (double*)malloc(sizeof(double) * N * V);
  double* nw = (double*)malloc(sizeof(double) * N * V);
  double ca[3];
  lap_coef(p, ca);
  for (int st = 0; st < nsteps; ++st) {
    int64_t step = step0 + st;
    or_mart_potential(p, eta, R);
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N; ++idx) {
      int x = (int)(idx / ((long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
      for (int v = 0; v < V; ++v) {
        double tg, tc, te, td;
        double lapv = lap7(eta + v * N, n0, n1, n2, x, y, z, ca);
        double Kv = kdisl(p, dstress, N, idx, v);
        double rhs = mart_rhs(p, eta, N, idx, v, lapv, R[v * N + idx], Kv, &tg, &tc, &te, &td);
        double xi = p->noise_amp != 0.0 ? noise_at(p, step, (uint32_t)idx, v) : 0.0;
        double e = eta[v * N + idx];
        double en;
        if (p->mode == GS_MODE_REFCOMPAT)
          en = e + p->dt * (rhs + p->noise_amp * xi);
        else
          en = e + p->dt * rhs + p->noise_amp * xi;
        if (defect) en = en * (1.0 - defect[idx]);
        nw[v * N + idx] = en;
      }
    }
    memcpy(eta, nw, sizeof(double) * N * V);
  }
  free(R);
  free(nw);
  return 0;
}

int or_mart_stats(const gs_params* p, const double* eta, const double* defect, const double* dstress, gs_stats* st) {
  (void)defect;
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz, V = p->nvariants;
  const long N = (long)n0 * n1 * n2;
  const double dV = p->dx * p->dy * p->dz;
  double* R = (double*)malloc(sizeof(double) * N * V);
  or_mart_potential(p, eta, R);
  double ca[3], cg[3];
  lap_coef(p, ca);
  cg[0] = 1.0 / (p->dx * p->dx);
  cg[1] = 1.0 / (p->dy * p->dy);
  cg[2] = 1.0 / (p->dz * p->dz);
  double mass = 0, eel = 0, ech = 0, egr = 0, eap = 0, sg = 0, sc = 0, se = 0, sd = 0;
  double e2[GS_MAX_V] = {0}, vf[GS_MAX_V] = {0};
  const double A2 = p->landau[0], A4 = p->landau[1], A6 = p->landau[2], Ac = p->landau[3];
#pragma omp parallel for schedule(static) reduction(+ : mass, eel, ech, egr, eap, sg, sc, se, sd, e2[:GS_MAX_V], vf[:GS_MAX_V])
  for (long idx = 0; idx < N; ++idx) {
    int x = (int)(idx / ((long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
    double s2 = 0, s4 = 0, pair = 0;
    for (int v = 0; v < V; ++v) {
      double e = eta[v * N + idx];
      double tg, tc, te, td;
      double lapv = lap7(eta + v * N, n0, n1, n2, x, y, z, ca);
      double Kv = kdisl(p, dstress, N, idx, v);
      mart_rhs(p, eta, N, idx, v, lapv, R[v * N + idx], Kv, &tg, &tc, &te, &td);
      sg += tg;
      sc += tc;
      se += te;
      sd += td;
      mass += e;
      e2[v] += e * e;
      vf[v] += fabs(e) > 0.5 ? 1.0 : 0.0;
      eel += 0.5 * p->weight_elastic * e * e * R[v * N + idx];
      egr += -0.5 * p->kappa * e * lap7(eta + v * N, n0, n1, n2, x, y, z, cg);
      eap += -(contract33(p->applied_stress, p->eigenstrain[v]) + p->weight_dislocation * Kv) * e * e;
      pair += s2 * e * e;
      s2 += e * e;
      s4 += e * e * e * e;
    }
    ech += A2 / 2 * s2 - A4 / 4 * s4 + A6 / 6 * s2 * s2 * s2 + Ac * pair;
  }
  memset(st, 0, sizeof(*st));
  st->mass = mass;
  st->eta_mean = mass / ((double)N * V);
  for (int v = 0; v < V; ++v) {
    st->eta2[v] = e2[v] / N;
    st->vf[v] = vf[v] / N;
  }
  st->e_el = eel * dV;
  st->e_chem = ech * dV;
  st->e_grad = egr * dV;
  st->e_appl = eap * dV;
  st->e_tot = st->e_el + st->e_chem + st->e_grad + st->e_appl;
  st->gradient_mean = sg / ((double)N * V);
  st->chemical_mean = sc / ((double)N * V);
  st->elastic_mean = se / ((double)N * V);
  st->dislocation_mean = sd / ((double)N * V);
  free(R);
  return 0;
}

/* ------------------------------------------------------------------ */
/* precipitate                                                         */
/* ------------------------------------------------------------------ */
/* mu_c = A1 (c - c1) + A2/2 sum eta^2   (LocalConFreeEnergy, :118-127)
 * g_v  = (2A5 e + 4A6 e^3) t2 + 2A6 e t4 + 2A7 e t22 + A2 e (c - c2)
 *        - A3 e^3 + A4 e^5               (LocalEtaFreeEnergy, :136-162)  */
static double precip_mu(const gs_params* p, double c, const double* e, int V) {
  double s = 0;
  for (int v = 0; v < V; ++v) s += (p->coef[2] / 2.0) * e[v] * e[v];
  return s + p->coef[1] * (c - p->c1);
}
static double precip_g(const gs_params* p, double c, const double* e, int V, int v) {
  double t2 = 0, t4 = 0, t22 = 0;
  for (int i = 0; i < V; ++i)
    if (i != v) {
      t2 += e[i] * e[i];
      t4 += e[i] * e[i] * e[i] * e[i];
    }
  for (int i = 0; i < V; ++i)
    for (int j = 0; j < V; ++j)
      if (v != i && v != j && i != j) t22 += e[i] * e[i] * e[j] * e[j];
  double x = e[v];
  const double* A = p->coef;
  return (2.0 * A[5] * x + 4.0 * A[6] * x * x * x) * t2 + (2.0 * A[6] * x) * t4 + (2.0 * A[7] * x) * t22 +
         (A[2] * x * (c - p->c2)) - (A[3] * x * x * x) + (A[4] * x * x * x * x * x);
}
static double precip_f(const gs_params* p, double c, const double* e, int V) {
  const double* A = p->coef;
  double f = A[1] / 2.0 * (c - p->c1) * (c - p->c1);
  for (int i = 0; i < V; ++i) {
    double e2 = e[i] * e[i];
    f += A[2] / 2.0 * (c - p->c2) * e2 - A[3] / 4.0 * e2 * e2 + A[4] / 6.0 * e2 * e2 * e2;
    for (int j = i + 1; j < V; ++j) {
      double f2 = e[j] * e[j];
      f += A[5] * e2 * f2 + A[6] * (e2 * e2 * f2 + e2 * f2 * f2);
      for (int k = j + 1; k < V; ++k) f += 2.0 * A[7] * e2 * f2 * e[k] * e[k];
    }
  }
  return f;
}

static double precip_escale(const gs_params* p) { return p->xi * p->weight_elastic; }

static void precip_potential(const gs_params* p, const double* c, const double* eta, double* R, int* F) {
  const long N = (long)p->nx * p->ny * p->nz;
  const int V = p->nvariants;
  *F = V + (p->c_elastic ? 1 : 0);
  double* phi = (double*)malloc(sizeof(double) * N * (*F));
  for (long i = 0; i < N * V; ++i) phi[i] = eta[i] * eta[i];
  if (p->c_elastic) memcpy(phi + (long)V * N, c, sizeof(double) * N);
  elastic_potential(p, 2, phi, *F, R, *F);
  free(phi);
}

int or_precip_run(const gs_params* p, double* c, double* eta, int nsteps, int64_t step0) {
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz, V = p->nvariants;
  const long N = (long)n0 * n1 * n2;
  const int ref = p->mode == GS_MODE_REFCOMPAT;
  double* R = (double*)malloc(sizeof(double) * N * (V + 1));
  cplx* cs = (cplx*)malloc(sizeof(cplx) * N);
  cplx* mus = (cplx*)malloc(sizeof(cplx) * N);
  cplx* es = (cplx*)malloc(sizeof(cplx) * N * V);
  cplx* gs = (cplx*)malloc(sizeof(cplx) * N * V);
  const double Es = precip_escale(p);
  const double an = p->noise_amp * (ref ? 1e-4 : 1.0);
  for (int st = 0; st < nsteps; ++st) {
    int64_t step = step0 + st;
    int F;
    precip_potential(p, c, eta, R, &F);
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N; ++idx) {
      double e[GS_MAX_V];
      for (int v = 0; v < V; ++v) e[v] = eta[v * N + idx];
      double mu = precip_mu(p, c[idx], e, V);
      if (p->c_elastic && !ref) mu += Es * R[(long)V * N + idx];
      if (an != 0.0) mu += an * noise_at(p, step, (uint32_t)idx, V);
      mus[idx] = mu;
      cs[idx] = c[idx];
      for (int v = 0; v < V; ++v) {
        double g = precip_g(p, c[idx], e, V, v) + Es * 2.0 * e[v] * R[v * N + idx];
        if (an != 0.0) g += an * noise_at(p, step, (uint32_t)idx, v);
        gs[v * N + idx] = g;
        es[v * N + idx] = e[v];
      }
    }
    or_fft3((double*)cs, n0, n1, n2, -1);
    or_fft3((double*)mus, n0, n1, n2, -1);
    for (int v = 0; v < V; ++v) {
      or_fft3((double*)(es + v * N), n0, n1, n2, -1);
      or_fft3((double*)(gs + v * N), n0, n1, n2, -1);
    }
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N; ++idx) {
      int x = (int)(idx / ((long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
      int mx = ref ? fold_ref(x, n0) : fold_base(x, n0);
      int my = ref ? fold_ref(y, n1) : fold_base(y, n1);
      int mz = ref ? fold_ref(z, n2) : fold_base(z, n2);
      double K = ksym(p, mx, my, mz);
      const double dt = p->dt, M = p->mobility_c, L = p->mobility_eta;
      cs[idx] = (cs[idx] - M * K * dt * mus[idx]) / (1.0 + dt * M * p->kappa_c * K * K);
      for (int v = 0; v < V; ++v)
        es[v * N + idx] = (es[v * N + idx] - dt * L * gs[v * N + idx]) / (1.0 + dt * L * p->kappa_eta * K);
    }
    or_fft3((double*)cs, n0, n1, n2, +1);
    for (long i = 0; i < N; ++i) c[i] = creal(cs[i]) / (double)N;
    for (int v = 0; v < V; ++v) {
      or_fft3((double*)(es + v * N), n0, n1, n2, +1);
      for (long i = 0; i < N; ++i) eta[v * N + i] = creal(es[v * N + i]) / (double)N;
    }
  }
  free(R);
  free(cs);
  free(mus);
  free(es);
  free(gs);
  return 0;
}

int or_precip_stats(const gs_params* p, const double* c, const double* eta, gs_stats* st) {
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz, V = p->nvariants;
  const long N = (long)n0 * n1 * n2;
  const double dV = p->dx * p->dy * p->dz;
  double* R = (double*)malloc(sizeof(double) * N * (V + 1));
  int F;
  precip_potential(p, c, eta, R, &F);
  const double Es = precip_escale(p);
  double cg[3] = {1.0 / (p->dx * p->dx), 1.0 / (p->dy * p->dy), 1.0 / (p->dz * p->dz)};
  double mass = 0, eel = 0, ech = 0, egr = 0, es = 0;
  double e2[GS_MAX_V] = {0}, vf[GS_MAX_V] = {0};
#pragma omp parallel for schedule(static) reduction(+ : mass, eel, ech, egr, es, e2[:GS_MAX_V], vf[:GS_MAX_V])
  for (long idx = 0; idx < N; ++idx) {
    int x = (int)(idx / ((long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
    double e[GS_MAX_V];
    for (int v = 0; v < V; ++v) e[v] = eta[v * N + idx];
    mass += c[idx];
    ech += precip_f(p, c[idx], e, V);
    egr += -0.5 * p->kappa_c * c[idx] * lap7(c, n0, n1, n2, x, y, z, cg);
    for (int v = 0; v < V; ++v) {
      es += e[v];
      e2[v] += e[v] * e[v];
      vf[v] += fabs(e[v]) > 0.5 ? 1.0 : 0.0;
      eel += 0.5 * Es * e[v] * e[v] * R[v * N + idx];
      egr += -0.5 * p->kappa_eta * e[v] * lap7(eta + v * N, n0, n1, n2, x, y, z, cg);
    }
    if (p->c_elastic) eel += 0.5 * Es * c[idx] * R[(long)V * N + idx];
  }
  memset(st, 0, sizeof(*st));
  st->mass = mass;
  st->c_mean = mass / N;
  st->eta_mean = es / ((double)N * V);
  for (int v = 0; v < V; ++v) {
    st->eta2[v] = e2[v] / N;
    st->vf[v] = vf[v] / N;
  }
  st->e_el = eel * dV;
  st->e_chem = ech * dV;
  st->e_grad = egr * dV;
  st->e_tot = st->e_el + st->e_chem + st->e_grad;
  free(R);
  return 0;
}

/* ------------------------------------------------------------------ */
/* stress                                                              */
/* ------------------------------------------------------------------ */
int or_stress(const gs_params* p, const double* eta, double* stress, double* defect) {
  const long N = (long)p->nx * p->ny * p->nz;
  const int V = p->nvariants;
  double* S = (double*)malloc(sizeof(double) * N * V);
  for (long i = 0; i < N * V; ++i) S[i] = eta[i] * eta[i];
  elastic_potential(p, 1, S, V, stress, 6);
  for (long i = 0; i < 6 * N; ++i) stress[i] = -p->xi * stress[i];
  if (defect)
    for (long i = 0; i < N; ++i) {
      double d = 0;
      for (int v = 0; v < V; ++v)
        if (fabs(eta[v * N + i]) > 0.9) d = 1.0;
      defect[i] = d;
    }
  free(S);
  return 0;
}

/* ------------------------------------------------------------------ */
/* adjoint of the baseline martensite step                             */
/* ------------------------------------------------------------------ */
/* Phi(eta) = eta + dt RHS(eta) (+ noise), RHS_p = L kappa lap eta_p
 *   - L f'_p(eta) + el eta_p R_p + lin_p eta_p, el = -2 L w_el,
 *   lin_p = 2 L sigma_a:eps_p, R = B conv (eta^2).
 * (dPhi/deta)^T lam = lam + dt [L kappa lap lam - L H lam
 *   + el (R lam + 2 eta Q) + lin lam],  Q = B conv (eta lam),
 * H the Landau Hessian.  Parameter derivatives of Phi_p: kappa: dt L lap
 * eta_p; A2: -dt L eta_p; A4: dt L eta_p^3; A6: -dt L S^2 eta_p; Ac: -dt L
 * 2 eta_p (S - eta_p^2); eigenstrain scale s (eps -> s eps at s = 1):
 * dt (2 el eta_p R_p + lin_p eta_p).
 * Loss J = sum (eta_T - target)^2 + lam_el (E_el(T) - E_target)^2, or,
 * with seed != NULL, J = <seed, eta_T> + seed_e E_el(T). */
int or_mart_adjoint(const gs_params* p, const double* eta0, int nsteps, const double* target, double lam_el,
                    double e_target, const double* seed, double seed_e, double* grads, double* grad_eta0,
                    double* loss_out) {
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz, V = p->nvariants;
  const long long N = (long long)n0 * n1 * n2;
  const double dV = p->dx * p->dy * p->dz;
  double* st = (double*)malloc(sizeof(double) * N * V * (nsteps + 1));
  memcpy(st, eta0, sizeof(double) * N * V);
  for (int n = 0; n < nsteps; ++n) {
    memcpy(st + (long long)(n + 1) * N * V, st + (long long)n * N * V, sizeof(double) * N * V);
    or_mart_run(p, st + (long long)(n + 1) * N * V, NULL, NULL, 1, n);
  }
  const double* eT = st + (long long)nsteps * N * V;
  double* R = (double*)malloc(sizeof(double) * N * V);
  double* Q = (double*)malloc(sizeof(double) * N * V);
  double* u = (double*)malloc(sizeof(double) * N * V);
  double* lam = (double*)malloc(sizeof(double) * N * V);
  double* lnew = (double*)malloc(sizeof(double) * N * V);
  or_mart_potential(p, eT, R);
  double eel = 0, lf = 0;
  for (long long i = 0; i < N * V; ++i) eel += 0.5 * p->weight_elastic * eT[i] * eT[i] * R[i];
  eel *= dV;
  double ce;
  if (seed) {
    for (long long i = 0; i < N * V; ++i) lam[i] = seed[i];
    ce = seed_e;
  } else {
    for (long long i = 0; i < N * V; ++i) {
      const double d = eT[i] - target[i];
      lf += d * d;
      lam[i] = 2.0 * d;
    }
    ce = 2.0 * lam_el * (eel - e_target);
  }
  /* dE_el/deta_p = w_el dV 2 eta_p R_p */
  for (long long i = 0; i < N * V; ++i) lam[i] += ce * p->weight_elastic * dV * 2.0 * eT[i] * R[i];
  for (int g = 0; g < 6; ++g) grads[g] = 0;
  grads[5] += ce * 2.0 * eel; /* dE_el/ds = 2 E_el */
  if (loss_out) {
    loss_out[0] = seed ? 0.0 : lf + lam_el * (eel - e_target) * (eel - e_target);
    loss_out[1] = lf;
    loss_out[2] = eel;
  }
  const double L = p->mobility, dt = p->dt, kap = p->kappa;
  const double A2 = p->landau[0], A4 = p->landau[1], A6 = p->landau[2], Ac = p->landau[3];
  const double el = -2.0 * L * p->weight_elastic;
  double lin[GS_MAX_V];
  for (int v = 0; v < V; ++v) lin[v] = 2.0 * L * contract33(p->applied_stress, p->eigenstrain[v]);
  double cg[3] = {1.0 / (p->dx * p->dx), 1.0 / (p->dy * p->dy), 1.0 / (p->dz * p->dz)};
  for (int n = nsteps - 1; n >= 0; --n) {
    const double* e = st + (long long)n * N * V;
    or_mart_potential(p, e, R);
    for (long long i = 0; i < N * V; ++i) u[i] = e[i] * lam[i];
    elastic_potential(p, 0, u, V, Q, V);
    double g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0;
#pragma omp parallel for schedule(static) reduction(+ : g0, g1, g2, g3, g4, g5)
    for (long long idx = 0; idx < N; ++idx) {
      int x = (int)(idx / ((long long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
      double S = 0, el_dot = 0;
      for (int q = 0; q < V; ++q) {
        S += e[q * N + idx] * e[q * N + idx];
        el_dot += e[q * N + idx] * lam[q * N + idx];
      }
      for (int r = 0; r < V; ++r) {
        const double er = e[r * N + idx], lr = lam[r * N + idx];
        const double lapl = lap7(lam + (long long)r * N, n0, n1, n2, x, y, z, cg);
        double off = 0;
        for (int q = 0; q < V; ++q)
          if (q != r) off += e[q * N + idx] * lam[q * N + idx];
        const double Hl = (A2 - 3 * A4 * er * er + A6 * S * S + 2 * Ac * (S - er * er)) * lr +
                          4 * er * (A6 * S * el_dot + Ac * off);
        const double Rr = R[r * N + idx], Qr = Q[r * N + idx];
        lnew[r * N + idx] = lr + dt * (L * kap * lapl - L * Hl + el * (Rr * lr + 2 * er * Qr) + lin[r] * lr);
        const double lape = lap7(e + (long long)r * N, n0, n1, n2, x, y, z, cg);
        g0 += dt * L * lape * lr;
        g1 += -dt * L * er * lr;
        g2 += dt * L * er * er * er * lr;
        g3 += -dt * L * S * S * er * lr;
        g4 += -dt * L * 2 * er * (S - er * er) * lr;
        g5 += dt * (2 * el * er * Rr + lin[r] * er) * lr;
      }
    }
    grads[0] += g0;
    grads[1] += g1;
    grads[2] += g2;
    grads[3] += g3;
    grads[4] += g4;
    grads[5] += g5;
    memcpy(lam, lnew, sizeof(double) * N * V);
  }
  if (grad_eta0) memcpy(grad_eta0, lam, sizeof(double) * N * V);
  free(st);
  free(R);
  free(Q);
  free(u);
  free(lam);
  free(lnew);
  return 0;
}

/* ------------------------------------------------------------------ */
/* nuclei of the precipitate chain (src/dynamics_cores.cu:55-186)      */
/* ------------------------------------------------------------------ */
/* The reference's test, point by point: pow(0.0f + i - ox, 2) + ... <=
 * pow(0.0f + Radius, 2) in double, for the offset and its shifts by +-n
 * along one axis at a time (the seven || terms of RandomCores). */
static int core_hit(int i, int j, int k, int ox, int oy, int oz, int nx, int ny, int nz, double r2) {
  const double dx = i - ox, dy = j - oy, dz = k - oz;
#define SQ(a) ((a) * (a))
  return SQ(dx) + SQ(dy) + SQ(dz) <= r2 || SQ(dx + nx) + SQ(dy) + SQ(dz) <= r2 ||
         SQ(dx - nx) + SQ(dy) + SQ(dz) <= r2 || SQ(dx) + SQ(dy + ny) + SQ(dz) <= r2 ||
         SQ(dx) + SQ(dy - ny) + SQ(dz) <= r2 || SQ(dx) + SQ(dy) + SQ(dz + nz) <= r2 ||
         SQ(dx) + SQ(dy) + SQ(dz - nz) <= r2;
#undef SQ
}

int or_cores_paint(int nx, int ny, int nz, int V, int ncores, const int* centers, const int* variant, double radius,
                   double c_matrix, double c_core, float* eta, float* conc) {
  const long long N = (long long)nx * ny * nz;
  const double r = (double)(float)radius;
  const double r2 = r * r;
  for (long long c = 0; c < N; ++c) conc[c] = (float)c_matrix;
  for (long long c = 0; c < N * V; ++c) eta[c] = 0.0f;
  for (int q = 0; q < ncores; ++q)
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
          if (core_hit(i, j, k, centers[3 * q], centers[3 * q + 1], centers[3 * q + 2], nx, ny, nz, r2)) {
            const long long c = ((long long)i * ny + j) * nz + k;
            conc[c] = (float)c_core;
            eta[(long long)variant[q] * N + c] = 1.0f;
          }
  return 0;
}

int or_cores_marked(int nx, int ny, int nz, int ncores, const int* centers, double radius, int i, int j, int k) {
  const double r = (double)(float)radius;
  for (int q = 0; q < ncores; ++q)
    if (core_hit(i, j, k, centers[3 * q], centers[3 * q + 1], centers[3 * q + 2], nx, ny, nz, r * r)) return 1;
  return 0;
}

/* ------------------------------------------------------------------ */
/* adjoint of the precipitate run (baseline mode)                      */
/* ------------------------------------------------------------------ */
/* u <- Re IFFT(S(k) FFT(u)) / N for a real field, S real and even: the
 * semi-implicit factors are such symbols, so each is its own transpose. */
enum { SYM_DC, SYM_KDC, SYM_K2DC, SYM_DE, SYM_KDE };
static void apply_symbol(const gs_params* p, int sym, const double* u, double* out) {
  const int n0 = p->nx, n1 = p->ny, n2 = p->nz;
  const long N = (long)n0 * n1 * n2;
  const int ref = p->mode == GS_MODE_REFCOMPAT;
  const double dt = p->dt, M = p->mobility_c, L = p->mobility_eta;
  cplx* w = (cplx*)malloc(sizeof(cplx) * N);
  for (long i = 0; i < N; ++i) w[i] = u[i];
  or_fft3((double*)w, n0, n1, n2, -1);
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < N; ++idx) {
    int x = (int)(idx / ((long)n1 * n2)), y = (int)((idx / n2) % n1), z = (int)(idx % n2);
    int mx = ref ? fold_ref(x, n0) : fold_base(x, n0);
    int my = ref ? fold_ref(y, n1) : fold_base(y, n1);
    int mz = ref ? fold_ref(z, n2) : fold_base(z, n2);
    const double K = ksym(p, mx, my, mz);
    const double Dc = 1.0 / (1.0 + dt * M * p->kappa_c * K * K), De = 1.0 / (1.0 + dt * L * p->kappa_eta * K);
    double s = sym == SYM_DC ? Dc : sym == SYM_KDC ? K * Dc : sym == SYM_K2DC ? K * K * Dc : sym == SYM_DE ? De : K * De;
    w[idx] *= s;
  }
  or_fft3((double*)w, n0, n1, n2, +1);
  for (long i = 0; i < N; ++i) out[i] = creal(w[i]) / (double)N;
  free(w);
}

/* J = <seed_c, c_T> + <seed_eta, eta_T> of the run from (c0, eta0); the
 * gradients with respect to c0, eta0 and theta = (kappa_c, kappa_eta,
 * coef[1..7]).  One step is c' = Dc (c - dt M K mu), eta_p' = De (eta_p -
 * dt L g_p) in k space, mu = A1 (c - c1) + A2/2 sum eta^2 + Es R_c,
 * g_p = dh/deta_p + 2 Es eta_p R_p, R = B * (eta^2, c); the additive noise
 * drops out.  The transposes: Dc, K, De are real even symbols (their own
 * transposes) and B is symmetric, so R's transpose is the same convolution. */
int or_precip_adjoint(const gs_params* p, const double* c0, const double* eta0, int nsteps, const double* seed_c,
                      const double* seed_eta, double* grad_c0, double* grad_eta0, double* grads) {
  const int V = p->nvariants;
  const long N = (long)p->nx * p->ny * p->nz;
  const long S = N * (V + 1);
  double* st = (double*)malloc(sizeof(double) * S * (nsteps + 1));
  memcpy(st, c0, sizeof(double) * N);
  memcpy(st + N, eta0, sizeof(double) * N * V);
  for (int n = 0; n < nsteps; ++n) {
    memcpy(st + (n + 1) * S, st + n * S, sizeof(double) * S);
    or_precip_run(p, st + (n + 1) * S, st + (n + 1) * S + N, 1, n);
  }
  const double dt = p->dt, M = p->mobility_c, L = p->mobility_eta, Es = precip_escale(p);
  const double* A = p->coef;
  const int ce = p->c_elastic && p->mode != GS_MODE_REFCOMPAT;
  double* lc = (double*)malloc(sizeof(double) * N);
  double* le = (double*)malloc(sizeof(double) * N * V);
  double* ac = (double*)malloc(sizeof(double) * N);
  double* dmu = (double*)malloc(sizeof(double) * N);
  double* ae = (double*)malloc(sizeof(double) * N * V);
  double* dg = (double*)malloc(sizeof(double) * N * V);
  double* tmp = (double*)malloc(sizeof(double) * N);
  double* R = (double*)malloc(sizeof(double) * N * (V + 1));
  double* dR = (double*)malloc(sizeof(double) * N * (V + 1));
  double* dP = (double*)malloc(sizeof(double) * N * (V + 1));
  memcpy(lc, seed_c, sizeof(double) * N);
  memcpy(le, seed_eta, sizeof(double) * N * V);
  for (int k = 0; k < 9; ++k) grads[k] = 0;
  for (int n = nsteps - 1; n >= 0; --n) {
    const double* c = st + n * S;
    const double* eta = c + N;
    const double* c1 = st + (n + 1) * S;
    const double* eta1 = c1 + N;
    /* kappa gradients: dc'/dkappa_c = -dt M K^2 Dc c', deta'/dkappa_eta = -dt L K De eta' */
    apply_symbol(p, SYM_K2DC, c1, tmp);
    for (long i = 0; i < N; ++i) grads[0] += -dt * M * lc[i] * tmp[i];
    for (int v = 0; v < V; ++v) {
      apply_symbol(p, SYM_KDE, eta1 + v * N, tmp);
      for (long i = 0; i < N; ++i) grads[1] += -dt * L * le[v * N + i] * tmp[i];
    }
    apply_symbol(p, SYM_DC, lc, ac);
    apply_symbol(p, SYM_KDC, lc, dmu);
    for (long i = 0; i < N; ++i) dmu[i] *= -dt * M;
    for (int v = 0; v < V; ++v) {
      apply_symbol(p, SYM_DE, le + v * N, ae + v * N);
      for (long i = 0; i < N; ++i) dg[v * N + i] = -dt * L * ae[v * N + i];
    }
    int F;
    precip_potential(p, c, eta, R, &F);
    for (int v = 0; v < V; ++v)
      for (long i = 0; i < N; ++i) dR[v * N + i] = 2.0 * Es * eta[v * N + i] * dg[v * N + i];
    if (F > V)
      for (long i = 0; i < N; ++i) dR[(long)V * N + i] = ce ? Es * dmu[i] : 0.0;
    elastic_potential(p, 2, dR, F, dP, F);
    double g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0, g6 = 0, g7 = 0;
    for (long i = 0; i < N; ++i) {
      double e[GS_MAX_V], s2 = 0;
      for (int v = 0; v < V; ++v) {
        e[v] = eta[v * N + i];
        s2 += e[v] * e[v];
      }
      double nlc = ac[i] + A[1] * dmu[i] + (F > V ? dP[(long)V * N + i] : 0.0);
      g1 += dmu[i] * (c[i] - p->c1);
      g2 += dmu[i] * s2 / 2.0;
      for (int pp = 0; pp < V; ++pp) {
        const double x = e[pp], d = dg[pp * N + i];
        double t2 = 0, t4 = 0;
        for (int j = 0; j < V; ++j)
          if (j != pp) {
            t2 += e[j] * e[j];
            t4 += e[j] * e[j] * e[j] * e[j];
          }
        const double t22 = t2 * t2 - t4;
        nlc += A[2] * x * d;
        g2 += d * x * (c[i] - p->c2);
        g3 += -d * x * x * x;
        g4 += d * x * x * x * x * x;
        g5 += d * 2.0 * x * t2;
        g6 += d * (4.0 * x * x * x * t2 + 2.0 * x * t4);
        g7 += d * 2.0 * x * t22;
      }
      lc[i] = nlc;
      for (int q = 0; q < V; ++q) {
        const double x = e[q];
        double t2 = 0, t4 = 0;
        for (int j = 0; j < V; ++j)
          if (j != q) {
            t2 += e[j] * e[j];
            t4 += e[j] * e[j] * e[j] * e[j];
          }
        const double t22 = t2 * t2 - t4;
        double v = ae[q * N + i] + A[2] * x * dmu[i];
        v += ((2.0 * A[5] + 12.0 * A[6] * x * x) * t2 + 2.0 * A[6] * t4 + 2.0 * A[7] * t22 + A[2] * (c[i] - p->c2) -
              3.0 * A[3] * x * x + 5.0 * A[4] * x * x * x * x) *
             dg[q * N + i];
        for (int pp = 0; pp < V; ++pp)
          if (pp != q) {
            const double y = e[pp];
            double u2 = 0;
            for (int j = 0; j < V; ++j)
              if (j != pp) u2 += e[j] * e[j];
            v += ((2.0 * A[5] * y + 4.0 * A[6] * y * y * y) * 2.0 * x + 2.0 * A[6] * y * 4.0 * x * x * x +
                  2.0 * A[7] * y * 4.0 * x * (u2 - x * x)) *
                 dg[pp * N + i];
          }
        v += 2.0 * Es * R[q * N + i] * dg[q * N + i] + 2.0 * x * dP[q * N + i];
        le[q * N + i] = v;
      }
    }
    grads[2] += g1;
    grads[3] += g2;
    grads[4] += g3;
    grads[5] += g4;
    grads[6] += g5;
    grads[7] += g6;
    grads[8] += g7;
  }
  if (grad_c0) memcpy(grad_c0, lc, sizeof(double) * N);
  if (grad_eta0) memcpy(grad_eta0, le, sizeof(double) * N * V);
  free(st);
  free(lc);
  free(le);
  free(ac);
  free(dmu);
  free(ae);
  free(dg);
  free(tmp);
  free(R);
  free(dR);
  free(dP);
  return 0;
}
