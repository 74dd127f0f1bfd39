// gs_capi.cu -- C ABI of the B200 phase-field step (include/gs_capi.h).
//
// Owns the device state of one simulation and sequences the HBM sweeps of a
// step.  The reference's equivalent is Dynamics_mart::Initialize / Calculate
// / Get (src/dynamics_mart.cu:14-173,348-417,443-456) over Data<Real>
// buffers, cuFFT plans and cuRAND generators.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <string>
#include <algorithm>
#include <utility>
#include <mutex>
#include <vector>

#include "../../include/gs_capi.h"
#include "gs_adjoint.cuh"
#include "gs_padj.cuh"
#include "gs_launch.h"
#include "gs_mart.cuh"
#include "gs_precip.cuh"
#include "gs_sim.h"

using namespace gs;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";

int gs_set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int gs_cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return GS_OK;
  if (e == cudaErrorInvalidValue && gs::bounds_message()[0]) {  // a launch refused by the range check
    const int r = gs_set_error(GS_EINVAL, "%s: %s", what, gs::bounds_message());
    gs::clear_bounds_message();
    return r;
  }
  if (e == cudaErrorMemoryAllocation) return gs_set_error(GS_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    return gs_set_error(GS_ENODEV, "%s: %s", what, cudaGetErrorString(e));
  return gs_set_error(GS_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define GS_TRY(expr)             \
  do {                           \
    int rc__ = (expr);           \
    if (rc__ != GS_OK) return rc__; \
  } while (0)
#define GS_CU(expr, what) GS_TRY(gs_cuda_check((expr), (what)))

extern "C" int gs_version(void) { return GS_CAPI_VERSION; }
extern "C" size_t gs_sizeof_params(void) { return sizeof(gs_params); }
extern "C" size_t gs_sizeof_stats(void) { return sizeof(gs_stats); }

extern "C" int gs_set_device(int device) {
  GS_CU(cudaSetDevice(device), "cudaSetDevice");
  return GS_OK;
}

extern "C" int gs_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return GS_EINVAL;
  snprintf(buf, len, "%s", g_err);
  return GS_OK;
}

// ---------------------------------------------------------------------------
// defaults
// ---------------------------------------------------------------------------
static void set_cubic(gs_params* p, double c11, double c12, double c44) {
  memset(p->cijkl, 0, sizeof(p->cijkl));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) p->cijkl[i][i][j][j] = c12;
  for (int i = 0; i < 3; ++i) p->cijkl[i][i][i][i] = c11;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (i != j) {
        p->cijkl[i][j][i][j] = c44;
        p->cijkl[i][j][j][i] = c44;
      }
}

// default modulus of Dynamics_stress (src/dynamics_stress.cu:56-78)
static void set_stress_default_modulus(gs_params* p) {
  memset(p->cijkl, 0, sizeof(p->cijkl));
  double(*c)[3][3][3] = p->cijkl;
  c[0][0][0][0] = 5.39; c[1][1][1][1] = 5.39; c[2][2][2][2] = 5.22;
  c[0][0][1][1] = 3.39; c[1][1][2][2] = 3.56; c[2][2][0][0] = 3.56;
  c[0][1][0][1] = 0.6;  c[1][2][1][2] = 0.77; c[2][0][2][0] = 0.77;
  c[1][1][0][0] = 3.39; c[2][2][1][1] = 3.56; c[0][0][2][2] = 3.56;
  c[1][0][1][0] = 0.60; c[0][1][1][0] = 0.60; c[1][0][0][1] = 0.60;
  c[2][1][2][1] = 0.77; c[2][1][1][2] = 0.77; c[1][2][2][1] = 0.77;
  c[0][2][0][2] = 0.77; c[0][2][2][0] = 0.77; c[2][0][0][2] = 0.77;
}

static void tetragonal(gs_params* p, int nv, double along, double other) {
  memset(p->eigenstrain, 0, sizeof(p->eigenstrain));
  for (int v = 0; v < nv; ++v)
    for (int a = 0; a < 3; ++a) p->eigenstrain[v][a][a] = (a == v % 3) ? along : other;
}

extern "C" int gs_params_default(gs_params* p, int model, int mode) {
  if (!p) return gs_set_error(GS_EINVAL, "gs_params_default: null params");
  memset(p, 0, sizeof(*p));
  p->model = model;
  p->mode = mode;
  p->dtype = GS_DTYPE_F32;
  p->dx = p->dy = p->dz = 1.0;
  p->weight_elastic = 1.0;
  p->xi = 1.0;
  if (model == GS_MODEL_MART) {
    if (mode == GS_MODE_REFCOMPAT) {
      // src/dynamics_mart.cu:20-27,40,80-89
      p->nvariants = 4;
      p->nx = p->ny = p->nz = 64;
      p->dt = 0.01;
      p->transition_temperature = 450.0;
      p->temperature = 450.0;
      p->weight_gradient = 2.5;
      p->weight_chemical = 1.0;
      p->weight_elastic = 100000.0;
      p->weight_dislocation = 1.0;
      p->noise_amp = 0.0001;
      p->lpc[2] = 32.05;
      p->lpc[3] = 37.5;
      set_cubic(p, 3.5, 1.5, 1.0);
    } else {
      // 3D cubic-to-tetragonal, 3 variants, 256^3 (the headline workload)
      p->nvariants = 3;
      p->nx = p->ny = p->nz = 256;
      p->dt = 0.005;
      p->landau[0] = 0.2;
      p->landau[1] = 3.0;
      p->landau[2] = 2.0;
      p->landau[3] = 1.0;
      p->kappa = 0.5;
      p->mobility = 1.0;
      tetragonal(p, 3, 0.02, -0.01);
      set_cubic(p, 1.4, 0.84, 0.56);
      p->applied_stress[2][2] = 0.005;
      p->noise_amp = 1e-3;
      p->seed = 1;
    }
  } else if (model == GS_MODEL_PRECIPITATE) {
    p->nvariants = 4;
    if (mode == GS_MODE_REFCOMPAT) {
      // src/dynamics_precipitate.cu:20-29,55
      p->nx = p->ny = p->nz = 64;
      p->dt = 0.1;
      const double A[8] = {0, 54.0, -17.0, 7.0, 2.5, 0.2, 0.2, 0.2};
      memcpy(p->coef, A, sizeof(A));
      p->kappa_eta = 300.0;
      p->kappa_c = 300.0;
      p->mobility_c = 0.4;
      p->mobility_eta = 0.4;
      p->xi = 400.0;
      p->c1 = 0.1;
      p->c2 = 0.44;
      p->noise_amp = 1.0;
      set_cubic(p, 3.5, 1.5, 1.0);
    } else {
      // 3D precipitate, c + 4 variants, 256^3
      p->nx = p->ny = p->nz = 256;
      p->dt = 0.01;
      // f = A1/2 (c-c1)^2 + A2/2 (c2-c) S eta^2 - A3/4 S eta^4 + A4/6 S eta^6
      //     + A5 S_{p<q} eta_p^2 eta_q^2, written in the 7-coefficient form
      const double A[8] = {0, 2.0, -20.0, 16.0, 14.0, 1.0, 0.0, 0.0};
      memcpy(p->coef, A, sizeof(A));
      p->c1 = 0.05;
      p->c2 = 0.95;
      p->kappa_c = 1.5;
      p->kappa_eta = 1.0;
      p->mobility_c = 1.0;
      p->mobility_eta = 1.0;
      p->misfit_c = 0.01;
      p->c_elastic = 1;
      p->mass_projection = 1;
      tetragonal(p, 4, 0.005, -0.0025);
      set_cubic(p, 1.4, 0.84, 0.56);
      p->seed = 2;
    }
  } else if (model == GS_MODEL_STRESS) {
    p->nvariants = 4;
    p->nx = p->ny = p->nz = 64;
    p->dt = 1.0;
    if (mode == GS_MODE_REFCOMPAT) {
      p->xi = 4000.0;  // src/dynamics_stress.cu:34
      set_stress_default_modulus(p);
    } else {
      set_cubic(p, 1.4, 0.84, 0.56);
    }
  } else {
    return gs_set_error(GS_EINVAL, "gs_params_default: unknown model %d", model);
  }
  return GS_OK;
}

// ---------------------------------------------------------------------------
// geometry and constants
// ---------------------------------------------------------------------------
static int canonicalize(gs_sim* s) {
  const gs_params& p = s->p;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  if (nx < 1 || ny < 1 || nz < 1) return gs_set_error(GS_EINVAL, "grid %d %d %d", nx, ny, nz);
  const double d[3] = {p.dx, p.dy, p.dz};
  int n[3], perm[3];
  if (nz > 1) {
    n[0] = nx; n[1] = ny; n[2] = nz; perm[0] = 0; perm[1] = 1; perm[2] = 2;
  } else if (ny > 1) {
    n[0] = 1; n[1] = nx; n[2] = ny; perm[0] = 2; perm[1] = 0; perm[2] = 1;
  } else {
    n[0] = 1; n[1] = 1; n[2] = nx; perm[0] = 1; perm[1] = 2; perm[2] = 0;
  }
  for (int c = 0; c < 3; ++c) {
    s->perm[c] = perm[c];
    s->dcan[c] = d[perm[c]];
  }
  s->n0 = n[0];
  s->n1 = n[1];
  s->n2 = n[2];
  if (n[2] % 2 != 0) return gs_set_error(GS_ENOTSUP, "last non-unit axis must be even (got %d)", n[2]);
  s->h = n[2] / 2;
  s->N = (long long)n[0] * n[1] * n[2];
  if (!size_supported(s->h) || !size_supported(n[1]) || !size_supported(n[0]))
    return gs_set_error(GS_ENOTSUP, "grid %dx%dx%d: line lengths must be 1 or one of 2,4,6,8,12,16,24,32,48,64,96,128,256 (z: 2x that)",
                        nx, ny, nz);
  if (n[1] != 1 && n[1] % 2 != 0) return gs_set_error(GS_ENOTSUP, "middle axis must be 1 or even");
  return GS_OK;
}

// strain sets of the B contraction: 0 = variants x variants, 1 = 6 unit
// strains x variants, 2 = precipitate fields (eta_p^2 then c)
static void strain_sets(const gs_params& p, int which, double (*ea)[3][3], int* na, double (*eb)[3][3], int* nb) {
  const int V = p.nvariants;
  if (which == 1) {
    const int bi[6] = {0, 0, 0, 1, 1, 2}, bj[6] = {0, 1, 2, 1, 2, 2};
    for (int b = 0; b < 6; ++b) {
      memset(ea[b], 0, sizeof(double) * 9);
      if (p.mode == GS_MODE_REFCOMPAT || bi[b] == bj[b]) {
        ea[b][bi[b]][bj[b]] = 1.0;
      } else {
        ea[b][bi[b]][bj[b]] = 0.5;
        ea[b][bj[b]][bi[b]] = 0.5;
      }
    }
    *na = 6;
    for (int v = 0; v < V; ++v) memcpy(eb[v], p.eigenstrain[v], sizeof(double) * 9);
    *nb = V;
    return;
  }
  for (int v = 0; v < V; ++v) {
    memcpy(ea[v], p.eigenstrain[v], sizeof(double) * 9);
    memcpy(eb[v], p.eigenstrain[v], sizeof(double) * 9);
  }
  int F = V;
  if (which == 2 && p.c_elastic) {
    memset(ea[V], 0, sizeof(double) * 9);
    for (int i = 0; i < 3; ++i) ea[V][i][i] = p.misfit_c;
    memcpy(eb[V], ea[V], sizeof(double) * 9);
    F = V + 1;
  }
  *na = *nb = F;
}

// B(n) is invariant under a relabelling of the axes applied to n, C and the
// strains together, so the constants are expressed in the canonical axis
// order (canonical axis c = original axis perm[c]) and the kernels use the
// canonical wave vector directly.
template <typename T> void build_elastic(const gs_sim* s, int which, double scale, ElasticConst<T>& ec) {
  const gs_params& p = s->p;
  double ea0[GS_MAXG + 1][3][3], eb0[GS_MAXF + 1][3][3];
  int na, nb;
  strain_sets(p, which, ea0, &na, eb0, &nb);
  const int* pm = s->perm;
  double ea[GS_MAXG + 1][3][3], eb[GS_MAXF + 1][3][3], C[3][3][3][3];
  for (int a = 0; a < na; ++a)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ea[a][i][j] = ea0[a][pm[i]][pm[j]];
  for (int b = 0; b < nb; ++b)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) eb[b][i][j] = eb0[b][pm[i]][pm[j]];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) C[i][j][k][l] = p.cijkl[pm[i]][pm[j]][pm[k]][pm[l]];
  memset(&ec, 0, sizeof(ec));
  ec.na = na;
  ec.nb = nb;
  ec.refcompat = p.mode == GS_MODE_REFCOMPAT;
  // Omega^-1_ij = C_iklj n_k n_l on the six entries ij = 00 01 02 11 12 22,
  // symmetrised over ij (exact for a modulus with the major and minor
  // symmetries) and over kl (n_k n_l is symmetric)
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
  for (int e = 0; e < 6; ++e) {
    const int i = pa[e], j = pb[e];
    for (int q = 0; q < 6; ++q) {
      const int a = pa[q], b = pb[q];
      double v = 0.5 * (C[i][a][b][j] + C[j][a][b][i]);
      if (a != b) v += 0.5 * (C[i][b][a][j] + C[j][b][a][i]);
      ec.qs[e][q] = (T)v;
    }
  }
  auto sig = [&](const double e[3][3], T out[3][3]) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double acc = 0;
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) acc += C[i][j][k][l] * e[k][l];
        out[i][j] = (T)acc;
      }
  };
  for (int a = 0; a < na; ++a) sig(ea[a], ec.sa[a]);
  for (int b = 0; b < nb; ++b) sig(eb[b], ec.sb[b]);
  for (int a = 0; a < na; ++a)
    for (int b = 0; b < nb; ++b) {
      double acc = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) acc += C[i][j][k][l] * ea[a][i][j] * eb[b][k][l];
      ec.a0[a][b] = (T)acc;
    }
  const int nc[3] = {s->n0, s->n1, s->n2};
  for (int c = 0; c < 3; ++c) {
    const double d = s->dcan[c];
    ec.kscale[c] = (T)(ec.refcompat ? 2.0 * 3.14 * d / nc[c] : 2.0 * M_PI / (nc[c] * d));
  }
  ec.scale = (T)scale;
}

static double contract33(const double a[3][3], const double b[3][3]) {
  double s = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s += a[i][j] * b[i][j];
  return s;
}

template <typename T> static void build_mart_p(const gs_sim* s, const gs_params& p, int64_t step, MartConst<T>& mc);

template <typename T> void build_mart(const gs_sim* s, MartConst<T>& mc) { build_mart_p<T>(s, s->p, s->step, mc); }

template <typename T> static void build_mart_p(const gs_sim* s, const gs_params& p, int64_t step, MartConst<T>& mc) {
  memset(&mc, 0, sizeof(mc));
  const bool ref = p.mode == GS_MODE_REFCOMPAT;
  mc.V = p.nvariants;
  mc.refcompat = ref;
  mc.has_defect = s->defect != nullptr;
  mc.has_K = s->K != nullptr;
  mc.dt = (T)p.dt;
  const int nc[3] = {s->n0, s->n1, s->n2};
  for (int c = 0; c < 3; ++c) {
    const double d = s->dcan[c];
    if (nc[c] == 1) {
      mc.lapc[c] = 0;
      mc.gcoef[c] = 0;
    } else {
      mc.lapc[c] = (T)(ref ? p.weight_gradient / (2.0 * d) / 3.0 : p.mobility * p.kappa / (d * d));
      mc.gcoef[c] = (T)(1.0 / (d * d));
    }
  }
  mc.A2 = (T)p.landau[0];
  mc.A4 = (T)p.landau[1];
  mc.A6 = (T)p.landau[2];
  mc.Ac = (T)p.landau[3];
  mc.L = (T)p.mobility;
  mc.kappa = (T)p.kappa;
  mc.el = (T)(ref ? -p.weight_elastic : -2.0 * p.mobility * p.weight_elastic);
  for (int v = 0; v < p.nvariants; ++v) {
    const double sa = contract33(p.applied_stress, p.eigenstrain[v]);
    mc.lin[v] = (T)(ref ? 0.0 : 2.0 * p.mobility * sa);
    mc.appl[v] = (T)sa;
  }
  mc.kc = (T)(ref ? -25.0 * p.weight_dislocation : 2.0 * p.mobility * p.weight_dislocation);
  mc.wD = (T)p.weight_dislocation;
  const float a1 = 0.02f * ((float)p.temperature - (float)p.transition_temperature);
  mc.a1 = (T)a1;
  mc.a2 = (T)p.lpc[2];
  mc.a3 = (T)p.lpc[3];
  mc.s = (T)std::sqrt(std::fabs((double)a1 / (p.lpc[2] - p.lpc[3])));
  mc.wC = (T)p.weight_chemical;
  mc.noise = (T)(ref ? p.dt * p.noise_amp : p.noise_amp);
  mc.wel_half = (T)(0.5 * p.weight_elastic);
  mc.k0 = (uint32_t)(p.seed & 0xffffffffu);
  mc.k1 = (uint32_t)(p.seed >> 32);
  mc.sim = p.sim_id;
  mc.step = (uint32_t)step;
}

// twiddle tables w_n^m = exp(-2 pi i m / n), m < n, for n2, h, n1, n0
template <typename T> static int build_twiddles(gs_sim* s) {
  const int lens[4] = {s->n2, s->h, s->n1, s->n0};
  size_t total = 0;
  for (int i = 0; i < 4; ++i) {
    s->tw_off[i] = total;
    total += (size_t)lens[i];
  }
  std::vector<cplx<T>> host(total);
  for (int i = 0; i < 4; ++i)
    for (int m = 0; m < lens[i]; ++m) {
      const double a = 2.0 * M_PI * (double)m / (double)lens[i];
      host[s->tw_off[i] + m] = mk2((T)std::cos(a), (T)-std::sin(a));
    }
  GS_CU(cudaMalloc(&s->tw, total * sizeof(cplx<T>)), "cudaMalloc twiddles");
  GS_CU(cudaMemcpy(s->tw, host.data(), total * sizeof(cplx<T>), cudaMemcpyHostToDevice), "upload twiddles");
  GS_CU(cudaDeviceSynchronize(), "upload twiddles sync");
  return GS_OK;
}

template <typename T> static const cplx<T>* twp(const gs_sim* s, int which) {
  return reinterpret_cast<const cplx<T>*>(s->tw) + s->tw_off[which];
}

// ---------------------------------------------------------------------------
// octant table of B(k)
// ---------------------------------------------------------------------------
// B(k) is even in axis c when reflecting that axis maps the problem onto
// itself: the stresses sigma = C:eps have no shear component coupling c with
// another axis, and the quadratic form Omega^-1(n) keeps its parity.  Axes of
// extent 1 carry k = 0 only and need no check.
// the contraction a model's step runs through the table: martensite the
// variants x variants set, precipitate the (eta_p^2, c) set; -1: none
static int btab_which(const gs_sim* s) {
  return s->p.model == GS_MODEL_MART ? 0 : (s->p.model == GS_MODEL_PRECIPITATE ? 2 : -1);
}

static bool btab_symmetric(const gs_sim* s) {
  ElasticConst<double> ec;
  build_elastic<double>(s, btab_which(s), 1.0, ec);
  if (ec.na != ec.nb) return false;  // square sets only
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
  const int nc[3] = {s->n0, s->n1, s->n2};
  for (int c = 0; c < 3; ++c) {
    if (nc[c] == 1) continue;
    for (int f = 0; f < ec.nb; ++f)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          if ((i == c) != (j == c) && (ec.sa[f][i][j] != 0.0 || ec.sb[f][i][j] != 0.0)) return false;
    for (int e = 0; e < 6; ++e)
      for (int q = 0; q < 6; ++q) {
        const int pe = (pa[e] == c) + (pb[e] == c), pq = (pa[q] == c) + (pb[q] == c);
        if ((pe + pq) % 2 != 0 && ec.qs[e][q] != 0.0) return false;
      }
  }
  return true;
}

// (Re)build the table of the handle's current parameters (martensite only).
template <typename T> static int build_btab(gs_sim* s, cudaStream_t st) {
  const int which = btab_which(s);
  if (which < 0 || s->btab_state == -1) return GS_OK;
  if (!btab_symmetric(s)) {
    s->btab_state = -2;
    return GS_OK;
  }
  ElasticConst<T> ec;
  build_elastic<T>(s, which, 1.0 / (double)s->N, ec);
  s->btab_fields = ec.nb;
  const size_t npt = (size_t)(s->n0 / 2 + 1) * (s->n1 / 2 + 1) * (s->n2 / 2 + 1);
  const size_t bytes = npt * btab_stride(ec.nb) * sizeof(T);
  if (s->btab && s->btab_bytes != bytes) {
    cudaFree(s->btab);
    s->btab = nullptr;
  }
  if (!s->btab) {
    GS_CU(cudaMalloc(&s->btab, bytes), "cudaMalloc B table");
    s->btab_bytes = bytes;
  }
  GS_CU(launch_btab_fill<T>(ec, s->n0, s->n1, s->n2, reinterpret_cast<T*>(s->btab), st), "B table fill");
  GS_CU(cudaStreamSynchronize(st), "B table sync");
  s->btab_state = 1;
  return GS_OK;
}

static int ensure_btab(gs_sim* s, cudaStream_t st) {
  return s->p.dtype == GS_DTYPE_F64 ? build_btab<double>(s, st) : build_btab<float>(s, st);
}

template <typename T> static void set_btab(const gs_sim* s, XArgs<T>& xa) {
  xa.btab = reinterpret_cast<const T*>(s->btab);
  xa.bt_d1 = s->n1 / 2 + 1;
  xa.bt_d2 = s->n2 / 2 + 1;
  xa.bt_stride = btab_stride(s->btab_fields);
}

// ---------------------------------------------------------------------------
// the martensite step
// ---------------------------------------------------------------------------
// z forward (with the eta^2 prologue where square[f]) -> y forward -> x pass
// (B contraction, F inputs -> G outputs, into out_spec) -> y inverse.
template <typename T>
static int elastic_chain_g(gs_sim* s, const T* const* src, const int* square, int F, int which, double scale,
                           void* out_spec, int G, cudaStream_t st, const T* const* mul = nullptr,
                           bool z_ready = false) {
  const long long rows = (long long)s->n0 * s->n1;
  s->spec_ready = false;  // the chain transforms the spectrum buffer in place
  ZfwdArgs<T> za;
  memset(&za, 0, sizeof(za));
  for (int f = 0; f < F; ++f) {
    za.src[f] = src[f];
    za.square[f] = square[f];
    za.mul[f] = mul ? mul[f] : nullptr;
  }
  za.dst = reinterpret_cast<cplx<T>*>(s->spec);
  za.rows_per_field = rows;
  za.nrows = rows * F;
  za.tw_h = twp<T>(s, 1);
  za.tw_n2 = twp<T>(s, 0);
  if (!z_ready) {  // else the previous update left the z spectra of src^2 in place
    GS_CU(launch_zfwd<T>(za, s->h, st, s->sched.z_lines), "z forward pass");
    gs_mark(s, st, "z_forward");
    s->launches += 1;
  }
  YArgs<T> ya;
  ya.spec = reinterpret_cast<cplx<T>*>(s->spec);
  ya.n0 = s->n0;
  ya.n1 = s->n1;
  ya.h = s->h;
  ya.tw = twp<T>(s, 2);
  GS_CU(launch_ypass<T>(ya, s->n1, F, -1, st, s->sched.y_cols, s->sched.y_radix), "y forward pass");
  if (s->n1 > 1) gs_mark(s, st, "y_forward");
  XArgs<T> xa;
  memset(&xa, 0, sizeof(xa));
  xa.in = reinterpret_cast<cplx<T>*>(s->spec);
  xa.out = reinterpret_cast<cplx<T>*>(out_spec);
  xa.n0 = s->n0;
  xa.n1 = s->n1;
  xa.n2 = s->n2;
  xa.h = s->h;
  xa.F = F;
  xa.G = G;
  xa.tw = twp<T>(s, 3);
  build_elastic<T>(s, which, scale, xa.ec);
  if (s->btab_state == 1 && which == btab_which(s) && F == s->btab_fields && G == F) set_btab<T>(s, xa);
  xa.tz_req = s->sched.x_cols;
  GS_CU(launch_xcontract<T>(xa, st), "x contraction pass");
  gs_mark(s, st, "x_contraction");
  YArgs<T> yb = ya;
  yb.spec = reinterpret_cast<cplx<T>*>(out_spec);
  GS_CU(launch_ypass<T>(yb, s->n1, G, 1, st, s->sched.y_cols, s->sched.y_radix), "y inverse pass");
  if (s->n1 > 1) gs_mark(s, st, "y_inverse");
  s->launches += 1 + (s->n1 > 1 ? 2 : 0);
  return GS_OK;
}

template <typename T> int elastic_chain(gs_sim* s, const T* eta, cudaStream_t st, bool z_ready = false) {
  const int V = s->p.nvariants;
  const T* src[GS_MAXF];
  int sq[GS_MAXF];
  for (int f = 0; f < V; ++f) {
    src[f] = eta + (long long)f * s->N;
    sq[f] = 1;
  }
  return elastic_chain_g<T>(s, src, sq, V, 0, 1.0 / (double)s->N, s->spec, V, st, nullptr, z_ready);
}

template <typename T> static void fill_mart_args(gs_sim* s, MartArgs<T>& ma, const T* in, T* out) {
  memset(&ma, 0, sizeof(ma));
  ma.spec = reinterpret_cast<const cplx<T>*>(s->spec);
  ma.eta_in = in;
  ma.eta_out = out;
  ma.defect = reinterpret_cast<const T*>(s->defect);
  ma.K = reinterpret_cast<const T*>(s->K);
  ma.n0 = s->n0;
  ma.n1 = s->n1;
  ma.n2 = s->n2;
  ma.nrows = (long long)s->n0 * s->n1;
  ma.tw_h = twp<T>(s, 1);
  ma.tw_n2 = twp<T>(s, 0);
  build_mart<T>(s, ma.mc);
  ma.partials = s->partials;
  ma.fd_n1 = FastDiv((uint32_t)s->n1);
  ma.fd_upr = FastDiv((uint32_t)(s->n2 % 4 == 0 ? s->n2 / 4 : s->n2 / 2));
  ma.fd_v = FastDiv((uint32_t)s->p.nvariants);
  ma.lr_req = s->sched.update_rows;
}

template <typename T> static int mart_step(gs_sim* s, cudaStream_t st) {
  T* in = reinterpret_cast<T*>(s->eta[s->cur]);
  T* out = reinterpret_cast<T*>(s->eta[s->cur ^ 1]);
  const bool z_ready = s->spec_ready && s->spec_cur == s->cur;
  GS_TRY(elastic_chain<T>(s, in, st, z_ready));
  MartArgs<T> ma;
  fill_mart_args<T>(s, ma, in, out);
  if (s->fuse) ma.spec_next = reinterpret_cast<cplx<T>*>(s->spec);
  GS_CU(launch_mart_update<T>(ma, s->h, false, st, nullptr), "update pass");
  gs_mark(s, st, "update");
  s->launches += 1;
  if (!s->trial) {  // a trial step wrote only the spare field and the spectra
    s->cur ^= 1;
    s->step += 1;
  }
  if (s->fuse) {  // the spectra of the field just written (trial steps: timing only)
    s->spec_ready = true;
    s->spec_cur = s->cur;
  }
  return GS_OK;
}

// R_p of the current state into R ([V][N]): the chain and the statistics
// sweep with its R output (the state is not advanced)
template <typename T> static int mart_potential(gs_sim* s, void* R, cudaStream_t st) {
  T* in = reinterpret_cast<T*>(s->eta[s->cur]);
  GS_TRY(elastic_chain<T>(s, in, st));
  MartArgs<T> ma;
  fill_mart_args<T>(s, ma, in, nullptr);
  ma.r_out = reinterpret_cast<T*>(R);
  int nb = 0;
  GS_CU(launch_mart_update<T>(ma, s->h, true, st, &nb), "potential pass");
  return GS_OK;
}

template <typename T> static int mart_stats(gs_sim* s, gs_stats* o, cudaStream_t st) {
  T* in = reinterpret_cast<T*>(s->eta[s->cur]);
  GS_TRY(elastic_chain<T>(s, in, st));
  MartArgs<T> ma;
  fill_mart_args<T>(s, ma, in, nullptr);
  int nb = 0;
  GS_CU(launch_mart_update<T>(ma, s->h, true, st, &nb), "statistics pass");
  GS_CU(launch_reduce(s->partials, nb, ACC_N, s->red, st), "reduce");
  double acc[ACC_N];
  GS_CU(cudaMemcpyAsync(acc, s->red, sizeof(acc), cudaMemcpyDeviceToHost, st), "stats D2H");
  GS_CU(cudaStreamSynchronize(st), "stats sync");
  const int V = s->p.nvariants;
  const double N = (double)s->N;
  const double dV = s->p.dx * s->p.dy * s->p.dz;
  memset(o, 0, sizeof(*o));
  o->mass = acc[ACC_MASS];
  o->eta_mean = acc[ACC_MASS] / (N * V);
  for (int v = 0; v < V; ++v) {
    o->eta2[v] = acc[ACC_ETA2 + v] / N;
    o->vf[v] = acc[ACC_VF + v] / N;
  }
  o->e_el = acc[ACC_EEL] * dV;
  o->e_chem = acc[ACC_ECHEM] * dV;
  o->e_grad = acc[ACC_EGRAD] * dV;
  o->e_appl = acc[ACC_EAPPL] * dV;
  o->e_tot = o->e_el + o->e_chem + o->e_grad + o->e_appl;
  o->gradient_mean = acc[ACC_FGRAD] / (N * V);
  o->chemical_mean = acc[ACC_FCHEM] / (N * V);
  o->elastic_mean = acc[ACC_FEL] / (N * V);
  o->dislocation_mean = acc[ACC_FDISL] / (N * V);
  o->step = s->step;
  return GS_OK;
}

// ---------------------------------------------------------------------------
// the precipitate step (src/dynamics_precipitate.cu:278-289)
// ---------------------------------------------------------------------------
static int precip_nfields(const gs_sim* s) { return s->p.nvariants + (s->p.c_elastic ? 1 : 0); }

template <typename T> static void fill_ktab(gs_sim* s) {
  // K(k) per canonical axis: refcompat |k|^2 of the 3.14 vector (_gSquare,
  // src/gtensorb.cu:9-23), baseline the seven-point symbol 4/d^2 sin^2(pi m/n)
  const gs_params& p = s->p;
  const int nc[3] = {s->n0, s->n1, s->n2};
  std::vector<T> host;
  for (int c = 0; c < 3; ++c) {
    s->ktab_off[c] = host.size();
    const double d = s->dcan[c];
    for (int i = 0; i < nc[c]; ++i) {
      double v = 0;
      if (nc[c] > 1) {
        if (p.mode == GS_MODE_REFCOMPAT) {
          const int m = i < nc[c] / 2 ? i : i - nc[c];
          const double k = 2.0 * 3.14 * d / nc[c] * m;
          v = k * k;
        } else {
          const double sn = std::sin(M_PI * (double)i / nc[c]);
          v = 4.0 / (d * d) * sn * sn;
        }
      }
      host.push_back((T)v);
    }
  }
  cudaMemcpy(s->ktab, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
  cudaDeviceSynchronize();  // the copy above may return before its DMA lands
}

template <typename T> static int precip_potential(gs_sim* s, cudaStream_t st) {
  const int V = s->p.nvariants, F1 = precip_nfields(s);
  const T* eta = reinterpret_cast<const T*>(s->eta[0]);
  const T* src[GS_MAXF + 1];
  int sq[GS_MAXF + 1];
  for (int f = 0; f < V; ++f) {
    src[f] = eta + (long long)f * s->N;
    sq[f] = 1;
  }
  if (F1 > V) {
    src[V] = reinterpret_cast<const T*>(s->conc);
    sq[V] = 0;
  }
  GS_TRY(elastic_chain_g<T>(s, src, sq, F1, 2, 1.0 / (double)s->N, s->spec, F1, st));
  ZinvArgs<T> zi;
  memset(&zi, 0, sizeof(zi));
  zi.spec = reinterpret_cast<const cplx<T>*>(s->spec);
  for (int f = 0; f < F1; ++f) zi.dst[f] = reinterpret_cast<T*>(s->rbuf) + (long long)f * s->N;
  zi.rows_per_field = (long long)s->n0 * s->n1;
  zi.nrows = zi.rows_per_field * F1;
  zi.tw_h = twp<T>(s, 1);
  zi.tw_n2 = twp<T>(s, 0);
  zi.offset_field = -1;
  GS_CU(launch_zinv<T>(zi, s->h, st), "z inverse (elastic potential)");
  gs_mark(s, st, "z_inverse_potential");
  s->launches += 1;
  return GS_OK;
}

template <typename T> static int precip_step(gs_sim* s, cudaStream_t st) {
  const gs_params& p = s->p;
  const int V = p.nvariants;
  const long long N = s->N;
  const bool ref = p.mode == GS_MODE_REFCOMPAT;
  const int F1 = precip_nfields(s);
  T* eta = reinterpret_cast<T*>(s->eta[0]);
  T* c = reinterpret_cast<T*>(s->conc);
  T* mu = reinterpret_cast<T*>(s->mubuf);
  T* g = mu + N;
  PrecipLocalArgs<T> la;
  memset(&la, 0, sizeof(la));
  la.c = c;
  la.eta = eta;
  la.R = reinterpret_cast<const T*>(s->rbuf);
  la.mu = mu;
  la.g = g;
  la.N = N;
  la.V = V;
  la.c_elastic = p.c_elastic && !ref;
  for (int i = 0; i < 8; ++i) la.A[i] = (T)p.coef[i];
  la.c1 = (T)p.c1;
  la.c2 = (T)p.c2;
  la.Es = (T)(p.xi * p.weight_elastic);
  la.an = (T)(p.noise_amp * (ref ? 1e-4 : 1.0));
  la.k0 = (uint32_t)(p.seed & 0xffffffffu);
  la.k1 = (uint32_t)(p.seed >> 32);
  la.sim = p.sim_id;
  la.step = (uint32_t)s->step;
  la.fold = 1;  // the sweeps form u_p = eta_p - dt L g_p (see k_precip_mid)
  la.dtL = (T)(p.dt * p.mobility_eta);
  const int F2 = V + 2, G2 = V + 1;
  const long long rows = (long long)s->n0 * s->n1;
  // chain 1 to its y inverse, then one sweep: z C2R of R, local terms, z R2C
  // of the update fields (k_precip_mid); rows too wide for one block take the
  // separate passes
  bool fused = false;
  {
    const T* src[GS_MAXF + 1];
    int sq[GS_MAXF + 1];
    for (int f = 0; f < V; ++f) {
      src[f] = eta + (long long)f * N;
      sq[f] = 1;
    }
    if (F1 > V) {
      src[V] = c;
      sq[V] = 0;
    }
    // the previous step's fused z inverse may have left the z spectra of
    // [eta_p^2, c] in the spectrum buffer
    const bool z_ready = s->spec_ready && s->spec_cur == 0;
    GS_TRY(elastic_chain_g<T>(s, src, sq, F1, 2, 1.0 / (double)N, s->spec, F1, st, nullptr, z_ready));
    PrecipMidArgs<T> pm;
    memset(&pm, 0, sizeof(pm));
    pm.rspec = reinterpret_cast<const cplx<T>*>(s->spec);
    pm.c = c;
    pm.eta = eta;
    pm.dst = reinterpret_cast<cplx<T>*>(s->spec2);
    pm.lr_req = s->sched.update_rows;
    pm.nrows = rows;
    pm.n2 = s->n2;
    pm.F1 = F1;
    pm.tw_h = twp<T>(s, 1);
    pm.tw_n2 = twp<T>(s, 0);
    pm.loc = la;
    const cudaError_t e = launch_precip_mid<T>(pm, s->h, st);
    if (e == cudaSuccess) {
      fused = true;
      gs_mark(s, st, "precip_mid");
      s->launches += 1;
    } else if (e != cudaErrorInvalidConfiguration) {
      GS_CU(e, "precipitate middle sweep");
    }
  }
  if (!fused) {
    ZinvArgs<T> zr;
    memset(&zr, 0, sizeof(zr));
    zr.spec = reinterpret_cast<const cplx<T>*>(s->spec);
    for (int f = 0; f < F1; ++f) zr.dst[f] = reinterpret_cast<T*>(s->rbuf) + (long long)f * N;
    zr.rows_per_field = rows;
    zr.nrows = rows * F1;
    zr.tw_h = twp<T>(s, 1);
    zr.tw_n2 = twp<T>(s, 0);
    zr.offset_field = -1;
    GS_CU(launch_zinv<T>(zr, s->h, st), "z inverse (elastic potential)");
    gs_mark(s, st, "z_inverse_potential");
    GS_CU(launch_precip_local<T>(la, st), "precipitate local terms");
    gs_mark(s, st, "precip_local");
    s->launches += 2;
  }
  // chain 2: [c, mu, u_0, u_1, ...] -> k-space update -> [c', eta'] (u_p
  // formed by the local terms in place of g_p)
  ZfwdArgs<T> za;
  memset(&za, 0, sizeof(za));
  za.src[0] = c;
  za.src[1] = mu;
  for (int v = 0; v < V; ++v) za.src[2 + v] = g + (long long)v * N;
  za.dst = reinterpret_cast<cplx<T>*>(s->spec2);
  za.rows_per_field = rows;
  za.nrows = rows * F2;
  za.tw_h = twp<T>(s, 1);
  za.tw_n2 = twp<T>(s, 0);
  if (!fused) {
    GS_CU(launch_zfwd<T>(za, s->h, st, s->sched.z_lines), "z forward (update fields)");
    gs_mark(s, st, "z_forward_update_fields");
    s->launches += 1;
  }
  YArgs<T> ya;
  ya.spec = reinterpret_cast<cplx<T>*>(s->spec2);
  ya.n0 = s->n0;
  ya.n1 = s->n1;
  ya.h = s->h;
  ya.tw = twp<T>(s, 2);
  GS_CU(launch_ypass<T>(ya, s->n1, F2, -1, st, s->sched.y_cols, s->sched.y_radix), "y forward (update fields)");
  if (s->n1 > 1) gs_mark(s, st, "y_forward_update_fields");
  XArgs<T> xa;
  memset(&xa, 0, sizeof(xa));
  xa.in = reinterpret_cast<cplx<T>*>(s->spec2);
  xa.out = reinterpret_cast<cplx<T>*>(s->spec2);
  xa.n0 = s->n0;
  xa.n1 = s->n1;
  xa.n2 = s->n2;
  xa.h = s->h;
  // the (c, mu) pair -> c', then one u_p per grid-z slice -> eta_p', written
  // to the chain-1 spectrum buffer (free by now), not in place
  xa.out = reinterpret_cast<cplx<T>*>(s->spec);
  xa.F = 2;
  xa.G = 1;
  xa.nsim = 1;
  xa.tz_req = s->sched.x_cols;
  xa.tw = twp<T>(s, 3);
  xa.pu.V = V;
  xa.pu.mass_proj = p.mass_projection;
  xa.pu.dtM = (T)(p.dt * p.mobility_c);
  xa.pu.dtL = (T)(p.dt * p.mobility_eta);
  xa.pu.kc = (T)p.kappa_c;
  xa.pu.ke = (T)p.kappa_eta;
  xa.pu.scale = (T)(1.0 / (double)N);
  for (int c3 = 0; c3 < 3; ++c3) xa.pu.ktab[c3] = reinterpret_cast<const T*>(s->ktab) + s->ktab_off[c3];
  GS_CU(launch_xprecip<T>(xa, st), "x pass (k-space update of c)");
  {
    const long long fs = (long long)s->n0 * s->n1 * s->h;  // complex values per field
    XArgs<T> xe = xa;
    xe.in = reinterpret_cast<cplx<T>*>(s->spec2) + 2 * fs;
    xe.out = reinterpret_cast<cplx<T>*>(s->spec) + fs;
    xe.F = 1;
    xe.G = 1;
    xe.nsim = V;
    GS_CU(launch_xprecip_eta<T>(xe, st), "x pass (k-space update of eta)");
  }
  gs_mark(s, st, "x_kspace_update");
  YArgs<T> yo = ya;
  yo.spec = reinterpret_cast<cplx<T>*>(s->spec);
  GS_CU(launch_ypass<T>(yo, s->n1, G2, 1, st, s->sched.y_cols, s->sched.y_radix), "y inverse (update fields)");
  if (s->n1 > 1) gs_mark(s, st, "y_inverse_update_fields");
  // z inverse of [c', eta'] fused with the next step's chain-1 z forward
  // (rows whose lines exceed one block take the plain z inverse)
  PrecipZArgs<T> pz;
  memset(&pz, 0, sizeof(pz));
  pz.spec = reinterpret_cast<cplx<T>*>(s->spec);
  pz.c = c;
  pz.eta = eta;
  pz.nrows = rows;
  pz.N = N;
  pz.V = V;
  pz.F1 = F1;
  pz.mass = p.mass_projection;
  pz.offset = s->mass0 / (double)N;
  pz.tw_h = twp<T>(s, 1);
  pz.tw_n2 = twp<T>(s, 0);
  const cudaError_t ez = launch_precip_zinv_fwd<T>(pz, s->h, st);
  if (ez == cudaSuccess) {
    gs_mark(s, st, "z_inverse_c_eta_next_z_forward");
    s->spec_ready = true;  // the next step skips its z forward
    s->spec_cur = 0;
  } else {
    if (ez != cudaErrorInvalidConfiguration) GS_CU(ez, "z inverse (c, eta) + next z forward");
    ZinvArgs<T> zi;
    memset(&zi, 0, sizeof(zi));
    zi.spec = reinterpret_cast<const cplx<T>*>(s->spec);
    zi.dst[0] = c;
    for (int v = 0; v < V; ++v) zi.dst[1 + v] = eta + (long long)v * N;
    zi.rows_per_field = rows;
    zi.nrows = rows * G2;
    zi.tw_h = twp<T>(s, 1);
    zi.tw_n2 = twp<T>(s, 0);
    zi.offset_field = p.mass_projection ? 0 : -1;
    zi.offset = s->mass0 / (double)N;
    GS_CU(launch_zinv<T>(zi, s->h, st), "z inverse (c, eta)");
    gs_mark(s, st, "z_inverse_c_eta");
  }
  s->launches += 3 + (s->n1 > 1 ? 2 : 0);
  s->step += 1;
  return GS_OK;
}

template <typename T> static int precip_stats(gs_sim* s, gs_stats* o, cudaStream_t st) {
  const gs_params& p = s->p;
  const int V = p.nvariants;
  GS_TRY(precip_potential<T>(s, st));
  PrecipStatsArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.c = reinterpret_cast<const T*>(s->conc);
  a.eta = reinterpret_cast<const T*>(s->eta[0]);
  a.R = reinterpret_cast<const T*>(s->rbuf);
  a.N = s->N;
  a.n0 = s->n0;
  a.n1 = s->n1;
  a.n2 = s->n2;
  a.V = V;
  a.c_elastic = p.c_elastic;
  for (int i = 0; i < 8; ++i) a.A[i] = (T)p.coef[i];
  a.c1 = (T)p.c1;
  a.c2 = (T)p.c2;
  a.Es = (T)(p.xi * p.weight_elastic);
  a.kc = (T)p.kappa_c;
  a.ke = (T)p.kappa_eta;
  const int nc[3] = {s->n0, s->n1, s->n2};
  for (int c = 0; c < 3; ++c) a.gcoef[c] = nc[c] > 1 ? (T)(1.0 / (s->dcan[c] * s->dcan[c])) : (T)0;
  a.partials = s->partials;
  int nb = 0;
  GS_CU(launch_precip_stats<T>(a, st, &nb), "precipitate statistics");
  GS_CU(launch_reduce(s->partials, nb, ACC_N, s->red, st), "reduce");
  double acc[ACC_N];
  GS_CU(cudaMemcpyAsync(acc, s->red, sizeof(acc), cudaMemcpyDeviceToHost, st), "stats D2H");
  GS_CU(cudaStreamSynchronize(st), "stats sync");
  const double N = (double)s->N, dV = p.dx * p.dy * p.dz;
  memset(o, 0, sizeof(*o));
  o->mass = acc[ACC_MASS];
  o->c_mean = acc[ACC_MASS] / N;
  o->eta_mean = acc[ACC_C] / (N * V);
  for (int v = 0; v < V; ++v) {
    o->eta2[v] = acc[ACC_ETA2 + v] / N;
    o->vf[v] = acc[ACC_VF + v] / N;
  }
  o->e_el = acc[ACC_EEL] * dV;
  o->e_chem = acc[ACC_ECHEM] * dV;
  o->e_grad = acc[ACC_EGRAD] * dV;
  o->e_tot = o->e_el + o->e_chem + o->e_grad;
  o->step = s->step;
  return GS_OK;
}

// ---------------------------------------------------------------------------
// the stress field (src/dynamics_stress.cu:147-194)
// ---------------------------------------------------------------------------
template <typename T> static int stress_step(gs_sim* s, cudaStream_t st) {
  const int V = s->p.nvariants;
  const T* eta = reinterpret_cast<const T*>(s->eta[0]);
  const T* src[GS_MAXF];
  int sq[GS_MAXF];
  for (int f = 0; f < V; ++f) {
    src[f] = eta + (long long)f * s->N;
    sq[f] = 1;
  }
  // sigma_b = -Xi IFFT(sum_v B_bv FFT(eta_v^2) / N)
  GS_TRY(elastic_chain_g<T>(s, src, sq, V, 1, -s->p.xi / (double)s->N, s->spec2, 6, st));
  ZinvArgs<T> zi;
  memset(&zi, 0, sizeof(zi));
  zi.spec = reinterpret_cast<const cplx<T>*>(s->spec2);
  for (int b = 0; b < 6; ++b) zi.dst[b] = reinterpret_cast<T*>(s->stressbuf) + (long long)b * s->N;
  zi.rows_per_field = (long long)s->n0 * s->n1;
  zi.nrows = zi.rows_per_field * 6;
  zi.tw_h = twp<T>(s, 1);
  zi.tw_n2 = twp<T>(s, 0);
  zi.offset_field = -1;
  GS_CU(launch_zinv<T>(zi, s->h, st), "z inverse (stress)");
  gs_mark(s, st, "z_inverse_stress");
  GS_CU(launch_defect<T>(eta, reinterpret_cast<T*>(s->defect), s->N, V, st), "defect mask");
  gs_mark(s, st, "defect_mask");
  s->launches += 2;
  s->step += 1;
  return GS_OK;
}

// ---------------------------------------------------------------------------
// lifecycle
// ---------------------------------------------------------------------------
static size_t elt(const gs_sim* s) { return s->p.dtype == GS_DTYPE_F64 ? 8 : 4; }

static void free_snaps(gs_sim* s);

static void free_sim(gs_sim* s) {
  if (!s) return;
  free_snaps(s);
  if (s->up_stream) cudaStreamSynchronize(s->up_stream);
  if (s->stage) cudaFree(s->stage);
  if (s->up_stream) cudaStreamDestroy(s->up_stream);
  if (s->up_done) cudaEventDestroy(s->up_done);
  if (s->stage_free) cudaEventDestroy(s->stage_free);
  void* ptrs[] = {s->eta[0], s->eta[1], s->spec, s->spec2, s->defect, s->K, s->conc, s->rbuf, s->mubuf,
                  s->stressbuf, s->ktab, s->tw, s->partials, s->red, s->btab, s->d_mcs, s->d_simscale};
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (s->own_stream) cudaStreamDestroy(s->own_stream);
  for (int i = 0; i < gs_sim::kMaxMarks; ++i)
    if (s->marks[i]) cudaEventDestroy(s->marks[i]);
  gs_plain_free(s);
  gs_cufft_free(s);
  delete s;
}

template <typename T> __global__ void k_fill(T* p, long long n, T v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

static int dalloc(void** p, size_t bytes, const char* what) {
  GS_CU(cudaMalloc(p, bytes), what);
  GS_CU(cudaMemset(*p, 0, bytes), what);
  return GS_OK;
}

extern "C" int gs_sim_create(const gs_params* p, gs_sim** out) {
  if (!p || !out) return gs_set_error(GS_EINVAL, "gs_sim_create: null argument");
  *out = nullptr;
  if (p->model != GS_MODEL_MART && p->model != GS_MODEL_PRECIPITATE && p->model != GS_MODEL_STRESS)
    return gs_set_error(GS_EINVAL, "unknown model %d", p->model);
  if (p->nvariants < 1 || p->nvariants > GS_MAX_V)
    return gs_set_error(GS_EINVAL, "nvariants %d outside 1..%d", p->nvariants, GS_MAX_V);
  if (p->dtype != GS_DTYPE_F32 && p->dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", p->dtype);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return gs_set_error(GS_ENODEV, "no CUDA device visible");
  }
  gs_sim* s = new gs_sim();
  s->p = *p;
  int rc = canonicalize(s);
  if (rc != GS_OK) {
    delete s;
    return rc;
  }
  const size_t fb = (size_t)s->N * elt(s);
  const int V = p->nvariants;
  auto fail = [&](int code) {
    free_sim(s);
    return code;
  };
  if ((rc = gs_cuda_check(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking), "stream")) != GS_OK)
    return fail(rc);
  if ((rc = dalloc(&s->eta[0], fb * V, "eta")) != GS_OK) return fail(rc);
  if (p->model == GS_MODEL_MART) {
    if ((rc = dalloc(&s->eta[1], fb * V, "eta pair")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->spec, fb * V, "spectrum")) != GS_OK) return fail(rc);
  } else if (p->model == GS_MODEL_PRECIPITATE) {
    const int F1 = precip_nfields(s);
    if ((rc = dalloc(&s->conc, fb, "concentration")) != GS_OK) return fail(rc);
    // chain 1 (F1 fields), then the V + 1 outputs of the k-space update
    if ((rc = dalloc(&s->spec, fb * (V + 1), "spectrum")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->rbuf, fb * F1, "elastic potentials")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->mubuf, fb * (V + 1), "local terms")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->spec2, fb * (2 * V + 2), "update spectra")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->ktab, elt(s) * (size_t)(s->n0 + s->n1 + s->n2), "K table")) != GS_OK) return fail(rc);
    if (p->dtype == GS_DTYPE_F64)
      fill_ktab<double>(s);
    else
      fill_ktab<float>(s);
    // the reference's default concentration c1 + (c2 - c1)/3 (src/dynamics_precipitate.cu:42-47)
    const double c0 = p->c1 + (p->c2 - p->c1) / 3.0;
    if (p->dtype == GS_DTYPE_F64)
      k_fill<double><<<256, 256>>>(reinterpret_cast<double*>(s->conc), s->N, c0);
    else
      k_fill<float><<<256, 256>>>(reinterpret_cast<float*>(s->conc), s->N, (float)c0);
    if ((rc = gs_cuda_check(cudaDeviceSynchronize(), "init concentration")) != GS_OK) return fail(rc);
    s->mass0 = (p->dtype == GS_DTYPE_F64 ? c0 : (double)(float)c0) * (double)s->N;
  } else {
    if ((rc = dalloc(&s->spec, fb * V, "spectrum")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->spec2, fb * 6, "stress spectra")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->stressbuf, fb * 6, "stress")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&s->defect, fb, "defect")) != GS_OK) return fail(rc);
  }
  rc = p->dtype == GS_DTYPE_F64 ? build_twiddles<double>(s) : build_twiddles<float>(s);
  if (rc != GS_OK) return fail(rc);
  s->partials_cap = (size_t)s->n0 * s->n1 + 148 * 16 + 1;
  if ((rc = gs_cuda_check(cudaMalloc(&s->partials, s->partials_cap * ACC_N * sizeof(double)), "partials")) != GS_OK)
    return fail(rc);
  if ((rc = gs_cuda_check(cudaMalloc(&s->red, 64 * sizeof(double)), "reduce out")) != GS_OK) return fail(rc);
  if ((rc = ensure_btab(s, s->own_stream)) != GS_OK) return fail(rc);
  *out = s;
  return GS_OK;
}

extern "C" int gs_sim_destroy(gs_sim* s) {
  if (!s) return GS_OK;
  cudaDeviceSynchronize();
  free_sim(s);
  return GS_OK;
}

template <typename T> static std::vector<T> to_type(const void* host, size_t count, int dtype) {
  std::vector<T> v(count);
  if (dtype == GS_DTYPE_F64) {
    const double* h = static_cast<const double*>(host);
    for (size_t i = 0; i < count; ++i) v[i] = (T)h[i];
  } else {
    const float* h = static_cast<const float*>(host);
    for (size_t i = 0; i < count; ++i) v[i] = (T)h[i];
  }
  return v;
}

static int upload(gs_sim* s, void* dst, const void* host, size_t count, int dtype) {
  const int want = s->p.dtype;
  if (dtype == want) {
    GS_CU(cudaMemcpy(dst, host, count * elt(s), cudaMemcpyHostToDevice), "upload");
    GS_CU(cudaDeviceSynchronize(), "upload sync");
    return GS_OK;
  }
  if (want == GS_DTYPE_F64) {
    auto v = to_type<double>(host, count, dtype);
    GS_CU(cudaMemcpy(dst, v.data(), count * 8, cudaMemcpyHostToDevice), "upload");
  } else {
    auto v = to_type<float>(host, count, dtype);
    GS_CU(cudaMemcpy(dst, v.data(), count * 4, cudaMemcpyHostToDevice), "upload");
  }
  // a pageable cudaMemcpy may return before its last DMA lands; the passes
  // run on non-blocking streams, so wait for it here
  GS_CU(cudaDeviceSynchronize(), "upload sync");
  return GS_OK;
}

static int download(gs_sim* s, const void* src, void* host, size_t count, int dtype) {
  const int have = s->p.dtype;
  if (dtype == have) {
    GS_CU(cudaMemcpy(host, src, count * elt(s), cudaMemcpyDeviceToHost), "download");
    return GS_OK;
  }
  if (have == GS_DTYPE_F64) {
    std::vector<double> v(count);
    GS_CU(cudaMemcpy(v.data(), src, count * 8, cudaMemcpyDeviceToHost), "download");
    float* h = static_cast<float*>(host);
    for (size_t i = 0; i < count; ++i) h[i] = (float)v[i];
  } else {
    std::vector<float> v(count);
    GS_CU(cudaMemcpy(v.data(), src, count * 4, cudaMemcpyDeviceToHost), "download");
    double* h = static_cast<double*>(host);
    for (size_t i = 0; i < count; ++i) h[i] = (double)v[i];
  }
  return GS_OK;
}

// K_p(x) = sigma(x):eps_p from the 6-component form xx xy xz yy yz zz (the
// 3x3 remap of src/dynamics_mart.cu:128-150 and the contraction of
// DislocationForceInit, :305-321, which the reference runs on the host),
// in double with separately rounded products and sums, rounded to T at the end.
struct KCoef {
  double c[GS_MAX_V][6];  // multipliers of xx xy xz yy yz zz per variant
};
template <typename S, typename T>
__global__ void k_stress_to_K(const S* __restrict__ sig, long long N, int V, KCoef kc, T* __restrict__ K) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double s6[6];
#pragma unroll
    for (int b = 0; b < 6; ++b) s6[b] = (double)sig[(long long)b * N + i];
    for (int v = 0; v < V; ++v) {
      double acc = __dmul_rn(s6[0], kc.c[v][0]);
#pragma unroll
      for (int b = 1; b < 6; ++b) acc = __dadd_rn(acc, __dmul_rn(s6[b], kc.c[v][b]));
      K[(long long)v * N + i] = (T)acc;
    }
  }
}

// sig: device stress [6][N] of type sig_dtype
static int stress_to_K(gs_sim* s, const void* sig, int sig_dtype, cudaStream_t st) {
  const int V = s->p.nvariants;
  const long long N = s->N;
  KCoef kc;
  for (int v = 0; v < V; ++v) {
    const double(*e)[3] = s->p.eigenstrain[v];
    kc.c[v][0] = e[0][0];
    kc.c[v][1] = e[0][1] + e[1][0];
    kc.c[v][2] = e[0][2] + e[2][0];
    kc.c[v][3] = e[1][1];
    kc.c[v][4] = e[1][2] + e[2][1];
    kc.c[v][5] = e[2][2];
  }
  if (!s->K) GS_CU(cudaMalloc(&s->K, (size_t)N * V * elt(s)), "cudaMalloc K");
  long long nb = (N + 255) / 256;
  if (nb > 148 * 16) nb = 148 * 16;
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  if (sig_dtype == GS_DTYPE_F64) {
    if (f64)
      k_stress_to_K<double, double><<<(unsigned)nb, 256, 0, st>>>(static_cast<const double*>(sig), N, V, kc,
                                                                   static_cast<double*>(s->K));
    else
      k_stress_to_K<double, float><<<(unsigned)nb, 256, 0, st>>>(static_cast<const double*>(sig), N, V, kc,
                                                                  static_cast<float*>(s->K));
  } else {
    if (f64)
      k_stress_to_K<float, double><<<(unsigned)nb, 256, 0, st>>>(static_cast<const float*>(sig), N, V, kc,
                                                                  static_cast<double*>(s->K));
    else
      k_stress_to_K<float, float><<<(unsigned)nb, 256, 0, st>>>(static_cast<const float*>(sig), N, V, kc,
                                                                 static_cast<float*>(s->K));
  }
  GS_CU(cudaGetLastError(), "stress to K");
  GS_CU(cudaStreamSynchronize(st), "stress to K sync");
  return GS_OK;
}

// drop a captured step (its launches hold pointers and tile sizes)
static void sim_graph_reset(gs_sim* s) {
  if (s->gexec) {
    cudaGraphExecDestroy(s->gexec);
    s->gexec = nullptr;
  }
}

extern "C" int gs_sim_set_field(gs_sim* s, const char* name, const void* host, size_t count, int dtype) {
  if (!s || !name || !host) return gs_set_error(GS_EINVAL, "gs_sim_set_field: null argument");
  sim_graph_reset(s);
  s->spec_ready = false;
  if (std::string(name) == "eta") s->staged = false;  // a field set given now replaces a staged one
  gs_cufft_invalidate(s);
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", dtype);
  const int V = s->p.nvariants;
  const size_t N = (size_t)s->N;
  const std::string nm(name);
  if (nm == "eta") {
    if (count != N * V) return gs_set_error(GS_EINVAL, "eta: %zu values, expected %zu", count, N * V);
    return upload(s, s->eta[s->cur], host, count, dtype);
  }
  if (nm == "concentration") {
    if (s->p.model != GS_MODEL_PRECIPITATE) return gs_set_error(GS_EINVAL, "concentration: not a precipitate model");
    if (count != N) return gs_set_error(GS_EINVAL, "concentration: %zu values, expected %zu", count, N);
    GS_TRY(upload(s, s->conc, host, count, dtype));
    // FP64 mass of the values as stored on the device (the projection target)
    double m = 0, cmp = 0;
    for (size_t i = 0; i < N; ++i) {
      double x = dtype == GS_DTYPE_F64 ? static_cast<const double*>(host)[i] : static_cast<const float*>(host)[i];
      if (s->p.dtype == GS_DTYPE_F32) x = (double)(float)x;
      const double t = m + x;
      cmp += std::fabs(m) >= std::fabs(x) ? (m - t) + x : (x - t) + m;
      m = t;
    }
    s->mass0 = m + cmp;
    return GS_OK;
  }
  if (nm == "defect") {
    if (s->p.model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "defect is an input of the martensite model only");
    if (count != N) return gs_set_error(GS_EINVAL, "defect: %zu values, expected %zu", count, N);
    if (!s->defect) GS_CU(cudaMalloc(&s->defect, N * elt(s)), "cudaMalloc defect");
    return upload(s, s->defect, host, count, dtype);
  }
  if (nm == "dislocationstress") {
    if (count != 6 * N) return gs_set_error(GS_EINVAL, "dislocationstress: %zu values, expected %zu", count, 6 * N);
    const size_t eb = dtype == GS_DTYPE_F64 ? 8 : 4;
    void* sig = nullptr;
    GS_CU(cudaMalloc(&sig, 6 * N * eb), "cudaMalloc stress upload");
    int rc = gs_cuda_check(cudaMemcpy(sig, host, 6 * N * eb, cudaMemcpyHostToDevice), "upload stress");
    if (rc == GS_OK) rc = gs_cuda_check(cudaDeviceSynchronize(), "upload stress sync");
    if (rc == GS_OK) rc = stress_to_K(s, sig, dtype, s->own_stream);
    cudaFree(sig);
    return rc;
  }
  return gs_set_error(GS_EINVAL, "unknown field '%s'", name);
}

extern "C" int gs_sim_get_field(gs_sim* s, const char* name, void* host, size_t count, int dtype) {
  if (!s || !name || !host) return gs_set_error(GS_EINVAL, "gs_sim_get_field: null argument");
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", dtype);
  GS_CU(cudaStreamSynchronize(s->own_stream), "sync");
  GS_CU(cudaDeviceSynchronize(), "sync");
  const int V = s->p.nvariants;
  const size_t N = (size_t)s->N;
  const std::string nm(name);
  if (nm == "eta") {
    if (count != N * V) return gs_set_error(GS_EINVAL, "eta: %zu values, expected %zu", count, N * V);
    return download(s, s->eta[s->cur], host, count, dtype);
  }
  if (nm == "defect") {
    if (!s->defect) return gs_set_error(GS_EINVAL, "defect not set");
    if (count != N) return gs_set_error(GS_EINVAL, "defect: %zu values, expected %zu", count, N);
    return download(s, s->defect, host, count, dtype);
  }
  if (nm == "concentration") {
    if (!s->conc) return gs_set_error(GS_EINVAL, "concentration: not a precipitate model");
    if (count != N) return gs_set_error(GS_EINVAL, "concentration: %zu values, expected %zu", count, N);
    return download(s, s->conc, host, count, dtype);
  }
  if (nm == "stress") {
    if (!s->stressbuf) return gs_set_error(GS_EINVAL, "stress: not a stress model");
    if (count != 6 * N) return gs_set_error(GS_EINVAL, "stress: %zu values, expected %zu", count, 6 * N);
    return download(s, s->stressbuf, host, count, dtype);
  }
  if (nm == "elastic_potential") {
    const bool f64 = s->p.dtype == GS_DTYPE_F64;
    if (s->p.model == GS_MODEL_PRECIPITATE) {
      const size_t F1 = (size_t)precip_nfields(s);
      if (count != F1 * N) return gs_set_error(GS_EINVAL, "elastic_potential: %zu values, expected %zu", count, F1 * N);
      GS_TRY(f64 ? precip_potential<double>(s, s->own_stream) : precip_potential<float>(s, s->own_stream));
      GS_CU(cudaStreamSynchronize(s->own_stream), "sync");
      return download(s, s->rbuf, host, count, dtype);
    }
    if (s->p.model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "elastic_potential: martensite or precipitate");
    if (count != (size_t)V * N) return gs_set_error(GS_EINVAL, "elastic_potential: %zu values, expected %zu", count,
                                                    (size_t)V * N);
    void* R = nullptr;
    GS_CU(cudaMalloc(&R, (size_t)V * N * elt(s)), "cudaMalloc potential");
    int rc = f64 ? mart_potential<double>(s, R, s->own_stream) : mart_potential<float>(s, R, s->own_stream);
    if (rc == GS_OK) rc = gs_cuda_check(cudaStreamSynchronize(s->own_stream), "sync");
    if (rc == GS_OK) rc = download(s, R, host, count, dtype);
    cudaFree(R);
    return rc;
  }
  return gs_set_error(GS_EINVAL, "unknown field '%s'", name);
}

extern "C" int gs_sim_set_scalar(gs_sim* s, const char* name, double value) {
  if (!s || !name) return gs_set_error(GS_EINVAL, "gs_sim_set_scalar: null argument");
  const std::string nm(name);
  if (nm == "temperature") {
    s->p.temperature = value;
    return GS_OK;
  }
  if (nm == "step") {
    s->step = (int64_t)value;
    return GS_OK;
  }
  return gs_set_error(GS_EINVAL, "unknown scalar '%s'", name);
}

static cudaStream_t pick_stream(gs_sim* s, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
}

template <typename T> static int batch_group_step(gs_sim* g, cudaStream_t st);
template <typename T> static int batch_upload_consts(gs_sim* g);

// gs_sim_use_graph: the martensite step as a one-simulation group whose
// constants (noise step counter included) live in device memory, so that a
// captured graph of two steps (the field pair swaps back) replays exactly.
template <typename T> static int sim_graph_steps(gs_sim* s, int nsteps, cudaStream_t st) {
  if (!s->d_mcs) {
    GS_CU(cudaMalloc(&s->d_mcs, sizeof(MartConst<T>)), "cudaMalloc step constants");
    GS_CU(cudaMalloc(&s->d_simscale, sizeof(T)), "cudaMalloc step scale");
  }
  s->nb = 1;
  s->bp.assign(1, s->p);
  s->bstep.assign(1, s->step);
  // steps queued by an earlier call still read the constants: let them finish
  GS_CU(cudaStreamSynchronize(st), "sync before constants");
  GS_TRY(batch_upload_consts<T>(s));  // current temperature and step counter
  int done = 0;
  const bool ready = !s->fuse || (s->spec_ready && s->spec_cur == s->cur);
  if (!s->gexec || s->gexec_stream != st || s->gexec_cur != s->cur || !ready) {
    sim_graph_reset(s);
    // direct steps first (kernel attributes are set outside any capture)
    GS_TRY(batch_group_step<T>(s, st));
    GS_TRY(batch_group_step<T>(s, st));
    done = 2;
    const int cur = s->cur;
    const int64_t step = s->step;
    const std::vector<int64_t> bstep = s->bstep;
    cudaGraph_t graph;
    GS_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    int rc = batch_group_step<T>(s, st);
    if (rc == GS_OK) rc = batch_group_step<T>(s, st);
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    s->cur = cur;  // the capture ran nothing
    s->step = step;
    s->bstep = bstep;
    if (rc != GS_OK) return rc;
    GS_CU(e, "end capture");
    GS_CU(cudaGraphInstantiate(&s->gexec, graph, 0), "instantiate graph");
    cudaGraphDestroy(graph);
    s->gexec_stream = st;
    s->gexec_cur = cur;
  }
  for (; done + 2 <= nsteps; done += 2) {
    GS_CU(cudaGraphLaunch(s->gexec, st), "graph launch");
    s->step += 2;
    s->bstep[0] += 2;
  }
  for (; done < nsteps; ++done) GS_TRY(batch_group_step<T>(s, st));
  return GS_OK;
}

static int step_once(gs_sim* s, cudaStream_t st) {
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  if (s->p.model == GS_MODEL_MART) return f64 ? mart_step<double>(s, st) : mart_step<float>(s, st);
  if (s->p.model == GS_MODEL_PRECIPITATE) return f64 ? precip_step<double>(s, st) : precip_step<float>(s, st);
  return f64 ? stress_step<double>(s, st) : stress_step<float>(s, st);
}

// GS_TIMING (read once per process): unset, empty or "0" = off; "1" = one
// JSON line per step on stderr with the device time of every pass (CUDA
// events on the stepping stream, direct launches, the host waits for each
// step); any other value = the path of a file the lines are appended to.
static const char* timing_target() {
  static const char* const v = [] {
    const char* e = getenv("GS_TIMING");
    return (e && *e && strcmp(e, "0") != 0) ? e : static_cast<const char*>(nullptr);
  }();
  return v;
}

static int timed_steps(gs_sim* s, int nsteps, cudaStream_t st, const char* target) {
  for (int i = 0; i < gs_sim::kMaxMarks; ++i)
    if (!s->marks[i]) GS_CU(cudaEventCreate(&s->marks[i]), "event create");
  static const char* const models[4] = {"", "martensite", "precipitate", "stress"};
  for (int k = 0; k < nsteps; ++k) {
    const int64_t step = s->step;
    s->nmarks = 0;
    s->profiling = true;
    gs_mark(s, st);
    const int rc = step_once(s, st);
    s->profiling = false;
    if (rc != GS_OK) return rc;
    GS_CU(cudaEventSynchronize(s->marks[s->nmarks - 1]), "event sync");
    std::string line = "{\"gs_timing\": 1, \"model\": \"";
    line += models[s->p.model >= 1 && s->p.model <= 3 ? s->p.model : 0];
    char buf[256];
    snprintf(buf, sizeof(buf), "\", \"step\": %lld, \"grid\": [%d, %d, %d], \"variants\": %d, \"dtype\": \"%s\", \"passes\": [",
             (long long)step, s->p.nx, s->p.ny, s->p.nz, s->p.nvariants, s->p.dtype == GS_DTYPE_F64 ? "f64" : "f32");
    line += buf;
    double total = 0;
    for (int i = 0; i + 1 < s->nmarks; ++i) {
      float ms = 0;
      GS_CU(cudaEventElapsedTime(&ms, s->marks[i], s->marks[i + 1]), "elapsed");
      total += ms;
      snprintf(buf, sizeof(buf), "%s{\"name\": \"%s\", \"ms\": %.6f}", i ? ", " : "",
               s->mark_names[i + 1] ? s->mark_names[i + 1] : "pass", ms);
      line += buf;
    }
    snprintf(buf, sizeof(buf), "], \"step_ms\": %.6f}\n", total);
    line += buf;
    if (strcmp(target, "1") == 0) {
      fputs(line.c_str(), stderr);
    } else if (FILE* f = fopen(target, "a")) {
      fputs(line.c_str(), f);
      fclose(f);
    } else {
      return gs_set_error(GS_EINVAL, "GS_TIMING: cannot append to '%s'", target);
    }
  }
  return GS_OK;
}

// a field set staged by gs_sim_stage_field_async becomes the current one:
// the stepping stream waits for its copy, the buffers swap, and the buffer
// handed to the stage is free once the stepping stream passes this point
static int take_staged(gs_sim* s, cudaStream_t st) {
  if (!s->staged) return GS_OK;
  GS_CU(cudaStreamWaitEvent(st, s->up_done, 0), "wait for the staged upload");
  std::swap(s->eta[s->cur], s->stage);
  sim_graph_reset(s);
  s->spec_ready = false;
  gs_cufft_invalidate(s);
  GS_CU(cudaEventRecord(s->stage_free, st), "stage free");
  s->staged = false;
  return GS_OK;
}

extern "C" int gs_sim_stage_field_async(gs_sim* s, const char* name, const void* host, size_t count, int dtype) {
  if (!s || !name || !host) return gs_set_error(GS_EINVAL, "gs_sim_stage_field_async: null argument");
  if (std::string(name) != "eta") return gs_set_error(GS_EINVAL, "gs_sim_stage_field_async: only \"eta\"");
  if (s->p.model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "gs_sim_stage_field_async: martensite only");
  if (dtype != s->p.dtype) return gs_set_error(GS_EINVAL, "gs_sim_stage_field_async: dtype must be the simulation's");
  const size_t n = (size_t)s->N * s->p.nvariants;
  if (count != n) return gs_set_error(GS_EINVAL, "eta: %zu values, expected %zu", count, n);
  if (s->staged) return gs_set_error(GS_EINVAL, "gs_sim_stage_field_async: a staged field set waits for a step");
  if (!s->stage) {
    GS_CU(cudaMalloc(&s->stage, n * elt(s)), "cudaMalloc staging field set");
    GS_CU(cudaStreamCreateWithFlags(&s->up_stream, cudaStreamNonBlocking), "upload stream");
    GS_CU(cudaEventCreateWithFlags(&s->up_done, cudaEventDisableTiming), "event");
    GS_CU(cudaEventCreateWithFlags(&s->stage_free, cudaEventDisableTiming), "event");
    GS_CU(cudaEventRecord(s->stage_free, s->own_stream), "event");
  }
  // the stage may still be the buffer an earlier step read or a snapshot copied
  GS_CU(cudaStreamWaitEvent(s->up_stream, s->stage_free, 0), "wait for a free stage");
  GS_CU(cudaMemcpyAsync(s->stage, host, n * elt(s), cudaMemcpyHostToDevice, s->up_stream), "staged upload");
  GS_CU(cudaEventRecord(s->up_done, s->up_stream), "event");
  s->staged = true;
  return GS_OK;
}

static int gs_sim_step_body(gs_sim* s, int nsteps, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_sim_step(gs_sim* s, int nsteps, void* stream) {
  return bc_after(gs_sim_step_body(s, nsteps, stream), static_cast<cudaStream_t>(stream));
}

static int gs_sim_step_body(gs_sim* s, int nsteps, void* stream) {
  if (!s) return gs_set_error(GS_EINVAL, "gs_sim_step: null sim");
  if (nsteps < 0) return gs_set_error(GS_EINVAL, "nsteps %d", nsteps);
  cudaStream_t st = pick_stream(s, stream);
  s->launches = 0;
  GS_TRY(take_staged(s, st));
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  if (const char* tt = timing_target())
    if (!s->profiling && !s->trial) return timed_steps(s, nsteps, st, tt);
  if (s->use_graph && s->p.model == GS_MODEL_MART && !s->plain && nsteps >= 2)
    return f64 ? sim_graph_steps<double>(s, nsteps, st) : sim_graph_steps<float>(s, nsteps, st);
  for (int i = 0; i < nsteps; ++i) GS_TRY(step_once(s, st));
  return GS_OK;
}

extern "C" int gs_sim_stats(gs_sim* s, gs_stats* out, void* stream) {
  if (!s || !out) return gs_set_error(GS_EINVAL, "gs_sim_stats: null argument");
  cudaStream_t st = pick_stream(s, stream);
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  if (s->p.model == GS_MODEL_MART) return f64 ? mart_stats<double>(s, out, st) : mart_stats<float>(s, out, st);
  if (s->p.model == GS_MODEL_PRECIPITATE)
    return f64 ? precip_stats<double>(s, out, st) : precip_stats<float>(s, out, st);
  memset(out, 0, sizeof(*out));
  out->step = s->step;
  return GS_OK;
}

extern "C" int gs_sim_device_field(gs_sim* s, const char* name, void** dptr, size_t* bytes) {
  if (!s || !name || !dptr) return gs_set_error(GS_EINVAL, "gs_sim_device_field: null argument");
  const std::string nm(name);
  const size_t fb = (size_t)s->N * elt(s);
  if (nm == "eta") {
    *dptr = s->eta[s->cur];
    if (bytes) *bytes = fb * s->p.nvariants;
    return GS_OK;
  }
  if (nm == "spectrum") {
    *dptr = s->spec;
    if (bytes) *bytes = fb * s->p.nvariants;
    return GS_OK;
  }
  if (nm == "btable") {  // octant table of B(k); NULL when B is formed on the fly
    const bool on = s->btab_state == 1;
    *dptr = on ? s->btab : nullptr;
    if (bytes) *bytes = on ? s->btab_bytes : 0;
    return GS_OK;
  }
  return gs_set_error(GS_EINVAL, "unknown device field '%s'", name);
}

extern "C" int64_t gs_sim_launch_count(const gs_sim* s) { return s ? s->launches : 0; }

extern "C" int gs_sim_use_graph(gs_sim* s, int on) {
  if (!s) return gs_set_error(GS_EINVAL, "null sim");
  s->use_graph = on;
  if (!on) sim_graph_reset(s);
  return GS_OK;
}

// instances used by the comparator translation unit
template void build_elastic<float>(const gs_sim*, int, double, ElasticConst<float>&);
template void build_elastic<double>(const gs_sim*, int, double, ElasticConst<double>&);
template void build_mart<float>(const gs_sim*, MartConst<float>&);
template void build_mart<double>(const gs_sim*, MartConst<double>&);

extern "C" int gs_sim_profile_step(gs_sim* s, void* stream, double* pass_ms, int max_pass, int* npass) {
  if (!s || !pass_ms || !npass) return gs_set_error(GS_EINVAL, "gs_sim_profile_step: null argument");
  cudaStream_t st = pick_stream(s, stream);
  for (int i = 0; i < gs_sim::kMaxMarks; ++i)
    if (!s->marks[i]) GS_CU(cudaEventCreate(&s->marks[i]), "event create");
  s->nmarks = 0;
  s->profiling = true;
  gs_mark(s, st);
  int rc = gs_sim_step(s, 1, stream);
  s->profiling = false;
  if (rc != GS_OK) return rc;
  GS_CU(cudaEventSynchronize(s->marks[s->nmarks - 1]), "event sync");
  const int n = s->nmarks - 1 < max_pass ? s->nmarks - 1 : max_pass;
  for (int i = 0; i < n; ++i) {
    float ms = 0;
    GS_CU(cudaEventElapsedTime(&ms, s->marks[i], s->marks[i + 1]), "elapsed");
    pass_ms[i] = ms;
  }
  *npass = n;
  return GS_OK;
}

extern "C" const char* gs_sim_pass_name(const gs_sim* s, int i) {
  if (!s || i < 0 || i + 1 >= s->nmarks) return nullptr;
  return s->mark_names[i + 1];
}

// ---------------------------------------------------------------------------
// batched ensembles: many independent martensite simulations, one launch per
// pass per shape group, optionally replayed as a captured CUDA graph
// ---------------------------------------------------------------------------
struct gs_batch {
  std::vector<gs_sim*> groups;
  std::vector<std::pair<int, int>> where;  // sim -> (group, slot)
  cudaStream_t stream = nullptr;
  int use_graph = 0;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t exec_stream = nullptr;
  std::vector<int> exec_cur;  // which field of each pair the graph reads first
  int64_t launches = 0;
  // the groups are independent: each steps on a branch stream of its own,
  // forked from and joined to the caller's stream by events (in a captured
  // graph: parallel branches), so one group's passes fill the GPU while
  // another's run their last waves
  bool concurrent = true;
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> joined;
  cudaEvent_t forked = nullptr;
};

// ratio r with b = r a for every eigenstrain component (-1 if not proportional)
static double strain_ratio(const gs_params& a, const gs_params& b) {
  double na = 0, dot = 0;
  for (int v = 0; v < a.nvariants; ++v)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        na += a.eigenstrain[v][i][j] * a.eigenstrain[v][i][j];
        dot += a.eigenstrain[v][i][j] * b.eigenstrain[v][i][j];
      }
  if (na == 0) return -1;
  const double r = dot / na;
  for (int v = 0; v < a.nvariants; ++v)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        if (std::fabs(b.eigenstrain[v][i][j] - r * a.eigenstrain[v][i][j]) > 1e-12 * (1 + std::fabs(r)))
          return -1;
  return r;
}

static bool same_group(const gs_params& a, const gs_params& b) {
  return a.model == b.model && a.mode == b.mode && a.dtype == b.dtype && a.nvariants == b.nvariants &&
         a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.dx == b.dx && a.dy == b.dy && a.dz == b.dz &&
         a.dt == b.dt && memcmp(a.cijkl, b.cijkl, sizeof(a.cijkl)) == 0 && strain_ratio(a, b) > 0;
}

template <typename T> static int batch_upload_consts(gs_sim* g) {
  std::vector<MartConst<T>> mcs(g->nb);
  std::vector<T> sc(g->nb);
  for (int k = 0; k < g->nb; ++k) {
    build_mart_p<T>(g, g->bp[k], g->bstep[k], mcs[k]);
    const double r = strain_ratio(g->bp[0], g->bp[k]);
    sc[k] = (T)(r * r);  // B is bilinear in the eigenstrains
  }
  GS_CU(cudaMemcpy(g->d_mcs, mcs.data(), sizeof(MartConst<T>) * g->nb, cudaMemcpyHostToDevice), "upload constants");
  GS_CU(cudaMemcpy(g->d_simscale, sc.data(), sizeof(T) * g->nb, cudaMemcpyHostToDevice), "upload scales");
  // a pageable copy may return before its DMA lands, and the steps run on
  // non-blocking streams: wait for it
  GS_CU(cudaDeviceSynchronize(), "upload constants sync");
  return GS_OK;
}

template <typename T> static int batch_group_step(gs_sim* g, cudaStream_t st) {
  const int V = g->p.nvariants, VT = V * g->nb;
  const long long rows = (long long)g->n0 * g->n1;
  T* in = reinterpret_cast<T*>(g->eta[g->cur]);
  T* out = reinterpret_cast<T*>(g->eta[g->cur ^ 1]);
  ZfwdArgs<T> za;
  memset(&za, 0, sizeof(za));
  za.src0 = in;
  za.fstride = g->N;
  za.square0 = 1;
  za.dst = reinterpret_cast<cplx<T>*>(g->spec);
  za.rows_per_field = rows;
  za.nrows = rows * VT;
  za.tw_h = twp<T>(g, 1);
  za.tw_n2 = twp<T>(g, 0);
  const bool z_ready = g->spec_ready && g->spec_cur == g->cur;
  g->spec_ready = false;
  if (!z_ready) {
    GS_CU(launch_zfwd<T>(za, g->h, st, g->sched.z_lines), "batch z forward");
    g->launches += 1;
  }
  YArgs<T> ya;
  ya.spec = reinterpret_cast<cplx<T>*>(g->spec);
  ya.n0 = g->n0;
  ya.n1 = g->n1;
  ya.h = g->h;
  ya.tw = twp<T>(g, 2);
  GS_CU(launch_ypass<T>(ya, g->n1, VT, -1, st, g->sched.y_cols, g->sched.y_radix), "batch y forward");
  XArgs<T> xa;
  memset(&xa, 0, sizeof(xa));
  xa.in = reinterpret_cast<cplx<T>*>(g->spec);
  xa.out = reinterpret_cast<cplx<T>*>(g->spec);
  xa.n0 = g->n0;
  xa.n1 = g->n1;
  xa.n2 = g->n2;
  xa.h = g->h;
  xa.F = V;
  xa.G = V;
  xa.nsim = g->nb;
  xa.simscale = reinterpret_cast<const T*>(g->d_simscale);
  xa.tw = twp<T>(g, 3);
  build_elastic<T>(g, 0, 1.0 / (double)g->N, xa.ec);
  if (g->btab_state == 1) set_btab<T>(g, xa);
  xa.tz_req = g->sched.x_cols;
  GS_CU(launch_xcontract<T>(xa, st), "batch x pass");
  GS_CU(launch_ypass<T>(ya, g->n1, VT, 1, st, g->sched.y_cols, g->sched.y_radix), "batch y inverse");
  MartArgs<T> ma;
  fill_mart_args<T>(g, ma, in, out);
  ma.mcs = reinterpret_cast<MartConst<T>*>(g->d_mcs);
  if (g->fuse) ma.spec_next = reinterpret_cast<cplx<T>*>(g->spec);
  GS_CU(launch_mart_update<T>(ma, g->h, false, st, nullptr, g->nb), "batch update");
  if (g->trial) {  // the state (fields, counters) is left as it was
    g->spec_ready = g->fuse;
    g->spec_cur = g->cur;
    return GS_OK;
  }
  GS_CU(launch_bump_step<T>(reinterpret_cast<MartConst<T>*>(g->d_mcs), g->nb, st), "batch step counter");
  g->launches += 3 + (g->n1 > 1 ? 2 : 0);
  g->cur ^= 1;
  g->step += 1;
  for (auto& k : g->bstep) k += 1;
  g->spec_ready = g->fuse;
  g->spec_cur = g->cur;
  return GS_OK;
}

static int batch_step_once(gs_batch* b, cudaStream_t st) {
  const size_t ng = b->groups.size();
  if (!b->concurrent || ng < 2) {
    for (gs_sim* g : b->groups) {
      int rc = g->p.dtype == GS_DTYPE_F64 ? batch_group_step<double>(g, st) : batch_group_step<float>(g, st);
      if (rc != GS_OK) return rc;
    }
    return GS_OK;
  }
  if (b->branch.size() != ng) {  // created on the first direct step, never during a capture
    for (size_t k = b->branch.size(); k < ng; ++k) {
      cudaStream_t bs;
      cudaEvent_t ev;
      GS_CU(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking), "branch stream");
      GS_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "branch event");
      b->branch.push_back(bs);
      b->joined.push_back(ev);
    }
    if (!b->forked) GS_CU(cudaEventCreateWithFlags(&b->forked, cudaEventDisableTiming), "fork event");
  }
  GS_CU(cudaEventRecord(b->forked, st), "fork");
  for (size_t k = 0; k < ng; ++k) {
    gs_sim* g = b->groups[k];
    GS_CU(cudaStreamWaitEvent(b->branch[k], b->forked, 0), "branch wait");
    int rc = g->p.dtype == GS_DTYPE_F64 ? batch_group_step<double>(g, b->branch[k])
                                        : batch_group_step<float>(g, b->branch[k]);
    if (rc != GS_OK) return rc;
    GS_CU(cudaEventRecord(b->joined[k], b->branch[k]), "branch done");
  }
  for (size_t k = 0; k < ng; ++k) GS_CU(cudaStreamWaitEvent(st, b->joined[k], 0), "join");
  return GS_OK;
}

extern "C" int gs_batch_create(const gs_params* params, int nsims, gs_batch** out) {
  if (!params || !out || nsims < 1) return gs_set_error(GS_EINVAL, "gs_batch_create: bad arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return gs_set_error(GS_ENODEV, "no CUDA device visible");
  }
  gs_batch* b = new gs_batch();
  auto fail = [&](int rc) {
    gs_batch_destroy(b);
    return rc;
  };
  for (int i = 0; i < nsims; ++i) {
    const gs_params& p = params[i];
    if (p.model != GS_MODEL_MART) return fail(gs_set_error(GS_ENOTSUP, "batches hold martensite simulations"));
    if (p.nvariants < 1 || p.nvariants > GS_MAX_V) return fail(gs_set_error(GS_EINVAL, "sim %d: nvariants", i));
    int gi = -1;
    for (size_t k = 0; k < b->groups.size(); ++k)
      if (same_group(b->groups[k]->bp[0], p)) gi = (int)k;
    if (gi < 0) {
      gs_sim* g = new gs_sim();
      g->p = p;
      g->nb = 0;
      int rc = canonicalize(g);
      if (rc != GS_OK) {
        delete g;
        return fail(rc);
      }
      b->groups.push_back(g);
      gi = (int)b->groups.size() - 1;
    }
    gs_sim* g = b->groups[gi];
    b->where.push_back({gi, g->nb});
    g->bp.push_back(p);
    g->bstep.push_back(0);
    g->nb += 1;
  }
  if (gs_cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream") != GS_OK)
    return fail(GS_ECUDA);
  for (gs_sim* g : b->groups) {
    const size_t fb = (size_t)g->N * elt(g) * g->p.nvariants * g->nb;
    int rc;
    if ((rc = dalloc(&g->eta[0], fb, "batch eta")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&g->eta[1], fb, "batch eta pair")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&g->spec, fb, "batch spectrum")) != GS_OK) return fail(rc);
    const size_t mcb = g->p.dtype == GS_DTYPE_F64 ? sizeof(MartConst<double>) : sizeof(MartConst<float>);
    if ((rc = dalloc(&g->d_mcs, mcb * g->nb, "batch constants")) != GS_OK) return fail(rc);
    if ((rc = dalloc(&g->d_simscale, elt(g) * g->nb, "batch scales")) != GS_OK) return fail(rc);
    rc = g->p.dtype == GS_DTYPE_F64 ? build_twiddles<double>(g) : build_twiddles<float>(g);
    if (rc != GS_OK) return fail(rc);
    rc = g->p.dtype == GS_DTYPE_F64 ? batch_upload_consts<double>(g) : batch_upload_consts<float>(g);
    if (rc != GS_OK) return fail(rc);
    g->partials_cap = (size_t)g->n0 * g->n1 + 148 * 16 + 1;
    if ((rc = gs_cuda_check(cudaMalloc(&g->partials, g->partials_cap * ACC_N * sizeof(double)), "partials")) != GS_OK)
      return fail(rc);
    if ((rc = gs_cuda_check(cudaMalloc(&g->red, 64 * sizeof(double)), "reduce out")) != GS_OK) return fail(rc);
    if ((rc = ensure_btab(g, b->stream)) != GS_OK) return fail(rc);
    g->own_stream = nullptr;
  }
  *out = b;
  return GS_OK;
}

extern "C" int gs_batch_destroy(gs_batch* b) {
  if (!b) return GS_OK;
  cudaDeviceSynchronize();
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (gs_sim* g : b->groups) {
    free_sim(g);  // frees the per-sim constants too
  }
  for (cudaStream_t bs : b->branch) cudaStreamDestroy(bs);
  for (cudaEvent_t ev : b->joined) cudaEventDestroy(ev);
  if (b->forked) cudaEventDestroy(b->forked);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return GS_OK;
}

extern "C" int gs_batch_groups(const gs_batch* b) { return b ? (int)b->groups.size() : 0; }

extern "C" int gs_batch_set_concurrent(gs_batch* b, int on) {
  if (!b) return gs_set_error(GS_EINVAL, "gs_batch_set_concurrent: null handle");
  if (b->concurrent != (on != 0) && b->exec) {  // the captured graph has the other shape
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  b->concurrent = on != 0;
  return GS_OK;
}
extern "C" int64_t gs_batch_launch_count(const gs_batch* b) { return b ? b->launches : 0; }

extern "C" int gs_batch_use_graph(gs_batch* b, int on) {
  if (!b) return gs_set_error(GS_EINVAL, "null batch");
  b->use_graph = on;
  return GS_OK;
}

static int batch_slot(gs_batch* b, int sim, gs_sim** g, int* slot) {
  if (!b || sim < 0 || sim >= (int)b->where.size()) return gs_set_error(GS_EINVAL, "sim index %d", sim);
  *g = b->groups[b->where[sim].first];
  *slot = b->where[sim].second;
  return GS_OK;
}

extern "C" int gs_batch_set_field(gs_batch* b, int sim, const char* name, const void* host, size_t count, int dtype) {
  gs_sim* g;
  int slot;
  GS_TRY(batch_slot(b, sim, &g, &slot));
  if (!name || !host || std::string(name) != "eta") return gs_set_error(GS_EINVAL, "batches take the field eta");
  const size_t n = (size_t)g->N * g->p.nvariants;
  if (count != n) return gs_set_error(GS_EINVAL, "eta: %zu values, expected %zu", count, n);
  GS_CU(cudaStreamSynchronize(b->stream), "sync");
  char* dst = static_cast<char*>(g->eta[g->cur]) + (size_t)slot * n * elt(g);
  g->spec_ready = false;  // the fused spectra no longer match the field
  if (b->exec) {          // a captured step starts from fused spectra
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  return upload(g, dst, host, count, dtype);
}

extern "C" int gs_batch_get_field(gs_batch* b, int sim, const char* name, void* host, size_t count, int dtype) {
  gs_sim* g;
  int slot;
  GS_TRY(batch_slot(b, sim, &g, &slot));
  if (!name || !host || std::string(name) != "eta") return gs_set_error(GS_EINVAL, "batches hold the field eta");
  const size_t n = (size_t)g->N * g->p.nvariants;
  if (count != n) return gs_set_error(GS_EINVAL, "eta: %zu values, expected %zu", count, n);
  GS_CU(cudaStreamSynchronize(b->stream), "sync");
  const char* src = static_cast<const char*>(g->eta[g->cur]) + (size_t)slot * n * elt(g);
  return download(g, src, host, count, dtype);
}

static int gs_batch_step_body(gs_batch* b, int nsteps, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_batch_step(gs_batch* b, int nsteps, void* stream) {
  return bc_after(gs_batch_step_body(b, nsteps, stream), static_cast<cudaStream_t>(stream));
}

static int gs_batch_step_body(gs_batch* b, int nsteps, void* stream) {
  if (!b || nsteps < 0) return gs_set_error(GS_EINVAL, "gs_batch_step: bad arguments");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  for (gs_sim* g : b->groups) g->launches = 0;
  int done = 0;
  if (b->use_graph && nsteps >= 2) {
    // the first steps run directly (kernel attributes are set outside any
    // capture); then a graph of two steps (the field pair swaps back) replays
    bool ready = true;  // the captured steps start from fused spectra
    for (gs_sim* g : b->groups) ready = ready && (!g->fuse || (g->spec_ready && g->spec_cur == g->cur));
    if (!b->exec || b->exec_stream != st || !ready) {
      if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
      }
      GS_TRY(batch_step_once(b, st));
      GS_TRY(batch_step_once(b, st));
      done = 2;
      std::vector<int> cur;
      std::vector<int64_t> steps;
      std::vector<std::vector<int64_t>> bsteps;
      for (gs_sim* g : b->groups) {
        cur.push_back(g->cur);
        steps.push_back(g->step);
        bsteps.push_back(g->bstep);
      }
      cudaGraph_t graph;
      GS_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
      int rc = batch_step_once(b, st);
      if (rc == GS_OK) rc = batch_step_once(b, st);
      cudaError_t e = cudaStreamEndCapture(st, &graph);
      if (rc != GS_OK) return rc;
      GS_CU(e, "end capture");
      GS_CU(cudaGraphInstantiate(&b->exec, graph, 0), "instantiate graph");
      cudaGraphDestroy(graph);
      b->exec_stream = st;
      for (size_t k = 0; k < b->groups.size(); ++k) {  // the capture did not run
        b->groups[k]->cur = cur[k];
        b->groups[k]->step = steps[k];
        b->groups[k]->bstep = bsteps[k];
      }
      b->exec_cur = cur;
    }
    // the graph's buffers are fixed: after an odd number of direct steps the
    // field pairs are swapped, and one more direct step swaps them back
    if (nsteps - done >= 1 && !b->groups.empty() && b->groups[0]->cur != b->exec_cur[0]) {
      GS_TRY(batch_step_once(b, st));
      ++done;
    }
    while (nsteps - done >= 2) {
      GS_CU(cudaGraphLaunch(b->exec, st), "graph launch");
      for (gs_sim* g : b->groups) {
        g->step += 2;
        for (auto& k : g->bstep) k += 2;
      }
      done += 2;
    }
  }
  for (; done < nsteps; ++done) GS_TRY(batch_step_once(b, st));
  b->launches = 0;
  for (gs_sim* g : b->groups) b->launches += g->launches;
  return GS_OK;
}

extern "C" int gs_batch_stats(gs_batch* b, int sim, gs_stats* out, void* stream) {
  gs_sim* g;
  int slot;
  GS_TRY(batch_slot(b, sim, &g, &slot));
  if (!out) return gs_set_error(GS_EINVAL, "null stats");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  // a single-simulation view of slot `slot`
  gs_sim view = *g;
  view.p = g->bp[slot];
  view.nb = 1;
  view.btab_state = -2;  // the group's table holds the group's B, not this sim's
  view.step = g->bstep[slot];
  const size_t n = (size_t)g->N * g->p.nvariants * elt(g);
  view.eta[view.cur] = static_cast<char*>(g->eta[g->cur]) + slot * n;
  int rc = g->p.dtype == GS_DTYPE_F64 ? mart_stats<double>(&view, out, st) : mart_stats<float>(&view, out, st);
  return rc;  // the view shares g's buffers: nothing to free
}

// ---------------------------------------------------------------------------
// a martensite step that allocates nothing
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory at the moment they want a step:
// a host that hands every byte of the GPU to its own pool allocator up front,
// a real-time loop that must not touch the allocator, or a plugin living in a
// process whose device memory is owned by someone else.  gs_mart_step_noalloc
// serves them: the caller passes the field buffers, and the one piece of
// scratch the step needs (the packed spectra and the twiddle tables) lives in
// this file-scope array, which every GPU that loads the library keeps until
// the process exits.  The array's name means a host stand-in in host code;
// its device address is taken once per device with cudaGetSymbolAddress.
static constexpr size_t kNoallocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

static constexpr int kNoallocMaxDev = 64;
static void* g_noalloc_ptr[kNoallocMaxDev] = {};
static std::mutex g_noalloc_mu;

static int noalloc_scratch(void** out) {
  int dev = 0;
  GS_CU(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoallocMaxDev) return gs_set_error(GS_ENODEV, "device %d beyond %d", dev, kNoallocMaxDev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    GS_CU(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress of the no-allocation scratch");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return GS_OK;
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

static int check_device_buffer(const void* p, int dev, const char* what) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: %s is not a CUDA pointer", what);
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: %s is not device memory", what);
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: %s lives on device %d, the current device is %d", what,
                        a.device, dev);
  return GS_OK;
}

template <typename T> static int noalloc_step(gs_sim& s, const void* in, void* out, cudaStream_t st) {
  // twiddle tables as build_twiddles makes them, written into the scratch
  const int lens[4] = {s.n2, s.h, s.n1, s.n0};
  constexpr int kMaxTw = 512 + 256 + 256 + 256;
  cplx<T> host[kMaxTw];
  size_t total = 0;
  for (int i = 0; i < 4; ++i) {
    s.tw_off[i] = total;
    total += (size_t)lens[i];
  }
  if (total > (size_t)kMaxTw) return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: twiddle table too long");
  for (int i = 0; i < 4; ++i)
    for (int m = 0; m < lens[i]; ++m) {
      const double a = 2.0 * M_PI * (double)m / (double)lens[i];
      host[s.tw_off[i] + m] = mk2((T)std::cos(a), (T)-std::sin(a));
    }
  GS_CU(cudaMemcpyAsync(s.tw, host, total * sizeof(cplx<T>), cudaMemcpyHostToDevice, st), "upload twiddles");
  s.eta[0] = const_cast<void*>(in);
  s.eta[1] = out;
  s.cur = 0;
  int rc = mart_step<T>(&s, st);
  // return only once the step has finished, so that calls made one after
  // another from one host thread never share the scratch on the GPU
  const cudaError_t e = cudaStreamSynchronize(st);
  if (rc != GS_OK) return rc;
  return gs_cuda_check(e, "gs_mart_step_noalloc");
}

extern "C" size_t gs_mart_step_noalloc_max_bytes(void) { return kNoallocScratchBytes; }

static int gs_mart_step_noalloc_body(const gs_params* p, const void* eta_in, void* eta_out, int64_t step, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_mart_step_noalloc(const gs_params* p, const void* eta_in, void* eta_out, int64_t step, void* stream) {
  return bc_after(gs_mart_step_noalloc_body(p, eta_in, eta_out, step, stream), static_cast<cudaStream_t>(stream));
}

static int gs_mart_step_noalloc_body(const gs_params* p, const void* eta_in, void* eta_out, int64_t step,
                                    void* stream) {
  if (!p || !eta_in || !eta_out) return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: null argument");
  if (p->model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: model must be martensite");
  if (p->nvariants < 1 || p->nvariants > GS_MAX_V)
    return gs_set_error(GS_EINVAL, "nvariants %d outside 1..%d", p->nvariants, GS_MAX_V);
  if (p->dtype != GS_DTYPE_F32 && p->dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", p->dtype);
  if (step < 0) return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: step %lld", (long long)step);
  gs_sim s;  // a view: every pointer below is the caller's or the static scratch
  s.p = *p;
  s.btab_state = -1;  // B formed on the fly: no table to allocate
  s.fuse = false;      // nothing carries the spectrum to a next call
  GS_TRY(canonicalize(&s));
  const size_t eb = elt(&s);
  const size_t fields = (size_t)s.N * p->nvariants * eb;
  const size_t tw_bytes = (size_t)(s.n2 + s.h + s.n1 + s.n0) * 2 * eb;
  const size_t need = align256(fields) + align256(tw_bytes);
  if (need > kNoallocScratchBytes)
    return gs_set_error(GS_EINVAL,
                        "gs_mart_step_noalloc: grid %dx%dx%d with %d variants needs %zu bytes of scratch; the "
                        "static scratch holds %zu",
                        p->nx, p->ny, p->nz, p->nvariants, need, kNoallocScratchBytes);
  // the kernels move fields in 16-byte vectors (float4 / double2)
  if ((reinterpret_cast<uintptr_t>(eta_in) | reinterpret_cast<uintptr_t>(eta_out)) & 15u)
    return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: eta_in and eta_out must be 16-byte aligned");
  const char* a = static_cast<const char*>(eta_in);
  const char* b = static_cast<const char*>(eta_out);
  if (a < b + fields && b < a + fields)
    return gs_set_error(GS_EINVAL, "gs_mart_step_noalloc: eta_in and eta_out overlap");
  int dev = 0;
  GS_CU(cudaGetDevice(&dev), "cudaGetDevice");
  GS_TRY(check_device_buffer(eta_in, dev, "eta_in"));
  GS_TRY(check_device_buffer(eta_out, dev, "eta_out"));
  void* scratch = nullptr;
  GS_TRY(noalloc_scratch(&scratch));
  char* base = static_cast<char*>(scratch);
  s.spec = base;
  s.tw = base + align256(fields);
  s.step = step;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dtype == GS_DTYPE_F64 ? noalloc_step<double>(s, eta_in, eta_out, st)
                                  : noalloc_step<float>(s, eta_in, eta_out, st);
}

// ---------------------------------------------------------------------------
// adjoint of the martensite run (checkpoint every K steps, recompute)
// ---------------------------------------------------------------------------
// Forward: the trajectory eta_0 .. eta_T with eta_{jK} kept as checkpoints
// and the last segment's states and elastic potentials kept whole.
// Backward, segment by segment from the last: recompute the segment's states
// eta_n and potentials R_n from its checkpoint (the same passes as the
// forward step, with R written out by the update), then per step n the chain
// Q = B * (eta_n lam) and the transposed update (gs_adjoint.cuh), whose
// per-step FP64 sums give the parameter gradients.
struct gs_adjoint {
  gs_sim* s = nullptr;
  int nsteps = 0, K = 0, nseg = 0;
  std::vector<void*> ckpt, seg_eta, seg_R;
  void* lam[2] = {nullptr, nullptr};
  void* target = nullptr;
  void* etaT = nullptr;
  void* RT = nullptr;
  double* gsum = nullptr;  // [nsteps][ADJ_N]
  int seg_valid = -1;      // segment held in seg_eta / seg_R
  const void* z_ready = nullptr;  // field whose z spectra the last update left in spec
  // the forward steps and the reverse sweep replayed as CUDA graphs after a
  // first direct run (gs_adjoint_use_graph)
  bool use_graph = true, warm = false;
  cudaGraphExec_t gfwd = nullptr, gbwd = nullptr;
  cudaStream_t gstream = nullptr;
  int64_t nl_fwd = 0, nl_bwd = 0;  // kernel launches inside each graph
  int ret_fwd = 0, ret_bwd = 0;     // what each body returned (kept for replays)
  bool forward_done = false, have_target = false;
  double lam_el = 0, e_target = 0, e_el_T = 0;
  size_t bytes = 0;
};

static void adj_graph_reset(gs_adjoint* a) {
  if (a->gfwd) cudaGraphExecDestroy(a->gfwd);
  if (a->gbwd) cudaGraphExecDestroy(a->gbwd);
  a->gfwd = a->gbwd = nullptr;
}

static void free_adjoint(gs_adjoint* a) {
  if (!a) return;
  adj_graph_reset(a);
  auto f = [](void* p) {
    if (p) cudaFree(p);
  };
  for (void* p : a->ckpt) f(p);
  for (void* p : a->seg_eta) f(p);
  for (void* p : a->seg_R) f(p);
  f(a->lam[0]);
  f(a->lam[1]);
  f(a->target);
  f(a->etaT);
  f(a->RT);
  f(a->gsum);
  if (a->s) {
    cudaDeviceSynchronize();
    free_sim(a->s);
  }
  delete a;
}

static int adj_check_params(const gs_params* p) {
  if (p->model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "adjoint: martensite model only");
  if (p->mode != GS_MODE_BASELINE) return gs_set_error(GS_ENOTSUP, "adjoint: baseline mode only");
  return GS_OK;
}

extern "C" int gs_adjoint_create(const gs_params* p, int nsteps, int checkpoint_every, gs_adjoint** out) {
  if (!p || !out) return gs_set_error(GS_EINVAL, "gs_adjoint_create: null argument");
  *out = nullptr;
  GS_TRY(adj_check_params(p));
  if (nsteps < 1) return gs_set_error(GS_EINVAL, "adjoint: nsteps %d", nsteps);
  if (checkpoint_every < 1) return gs_set_error(GS_EINVAL, "adjoint: checkpoint_every %d", checkpoint_every);
  gs_adjoint* a = new gs_adjoint();
  int rc = gs_sim_create(p, &a->s);
  if (rc != GS_OK) {
    delete a;
    return rc;
  }
  a->nsteps = nsteps;
  a->K = checkpoint_every < nsteps ? checkpoint_every : nsteps;
  a->nseg = (nsteps + a->K - 1) / a->K;
  const size_t fb = (size_t)a->s->N * p->nvariants * elt(a->s);
  auto fail = [&](int code) {
    free_adjoint(a);
    return code;
  };
  auto get = [&](void** q, size_t b, const char* what) {
    const int r = dalloc(q, b, what);
    if (r == GS_OK) a->bytes += b;
    return r;
  };
  a->ckpt.assign(a->nseg, nullptr);
  a->seg_eta.assign(a->K, nullptr);
  a->seg_R.assign(a->K, nullptr);
  for (int j = 0; j < a->nseg; ++j)
    if ((rc = get(&a->ckpt[j], fb, "adjoint checkpoint")) != GS_OK) return fail(rc);
  for (int i = 0; i < a->K; ++i) {
    if (i > 0 && (rc = get(&a->seg_eta[i], fb, "adjoint segment")) != GS_OK) return fail(rc);
    if ((rc = get(&a->seg_R[i], fb, "adjoint potentials")) != GS_OK) return fail(rc);
  }
  if ((rc = get(&a->lam[0], fb, "adjoint lambda")) != GS_OK) return fail(rc);
  if ((rc = get(&a->lam[1], fb, "adjoint lambda")) != GS_OK) return fail(rc);
  if ((rc = get(&a->etaT, fb, "final state")) != GS_OK) return fail(rc);
  if ((rc = get(&a->RT, fb, "final potentials")) != GS_OK) return fail(rc);
  if ((rc = get(reinterpret_cast<void**>(&a->gsum), (size_t)nsteps * ADJ_N * sizeof(double), "adjoint sums")) !=
      GS_OK)
    return fail(rc);
  // the handle's own simulation buffers
  a->bytes += fb * 3 + a->s->partials_cap * ACC_N * sizeof(double);
  *out = a;
  return GS_OK;
}

extern "C" int gs_adjoint_destroy(gs_adjoint* a) {
  free_adjoint(a);
  return GS_OK;
}

extern "C" size_t gs_adjoint_device_bytes(const gs_adjoint* a) { return a ? a->bytes : 0; }

extern "C" int gs_adjoint_set_params(gs_adjoint* a, const gs_params* p) {
  if (!a || !p) return gs_set_error(GS_EINVAL, "gs_adjoint_set_params: null argument");
  GS_TRY(adj_check_params(p));
  const gs_params& o = a->s->p;
  if (p->nx != o.nx || p->ny != o.ny || p->nz != o.nz || p->nvariants != o.nvariants || p->dtype != o.dtype)
    return gs_set_error(GS_EINVAL, "adjoint: grid, variant count and dtype are fixed at creation");
  a->s->p = *p;
  a->forward_done = false;
  adj_graph_reset(a);  // the captured launches hold the old constants
  a->s->btab_state = 0;
  return ensure_btab(a->s, a->s->own_stream);
}

extern "C" int gs_adjoint_set_loss(gs_adjoint* a, const void* target, int dtype, double lam_el, double e_target) {
  if (!a || !target) return gs_set_error(GS_EINVAL, "gs_adjoint_set_loss: null argument");
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", dtype);
  if (!a->target) {
    const size_t fb = (size_t)a->s->N * a->s->p.nvariants * elt(a->s);
    GS_TRY(dalloc(&a->target, fb, "adjoint target"));
    a->bytes += fb;
  }
  GS_TRY(upload(a->s, a->target, target, (size_t)a->s->N * a->s->p.nvariants, dtype));
  a->lam_el = lam_el;
  a->e_target = e_target;
  a->have_target = true;
  return GS_OK;
}

// location of eta_n during the forward run or a recompute of seg_valid
static void* adj_eta(gs_adjoint* a, int n) {
  if (n == a->nsteps) return a->etaT;
  const int j = n / a->K, i = n % a->K;
  if (i == 0) return a->ckpt[j];
  if (j == a->seg_valid) return a->seg_eta[i];
  return a->s->eta[n & 1];
}

// one forward step in -> out; the update also leaves the z spectra of out^2
// in the spectrum buffer, which the next step from out takes as its z forward
template <typename T>
static int adj_fwd_step(gs_adjoint* a, const void* in, void* out, void* r_out, int n, cudaStream_t st) {
  gs_sim* s = a->s;
  s->step = n;
  GS_TRY(elastic_chain<T>(s, reinterpret_cast<const T*>(in), st, a->z_ready == in));
  MartArgs<T> ma;
  fill_mart_args<T>(s, ma, reinterpret_cast<const T*>(in), reinterpret_cast<T*>(out));
  ma.r_out = reinterpret_cast<T*>(r_out);
  ma.spec_next = reinterpret_cast<cplx<T>*>(s->spec);
  GS_CU(launch_mart_update<T>(ma, s->h, false, st, nullptr), "update pass");
  s->launches += 1;
  a->z_ready = out;
  return GS_OK;
}

// The reverse sweep from lam[0] (the seed) to dJ/deta_0, segment by segment;
// returns the index of the lam buffer that holds dJ/deta_0.  Its launches
// depend only on the handle's sizes and parameters, so it can be captured.
template <typename T> static int adj_sweep(gs_adjoint* a, cudaStream_t st) {
  gs_sim* s = a->s;
  const int V = s->p.nvariants;
  const long long N = s->N;
  int c = 0;
  const T* src[GS_MAXF];
  const T* mul[GS_MAXF];
  int sq[GS_MAXF];
  for (int j = a->nseg - 1; j >= 0; --j) {
    const int n0 = j * a->K, len = (j == a->nseg - 1) ? a->nsteps - n0 : a->K;
    if (a->seg_valid != j) {  // recompute eta_n and R_n of the segment
      a->seg_valid = j;
      a->z_ready = nullptr;  // the backward chains used the spectrum buffer
      for (int i = 0; i < len; ++i) {
        void* in = i == 0 ? a->ckpt[j] : a->seg_eta[i];
        void* out = i + 1 < len ? a->seg_eta[i + 1] : s->eta[0];
        GS_TRY(adj_fwd_step<T>(a, in, out, a->seg_R[i], n0 + i, st));
      }
    }
    for (int i = len - 1; i >= 0; --i) {
      const int n = n0 + i;
      const T* eta = reinterpret_cast<const T*>(i == 0 ? a->ckpt[j] : a->seg_eta[i]);
      const T* lin = reinterpret_cast<const T*>(a->lam[c]);
      for (int f = 0; f < V; ++f) {
        src[f] = eta + (long long)f * N;
        mul[f] = lin + (long long)f * N;
        sq[f] = 0;
      }
      GS_TRY(elastic_chain_g<T>(s, src, sq, V, 0, 1.0 / (double)N, s->spec, V, st, mul));
      AdjArgs<T> aa;
      memset(&aa, 0, sizeof(aa));
      aa.spec = reinterpret_cast<const cplx<T>*>(s->spec);
      aa.eta = eta;
      aa.lam_in = lin;
      aa.lam_out = reinterpret_cast<T*>(a->lam[c ^ 1]);
      aa.R = reinterpret_cast<const T*>(a->seg_R[i]);
      aa.n0 = s->n0;
      aa.n1 = s->n1;
      aa.n2 = s->n2;
      aa.nrows = (long long)s->n0 * s->n1;
      aa.tw_h = twp<T>(s, 1);
      aa.tw_n2 = twp<T>(s, 0);
      s->step = n;
      build_mart<T>(s, aa.mc);
      aa.partials = s->partials;
      aa.fd_n1 = FastDiv((uint32_t)s->n1);
      aa.fd_upr = FastDiv((uint32_t)(s->n2 % 4 == 0 ? s->n2 / 4 : s->n2 / 2));
      aa.fd_v = FastDiv((uint32_t)V);
      int nbk = 0;
      GS_CU(launch_adj_update<T>(aa, s->h, st, &nbk), "adjoint update");
      GS_CU(launch_reduce(s->partials, nbk, ADJ_N, a->gsum + (size_t)n * ADJ_N, st), "adjoint reduce");
      s->launches += 2;
      c ^= 1;
    }
  }
  return c;
}

// The forward steps eta_0 -> eta_T of the run (checkpoints, last segment).
template <typename T> static int adj_steps(gs_adjoint* a, cudaStream_t st) {
  a->seg_valid = a->nseg - 1;
  a->z_ready = nullptr;
  for (int n = 0; n < a->nsteps; ++n) {
    void* r_out = n / a->K == a->nseg - 1 ? a->seg_R[n % a->K] : nullptr;
    GS_TRY(adj_fwd_step<T>(a, adj_eta(a, n), adj_eta(a, n + 1), r_out, n, st));
  }
  return GS_OK;
}

// Run body directly the first time (kernel attributes are set outside any
// capture), then capture it once as a CUDA graph and replay that graph.
// body's host-side effects are the same on every run, so replaying leaves
// the handle as a direct run would; *ret holds body's result from the last
// direct run or capture, which a replay repeats.
template <class F>
static int adj_graph(gs_adjoint* a, cudaGraphExec_t* ex, int* ret, int64_t* nlaunch, cudaStream_t st, F body,
                     bool allowed = true) {
  if (!a->use_graph || !a->warm || !allowed) {
    const int r = body();
    if (r < 0) return r;
    *ret = r;
    return GS_OK;
  }
  if (!*ex || a->gstream != st) {
    if (*ex) cudaGraphExecDestroy(*ex);
    *ex = nullptr;
    cudaGraph_t g;
    const int64_t l0 = a->s->launches;
    GS_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    const int r = body();
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (r < 0) return r;
    GS_CU(e, "end capture");
    GS_CU(cudaGraphInstantiate(ex, g, 0), "instantiate graph");
    cudaGraphDestroy(g);
    a->gstream = st;
    *ret = r;
    *nlaunch = a->s->launches - l0;
    a->s->launches = l0;
  }
  GS_CU(cudaGraphLaunch(*ex, st), "graph launch");
  a->s->launches += *nlaunch;
  return GS_OK;
}

template <typename T> static int adj_forward(gs_adjoint* a, cudaStream_t st) {
  gs_sim* s = a->s;
  GS_TRY(adj_graph(a, &a->gfwd, &a->ret_fwd, &a->nl_fwd, st, [&]() { return adj_steps<T>(a, st); }));
  a->seg_valid = a->nseg - 1;
  a->z_ready = a->etaT;
  // E_el and R at the final state
  GS_TRY(elastic_chain<T>(s, reinterpret_cast<const T*>(a->etaT), st, a->z_ready == a->etaT));
  a->z_ready = nullptr;
  MartArgs<T> ma;
  fill_mart_args<T>(s, ma, reinterpret_cast<const T*>(a->etaT), nullptr);
  ma.r_out = reinterpret_cast<T*>(a->RT);
  int nb = 0;
  GS_CU(launch_mart_update<T>(ma, s->h, true, st, &nb), "final statistics");
  GS_CU(launch_reduce(s->partials, nb, ACC_N, s->red, st), "reduce");
  double acc[ACC_N];
  GS_CU(cudaMemcpyAsync(acc, s->red, sizeof(acc), cudaMemcpyDeviceToHost, st), "stats D2H");
  GS_CU(cudaStreamSynchronize(st), "forward sync");
  a->e_el_T = acc[ACC_EEL] * s->p.dx * s->p.dy * s->p.dz;
  s->step = a->nsteps;
  a->forward_done = true;
  return GS_OK;
}

static int gs_adjoint_forward_body(gs_adjoint* a, const void* eta0, int dtype, void* eta_final, double* e_el_final,
                                   void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_adjoint_forward(gs_adjoint* a, const void* eta0, int dtype, void* eta_final, double* e_el_final,
                                  void* stream) {
  return bc_after(gs_adjoint_forward_body(a, eta0, dtype, eta_final, e_el_final, stream),
                  static_cast<cudaStream_t>(stream));
}

static int gs_adjoint_forward_body(gs_adjoint* a, const void* eta0, int dtype, void* eta_final, double* e_el_final,
                                  void* stream) {
  if (!a || !eta0) return gs_set_error(GS_EINVAL, "gs_adjoint_forward: null argument");
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", dtype);
  gs_sim* s = a->s;
  const size_t count = (size_t)s->N * s->p.nvariants;
  GS_TRY(upload(s, a->ckpt[0], eta0, count, dtype));
  cudaStream_t st = pick_stream(s, stream);
  s->launches = 0;
  GS_TRY(s->p.dtype == GS_DTYPE_F64 ? adj_forward<double>(a, st) : adj_forward<float>(a, st));
  if (e_el_final) *e_el_final = a->e_el_T;
  if (eta_final) GS_TRY(download(s, a->etaT, eta_final, count, dtype));
  return GS_OK;
}

template <typename T>
static int adj_backward(gs_adjoint* a, const void* seed_dev, double seed_e, double* loss, double* grads,
                        cudaStream_t st) {
  gs_sim* s = a->s;
  const gs_params& p = s->p;
  const int V = p.nvariants;
  const long long N = s->N;
  const double dV = p.dx * p.dy * p.dz;
  const double ce = seed_dev ? seed_e : 2.0 * a->lam_el * (a->e_el_T - a->e_target);
  AdjSeedArgs<T> sa;
  memset(&sa, 0, sizeof(sa));
  sa.eta = reinterpret_cast<const T*>(a->etaT);
  sa.R = reinterpret_cast<const T*>(a->RT);
  sa.target = seed_dev ? nullptr : reinterpret_cast<const T*>(a->target);
  sa.seed = reinterpret_cast<const T*>(seed_dev);
  sa.lam = reinterpret_cast<T*>(a->lam[0]);
  sa.n = N * V;
  sa.c = ce * p.weight_elastic * dV;
  sa.partials = s->partials;
  int nb = 0;
  GS_CU(launch_adj_seed<T>(sa, st, &nb), "adjoint seed");
  GS_CU(launch_reduce(s->partials, nb, 1, s->red, st), "reduce");
  double field = 0;
  GS_CU(cudaMemcpyAsync(&field, s->red, sizeof(double), cudaMemcpyDeviceToHost, st), "loss D2H");
  // the captured sweep starts with the last segment held (as after a forward run)
  const bool from_forward = a->seg_valid == a->nseg - 1;
  GS_TRY(adj_graph(a, &a->gbwd, &a->ret_bwd, &a->nl_bwd, st, [&]() { return adj_sweep<T>(a, st); }, from_forward));
  const int c = a->ret_bwd;
  a->seg_valid = 0;  // as the sweep leaves it
  std::vector<double> h((size_t)a->nsteps * ADJ_N);
  GS_CU(cudaMemcpyAsync(h.data(), a->gsum, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "sums D2H");
  GS_CU(cudaStreamSynchronize(st), "adjoint sync");
  // Neumaier sums over the steps
  double sum[ADJ_N], cmp[ADJ_N];
  for (int k = 0; k < ADJ_N; ++k) sum[k] = cmp[k] = 0;
  for (int n = 0; n < a->nsteps; ++n)
    for (int k = 0; k < ADJ_N; ++k) {
      const double x = h[(size_t)n * ADJ_N + k], t = sum[k] + x;
      cmp[k] += std::fabs(sum[k]) >= std::fabs(x) ? (sum[k] - t) + x : (x - t) + sum[k];
      sum[k] = t;
    }
  for (int k = 0; k < ADJ_N; ++k) sum[k] += cmp[k];
  const double dt = p.dt, L = p.mobility;
  grads[0] = dt * L * sum[ADJ_ETA_LAP];
  grads[1] = -dt * L * sum[ADJ_ETA_LAM];
  grads[2] = dt * L * sum[ADJ_ETA3_LAM];
  grads[3] = -dt * L * sum[ADJ_S2_ETA_LAM];
  grads[4] = -dt * L * sum[ADJ_AC_LAM];
  grads[5] = dt * sum[ADJ_S_LAM] + ce * 2.0 * a->e_el_T;
  if (loss) {
    loss[1] = seed_dev ? 0.0 : field;
    loss[2] = a->e_el_T;
    loss[0] = seed_dev ? 0.0 : field + a->lam_el * (a->e_el_T - a->e_target) * (a->e_el_T - a->e_target);
  }
  return c;  // index of the buffer holding dJ/deta_0
}

static int gs_adjoint_backward_body(gs_adjoint* a, const void* seed, int seed_dtype, double seed_e, double* loss,
                                    double* grads, void* grad_eta0, int grad_dtype, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_adjoint_backward(gs_adjoint* a, const void* seed, int seed_dtype, double seed_e, double* loss,
                                   double* grads, void* grad_eta0, int grad_dtype, void* stream) {
  return bc_after(gs_adjoint_backward_body(a, seed, seed_dtype, seed_e, loss, grads, grad_eta0, grad_dtype, stream),
                  static_cast<cudaStream_t>(stream));
}

static int gs_adjoint_backward_body(gs_adjoint* a, const void* seed, int seed_dtype, double seed_e, double* loss,
                                   double* grads, void* grad_eta0, int grad_dtype, void* stream) {
  if (!a || !grads) return gs_set_error(GS_EINVAL, "gs_adjoint_backward: null argument");
  if (!a->forward_done) return gs_set_error(GS_EINVAL, "gs_adjoint_backward: run gs_adjoint_forward first");
  if (!seed && !a->have_target) return gs_set_error(GS_EINVAL, "gs_adjoint_backward: no seed and no loss set");
  gs_sim* s = a->s;
  const size_t count = (size_t)s->N * s->p.nvariants;
  if (seed) {
    if (seed_dtype != GS_DTYPE_F32 && seed_dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", seed_dtype);
    GS_TRY(upload(s, a->lam[1], seed, count, seed_dtype));
  }
  if (grad_eta0 && grad_dtype != GS_DTYPE_F32 && grad_dtype != GS_DTYPE_F64)
    return gs_set_error(GS_EINVAL, "dtype %d", grad_dtype);
  cudaStream_t st = pick_stream(s, stream);
  s->launches = 0;
  const void* sd = seed ? a->lam[1] : nullptr;
  const int c = s->p.dtype == GS_DTYPE_F64 ? adj_backward<double>(a, sd, seed_e, loss, grads, st)
                                           : adj_backward<float>(a, sd, seed_e, loss, grads, st);
  if (c < 0) return c;
  a->warm = true;  // both sweeps have run directly: kernel attributes are set
  if (grad_eta0) GS_TRY(download(s, a->lam[c], grad_eta0, count, grad_dtype));
  return GS_OK;
}

extern "C" int gs_adjoint_use_graph(gs_adjoint* a, int on) {
  if (!a) return gs_set_error(GS_EINVAL, "gs_adjoint_use_graph: null handle");
  a->use_graph = on != 0;
  if (!on) adj_graph_reset(a);
  return GS_OK;
}

extern "C" int64_t gs_adjoint_launch_count(const gs_adjoint* a) { return a && a->s ? a->s->launches : 0; }

// ---------------------------------------------------------------------------
// autotuner of the tile schedule
// ---------------------------------------------------------------------------
// Coordinate descent over the four tile sizes of the martensite passes (z
// lines per block, y and x columns per block, update rows per block): each
// candidate is timed with CUDA events over `reps` trial steps, which write
// only the spare field of the pair and the spectra, so the simulation's
// state is untouched.  Candidates a launcher cannot take fall back to its
// default and time the same.  Two sweeps; the fastest schedule is kept.
template <class StepFn> static int tune(gs_sim* s, int reps, cudaStream_t st, StepFn trial_step, gs_schedule* out) {
  cudaEvent_t e0, e1;
  GS_CU(cudaEventCreate(&e0), "event");
  GS_CU(cudaEventCreate(&e1), "event");
  s->trial = true;
  auto time_sched = [&](const gs_schedule& sc, float* ms) -> int {
    s->sched = sc;
    GS_TRY(trial_step());  // warm: attributes, caches
    float best = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      GS_CU(cudaEventRecord(e0, st), "record");
      for (int i = 0; i < reps; ++i) GS_TRY(trial_step());
      GS_CU(cudaEventRecord(e1, st), "record");
      GS_CU(cudaEventSynchronize(e1), "sync");
      float t = 0;
      GS_CU(cudaEventElapsedTime(&t, e0, e1), "elapsed");
      if (t < best) best = t;
    }
    *ms = best;
    return GS_OK;
  };
  gs_schedule best = s->sched;
  float best_ms = 0;
  int rc = time_sched(best, &best_ms);
  const int cand[] = {1, 2, 4, 8, 16, 32, 64};
  for (int sweep = 0; sweep < 2 && rc == GS_OK; ++sweep) {
    for (int knob = 0; knob < 4 && rc == GS_OK; ++knob) {
      for (int c : cand) {
        gs_schedule sc = best;
        int* f = knob == 0 ? &sc.z_lines : knob == 1 ? &sc.y_cols : knob == 2 ? &sc.x_cols : &sc.update_rows;
        if (*f == c) continue;
        *f = c;
        float ms = 0;
        if ((rc = time_sched(sc, &ms)) != GS_OK) break;
        if (ms < 0.98f * best_ms) {
          best = sc;
          best_ms = ms;
        }
      }
    }
    // the radix split of the y lines: the default plan or its alternative
    // (the rounding differs between plans, within the step's accuracy bar)
    const int alt = ypass_alt_radix(s->n1);
    if (alt && rc == GS_OK) {
      gs_schedule sc = best;
      sc.y_radix = best.y_radix == alt ? 0 : alt;
      float ms = 0;
      if ((rc = time_sched(sc, &ms)) == GS_OK && ms < 0.98f * best_ms) {
        best = sc;
        best_ms = ms;
      }
    }
  }
  s->trial = false;
  s->spec_ready = false;  // the trial steps left other spectra behind
  s->sched = best;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != GS_OK) return rc;
  if (out) *out = best;
  return GS_OK;
}

extern "C" int gs_sim_set_schedule(gs_sim* s, const gs_schedule* sc) {
  if (!s || !sc) return gs_set_error(GS_EINVAL, "gs_sim_set_schedule: null argument");
  sim_graph_reset(s);
  if (sc->z_lines < 0 || sc->y_cols < 0 || sc->x_cols < 0 || sc->update_rows < 0)
    return gs_set_error(GS_EINVAL, "gs_sim_set_schedule: negative tile size");
  if (sc->y_radix != 0 && sc->y_radix != ypass_alt_radix(s->n1))
    return gs_set_error(GS_EINVAL, "gs_sim_set_schedule: y radix %d: 0 or %d for lines of %d", sc->y_radix,
                        ypass_alt_radix(s->n1), s->n1);
  s->sched = *sc;
  return GS_OK;
}

extern "C" int gs_sim_get_schedule(const gs_sim* s, gs_schedule* sc) {
  if (!s || !sc) return gs_set_error(GS_EINVAL, "gs_sim_get_schedule: null argument");
  *sc = s->sched;
  return GS_OK;
}

extern "C" int gs_sim_autotune(gs_sim* s, int reps, void* stream, gs_schedule* chosen) {
  if (!s) return gs_set_error(GS_EINVAL, "gs_sim_autotune: null sim");
  if (s->plain || s->p.model == GS_MODEL_STRESS)
    return gs_set_error(GS_ENOTSUP, "gs_sim_autotune: martensite and precipitate simulations only");
  if (reps < 1) reps = 1;
  sim_graph_reset(s);
  cudaStream_t st = pick_stream(s, stream);
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  if (s->p.model == GS_MODEL_MART)
    return tune(s, reps, st, [&]() { return f64 ? mart_step<double>(s, st) : mart_step<float>(s, st); }, chosen);
  // precipitate: the trial steps advance c and eta in place, so the state and
  // the step counter are kept aside and put back
  const size_t fb = (size_t)s->N * elt(s), V = (size_t)s->p.nvariants;
  void* keep = nullptr;
  GS_CU(cudaMalloc(&keep, fb * (V + 1)), "tuning state copy");
  const int64_t step0 = s->step;
  int rc = gs_cuda_check(cudaMemcpyAsync(keep, s->conc, fb, cudaMemcpyDeviceToDevice, st), "keep state");
  if (rc == GS_OK)
    rc = gs_cuda_check(
        cudaMemcpyAsync(static_cast<char*>(keep) + fb, s->eta[0], fb * V, cudaMemcpyDeviceToDevice, st), "keep state");
  if (rc == GS_OK)
    rc = tune(s, reps, st, [&]() { return f64 ? precip_step<double>(s, st) : precip_step<float>(s, st); }, chosen);
  cudaMemcpyAsync(s->conc, keep, fb, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->eta[0], static_cast<char*>(keep) + fb, fb * V, cudaMemcpyDeviceToDevice, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(keep);
  s->step = step0;
  if (rc == GS_OK) rc = gs_cuda_check(e, "restore state");
  return rc;
}

extern "C" int gs_batch_autotune(gs_batch* b, int reps, void* stream) {
  if (!b) return gs_set_error(GS_EINVAL, "gs_batch_autotune: null batch");
  if (reps < 1) reps = 1;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  if (b->exec) {  // a captured step holds the old tile sizes
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  for (gs_sim* g : b->groups) {
    const bool f64 = g->p.dtype == GS_DTYPE_F64;
    GS_TRY(tune(g, reps, st,
                [&]() { return f64 ? batch_group_step<double>(g, st) : batch_group_step<float>(g, st); }, nullptr));
  }
  return GS_OK;
}

extern "C" int gs_batch_get_schedule(const gs_batch* b, int group, gs_schedule* sc) {
  if (!b || !sc || group < 0 || group >= (int)b->groups.size())
    return gs_set_error(GS_EINVAL, "gs_batch_get_schedule: bad arguments");
  *sc = b->groups[group]->sched;
  return GS_OK;
}

// ---------------------------------------------------------------------------
// device-to-device hand-off between simulations
// ---------------------------------------------------------------------------
// The reference passes the stress stage's results to the martensite stage
// through files (dump stress / defect, then read dislocationstress / defect:
// scripts/in.precipitate.sh) and remaps them on the host
// (src/dynamics_mart.cu:128-154, :305-321).  Here they stay on the device.
extern "C" int gs_sim_take_field(gs_sim* dst, const char* dst_name, gs_sim* src, const char* src_name) {
  if (!dst || !src || !dst_name || !src_name) return gs_set_error(GS_EINVAL, "gs_sim_take_field: null argument");
  if (dst->p.nx != src->p.nx || dst->p.ny != src->p.ny || dst->p.nz != src->p.nz)
    return gs_set_error(GS_EINVAL, "gs_sim_take_field: grids differ");
  const std::string dn(dst_name), sn(src_name);
  GS_CU(cudaStreamSynchronize(src->own_stream), "sync source");
  GS_CU(cudaStreamSynchronize(dst->own_stream), "sync destination");
  sim_graph_reset(dst);
  dst->spec_ready = false;
  gs_cufft_invalidate(dst);
  const size_t N = (size_t)dst->N;
  if (dn == "dislocationstress" && sn == "stress") {
    if (dst->p.model != GS_MODEL_MART || !src->stressbuf)
      return gs_set_error(GS_EINVAL, "gs_sim_take_field: stress of a stress model into a martensite model");
    return stress_to_K(dst, src->stressbuf, src->p.dtype, dst->own_stream);
  }
  if (dn == "defect" && sn == "defect") {
    if (dst->p.model != GS_MODEL_MART || !src->defect)
      return gs_set_error(GS_EINVAL, "gs_sim_take_field: defect of a stress model into a martensite model");
    if (!dst->defect) GS_CU(cudaMalloc(&dst->defect, N * elt(dst)), "cudaMalloc defect");
    if (dst->p.dtype == src->p.dtype) {
      GS_CU(cudaMemcpy(dst->defect, src->defect, N * elt(dst), cudaMemcpyDeviceToDevice), "copy defect");
    } else {
      std::vector<char> tmp(N * elt(src));
      GS_TRY(download(src, src->defect, tmp.data(), N, src->p.dtype));
      GS_TRY(upload(dst, dst->defect, tmp.data(), N, src->p.dtype));
    }
    GS_CU(cudaDeviceSynchronize(), "copy defect sync");
    return GS_OK;
  }
  if (dn == "eta" && sn == "eta") {
    if (dst->p.nvariants != src->p.nvariants || dst->p.dtype != src->p.dtype)
      return gs_set_error(GS_EINVAL, "gs_sim_take_field: eta needs the same variants and dtype");
    GS_CU(cudaMemcpy(dst->eta[dst->cur], src->eta[src->cur], N * elt(dst) * dst->p.nvariants,
                     cudaMemcpyDeviceToDevice),
          "copy eta");
    GS_CU(cudaDeviceSynchronize(), "copy eta sync");
    return GS_OK;
  }
  return gs_set_error(GS_EINVAL, "gs_sim_take_field: cannot take '%s' from '%s'", dst_name, src_name);
}

// ---------------------------------------------------------------------------
// adjoint of the precipitate run (every state kept)
// ---------------------------------------------------------------------------
// The reverse sweep per step: one spectral pass over the pairs (lambda',
// state') gives D lambda', K D lambda' and K^a D state' of every field
// (PrecipAdjOp), the first pointwise sweep the local-term adjoints and the
// elastic sources dR, the elastic chain B * dR, the second sweep the new
// lambda; R of the state comes from its own chain.  gs_padj.cuh has the
// formulas; the oracle's or_precip_adjoint states the same in FP64.
struct gs_padjoint {
  gs_sim* s = nullptr;
  int nsteps = 0, F1 = 0;
  int K = 1, nseg = 1;     // a checkpoint every K steps; nseg segments
  void* ckpt = nullptr;    // [nseg + 1][V + 1][N]: the states at steps 0, K, 2K, ... and the final one
  void* seg = nullptr;     // [K - 1][V + 1][N]: the inner states of one segment (none when K = 1)
  int seg_valid = -1;      // the segment whose inner states seg holds (-1: none)
  void* lam[2] = {nullptr, nullptr};
  void* Y = nullptr;   // [3 (V + 1)] spectra
  void* Zr = nullptr;  // [3 (V + 1)][N]
  void* dP = nullptr;  // [F1][N]
  double* gsum = nullptr;  // [nsteps][PADJ_N]
  void* seed = nullptr;    // [V + 1][N]: dJ/d(c_T, eta_T)
  bool forward_done = false, seeded = false;
  size_t bytes = 0;
  // the reverse sweep replayed as one captured graph (after a first direct
  // run); captured with the mass-projection offset of its initial state
  bool use_graph = true, warm = false;
  cudaGraphExec_t gbwd = nullptr;
  cudaStream_t gstream = nullptr;
  int64_t nl_bwd = 0;
  double g_mass0 = 0;
};

static void padj_graph_reset(gs_padjoint* a) {
  if (a->gbwd) cudaGraphExecDestroy(a->gbwd);
  a->gbwd = nullptr;
}

static void free_padjoint(gs_padjoint* a) {
  if (!a) return;
  cudaDeviceSynchronize();
  padj_graph_reset(a);
  for (void* q : {a->ckpt, a->seg, a->lam[0], a->lam[1], a->Y, a->Zr, a->dP, (void*)a->gsum, a->seed})
    if (q) cudaFree(q);
  if (a->s) free_sim(a->s);
  delete a;
}

extern "C" int gs_precip_adjoint_create(const gs_params* p, int nsteps, int checkpoint_every, gs_padjoint** out) {
  if (!p || !out) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_create: null argument");
  *out = nullptr;
  if (p->model != GS_MODEL_PRECIPITATE) return gs_set_error(GS_EINVAL, "precipitate adjoint: precipitate model only");
  if (p->mode != GS_MODE_BASELINE) return gs_set_error(GS_ENOTSUP, "precipitate adjoint: baseline mode only");
  if (nsteps < 1) return gs_set_error(GS_EINVAL, "precipitate adjoint: nsteps %d", nsteps);
  if (checkpoint_every < 1 || checkpoint_every > nsteps)
    return gs_set_error(GS_EINVAL, "precipitate adjoint: checkpoint_every %d outside 1..%d", checkpoint_every, nsteps);
  gs_padjoint* a = new gs_padjoint();
  int rc = gs_sim_create(p, &a->s);
  if (rc != GS_OK) {
    delete a;
    return rc;
  }
  a->nsteps = nsteps;
  a->K = checkpoint_every;
  a->nseg = (nsteps + a->K - 1) / a->K;
  a->F1 = precip_nfields(a->s);
  const int V = p->nvariants;
  const size_t fb = (size_t)a->s->N * elt(a->s);
  auto get = [&](void** q, size_t b, const char* what) {
    const int r = dalloc(q, b, what);
    if (r == GS_OK) a->bytes += b;
    return r;
  };
  if ((rc = get(&a->ckpt, fb * (V + 1) * (a->nseg + 1), "adjoint checkpoints")) != GS_OK ||
      (a->K > 1 && (rc = get(&a->seg, fb * (V + 1) * (a->K - 1), "adjoint segment states")) != GS_OK) ||
      (rc = get(&a->lam[0], fb * (V + 1), "adjoint lambda")) != GS_OK ||
      (rc = get(&a->lam[1], fb * (V + 1), "adjoint lambda")) != GS_OK ||
      (rc = get(&a->seed, fb * (V + 1), "adjoint seed")) != GS_OK ||
      (rc = get(&a->Y, fb * 3 * (V + 1), "adjoint spectra")) != GS_OK ||
      (rc = get(&a->Zr, fb * 3 * (V + 1), "adjoint fields")) != GS_OK ||
      (rc = get(&a->dP, fb * a->F1, "adjoint elastic sources")) != GS_OK ||
      (rc = get(reinterpret_cast<void**>(&a->gsum), (size_t)nsteps * PADJ_N * sizeof(double), "adjoint sums")) !=
          GS_OK) {
    free_padjoint(a);
    return rc;
  }
  // the simulation's own buffers count too (fields, spectra, work arrays)
  const int F2 = 2 * V + 2;
  a->bytes += fb * ((size_t)V + 1 + (V + 1) + a->F1 + (V + 1) + F2);
  *out = a;
  return GS_OK;
}

extern "C" int gs_precip_adjoint_destroy(gs_padjoint* a) {
  free_padjoint(a);
  return GS_OK;
}

extern "C" size_t gs_precip_adjoint_device_bytes(const gs_padjoint* a) { return a ? a->bytes : 0; }

extern "C" int gs_precip_adjoint_use_graph(gs_padjoint* a, int on) {
  if (!a) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_use_graph: null handle");
  a->use_graph = on != 0;
  if (!a->use_graph) padj_graph_reset(a);
  return GS_OK;
}

// copy the simulation's state (c, eta) to / from a [V + 1][N] slot
static int padj_save(gs_padjoint* a, void* dst, cudaStream_t st) {
  gs_sim* s = a->s;
  const size_t fb = (size_t)s->N * elt(s);
  GS_CU(cudaMemcpyAsync(dst, s->conc, fb, cudaMemcpyDeviceToDevice, st), "keep state");
  GS_CU(cudaMemcpyAsync(static_cast<char*>(dst) + fb, s->eta[0], fb * s->p.nvariants, cudaMemcpyDeviceToDevice, st),
        "keep state");
  return GS_OK;
}
static int padj_load(gs_padjoint* a, const void* src, cudaStream_t st) {
  gs_sim* s = a->s;
  const size_t fb = (size_t)s->N * elt(s);
  s->spec_ready = false;  // the spectra left by the last step are not this state's
  GS_CU(cudaMemcpyAsync(s->conc, src, fb, cudaMemcpyDeviceToDevice, st), "restore state");
  GS_CU(cudaMemcpyAsync(s->eta[0], static_cast<const char*>(src) + fb, fb * s->p.nvariants, cudaMemcpyDeviceToDevice,
                        st),
        "restore state");
  return GS_OK;
}
static char* padj_slot(void* base, const gs_padjoint* a, int i) {
  return static_cast<char*>(base) + (size_t)i * (size_t)a->s->N * elt(a->s) * (a->s->p.nvariants + 1);
}

// the state of step n inside segment j (a0 = jK <= n <= b0): the two
// checkpoints at its ends, the inner states in seg
static char* padj_state(gs_padjoint* a, int j, int n) {
  const int a0 = j * a->K, b0 = std::min(a0 + a->K, a->nsteps);
  if (n == a0) return padj_slot(a->ckpt, a, j);
  if (n == b0) return padj_slot(a->ckpt, a, j + 1);
  return padj_slot(a->seg, a, n - a0 - 1);
}

// the inner states of segment j into seg, recomputed from checkpoint j with
// the forward's own step counters (the same bits as the forward's states)
static int padj_recompute(gs_padjoint* a, int j, cudaStream_t st) {
  gs_sim* s = a->s;
  const int a0 = j * a->K, b0 = std::min(a0 + a->K, a->nsteps);
  if (b0 - a0 > 1) {
    GS_TRY(padj_load(a, padj_slot(a->ckpt, a, j), st));
    s->step = a0;
    const bool f64 = s->p.dtype == GS_DTYPE_F64;
    for (int n = a0 + 1; n < b0; ++n) {
      GS_TRY(f64 ? precip_step<double>(s, st) : precip_step<float>(s, st));
      GS_TRY(padj_save(a, padj_state(a, j, n), st));
    }
  }
  a->seg_valid = j;
  return GS_OK;
}

static int gs_precip_adjoint_forward_body(gs_padjoint* a, const void* c0, const void* eta0, int dtype, void* c_final,
                                          void* eta_final, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_precip_adjoint_forward(gs_padjoint* a, const void* c0, const void* eta0, int dtype, void* c_final,
                                         void* eta_final, void* stream) {
  return bc_after(gs_precip_adjoint_forward_body(a, c0, eta0, dtype, c_final, eta_final, stream),
                  static_cast<cudaStream_t>(stream));
}

static int gs_precip_adjoint_forward_body(gs_padjoint* a, const void* c0, const void* eta0, int dtype, void* c_final,
                                         void* eta_final, void* stream) {
  if (!a) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_forward: null handle");
  if (!c0 != !eta0) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_forward: give both c0 and eta0, or neither");
  gs_sim* s = a->s;
  const int V = s->p.nvariants;
  const size_t N = (size_t)s->N;
  cudaStream_t st = pick_stream(s, stream);
  if (c0) {
    GS_TRY(gs_sim_set_field(s, "concentration", c0, N, dtype));
    GS_TRY(gs_sim_set_field(s, "eta", eta0, N * V, dtype));
  } else {  // again from the initial state of the previous forward run
    if (!a->forward_done) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_forward: no initial state yet");
    GS_TRY(padj_load(a, padj_slot(a->ckpt, a, 0), st));
  }
  s->step = 0;
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  const int last = a->nseg - 1, last0 = last * a->K;  // the last segment's inner states stay in seg
  for (int n = 0; n <= a->nsteps; ++n) {
    if (n % a->K == 0 || n == a->nsteps) GS_TRY(padj_save(a, padj_slot(a->ckpt, a, (n + a->K - 1) / a->K), st));
    else if (n > last0) GS_TRY(padj_save(a, padj_state(a, last, n), st));
    if (n < a->nsteps) GS_TRY(f64 ? precip_step<double>(s, st) : precip_step<float>(s, st));
  }
  GS_CU(cudaStreamSynchronize(st), "forward sync");
  a->seg_valid = a->nseg - 1;
  a->forward_done = true;
  if (c_final) GS_TRY(download(s, s->conc, c_final, N, dtype));
  if (eta_final) GS_TRY(download(s, s->eta[0], eta_final, N * V, dtype));
  return GS_OK;
}

// one reverse step n from lam[c] into lam[c ^ 1]; st0, st1: the states of
// steps n and n + 1
template <typename T>
static int padj_reverse_step(gs_padjoint* a, int n, const T* st0, const T* st1, int c, cudaStream_t st);

template <typename T> static int padj_backward(gs_padjoint* a, cudaStream_t st, int* cur) {
  int c = 0;
  for (int j = a->nseg - 1; j >= 0; --j) {
    if (a->seg_valid != j) GS_TRY(padj_recompute(a, j, st));
    const int a0 = j * a->K, b0 = std::min(a0 + a->K, a->nsteps);
    for (int n = b0 - 1; n >= a0; --n) {
      const T* st0 = reinterpret_cast<const T*>(padj_state(a, j, n));
      const T* st1 = reinterpret_cast<const T*>(padj_state(a, j, n + 1));
      GS_TRY(padj_reverse_step<T>(a, n, st0, st1, c, st));
      c ^= 1;
    }
  }
  *cur = c;
  return GS_OK;
}

template <typename T>
static int padj_reverse_step(gs_padjoint* a, int n, const T* st0, const T* st1, int c, cudaStream_t st) {
  gs_sim* s = a->s;
  const gs_params& p = s->p;
  const int V = p.nvariants, F1 = a->F1, FV = V + 1;
  const long long N = s->N, rows = (long long)s->n0 * s->n1;
  T* Zr = reinterpret_cast<T*>(a->Zr);
  {
    const T* lin = reinterpret_cast<const T*>(a->lam[c]);
    T* lout = reinterpret_cast<T*>(a->lam[c ^ 1]);
    // spectral pass over the pairs (lambda', state')
    ZfwdArgs<T> za;
    memset(&za, 0, sizeof(za));
    for (int f = 0; f < FV; ++f) {
      za.src[2 * f] = lin + (size_t)f * N;
      za.src[2 * f + 1] = st1 + (size_t)f * N;
    }
    za.dst = reinterpret_cast<cplx<T>*>(s->spec2);
    za.rows_per_field = rows;
    za.nrows = rows * 2 * FV;
    za.tw_h = twp<T>(s, 1);
    za.tw_n2 = twp<T>(s, 0);
    GS_CU(launch_zfwd<T>(za, s->h, st), "adjoint z forward");
    YArgs<T> ya;
    ya.spec = reinterpret_cast<cplx<T>*>(s->spec2);
    ya.n0 = s->n0;
    ya.n1 = s->n1;
    ya.h = s->h;
    ya.tw = twp<T>(s, 2);
    GS_CU(launch_ypass<T>(ya, s->n1, 2 * FV, -1, st), "adjoint y forward");
    XArgs<T> xa;
    memset(&xa, 0, sizeof(xa));
    xa.in = reinterpret_cast<cplx<T>*>(s->spec2);
    xa.out = reinterpret_cast<cplx<T>*>(a->Y);
    xa.n0 = s->n0;
    xa.n1 = s->n1;
    xa.n2 = s->n2;
    xa.h = s->h;
    xa.F = 2;
    xa.G = 3;
    xa.nsim = FV;
    xa.tw = twp<T>(s, 3);
    xa.pu.V = V;
    xa.pu.dtM = (T)(p.dt * p.mobility_c);
    xa.pu.dtL = (T)(p.dt * p.mobility_eta);
    xa.pu.kc = (T)p.kappa_c;
    xa.pu.ke = (T)p.kappa_eta;
    xa.pu.scale = (T)(1.0 / (double)N);
    for (int c3 = 0; c3 < 3; ++c3) xa.pu.ktab[c3] = reinterpret_cast<const T*>(s->ktab) + s->ktab_off[c3];
    GS_CU(launch_xprecip_adjoint<T>(xa, st), "adjoint x pass");
    YArgs<T> yb = ya;
    yb.spec = reinterpret_cast<cplx<T>*>(a->Y);
    GS_CU(launch_ypass<T>(yb, s->n1, 3 * FV, 1, st), "adjoint y inverse");
    for (int f0 = 0; f0 < 3 * FV; f0 += GS_MAXG + 1) {
      const int nf = 3 * FV - f0 < GS_MAXG + 1 ? 3 * FV - f0 : GS_MAXG + 1;
      ZinvArgs<T> zi;
      memset(&zi, 0, sizeof(zi));
      zi.spec = reinterpret_cast<const cplx<T>*>(a->Y) + (size_t)f0 * rows * s->h;
      for (int k = 0; k < nf; ++k) zi.dst[k] = Zr + (size_t)(f0 + k) * N;
      zi.rows_per_field = rows;
      zi.nrows = rows * nf;
      zi.tw_h = twp<T>(s, 1);
      zi.tw_n2 = twp<T>(s, 0);
      zi.offset_field = -1;
      GS_CU(launch_zinv<T>(zi, s->h, st), "adjoint z inverse");
    }
    // R of state n into rbuf
    {
      const T* src[GS_MAXF + 1];
      int sq[GS_MAXF + 1];
      for (int f = 0; f < V; ++f) {
        src[f] = st0 + (size_t)(1 + f) * N;
        sq[f] = 1;
      }
      if (F1 > V) {
        src[V] = st0;
        sq[V] = 0;
      }
      GS_TRY(elastic_chain_g<T>(s, src, sq, F1, 2, 1.0 / (double)N, s->spec, F1, st));
      ZinvArgs<T> zr;
      memset(&zr, 0, sizeof(zr));
      zr.spec = reinterpret_cast<const cplx<T>*>(s->spec);
      for (int f = 0; f < F1; ++f) zr.dst[f] = reinterpret_cast<T*>(s->rbuf) + (size_t)f * N;
      zr.rows_per_field = rows;
      zr.nrows = rows * F1;
      zr.tw_h = twp<T>(s, 1);
      zr.tw_n2 = twp<T>(s, 0);
      zr.offset_field = -1;
      GS_CU(launch_zinv<T>(zr, s->h, st), "adjoint potential");
    }
    PadjArgs<T> pa;
    memset(&pa, 0, sizeof(pa));
    pa.N = N;
    pa.V = V;
    pa.F = F1;
    pa.ce = p.c_elastic ? 1 : 0;
    for (int i = 0; i < 8; ++i) pa.A[i] = (T)p.coef[i];
    pa.c1 = (T)p.c1;
    pa.c2 = (T)p.c2;
    pa.Es = (T)(p.xi * p.weight_elastic);
    pa.dtM = (T)(p.dt * p.mobility_c);
    pa.dtL = (T)(p.dt * p.mobility_eta);
    pa.lc = lin;
    pa.le = lin + N;
    pa.zr = Zr;
    pa.c = st0;
    pa.eta = st0 + N;
    pa.R = reinterpret_cast<const T*>(s->rbuf);
    pa.dR = reinterpret_cast<T*>(s->mubuf);
    pa.dP = reinterpret_cast<const T*>(a->dP);
    pa.lc_out = lout;
    pa.le_out = lout + N;
    pa.partials = s->partials;
    int nb = 0;
    GS_CU(launch_padj<T>(pa, false, st, &nb), "adjoint local sources");
    GS_CU(launch_reduce(s->partials, nb, 2, a->gsum + (size_t)n * PADJ_N + PADJ_KC, st), "adjoint reduce");
    // B * dR
    {
      const T* src[GS_MAXF + 1];
      int sq[GS_MAXF + 1];
      for (int f = 0; f < F1; ++f) {
        src[f] = reinterpret_cast<const T*>(s->mubuf) + (size_t)f * N;
        sq[f] = 0;
      }
      GS_TRY(elastic_chain_g<T>(s, src, sq, F1, 2, 1.0 / (double)N, s->spec, F1, st));
      ZinvArgs<T> zp;
      memset(&zp, 0, sizeof(zp));
      zp.spec = reinterpret_cast<const cplx<T>*>(s->spec);
      for (int f = 0; f < F1; ++f) zp.dst[f] = reinterpret_cast<T*>(a->dP) + (size_t)f * N;
      zp.rows_per_field = rows;
      zp.nrows = rows * F1;
      zp.tw_h = twp<T>(s, 1);
      zp.tw_n2 = twp<T>(s, 0);
      zp.offset_field = -1;
      GS_CU(launch_zinv<T>(zp, s->h, st), "adjoint elastic transpose");
    }
    GS_CU(launch_padj<T>(pa, true, st, &nb), "adjoint lambda");
    GS_CU(launch_reduce(s->partials, nb, 7, a->gsum + (size_t)n * PADJ_N + PADJ_A1, st), "adjoint reduce");
  }
  return GS_OK;
}

extern "C" int gs_precip_adjoint_set_seed(gs_padjoint* a, const void* seed_c, const void* seed_eta, int dtype) {
  if (!a || !seed_c || !seed_eta) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_set_seed: null argument");
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", dtype);
  gs_sim* s = a->s;
  const size_t N = (size_t)s->N, fb = N * elt(s);
  GS_TRY(upload(s, a->seed, seed_c, N, dtype));
  GS_TRY(upload(s, static_cast<char*>(a->seed) + fb, seed_eta, N * s->p.nvariants, dtype));
  a->seeded = true;
  return GS_OK;
}

static int gs_precip_adjoint_backward_body(gs_padjoint* a, const void* seed_c, const void* seed_eta, int dtype,
                                           double* grads, void* grad_c0, void* grad_eta0, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_precip_adjoint_backward(gs_padjoint* a, const void* seed_c, const void* seed_eta, int dtype,
                                          double* grads, void* grad_c0, void* grad_eta0, void* stream) {
  return bc_after(gs_precip_adjoint_backward_body(a, seed_c, seed_eta, dtype, grads, grad_c0, grad_eta0, stream),
                  static_cast<cudaStream_t>(stream));
}

static int gs_precip_adjoint_backward_body(gs_padjoint* a, const void* seed_c, const void* seed_eta, int dtype,
                                          double* grads, void* grad_c0, void* grad_eta0, void* stream) {
  if (!a || !grads) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_backward: null argument");
  if (!a->forward_done) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_backward: run the forward first");
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "dtype %d", dtype);
  if (!seed_c != !seed_eta) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_backward: give both seeds, or neither");
  if (seed_c) GS_TRY(gs_precip_adjoint_set_seed(a, seed_c, seed_eta, dtype));
  if (!a->seeded) return gs_set_error(GS_EINVAL, "gs_precip_adjoint_backward: no seed set");
  gs_sim* s = a->s;
  const int V = s->p.nvariants;
  const size_t N = (size_t)s->N, fb = N * elt(s);
  cudaStream_t st = pick_stream(s, stream);
  const bool f64 = s->p.dtype == GS_DTYPE_F64;
  // the sweep: the seed into lambda, then every segment (recomputed from its
  // checkpoint unless its states are in seg) and its reverse steps
  auto body = [&](int* cur) -> int {
    GS_CU(cudaMemcpyAsync(a->lam[0], a->seed, fb * (V + 1), cudaMemcpyDeviceToDevice, st), "seed");
    return f64 ? padj_backward<double>(a, st, cur) : padj_backward<float>(a, st, cur);
  };
  // a replayed graph starts from the forward's last segment, as captured
  if (a->seg_valid != a->nseg - 1) GS_TRY(padj_recompute(a, a->nseg - 1, st));
  int c = 0;
  if (a->gbwd && (a->gstream != st || a->g_mass0 != s->mass0)) padj_graph_reset(a);
  if (!a->use_graph || !a->warm) {
    GS_TRY(body(&c));
    a->warm = true;  // kernel attributes are set: later sweeps may be captured
  } else {
    if (!a->gbwd) {
      cudaGraph_t g;
      const int64_t l0 = s->launches;
      const int64_t step0 = s->step;
      GS_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
      const int rc = body(&c);
      const cudaError_t e = cudaStreamEndCapture(st, &g);
      s->step = step0;
      if (rc != GS_OK) return rc;
      GS_CU(e, "end capture");
      GS_CU(cudaGraphInstantiate(&a->gbwd, g, 0), "instantiate graph");
      cudaGraphDestroy(g);
      a->gstream = st;
      a->g_mass0 = s->mass0;
      a->nl_bwd = s->launches - l0;
      s->launches = l0;
    } else {
      c = a->nsteps % 2;  // lambda swaps once per step
    }
    GS_CU(cudaGraphLaunch(a->gbwd, st), "graph launch");
    s->launches += a->nl_bwd;
  }
  // seg now holds segment 0 (the last one the sweep visits); the next sweep
  // recomputes the last segment first
  a->seg_valid = 0;
  std::vector<double> h((size_t)a->nsteps * PADJ_N);
  GS_CU(cudaMemcpyAsync(h.data(), a->gsum, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "sums D2H");
  GS_CU(cudaStreamSynchronize(st), "adjoint sync");
  for (int k = 0; k < PADJ_N; ++k) {
    double sum = 0, cmp = 0;
    for (int n = 0; n < a->nsteps; ++n) {
      const double x = h[(size_t)n * PADJ_N + k], t = sum + x;
      cmp += std::fabs(sum) >= std::fabs(x) ? (sum - t) + x : (x - t) + sum;
      sum = t;
    }
    grads[k] = sum + cmp;
  }
  if (grad_c0) GS_TRY(download(s, a->lam[c], grad_c0, N, dtype));
  if (grad_eta0) GS_TRY(download(s, static_cast<char*>(a->lam[c]) + fb, grad_eta0, N * V, dtype));
  return GS_OK;
}

extern "C" void gs_set_x_prefetch(int on) { set_x_prefetch(on != 0); }

extern "C" unsigned int gs_x_prefetch_timeouts(void) { return x_wait_timeouts(); }

// ---------------------------------------------------------------------------
// asynchronous field copies: a dump that overlaps the steps after it
// ---------------------------------------------------------------------------
// gs_sim_copy_field_async snapshots the field on the device (a device-to-
// device copy on the stepping stream, ordered after the steps already
// issued, so the next steps may overwrite the field at once), then copies the
// snapshot to page-locked staging memory on the simulation's copy stream.
// gs_sim_copy_field_wait waits for that copy and converts it into the
// caller's buffer.  Two copies can be in flight per simulation; a third
// waits (up to two minutes) for a gs_sim_copy_field_wait to free a slot.
struct gs_snapslot {
  void* dev = nullptr;
  size_t dev_bytes = 0;
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  cudaEvent_t taken = nullptr;   // snapshot done (stepping stream)
  cudaEvent_t landed = nullptr;  // staging copy done (copy stream)
  size_t count = 0;
  bool direct = false;  // copied straight into the caller's page-locked buffer
  int ticket = 0;       // 0: free
};

struct gs_snaps {
  static constexpr int kSlots = 2;
  gs_snapslot slot[kSlots];
  cudaStream_t copy = nullptr;
  int next = 1;
  std::mutex mu;
  std::condition_variable cv;
};

static void free_snaps(gs_sim* s) {
  gs_snaps* q = s->snaps;
  if (!q) return;
  for (gs_snapslot& sl : q->slot) {
    if (sl.landed) cudaEventSynchronize(sl.landed);
    if (sl.dev) cudaFree(sl.dev);
    if (sl.pinned) cudaFreeHost(sl.pinned);
    if (sl.taken) cudaEventDestroy(sl.taken);
    if (sl.landed) cudaEventDestroy(sl.landed);
  }
  if (q->copy) cudaStreamDestroy(q->copy);
  delete q;
  s->snaps = nullptr;
}

// device address and value count of a field the dumps ask for
static int field_source(gs_sim* s, const std::string& nm, const void** src, size_t* count) {
  const size_t N = (size_t)s->N;
  if (nm == "eta") {
    *src = s->eta[s->cur];
    *count = N * s->p.nvariants;
  } else if (nm == "concentration" && s->conc) {
    *src = s->conc;
    *count = N;
  } else if (nm == "stress" && s->stressbuf) {
    *src = s->stressbuf;
    *count = 6 * N;
  } else if (nm == "defect" && s->defect) {
    *src = s->defect;
    *count = N;
  } else {
    return gs_set_error(GS_EINVAL, "gs_sim_copy_field_async: no field '%s' in this simulation", nm.c_str());
  }
  return GS_OK;
}

extern "C" int gs_sim_copy_field_async(gs_sim* s, const char* name, void* stream, void* pinned_dst, int* ticket) {
  if (!s || !name || !ticket) return gs_set_error(GS_EINVAL, "gs_sim_copy_field_async: null argument");
  const void* src = nullptr;
  size_t count = 0;
  GS_TRY(field_source(s, name, &src, &count));
  if (!s->snaps) {
    gs_snaps* q = new gs_snaps();
    if (cudaStreamCreateWithFlags(&q->copy, cudaStreamNonBlocking) != cudaSuccess) {
      delete q;
      return gs_set_error(GS_ECUDA, "copy stream: %s", cudaGetErrorString(cudaGetLastError()));
    }
    s->snaps = q;
  }
  gs_snaps* q = s->snaps;
  std::unique_lock<std::mutex> lk(q->mu);
  auto free_slot = [q]() {
    for (int i = 0; i < gs_snaps::kSlots; ++i)
      if (!q->slot[i].ticket) return i;
    return -1;
  };
  if (!q->cv.wait_for(lk, std::chrono::seconds(120), [&] { return free_slot() >= 0; }))
    return gs_set_error(GS_ETIMEOUT, "gs_sim_copy_field_async: both copy slots still wait for gs_sim_copy_field_wait");
  gs_snapslot& sl = q->slot[free_slot()];
  const size_t bytes = count * elt(s);
  if (sl.dev_bytes < bytes) {
    if (sl.dev) cudaFree(sl.dev);
    sl.dev = nullptr;
    sl.dev_bytes = 0;
    GS_CU(cudaMalloc(&sl.dev, bytes), "snapshot buffer");
    sl.dev_bytes = bytes;
  }
  if (!pinned_dst && sl.pinned_bytes < bytes) {
    if (sl.pinned) cudaFreeHost(sl.pinned);
    sl.pinned = nullptr;
    sl.pinned_bytes = 0;
    GS_CU(cudaMallocHost(&sl.pinned, bytes), "page-locked staging");
    sl.pinned_bytes = bytes;
  }
  if (!sl.taken) GS_CU(cudaEventCreateWithFlags(&sl.taken, cudaEventDisableTiming), "event");
  if (!sl.landed) GS_CU(cudaEventCreateWithFlags(&sl.landed, cudaEventDisableTiming), "event");
  cudaStream_t st = pick_stream(s, stream);
  GS_CU(cudaMemcpyAsync(sl.dev, src, bytes, cudaMemcpyDeviceToDevice, st), "snapshot");
  GS_CU(cudaEventRecord(sl.taken, st), "event");
  GS_CU(cudaStreamWaitEvent(q->copy, sl.taken, 0), "event wait");
  GS_CU(cudaMemcpyAsync(pinned_dst ? pinned_dst : sl.pinned, sl.dev, bytes, cudaMemcpyDeviceToHost, q->copy),
        "snapshot D2H");
  GS_CU(cudaEventRecord(sl.landed, q->copy), "event");
  sl.direct = pinned_dst != nullptr;
  sl.count = count;
  sl.ticket = q->next++;
  if (q->next <= 0) q->next = 1;
  *ticket = sl.ticket;
  return GS_OK;
}

extern "C" int gs_sim_copy_field_wait(gs_sim* s, int ticket, void* host, size_t count, int dtype) {
  if (!s || ticket <= 0) return gs_set_error(GS_EINVAL, "gs_sim_copy_field_wait: bad argument");
  gs_snaps* q = s->snaps;
  if (!q) return gs_set_error(GS_EINVAL, "gs_sim_copy_field_wait: no copy in flight");
  gs_snapslot* sl = nullptr;
  {
    std::lock_guard<std::mutex> lk(q->mu);
    for (gs_snapslot& x : q->slot)
      if (x.ticket == ticket) sl = &x;
  }
  if (!sl) return gs_set_error(GS_EINVAL, "gs_sim_copy_field_wait: unknown ticket %d", ticket);
  int rc = GS_OK;
  if (sl->direct) {  // the values are already in the caller's buffer
    rc = gs_cuda_check(cudaEventSynchronize(sl->landed), "copy wait");
  } else if (!host || (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64)) {
    cudaEventSynchronize(sl->landed);
    rc = gs_set_error(GS_EINVAL, "gs_sim_copy_field_wait: a host buffer of dtype 0 or 1 is needed");
  } else if (count != sl->count) {
    cudaEventSynchronize(sl->landed);
    rc = gs_set_error(GS_EINVAL, "gs_sim_copy_field_wait: %zu values asked, the copy holds %zu", count, sl->count);
  } else if ((rc = gs_cuda_check(cudaEventSynchronize(sl->landed), "copy wait")) == GS_OK) {
    const bool f64 = s->p.dtype == GS_DTYPE_F64;
    if ((dtype == GS_DTYPE_F64) == f64) {
      memcpy(host, sl->pinned, count * elt(s));
    } else if (f64) {
      const double* a = static_cast<const double*>(sl->pinned);
      float* b = static_cast<float*>(host);
      for (size_t i = 0; i < count; ++i) b[i] = (float)a[i];
    } else {
      const float* a = static_cast<const float*>(sl->pinned);
      double* b = static_cast<double*>(host);
      for (size_t i = 0; i < count; ++i) b[i] = (double)a[i];
    }
  }
  {
    std::lock_guard<std::mutex> lk(q->mu);
    sl->ticket = 0;
  }
  q->cv.notify_all();
  return rc;
}

// An upload on a stream: the asynchronous counterpart of gs_sim_set_field for
// the field set ("eta") in the simulation's own dtype.  From page-locked
// memory the copy overlaps whatever else runs (a download of the previous
// state on the copy stream, say); the caller keeps `host` unchanged until
// the stream has passed the copy.
extern "C" int gs_sim_set_field_async(gs_sim* s, const char* name, const void* host, size_t count, int dtype,
                                      void* stream) {
  if (!s || !name || !host) return gs_set_error(GS_EINVAL, "gs_sim_set_field_async: null argument");
  if (std::string(name) != "eta") return gs_set_error(GS_EINVAL, "gs_sim_set_field_async: only \"eta\"");
  if (dtype != s->p.dtype) return gs_set_error(GS_EINVAL, "gs_sim_set_field_async: dtype must be the simulation's");
  const size_t n = (size_t)s->N * s->p.nvariants;
  if (count != n) return gs_set_error(GS_EINVAL, "eta: %zu values, expected %zu", count, n);
  sim_graph_reset(s);
  s->spec_ready = false;
  s->staged = false;  // a field set given now replaces a staged one
  gs_cufft_invalidate(s);
  cudaStream_t st = pick_stream(s, stream);
  GS_CU(cudaMemcpyAsync(s->eta[s->cur], host, n * elt(s), cudaMemcpyHostToDevice, st), "upload");
  return GS_OK;
}

// ---------------------------------------------------------------------------
// a simulation split into slabs along axis 0, one slab per rank
// ---------------------------------------------------------------------------
// The reference holds a whole grid on one device (one cuFFT plan over it,
// src/dynamics_mart.cu:113-117).  Here a martensite grid nx x ny x nz is cut
// into R slabs of nx/R x-planes.  A step is three local phases with two
// all-to-all transposes and a halo exchange between them, which the caller
// performs (NCCL through torch.distributed on GPUs, device copies when all
// slabs share one device):
//   begin: z forward of eta^2 (or the spectra the last update left), y
//          forward, pack the spectra by destination kz range
//          [R][V][nx/R][ny][h/R] into `send`; the slab's two face planes
//          [2][V][ny][nz] into `halo_send`;
//   xpass: unpack the received pieces into x-pencils [V][nx][ny][h/R] (all
//          x for this rank's kz range), x forward -> B contraction -> x
//          inverse, pack by destination x range into `send`;
//   end:   unpack into the slab's spectra, y inverse, the fused update with
//          the neighbours' face planes as halos (and the next z forward).
// Every line transform, table point and cell update is the single-grid
// kernels' own arithmetic, so the slabs reproduce the one-device step bit for
// bit.  No load of another device's memory is issued here.
struct gs_slab {
  gs_sim* loc = nullptr;  // this rank's slab: fields, local spectra, stream, twiddles of y and z
  gs_sim geo;             // the whole grid's geometry and parameters (no buffers)
  int rank = 0, nranks = 1, x0 = 0, hr = 0;
  void* pencil = nullptr;  // x-pencil spectra [V][nx][ny][h/R]
  void* twx = nullptr;     // twiddles of the whole x axis
  void* btab = nullptr;    // octant B table of the whole grid (null: B formed per k)
  int btab_fields = 0;
  bool z_ready = false;    // the slab's spectra hold the z transforms of eta[cur]^2
};

template <typename T>
__global__ void k_copy5(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst, long long n, int d1, int d2, int d3,
                        int d4, long long s0, long long s1, long long s2, long long s3, long long t0, long long t1,
                        long long t2, long long t3) {
  // dims (d0, d1, d2, d3, d4), innermost contiguous on both sides
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int i4 = (int)(r % d4);
    r /= d4;
    const int i3 = (int)(r % d3);
    r /= d3;
    const int i2 = (int)(r % d2);
    r /= d2;
    const int i1 = (int)(r % d1);
    const long long i0 = r / d1;
    dst[i0 * t0 + i1 * t1 + i2 * t2 + i3 * t3 + i4] = src[i0 * s0 + i1 * s1 + i2 * s2 + i3 * s3 + i4];
  }
}

template <typename T>
static int copy5(const void* src, void* dst, const int d[5], const long long ss[4], const long long ts[4],
                 cudaStream_t st) {
  const long long n = (long long)d[0] * d[1] * d[2] * d[3] * d[4];
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_copy5<T><<<(unsigned)blocks, 256, 0, st>>>(reinterpret_cast<const cplx<T>*>(src), reinterpret_cast<cplx<T>*>(dst),
                                                 n, d[1], d[2], d[3], d[4], ss[0], ss[1], ss[2], ss[3], ts[0], ts[1],
                                                 ts[2], ts[3]);
  GS_CU(cudaGetLastError(), "slab transpose copy");
  return GS_OK;
}

static void free_slab(gs_slab* sl) {
  if (!sl) return;
  cudaDeviceSynchronize();
  for (void* q : {sl->pencil, sl->twx, sl->btab})
    if (q) cudaFree(q);
  if (sl->loc) free_sim(sl->loc);
  delete sl;
}

template <typename T> static int slab_init(gs_slab* sl) {
  gs_sim& g = sl->geo;
  const int gn0 = g.n0;
  // twiddles of the whole x axis
  std::vector<cplx<T>> tw(gn0);
  for (int m = 0; m < gn0; ++m) {
    const double a = 2.0 * M_PI * (double)m / (double)gn0;
    tw[m] = mk2((T)std::cos(a), (T)-std::sin(a));
  }
  GS_CU(cudaMalloc(&sl->twx, sizeof(cplx<T>) * gn0), "cudaMalloc x twiddles");
  GS_CU(cudaMemcpy(sl->twx, tw.data(), sizeof(cplx<T>) * gn0, cudaMemcpyHostToDevice), "upload x twiddles");
  // the octant table of the whole grid (as build_btab makes it)
  if (btab_symmetric(&g)) {
    ElasticConst<T> ec;
    build_elastic<T>(&g, 0, 1.0 / (double)g.N, ec);
    sl->btab_fields = ec.nb;
    const size_t npt = (size_t)(g.n0 / 2 + 1) * (g.n1 / 2 + 1) * (g.n2 / 2 + 1);
    GS_CU(cudaMalloc(&sl->btab, npt * btab_stride(ec.nb) * sizeof(T)), "cudaMalloc B table");
    GS_CU(launch_btab_fill<T>(ec, g.n0, g.n1, g.n2, reinterpret_cast<T*>(sl->btab), sl->loc->own_stream),
          "B table fill");
  }
  const size_t pb = sizeof(cplx<T>) * (size_t)g.p.nvariants * gn0 * g.n1 * sl->hr;
  GS_CU(cudaMalloc(&sl->pencil, pb), "cudaMalloc x pencils");
  GS_CU(cudaStreamSynchronize(sl->loc->own_stream), "slab init");
  return GS_OK;
}

extern "C" int gs_slab_create(const gs_params* p, int rank, int nranks, gs_slab** out) {
  if (!p || !out) return gs_set_error(GS_EINVAL, "gs_slab_create: null argument");
  *out = nullptr;
  if (p->model != GS_MODEL_MART) return gs_set_error(GS_EINVAL, "gs_slab_create: martensite only");
  if (nranks < 1 || rank < 0 || rank >= nranks)
    return gs_set_error(GS_EINVAL, "gs_slab_create: rank %d of %d", rank, nranks);
  if (p->nx < 2 || p->ny < 2 || p->nz < 2)
    return gs_set_error(GS_ENOTSUP, "gs_slab_create: a 3D grid is split (got %dx%dx%d)", p->nx, p->ny, p->nz);
  if (p->nx % nranks != 0 || (p->nz / 2) % nranks != 0)
    return gs_set_error(GS_EINVAL, "gs_slab_create: nx %d and nz/2 %d must be multiples of %d ranks", p->nx,
                        p->nz / 2, nranks);
  gs_slab* sl = new gs_slab();
  sl->geo.p = *p;
  int rc = canonicalize(&sl->geo);
  if (rc != GS_OK) {
    delete sl;
    return rc;
  }
  sl->rank = rank;
  sl->nranks = nranks;
  sl->x0 = rank * (p->nx / nranks);
  sl->hr = sl->geo.h / nranks;
  gs_params lp = *p;
  lp.nx = p->nx / nranks;
  if ((rc = gs_sim_create(&lp, &sl->loc)) != GS_OK) {
    delete sl;
    return rc;
  }
  // the slab's own table would describe a grid of nx/R planes: the whole
  // grid's table replaces it
  if (sl->loc->btab) cudaFree(sl->loc->btab);
  sl->loc->btab = nullptr;
  sl->loc->btab_state = -1;
  rc = p->dtype == GS_DTYPE_F64 ? slab_init<double>(sl) : slab_init<float>(sl);
  if (rc != GS_OK) {
    free_slab(sl);
    return rc;
  }
  *out = sl;
  return GS_OK;
}

extern "C" int gs_slab_destroy(gs_slab* sl) {
  free_slab(sl);
  return GS_OK;
}

extern "C" int gs_slab_info(const gs_slab* sl, gs_slab_geometry* out) {
  if (!sl || !out) return gs_set_error(GS_EINVAL, "gs_slab_info: null argument");
  const gs_sim* l = sl->loc;
  out->rank = sl->rank;
  out->nranks = sl->nranks;
  out->x0 = sl->x0;
  out->nx_local = l->n0;
  out->kz0 = sl->rank * sl->hr;
  out->nkz_local = sl->hr;
  out->a2a_bytes = (size_t)l->N * l->p.nvariants * elt(l);  // the slab's spectra: [R][V][nx/R][ny][h/R] complex
  out->halo_bytes = 2 * (size_t)l->n1 * l->n2 * l->p.nvariants * elt(l);
  out->step = l->step;
  return GS_OK;
}

extern "C" int gs_slab_set_field(gs_slab* sl, const char* name, const void* host, size_t count, int dtype) {
  if (!sl) return gs_set_error(GS_EINVAL, "gs_slab_set_field: null handle");
  if (!name || std::string(name) != "eta") return gs_set_error(GS_EINVAL, "gs_slab_set_field: only \"eta\"");
  sl->z_ready = false;
  return gs_sim_set_field(sl->loc, name, host, count, dtype);
}

extern "C" int gs_slab_get_field(gs_slab* sl, const char* name, void* host, size_t count, int dtype) {
  if (!sl) return gs_set_error(GS_EINVAL, "gs_slab_get_field: null handle");
  return gs_sim_get_field(sl->loc, name, host, count, dtype);
}

extern "C" int gs_slab_set_step(gs_slab* sl, int64_t step) {
  if (!sl || step < 0) return gs_set_error(GS_EINVAL, "gs_slab_set_step: bad argument");
  sl->loc->step = step;
  return GS_OK;
}

template <typename T> static int slab_begin(gs_slab* sl, void* send, void* halo_send, cudaStream_t st) {
  gs_sim* l = sl->loc;
  const int V = l->p.nvariants, R = sl->nranks, n0r = l->n0, n1 = l->n1, h = l->h, hr = sl->hr;
  const T* eta = reinterpret_cast<const T*>(l->eta[l->cur]);
  if (!sl->z_ready) {
    ZfwdArgs<T> za;
    memset(&za, 0, sizeof(za));
    for (int f = 0; f < V; ++f) {
      za.src[f] = eta + (long long)f * l->N;
      za.square[f] = 1;
    }
    za.dst = reinterpret_cast<cplx<T>*>(l->spec);
    za.rows_per_field = (long long)n0r * n1;
    za.nrows = za.rows_per_field * V;
    za.tw_h = twp<T>(l, 1);
    za.tw_n2 = twp<T>(l, 0);
    GS_CU(launch_zfwd<T>(za, h, st, l->sched.z_lines), "slab z forward");
  }
  YArgs<T> ya;
  ya.spec = reinterpret_cast<cplx<T>*>(l->spec);
  ya.n0 = n0r;
  ya.n1 = n1;
  ya.h = h;
  ya.tw = twp<T>(l, 2);
  GS_CU(launch_ypass<T>(ya, n1, V, -1, st, l->sched.y_cols, l->sched.y_radix), "slab y forward");
  // [V][x][y][kz = r hr + k] -> send [r][V][x][y][k]
  const int d[5] = {R, V, n0r, n1, hr};
  const long long ss[4] = {hr, (long long)n0r * n1 * h, (long long)n1 * h, h};
  const long long ts[4] = {(long long)V * n0r * n1 * hr, (long long)n0r * n1 * hr, (long long)n1 * hr, hr};
  GS_TRY(copy5<T>(l->spec, send, d, ss, ts, st));
  // face planes: [0] = plane 0, [1] = plane nx/R - 1, each [V][ny][nz]
  const size_t plane = (size_t)n1 * l->n2 * sizeof(T);
  char* hs = static_cast<char*>(halo_send);
  GS_CU(cudaMemcpy2DAsync(hs, plane, eta, (size_t)l->N * sizeof(T), plane, V, cudaMemcpyDeviceToDevice, st),
        "slab face plane");
  GS_CU(cudaMemcpy2DAsync(hs + plane * V, plane, eta + (size_t)(n0r - 1) * n1 * l->n2, (size_t)l->N * sizeof(T), plane,
                          V, cudaMemcpyDeviceToDevice, st),
        "slab face plane");
  return GS_OK;
}

template <typename T> static int slab_xpass(gs_slab* sl, const void* recv, void* send, cudaStream_t st) {
  gs_sim* l = sl->loc;
  gs_sim& g = sl->geo;
  const int V = l->p.nvariants, R = sl->nranks, n0r = l->n0, n1 = l->n1, hr = sl->hr, gn0 = g.n0;
  // recv [s][V][x][y][k] -> pencil [V][s nx/R + x][y][k]
  const int d[5] = {R, V, n0r, n1, hr};
  const long long rs[4] = {(long long)V * n0r * n1 * hr, (long long)n0r * n1 * hr, (long long)n1 * hr, hr};
  const long long ps[4] = {(long long)n0r * n1 * hr, (long long)gn0 * n1 * hr, (long long)n1 * hr, hr};
  GS_TRY(copy5<T>(recv, sl->pencil, d, rs, ps, st));
  XArgs<T> xa;
  memset(&xa, 0, sizeof(xa));
  xa.in = reinterpret_cast<cplx<T>*>(sl->pencil);
  xa.out = reinterpret_cast<cplx<T>*>(sl->pencil);
  xa.n0 = gn0;
  xa.n1 = n1;
  xa.n2 = g.n2;
  xa.h = hr;
  xa.hg = g.h;
  xa.kz_off = sl->rank * hr;
  xa.F = V;
  xa.G = V;
  xa.tw = reinterpret_cast<const cplx<T>*>(sl->twx);
  build_elastic<T>(&g, 0, 1.0 / (double)g.N, xa.ec);
  if (sl->btab && sl->btab_fields == V) {
    xa.btab = reinterpret_cast<const T*>(sl->btab);
    xa.bt_d1 = n1 / 2 + 1;
    xa.bt_d2 = g.n2 / 2 + 1;
    xa.bt_stride = btab_stride(V);
  }
  xa.tz_req = l->sched.x_cols;
  GS_CU(launch_xcontract<T>(xa, st), "slab x pass");
  // pencil -> send [s][V][x][y][k] (destination s takes its x range)
  GS_TRY(copy5<T>(sl->pencil, send, d, ps, rs, st));
  return GS_OK;
}

template <typename T> static int slab_end(gs_slab* sl, const void* recv, const void* halo_recv, cudaStream_t st) {
  gs_sim* l = sl->loc;
  const int V = l->p.nvariants, R = sl->nranks, n0r = l->n0, n1 = l->n1, h = l->h, hr = sl->hr;
  // recv [r][V][x][y][k] -> spectra [V][x][y][r hr + k]
  const int d[5] = {R, V, n0r, n1, hr};
  const long long rs[4] = {(long long)V * n0r * n1 * hr, (long long)n0r * n1 * hr, (long long)n1 * hr, hr};
  const long long ss[4] = {hr, (long long)n0r * n1 * h, (long long)n1 * h, h};
  GS_TRY(copy5<T>(recv, l->spec, d, rs, ss, st));
  YArgs<T> ya;
  ya.spec = reinterpret_cast<cplx<T>*>(l->spec);
  ya.n0 = n0r;
  ya.n1 = n1;
  ya.h = h;
  ya.tw = twp<T>(l, 2);
  GS_CU(launch_ypass<T>(ya, n1, V, 1, st, l->sched.y_cols, l->sched.y_radix), "slab y inverse");
  T* in = reinterpret_cast<T*>(l->eta[l->cur]);
  T* out = reinterpret_cast<T*>(l->eta[l->cur ^ 1]);
  MartArgs<T> ma;
  fill_mart_args<T>(l, ma, in, out);
  build_mart_p<T>(&sl->geo, sl->geo.p, l->step, ma.mc);  // the whole grid's stencil and constants
  ma.spec_next = reinterpret_cast<cplx<T>*>(l->spec);
  ma.halo = reinterpret_cast<const T*>(halo_recv);
  ma.cell_off = (long long)sl->x0 * n1 * l->n2;
  GS_CU(launch_mart_update<T>(ma, h, false, st, nullptr), "slab update");
  l->cur ^= 1;
  l->step += 1;
  sl->z_ready = true;
  return GS_OK;
}

static int slab_check(gs_slab* sl, const void* a, const void* b, const char* what) {
  if (!sl || !a || !b) return gs_set_error(GS_EINVAL, "%s: null argument", what);
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15u)
    return gs_set_error(GS_EINVAL, "%s: buffers must be 16-byte aligned", what);
  return GS_OK;
}

static int gs_slab_begin_body(gs_slab* sl, void* send, void* halo_send, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_slab_begin(gs_slab* sl, void* send, void* halo_send, void* stream) {
  return bc_after(gs_slab_begin_body(sl, send, halo_send, stream), static_cast<cudaStream_t>(stream));
}

static int gs_slab_begin_body(gs_slab* sl, void* send, void* halo_send, void* stream) {
  GS_TRY(slab_check(sl, send, halo_send, "gs_slab_begin"));
  cudaStream_t st = pick_stream(sl->loc, stream);
  return sl->loc->p.dtype == GS_DTYPE_F64 ? slab_begin<double>(sl, send, halo_send, st)
                                          : slab_begin<float>(sl, send, halo_send, st);
}

static int gs_slab_xpass_body(gs_slab* sl, const void* recv, void* send, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_slab_xpass(gs_slab* sl, const void* recv, void* send, void* stream) {
  return bc_after(gs_slab_xpass_body(sl, recv, send, stream), static_cast<cudaStream_t>(stream));
}

static int gs_slab_xpass_body(gs_slab* sl, const void* recv, void* send, void* stream) {
  GS_TRY(slab_check(sl, recv, send, "gs_slab_xpass"));
  cudaStream_t st = pick_stream(sl->loc, stream);
  return sl->loc->p.dtype == GS_DTYPE_F64 ? slab_xpass<double>(sl, recv, send, st)
                                          : slab_xpass<float>(sl, recv, send, st);
}

static int gs_slab_end_body(gs_slab* sl, const void* recv, const void* halo_recv, void* stream);
// the bounds-check build waits here and reports index violations (GS_EBOUNDS)
extern "C" int gs_slab_end(gs_slab* sl, const void* recv, const void* halo_recv, void* stream) {
  return bc_after(gs_slab_end_body(sl, recv, halo_recv, stream), static_cast<cudaStream_t>(stream));
}

static int gs_slab_end_body(gs_slab* sl, const void* recv, const void* halo_recv, void* stream) {
  GS_TRY(slab_check(sl, recv, halo_recv, "gs_slab_end"));
  cudaStream_t st = pick_stream(sl->loc, stream);
  return sl->loc->p.dtype == GS_DTYPE_F64 ? slab_end<double>(sl, recv, halo_recv, st)
                                          : slab_end<float>(sl, recv, halo_recv, st);
}
