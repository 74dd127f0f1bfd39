// gs_mart.cuh -- last sweep of the martensite step: z-axis C2R of the
// elastic potential R_p fused with the explicit Euler TDGL update.
//
// Replaces, in one pass over the field set, the reference's Grad_Mart_Kernel
// (src/dynamics_mart.cu:181-188), ChemiFor_Mart_Kernel (:222-250), the
// elastic product -wE R eta (:291), the dislocation force (:326), the noise
// (:372), the Euler update (:385) and Block_Mart_Kernel (:333-338), plus the
// ~20 Data<T> expression sweeps between them (include/datamath.th).
#pragma once
#include "gs_passes.cuh"

namespace gs {

// FP64 accumulators of the statistics sweep
enum {
  ACC_MASS = 0, ACC_EEL, ACC_ECHEM, ACC_EGRAD, ACC_EAPPL,
  ACC_FGRAD, ACC_FCHEM, ACC_FEL, ACC_FDISL, ACC_C,
  ACC_ETA2 = 10,
  ACC_VF = ACC_ETA2 + 8,
  ACC_N = ACC_VF + 8
};

template <typename T> struct MartConst {
  int V, refcompat, has_defect, has_K;
  T dt;
  T lapc[3];   // RHS stencil coefficient per canonical axis
  T gcoef[3];  // 1/d^2 per canonical axis (gradient energy)
  T A2, A4, A6, Ac, L, kappa;
  T el;               // RHS += el * R_p * eta_p
  T lin[8];           // RHS += lin_p * eta_p
  T kc;               // RHS += kc * K_p(x) * eta_p
  T a1, a2, a3, s, wC;  // refcompat chemical force
  T noise;            // eta += noise * xi
  T wel_half;         // energy: wel_half * eta^2 * R
  T appl[8];          // energy: -(appl_p + wD K_p) eta_p^2
  T wD;
  uint32_t k0, k1, sim, step;
};

template <typename T> struct MartArgs {
  const cplx<T>* spec;  // R spectra [V][n0][n1][h]
  const T* eta_in;
  T* eta_out;
  const T* defect;  // [N] or null
  const T* K;       // [V][N] or null
  int n0, n1, n2, lr;
  long long nrows;  // n0*n1
  const cplx<T>* tw_h;
  const cplx<T>* tw_n2;
  MartConst<T> mc;
  double* partials;  // [gridDim.x][ACC_N], statistics sweep only
  FastDiv fd_n1, fd_upr, fd_v;  // y extent, update runs per row, variants
  MartConst<T>* mcs;  // batched: constants of sim blockIdx.y in device memory
  T* r_out;           // when set: R_p written out [V][N] (adjoint checkpoints)
  int lr_req;         // rows per block asked by the autotuner (0 = default)
  cplx<T>* spec_next;  // FUSE: packed z spectra of eta'^2 for the next step (may be spec)
  const T* r_in;       // !ZF: R_p in real space [V][N] (a library FFT's output)
  T* sq_out;           // !ZF and FUSE: eta'^2 [V][N] (the next step's FFT input)
  // HALO (a slab of a simulation split along axis 0): the planes beyond the
  // slab's faces [2][V][n1][n2] (the neighbour below, then above), and the
  // global index of the slab's first cell (the noise counter)
  const T* halo;
  long long cell_off;
};

// advance the step counter of every batched simulation (keeps a captured
// graph of one step replayable: the noise counter lives in device memory)
template <typename T> __global__ void k_bump_step(MartConst<T>* mcs, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) mcs[i].step += 1;
}

struct Neu {  // Neumaier compensated sum (Neumaier 1974)
  double s = 0, c = 0;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x))
      c += (s - t) + x;
    else
      c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ double get() const { return s + c; }
};

// block sum of acc[0..n) into partials[blockIdx.x*n + i]
__device__ __forceinline__ void block_reduce_store(Neu* acc, int n, double* out) {
  __shared__ double red[32];
  for (int i = 0; i < n; ++i) {
    double v = acc[i].get();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      const int nw = (blockDim.x + 31) >> 5;
      double w = threadIdx.x < nw ? red[threadIdx.x] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
      if (threadIdx.x == 0) out[(long long)blockIdx.x * n + i] = w;
    }
  }
}

// vector loads of CW consecutive values (CW = 2 or 4, 8/16-byte aligned)
template <int CW> __device__ __forceinline__ void ldv(const float* p, float (&o)[CW]) {
  if constexpr (CW == 4) {
    const float4 x = *reinterpret_cast<const float4*>(p);
    o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w;
  } else {
    const float2 x = *reinterpret_cast<const float2*>(p);
    o[0] = x.x; o[1] = x.y;
  }
}
template <int CW> __device__ __forceinline__ void ldv(const double* p, double (&o)[CW]) {
#pragma unroll
  for (int j = 0; j < CW; j += 2) {
    const double2 x = *reinterpret_cast<const double2*>(p + j);
    o[j] = x.x; o[j + 1] = x.y;
  }
}
template <int CW> __device__ __forceinline__ void stv(float* p, const float (&o)[CW]) {
  if constexpr (CW == 4)
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
  else
    *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
}
template <int CW> __device__ __forceinline__ void stv(double* p, const double (&o)[CW]) {
#pragma unroll
  for (int j = 0; j < CW; j += 2) *reinterpret_cast<double2*>(p + j) = make_double2(o[j], o[j + 1]);
}

// The baseline right-hand side and Euler step of two cells of one variant
// as packed FP32x2 operations: lane by lane the operations and the order of
// the scalar path in k_mart_update (the same bits), in half the instructions.
//   g   = lapc0 (x+ + x-) + (lapc1 (y+ + y-) + lapc2 (z+ + z-))
//   rhs = eta (lin' + kc K - L (P0 - cA eta^2) + el R) + g
//   eta' = (eta + dt rhs + noise xi) (1 - defect)
__device__ __forceinline__ float2 mart_upd2(const MartConst<float>& mc, float2 et, float2 xp, float2 xm, float2 yp,
                                            float2 ym, float2 zs, float2 P0, float2 R, float2 K, float2 xi,
                                            float2 dfc, float lqc, float cA) {
  auto b = [](float s) { return make_float2(s, s); };
  const float2 vx = __fadd2_rn(xp, xm), vy = __fadd2_rn(yp, ym);
  float2 g = __fmul2_rn(b(mc.lapc[2]), zs);
  g = __ffma2_rn(b(mc.lapc[1]), vy, g);
  g = __ffma2_rn(b(mc.lapc[0]), vx, g);
  const float2 e2 = __fmul2_rn(et, et);
  const float2 m = __ffma2_rn(b(mc.kc), K, b(lqc));
  const float2 t1 = __ffma2_rn(b(-cA), e2, P0);
  const float2 s1 = __ffma2_rn(b(mc.el), R, m);
  const float2 coef = __ffma2_rn(b(-mc.L), t1, s1);
  const float2 rhs = __ffma2_rn(et, coef, g);
  float2 en = __ffma2_rn(b(mc.dt), rhs, et);
  en = __ffma2_rn(b(mc.noise), xi, en);
  if (mc.has_defect) en = __fmul2_rn(en, dfc);
  return en;
}

// One row group per block: the inverse z FFT of R_p for every (variant,
// row) line leaves R in shared memory; then each thread updates a run of CW
// cells (a quad, or a pair when n2 = 2) for all variants at once, so the
// centre values, the Landau coupling sums and the defect mask are loaded and
// formed once per run, and one Philox block per variant serves the run.
template <int VM, bool STATS> struct UpdBlocks {  // resident blocks asked of the register allocator
  static constexpr int v = (VM <= 4 && !STATS) ? 3 : 1;
};

// FUSE: the next step's z forward runs here too.  Each thread overwrites the
// R values of its own cells with eta'^2 (only it reads them), and after the
// sweep every (variant, row) line transforms its shared-memory row into the
// packed spectrum of the next step, in the rows of the spectrum buffer this
// block alone read: the next step then starts at the y forward pass.
//
// ZF = false: the same update without the z transforms, for the cuFFT
// comparator step -- R_p is read from a.r_in (real space) and, with FUSE,
// eta'^2 is written to a.sq_out for the library's next forward transform.
//
// HALO: the field is a slab of a grid split along axis 0; the x neighbours
// across its two faces come from a.halo, and the noise counter uses global
// cell indices.
template <typename T, int H, int VM, bool STATS, bool BATCH, bool FUSE = false, bool ZF = true, bool HALO = false>
__global__ void __launch_bounds__(256, UpdBlocks<VM, STATS>::v) k_mart_update(MartArgs<T> a) {
  using L = Line<T, H>;
  using V = cplx<T>;
  constexpr int CW = (2 * H) % 4 == 0 ? 4 : 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const MartConst<T>& mc = BATCH ? a.mcs[blockIdx.y] : a.mc;
  if (BATCH) {  // fields of sim blockIdx.y
    const long long off = (long long)blockIdx.y * mc.V * a.nrows * a.n2;
    a.spec += off / 2;
    a.eta_in += off;
    a.eta_out += off;
    if (FUSE) a.spec_next += off / 2;
  }
  const int Vn = mc.V;
  // logical extents (values): every field set of the launch (gridDim.y sims
  // when batched) and this block's simulation's offset in them
  GS_BC_DECL(const long long fext = (long long)(BATCH ? gridDim.y : 1) * Vn * a.nrows * a.n2,
             foff = BATCH ? (long long)blockIdx.y * Vn * a.nrows * a.n2 : 0,
             next = (long long)a.nrows * a.n2)
  if constexpr (ZF) {
    GS_BC_SMEM_GUARD((long long)(blockDim.x / L::P) * L::PAD, V, BC_UPD_SMEM)
    const int line = threadIdx.x / L::P, t = threadIdx.x % L::P;
    const int v = line % Vn, rr = line / Vn;
    const long long row = (long long)blockIdx.x * a.lr + rr;
    const bool act = rr < a.lr && row < a.nrows;
    V* sl = smb + line * L::PAD;
    const V* srow = a.spec + ((long long)v * a.nrows + (act ? row : 0)) * H;
    V r[L::R1];
    zinv_row<T, H>(srow, act, t, sl, a.tw_h, a.tw_n2, r,
                   GS_BCX(foff / 2 + ((long long)v * a.nrows + (act ? row : 0)) * H), GS_BCX(fext / 2));
    __syncthreads();
#pragma unroll
    for (int i = 0; i < L::R1; ++i) sl[L::out_pos(t, i)] = r[i];
    __syncthreads();
  }
  Neu acc[STATS ? ACC_N : 1];
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  // one simulation's field set holds fewer than 2^31 values (256 x 256 x
  // 512 x 8 at most), so cell offsets are 32-bit
  const int N = (int)(a.nrows * n2);
  const int upr = n2 / CW;
  const int nunits = a.lr * upr;
  // unit w -> (row rr, run u); runs of one row are consecutive so
  // neighbouring threads touch neighbouring cells
#pragma unroll 1
  for (int w = threadIdx.x; w < nunits; w += blockDim.x) {
    const int rr = (int)a.fd_upr.div((uint32_t)w), u = w - rr * upr;
    const int row = blockIdx.x * a.lr + rr;
    if (row >= a.nrows) continue;
    const int x = (int)a.fd_n1.div((uint32_t)row), y = row - x * n1;
    const int z0 = u * CW;
    const int cell = row * n2 + z0;
    // neighbour offsets relative to the run, the same for every variant
    const int sx = n1 * n2;
    const int oxp = x + 1 == n0 ? -(n0 - 1) * sx : sx, oxm = x == 0 ? (n0 - 1) * sx : -sx;
    const int oyp = y + 1 == n1 ? -(n1 - 1) * n2 : n2, oym = y == 0 ? (n1 - 1) * n2 : -n2;
    const int ozl = (z0 == 0 ? n2 - 1 : z0 - 1) - z0, ozr = (z0 + CW == n2 ? 0 : z0 + CW) - z0;
    const bool hlo = HALO && x == 0, hhi = HALO && x == n0 - 1;  // neighbour plane from the halo
    const long long hplane = (long long)n1 * n2;
    const int yz = cell - x * sx;
    const long long gcell = HALO ? (long long)cell + a.cell_off : (long long)cell;
    T e[VM][CW];
#pragma unroll
    for (int p = 0; p < VM; ++p)
      if (p < Vn) ldv<CW>(a.eta_in + GS_BCR(foff, p * N + cell, CW, fext, BC_UPD_ETA), e[p]);
    T s2[CW], s4[CW], pr[CW], P0[CW];
#pragma unroll
    for (int j = 0; j < CW; ++j) {
      T a2 = 0, a4 = 0, ap = 0;
#pragma unroll
      for (int p = 0; p < VM; ++p)
        if (p < Vn) {
          const T e2 = e[p][j] * e[p][j];
          ap += a2 * e2;
          a2 += e2;
          a4 += e2 * e2;
        }
      s2[j] = a2;
      s4[j] = a4;
      pr[j] = ap;
      // the part of the baseline Landau factor shared by every variant of
      // the cell: A2 + 2 Ac S + A6 S^2, S = sum of eta^2
      P0[j] = mc.A2 + a2 * ((T)2 * mc.Ac + mc.A6 * a2);
    }
    // baseline factored update (not the statistics sweep): per variant
    //   rhs = g + eta (m - L (P0 - (A4 + 2 Ac) eta^2) + el R),
    // g the stencil's neighbour sums, its centre term -2 sum(lapc) eta folded
    // into m = lin_p - 2 sum(lapc) (+ kc K_p)
    const T cA = mc.A4 + (T)2 * mc.Ac;
    const T lapsum2 = (T)2 * (mc.lapc[0] + mc.lapc[1] + mc.lapc[2]);
    T dfc[CW];
#pragma unroll
    for (int j = 0; j < CW; ++j) dfc[j] = 1;
    if (mc.has_defect) {
      ldv<CW>(a.defect + GS_BCR(0, cell, CW, next, BC_UPD_AUX), dfc);
#pragma unroll
      for (int j = 0; j < CW; ++j) dfc[j] = (T)1 - dfc[j];
    }
    // a run of 2 (n2 = 2 mod 4) may sit in the upper half of its Philox quad
    const bool hi_pair = CW == 2 && (gcell & 2);
#pragma unroll
    for (int q = 0; q < VM; ++q) {
      if (q >= Vn) break;
      const T* eq = a.eta_in + q * N + cell;
      GS_BC_DECL(const long long qoff = foff + (long long)q * N + cell, hext = 2 * Vn * hplane)
      T vxp[CW], vxm[CW], vyp[CW], vym[CW];
      ldv<CW>(hhi ? a.halo + GS_BCR(0, (long long)(Vn + q) * hplane + yz, CW, hext, BC_UPD_HALO)
                  : eq + GS_BCR(qoff, oxp, CW, fext, BC_UPD_ETA), vxp);
      ldv<CW>(hlo ? a.halo + GS_BCR(0, (long long)q * hplane + yz, CW, hext, BC_UPD_HALO)
                  : eq + GS_BCR(qoff, oxm, CW, fext, BC_UPD_ETA), vxm);
      ldv<CW>(eq + GS_BCR(qoff, oyp, CW, fext, BC_UPD_ETA), vyp);
      ldv<CW>(eq + GS_BCR(qoff, oym, CW, fext, BC_UPD_ETA), vym);
      const T el_ = eq[GS_BCO(qoff, ozl, fext, BC_UPD_ETA)], er_ = eq[GS_BCO(qoff, ozr, fext, BC_UPD_ETA)];
      const T* Rq = ZF ? reinterpret_cast<const T*>(smb + (rr * Vn + q) * L::PAD) + z0 : nullptr;
      T Rl[CW];
      if constexpr (ZF) {
        if constexpr (sizeof(T) == 4 && CW == 4 && L::PAD % 2 == 0) {
          // 16-byte shared-memory load: the line starts on a 16-byte boundary
          // when its padded length is even, and z0 is a multiple of 4
          const float4 R4 = *reinterpret_cast<const float4*>(Rq);
          Rl[0] = R4.x; Rl[1] = R4.y; Rl[2] = R4.z; Rl[3] = R4.w;
        } else {
#pragma unroll
          for (int j = 0; j < CW; ++j) Rl[j] = Rq[j];
        }
      } else {
        ldv<CW>(a.r_in + GS_BCR(0, q * N + cell, CW, (long long)Vn * next, BC_UPD_AUX), Rl);
      }
      T Kq[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) Kq[j] = 0;
      if (mc.has_K) ldv<CW>(a.K + GS_BCR(0, q * N + cell, CW, (long long)Vn * next, BC_UPD_AUX), Kq);
      T xi[4] = {0, 0, 0, 0};
      if (!STATS && mc.noise != (T)0)
        normal_quad<T>((uint32_t)(gcell >> 2), mc.step, mc.sim, (uint32_t)q, mc.k0, mc.k1, xi);
      const T lq = mc.lin[q];
      const T lqc = lq - lapsum2;
      T out[CW], rv[CW];
      bool done = false;  // the packed FP32 path below advanced the run
      if constexpr (sizeof(T) == 4 && CW == 4 && !STATS) {
        if (!mc.refcompat) {
          // z neighbour sums, then cells (0, 1) and (2, 3) as packed pairs
          const float zs[4] = {el_ + e[q][1], e[q][0] + e[q][2], e[q][1] + e[q][3], e[q][2] + er_};
#pragma unroll
          for (int j = 0; j < 4; j += 2) {
            const float2 en = mart_upd2(mc, make_float2(e[q][j], e[q][j + 1]), make_float2(vxp[j], vxp[j + 1]),
                                        make_float2(vxm[j], vxm[j + 1]), make_float2(vyp[j], vyp[j + 1]),
                                        make_float2(vym[j], vym[j + 1]), make_float2(zs[j], zs[j + 1]),
                                        make_float2(P0[j], P0[j + 1]), make_float2(Rl[j], Rl[j + 1]),
                                        make_float2(Kq[j], Kq[j + 1]), make_float2(xi[j], xi[j + 1]),
                                        make_float2(dfc[j], dfc[j + 1]), lqc, cA);
            out[j] = en.x;
            out[j + 1] = en.y;
            rv[j] = Rl[j];
            rv[j + 1] = Rl[j + 1];
          }
          done = true;
        }
      }
#pragma unroll
      for (int j = 0; j < CW; ++j) {
        if (done) break;
        const T et = e[q][j];
        const T zlv = j == 0 ? el_ : e[q][j - 1];
        const T zrv = j == CW - 1 ? er_ : e[q][j + 1];
        const T xij = CW == 2 ? (hi_pair ? xi[j + 2 < 4 ? j + 2 : 3] : xi[j]) : xi[j];
        if (!STATS && !mc.refcompat) {
          const T Rv = Rl[j];
          const T e2 = et * et;
          const T g = mc.lapc[0] * (vxp[j] + vxm[j]) + (mc.lapc[1] * (vyp[j] + vym[j]) + mc.lapc[2] * (zlv + zrv));
          const T m = lqc + mc.kc * Kq[j];
          const T coef = -mc.L * (P0[j] - cA * e2) + (mc.el * Rv + m);
          const T rhs = et * coef + g;
          T en = et + mc.dt * rhs + mc.noise * xij;
          if (mc.has_defect) en *= dfc[j];
          out[j] = en;
          rv[j] = Rv;
          continue;
        }
        const T d0 = vxp[j] + vxm[j] - 2 * et, d1 = vyp[j] + vym[j] - 2 * et, d2 = zlv + zrv - 2 * et;
        const T grad = mc.lapc[0] * d0 + mc.lapc[1] * d1 + mc.lapc[2] * d2;
        T chem;
        if (mc.refcompat) {
          const T se = mc.s * et;
          chem = et >= (T)0 ? -mc.wC * se * (mc.a1 - mc.a2 * se * se + mc.a3 * mc.s * mc.s * s2[j])
                            : (T)1000 * mc.wC * mc.a2 * et * et;
        } else {
          const T e2 = et * et;
          chem = -mc.L * (mc.A2 * et - mc.A4 * e2 * et + mc.A6 * s2[j] * s2[j] * et +
                          (T)2 * mc.Ac * et * (s2[j] - e2));
        }
        const T Rv = Rl[j];
        rv[j] = Rv;
        const T el = mc.el * Rv * et;
        const T lin = (lq + mc.kc * Kq[j]) * et;
        const T rhs = grad + chem + el + lin;
        T en = et + mc.dt * rhs + mc.noise * xij;
        if (mc.has_defect) en *= dfc[j];
        out[j] = en;
        if (STATS) {
          acc[ACC_MASS].add((double)et);
          acc[ACC_ETA2 + q].add((double)et * (double)et);
          acc[ACC_VF + q].add(fabs((double)et) > 0.5 ? 1.0 : 0.0);
          acc[ACC_EEL].add((double)mc.wel_half * (double)et * (double)et * (double)Rv);
          const double lg = (double)mc.gcoef[0] * d0 + (double)mc.gcoef[1] * d1 + (double)mc.gcoef[2] * d2;
          acc[ACC_EGRAD].add(-0.5 * (double)mc.kappa * (double)et * lg);
          acc[ACC_EAPPL].add(-((double)mc.appl[q] + (double)mc.wD * Kq[j]) * (double)et * (double)et);
          if (q == 0)
            acc[ACC_ECHEM].add((double)mc.A2 / 2 * s2[j] - (double)mc.A4 / 4 * s4[j] +
                               (double)mc.A6 / 6 * (double)s2[j] * s2[j] * s2[j] + (double)mc.Ac * pr[j]);
          acc[ACC_FGRAD].add((double)grad);
          acc[ACC_FCHEM].add((double)chem);
          acc[ACC_FEL].add((double)el);
          acc[ACC_FDISL].add((double)lin);
        }
      }
      if (!STATS) stv<CW>(a.eta_out + GS_BCR(foff, q * N + cell, CW, fext, BC_UPD_ETA_OUT), out);
      if (!BATCH && a.r_out) stv<CW>(a.r_out + GS_BCR(0, q * N + cell, CW, (long long)Vn * next, BC_UPD_AUX), rv);
      if (FUSE) {
        if constexpr (ZF) {
          T* sq = const_cast<T*>(Rq);
          if constexpr (sizeof(T) == 4 && CW == 4) {
            const float2 a = __fmul2_rn(make_float2(out[0], out[1]), make_float2(out[0], out[1]));
            const float2 b = __fmul2_rn(make_float2(out[2], out[3]), make_float2(out[2], out[3]));
            if constexpr (L::PAD % 2 == 0) {  // 16-byte aligned (as the load above)
              *reinterpret_cast<float4*>(sq) = make_float4(a.x, a.y, b.x, b.y);
            } else {  // 8-byte aligned: a line holds whole complex values
              reinterpret_cast<float2*>(sq)[0] = a;
              reinterpret_cast<float2*>(sq)[1] = b;
            }
          } else {
#pragma unroll
            for (int j = 0; j < CW; ++j) sq[j] = out[j] * out[j];
          }
        } else {
          T o2[CW];
#pragma unroll
          for (int j = 0; j < CW; ++j) o2[j] = out[j] * out[j];
          stv<CW>(a.sq_out + GS_BCR(0, q * N + cell, CW, (long long)Vn * next, BC_UPD_AUX), o2);
        }
      }
    }
  }
  if (STATS) block_reduce_store(acc, ACC_N, a.partials);
  if (FUSE && ZF) {
    __syncthreads();
    const int line = threadIdx.x / L::P, t = threadIdx.x % L::P;
    const int v = line % Vn, rr = line / Vn;
    const long long row = (long long)blockIdx.x * a.lr + rr;
    const bool act = rr < a.lr && row < a.nrows;
    V* sl = smb + line * L::PAD;
    V x[L::R1];
#pragma unroll
    for (int r = 0; r < L::R1; ++r) x[r] = sl[L::in_pos(t, r)];
    __syncthreads();
    zfwd_line<T, H>(x, t, sl, act ? a.spec_next + ((long long)v * a.nrows + row) * H : nullptr, a.tw_h, a.tw_n2,
                    GS_BCX(foff / 2 + ((long long)v * a.nrows + row) * H), GS_BCX(fext / 2));
  }
}

// Sum per-block partials [nb][n] into out[n] with Neumaier compensation.
__global__ void k_reduce_partials(const double* __restrict__ partials, int nb, int n, double* __restrict__ out);

}  // namespace gs
