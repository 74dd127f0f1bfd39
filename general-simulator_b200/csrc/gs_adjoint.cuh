// gs_adjoint.cuh -- the transposed (adjoint) martensite step.
//
// The forward step (baseline mode) is eta' = Phi(eta) = eta + dt RHS(eta)
// + noise with, per variant r,
//   RHS_r = L kappa lap eta_r - L f'_r(eta) + el eta_r R_r + lin_r eta_r,
//   R = B * (eta^2) (the Khachaturyan convolution), el = -2 L w_el.
// Its vector-Jacobian product with lam = dJ/deta' is
//   lam_r + dt [L kappa lap lam_r - L (H lam)_r + el (R_r lam_r + 2 eta_r Q_r)
//               + lin_r lam_r],   Q = B * (eta lam),
// because lap is self-adjoint on the periodic grid and B(k) is real, even
// and symmetric, so the transpose of the FFT convolution is the same
// convolution.  H is the Landau Hessian,
//   (H lam)_r = (A2 - 3 A4 eta_r^2 + A6 S^2 + 2 Ac (S - eta_r^2)) lam_r
//             + 4 eta_r (A6 S (eta . lam) + Ac sum_{q != r} eta_q lam_q),
// S = sum_q eta_q^2.  The noise is additive and drops out.  The same sweep
// accumulates lam . dPhi/dtheta for theta = kappa, A2, A4, A6, Ac and the
// eigenstrain scale s (eps -> s eps, so R ~ s^2 and lin ~ s).
//
// Q arrives as packed spectra after the y inverse (the forward chain with
// eta lam as its z input), exactly like R in the forward update; its z
// inverse runs here, in shared memory, before the cell sweep.
#pragma once
#include "gs_mart.cuh"

namespace gs {

// raw sums of the sweep; the host scales them into dJ/dtheta
enum { ADJ_ETA_LAP = 0, ADJ_ETA_LAM, ADJ_ETA3_LAM, ADJ_S2_ETA_LAM, ADJ_AC_LAM, ADJ_S_LAM, ADJ_N };

template <typename T> struct AdjArgs {
  const cplx<T>* spec;  // Q spectra [V][n0][n1][h]
  const T* eta;         // eta_n [V][N]
  const T* lam_in;      // dJ/deta_{n+1} [V][N]
  T* lam_out;           // dJ/deta_n [V][N]
  const T* R;           // R_n [V][N]
  int n0, n1, n2, lr;
  long long nrows;
  const cplx<T>* tw_h;
  const cplx<T>* tw_n2;
  MartConst<T> mc;
  double* partials;  // [gridDim.x][ADJ_N]
  FastDiv fd_n1, fd_upr, fd_v;
};

template <typename T, int H, int VM>
__global__ void __launch_bounds__(256, VM <= 4 ? 2 : 1) k_adj_update(AdjArgs<T> a) {
  using L = Line<T, H>;
  using V = cplx<T>;
  constexpr int CW = (2 * H) % 4 == 0 ? 4 : 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const MartConst<T>& mc = a.mc;
  const int Vn = mc.V;
  GS_BC_SMEM_GUARD((long long)(blockDim.x / L::P) * L::PAD, V, BC_UPD_SMEM)
  GS_BC_DECL(const long long fext = (long long)Vn * a.nrows * a.n2)
  {
    const int line = threadIdx.x / L::P, t = threadIdx.x % L::P;
    const int v = line % Vn, rr = line / Vn;
    const long long row = (long long)blockIdx.x * a.lr + rr;
    const bool act = rr < a.lr && row < a.nrows;
    V* sl = smb + line * L::PAD;
    const V* srow = a.spec + ((long long)v * a.nrows + (act ? row : 0)) * H;
    V r[L::R1];
    zinv_row<T, H>(srow, act, t, sl, a.tw_h, a.tw_n2, r, GS_BCX(((long long)v * a.nrows + (act ? row : 0)) * H),
                   GS_BCX(fext / 2));
    __syncthreads();
#pragma unroll
    for (int i = 0; i < L::R1; ++i) sl[L::out_pos(t, i)] = r[i];
    __syncthreads();
  }
  double acc[ADJ_N];
#pragma unroll
  for (int i = 0; i < ADJ_N; ++i) acc[i] = 0;
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const long long N = a.nrows * n2;
  const int upr = n2 / CW;
  const int nunits = a.lr * upr;
  // one thread per run of CW cells, all variants: the centre values of eta
  // and lambda and the sums S, eta.lambda are loaded and formed once
#pragma unroll 1
  for (int w = threadIdx.x; w < nunits; w += blockDim.x) {
    const int rr = (int)a.fd_upr.div((uint32_t)w), u = w - rr * upr;
    const long long row = (long long)blockIdx.x * a.lr + rr;
    if (row >= a.nrows) continue;
    const int x = (int)a.fd_n1.div((uint32_t)row), y = (int)(row - (long long)x * n1);
    const int xp = x + 1 == n0 ? 0 : x + 1, xm = x == 0 ? n0 - 1 : x - 1;
    const int yp = y + 1 == n1 ? 0 : y + 1, ym = y == 0 ? n1 - 1 : y - 1;
    const int z0 = u * CW;
    const long long rowb = row * n2, cell = rowb + z0;
    const long long oxp = ((long long)xp * n1 + y) * n2 + z0 - cell, oxm = ((long long)xm * n1 + y) * n2 + z0 - cell;
    const long long oyp = ((long long)x * n1 + yp) * n2 + z0 - cell, oym = ((long long)x * n1 + ym) * n2 + z0 - cell;
    const int ozl = (z0 == 0 ? n2 - 1 : z0 - 1) - z0, ozr = (z0 + CW == n2 ? 0 : z0 + CW) - z0;
    T e[VM][CW], l[VM][CW];
#pragma unroll
    for (int p = 0; p < VM; ++p)
      if (p < Vn) {
        ldv<CW>(a.eta + GS_BCR(0, (long long)p * N + cell, CW, fext, BC_UPD_ETA), e[p]);
        ldv<CW>(a.lam_in + GS_BCR(0, (long long)p * N + cell, CW, fext, BC_UPD_ETA), l[p]);
      }
    T S[CW], ed[CW];
#pragma unroll
    for (int j = 0; j < CW; ++j) {
      T s2 = 0, sd = 0;
#pragma unroll
      for (int p = 0; p < VM; ++p)
        if (p < Vn) {
          s2 += e[p][j] * e[p][j];
          sd += e[p][j] * l[p][j];
        }
      S[j] = s2;
      ed[j] = sd;
    }
#pragma unroll
    for (int q = 0; q < VM; ++q) {
      if (q >= Vn) break;
      const T* lq_ = a.lam_in + (long long)q * N + cell;
      GS_BC_DECL(const long long qoff = (long long)q * N + cell)
      T vxp[CW], vxm[CW], vyp[CW], vym[CW], Rq[CW];
      ldv<CW>(lq_ + GS_BCR(qoff, oxp, CW, fext, BC_UPD_ETA), vxp);
      ldv<CW>(lq_ + GS_BCR(qoff, oxm, CW, fext, BC_UPD_ETA), vxm);
      ldv<CW>(lq_ + GS_BCR(qoff, oyp, CW, fext, BC_UPD_ETA), vyp);
      ldv<CW>(lq_ + GS_BCR(qoff, oym, CW, fext, BC_UPD_ETA), vym);
      ldv<CW>(a.R + GS_BCR(0, (long long)q * N + cell, CW, fext, BC_UPD_AUX), Rq);
      const T zl_ = lq_[GS_BCO(qoff, ozl, fext, BC_UPD_ETA)], zr_ = lq_[GS_BCO(qoff, ozr, fext, BC_UPD_ETA)];
      const T* Qq = reinterpret_cast<const T*>(smb + (rr * Vn + q) * L::PAD) + z0;
      const T linq = mc.lin[q];
      T out[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) {
        const T eq = e[q][j], lq = l[q][j];
        const T zlv = j == 0 ? zl_ : l[q][j - 1];
        const T zrv = j == CW - 1 ? zr_ : l[q][j + 1];
        const T d0 = vxp[j] + vxm[j] - 2 * lq, d1 = vyp[j] + vym[j] - 2 * lq, d2 = zlv + zrv - 2 * lq;
        const T gl = mc.lapc[0] * d0 + mc.lapc[1] * d1 + mc.lapc[2] * d2;  // L kappa lap lam
        const T lap = mc.gcoef[0] * d0 + mc.gcoef[1] * d1 + mc.gcoef[2] * d2;
        const T e2 = eq * eq;
        const T off = ed[j] - eq * lq;
        const T Hl = (mc.A2 - 3 * mc.A4 * e2 + mc.A6 * S[j] * S[j] + 2 * mc.Ac * (S[j] - e2)) * lq +
                     4 * eq * (mc.A6 * S[j] * ed[j] + mc.Ac * off);
        const T Rv = Rq[j], Qv = Qq[j];
        out[j] = lq + mc.dt * (gl - mc.L * Hl + mc.el * (Rv * lq + 2 * eq * Qv) + linq * lq);
        const double el_ = (double)eq * (double)lq;
        acc[ADJ_ETA_LAP] += (double)eq * (double)lap;
        acc[ADJ_ETA_LAM] += el_;
        acc[ADJ_ETA3_LAM] += (double)e2 * el_;
        acc[ADJ_S2_ETA_LAM] += (double)S[j] * (double)S[j] * el_;
        acc[ADJ_AC_LAM] += 2.0 * ((double)S[j] - (double)e2) * el_;
        acc[ADJ_S_LAM] += (2.0 * (double)mc.el * (double)Rv + (double)linq) * el_;
      }
      stv<CW>(a.lam_out + GS_BCR(0, (long long)q * N + cell, CW, fext, BC_UPD_ETA_OUT), out);
    }
  }
  Neu nacc[ADJ_N];
#pragma unroll
  for (int i = 0; i < ADJ_N; ++i) nacc[i].add(acc[i]);
  block_reduce_store(nacc, ADJ_N, a.partials);
}

// Seed of the backward sweep at the final state:
//   lam = g + c * 2 eta R, g = 2 (eta - target) (loss mode) or the caller's
//   seed; partials[b] = block sums of (eta - target)^2 (loss mode).
template <typename T> struct AdjSeedArgs {
  const T* eta;
  const T* R;
  const T* target;  // loss mode, else null
  const T* seed;    // seed mode, else null
  T* lam;
  long long n;
  double c;         // dJ/dE_el * w_el * dV
  double* partials;
};

template <typename T> __global__ void k_adj_seed(AdjSeedArgs<T> a) {
  Neu acc[1];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
    const double e = (double)a.eta[i];
    double g = 0;
    if (a.target) {
      const double d = e - (double)a.target[i];
      acc[0].add(d * d);
      g = 2.0 * d;
    } else if (a.seed) {
      g = (double)a.seed[i];
    }
    a.lam[i] = (T)(g + a.c * 2.0 * e * (double)a.R[i]);
  }
  block_reduce_store(acc, 1, a.partials);
}

template <typename T> cudaError_t launch_adj_update(AdjArgs<T>& a, int H, cudaStream_t s, int* nblocks);
template <typename T> cudaError_t launch_adj_seed(AdjSeedArgs<T>& a, cudaStream_t s, int* nblocks);

}  // namespace gs
