// gs_passes.cuh -- the HBM sweeps of one phase-field step.
//
// Spectral layout ("packed half-complex"): a real field r[n0][n1][n2] has
// the spectrum P[n0][n1][h] (h = n2/2 complex), exactly the bytes of r.
//   z level: row (x,y): slot k in [1,h) holds S_k; slot 0 holds (S_0, S_h),
//            both real.
//   y level (after the y pass), kz slot 0 at fixed x holds two real-input
//            sequences a = S_0(y), b = S_h(y) packed as u = a + i b.  Their
//            y spectra A, B are Hermitian; slot j in [1,n1/2) holds A(j),
//            slot n1/2 + j holds B(j), slot 0 holds (A(0), A(n1/2)) and slot
//            n1/2 holds (B(0), B(n1/2)), all real.
//   x level: columns (ky slot, kz slot); the two columns (0,0) and (n1/2,0)
//            hold two real x sequences each (packed again) and are unpacked
//            with their Hermitian partner kx -> n0-kx inside the x pass.
// Every unpack is local to the line being transformed, so the passes keep
// power-of-two line lengths and coalesced tiles, and the spectrum never
// needs more bytes than the field.
//
// The reference computes the same spectra with cufftPlanMany C2C (complex
// copies of the real fields, twice the bytes) and a separate kernel per term
// (src/dynamics_mart.cu:281-303).
#pragma once
#include "gs_common.cuh"
#include "gs_fft.cuh"
#include "gs_philox.cuh"

namespace gs {

// ---------------------------------------------------------------------------
// B(n): the Khachaturyan tensor for one wave vector (src/gtensorb.cu:110-182),
// evaluated in registers from per-simulation constants instead of streamed
// from a [V][V][N] array.
// ---------------------------------------------------------------------------
// 1/sqrt and 1/x: hardware approximations in FP32 (within 2 ulp), exact in FP64
__device__ __forceinline__ float gs_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double gs_rsqrt(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float gs_rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double gs_rcp(double x) { return 1.0 / x; }

// out[g] += w * sum_f B_gf(k) in[f] for the Khachaturyan
//   B_gf(n) = C:ea_g:eb_f - (sigma_g n) . Omega(n) . (sigma_f n),
//   Omega(n)^-1_ij = C_iklj n_k n_l,
// evaluated as  out_g = sum_f a0_gf in_f - v_g . Omega (sum_f w_f in_f)
// with w_f = sigma_f n, v_g = sigma_g n (sigma = C:eps is symmetric), so
// no B entry is ever formed.  Omega^-1 is symmetric for a modulus with the
// major and minor symmetries; its six entries and the cofactor inverse
// follow src/gtensorb.cu:121-157 (|det| < 1e-8 -> Omega = 0 in the
// reference's rule).  k and the constants are in the canonical axis order.
template <typename T, int FM, int GM>
__device__ __forceinline__ void contract_k(const ElasticConst<T>& ec, const T k[3], const cplx<T> (&in)[FM],
                                           cplx<T> (&out)[GM], T w) {
  const T kk = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  T n[3] = {0, 0, 0};
  if (ec.refcompat) {
    if (!(kk <= (T)0.0000005 * (T)0.0000005)) {
      const T im = gs_rsqrt(kk);
      n[0] = k[0] * im;
      n[1] = k[1] * im;
      n[2] = k[2] * im;
    }
  } else {
    if (kk == (T)0) return;  // B(0) = 0
    const T im = gs_rsqrt(kk);
    n[0] = k[0] * im;
    n[1] = k[1] * im;
    n[2] = k[2] * im;
  }
  const T nn[6] = {n[0] * n[0], n[0] * n[1], n[0] * n[2], n[1] * n[1], n[1] * n[2], n[2] * n[2]};
  T m[6];  // m00 m01 m02 m11 m12 m22
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    T sacc = 0;
#pragma unroll
    for (int q = 0; q < 6; ++q) sacc += ec.qs[e][q] * nn[q];
    m[e] = sacc;
  }
  const T c00 = m[3] * m[5] - m[4] * m[4], c01 = m[2] * m[4] - m[1] * m[5], c02 = m[1] * m[4] - m[2] * m[3];
  const T c11 = m[0] * m[5] - m[2] * m[2], c12 = m[1] * m[2] - m[0] * m[4], c22 = m[0] * m[3] - m[1] * m[1];
  const T det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  const bool ok = ec.refcompat ? (det >= (T)1e-8 || det <= (T)-1e-8) : (det != (T)0);
  const T id = ok ? gs_rcp(det) : (T)0;
  const T o00 = c00 * id, o01 = c01 * id, o02 = c02 * id, o11 = c11 * id, o12 = c12 * id, o22 = c22 * id;
  // u = sum_f (sigma_f n) in_f
  cplx<T> u0 = mk2((T)0, (T)0), u1 = u0, u2 = u0;
#pragma unroll
  for (int f = 0; f < FM; ++f) {
    if (f < ec.nb) {
      const T w0 = ec.sb[f][0][0] * n[0] + ec.sb[f][0][1] * n[1] + ec.sb[f][0][2] * n[2];
      const T w1 = ec.sb[f][1][0] * n[0] + ec.sb[f][1][1] * n[1] + ec.sb[f][1][2] * n[2];
      const T w2 = ec.sb[f][2][0] * n[0] + ec.sb[f][2][1] * n[1] + ec.sb[f][2][2] * n[2];
      u0 = u0 + in[f] * w0;
      u1 = u1 + in[f] * w1;
      u2 = u2 + in[f] * w2;
    }
  }
  const cplx<T> p0 = u0 * o00 + u1 * o01 + u2 * o02;
  const cplx<T> p1 = u0 * o01 + u1 * o11 + u2 * o12;
  const cplx<T> p2 = u0 * o02 + u1 * o12 + u2 * o22;
#pragma unroll
  for (int g = 0; g < GM; ++g) {
    if (g < ec.na) {
      const T v0 = ec.sa[g][0][0] * n[0] + ec.sa[g][0][1] * n[1] + ec.sa[g][0][2] * n[2];
      const T v1 = ec.sa[g][1][0] * n[0] + ec.sa[g][1][1] * n[1] + ec.sa[g][1][2] * n[2];
      const T v2 = ec.sa[g][2][0] * n[0] + ec.sa[g][2][1] * n[1] + ec.sa[g][2][2] * n[2];
      cplx<T> acc = mk2((T)0, (T)0) - (p0 * v0 + p1 * v1 + p2 * v2);
#pragma unroll
      for (int f = 0; f < FM; ++f)
        if (f < ec.nb) acc = acc + in[f] * ec.a0[g][f];
      out[g] = out[g] + acc * w;
    }
  }
}

// folded signed index of spectral index i on an axis of length n
__device__ __forceinline__ int fold_idx(int i, int n, int refcompat) {
  return refcompat ? (i < n / 2 ? i : i - n) : (2 * i < n ? i : i - n);
}

// out = scale * B(k) in at spectral index (ix, iy, iz) of the canonical grid.
// B is averaged over the sign of Nyquist components, so that the stored half
// spectrum stays Hermitian (equal to the real part of the reference's C2C
// inverse, which sees both signs through the conjugate partner).
template <typename T, int FM, int GM>
__device__ __forceinline__ void contract_at(const ElasticConst<T>& ec, const int (&nn)[3], int ix, int iy, int iz,
                                            const cplx<T> (&in)[FM], cplx<T> (&out)[GM], T mult = (T)1) {
  const int id[3] = {ix, iy, iz};
  int m[3];
  bool nyq = false;
  bool isnyq[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    m[c] = fold_idx(id[c], nn[c], ec.refcompat);
    isnyq[c] = (nn[c] > 1) && (nn[c] % 2 == 0) && (2 * id[c] == nn[c]);
    nyq |= isnyq[c];
  }
#pragma unroll
  for (int g = 0; g < GM; ++g) out[g] = mk2((T)0, (T)0);
  const T w = (nyq ? (T)0.5 * ec.scale : ec.scale) * mult;
  const int trips = nyq ? 2 : 1;
#pragma unroll 1
  for (int trip = 0; trip < trips; ++trip) {
    T k[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) k[c] = ec.kscale[c] * (T)((trip && isnyq[c]) ? -m[c] : m[c]);
    contract_k<T, FM, GM>(ec, k, in, out, w);
  }
}

// ---------------------------------------------------------------------------
// z forward: real rows -> packed half spectrum, with a fused prologue.
// ---------------------------------------------------------------------------
// z forward of one row held as H complex values v (in_pos order: the pairs
// (r[2m], r[2m+1]) of the real row): the length-H FFT, then the split into
// the packed half spectrum, written to dst (nullptr: the line is inactive).
// sl is the line's shared buffer (PAD values).  All threads of the block call it.
// Register of thread 0 of a line that holds the partner Z_{H-k} of its
// register i (out_pos order; i = 0 is k = 0, its own partner).
template <int R1, int R2> __device__ __forceinline__ constexpr int zfwd_partner0(int i) {
  return i / R2 == 0 ? (i % R2 == 0 ? 0 : R2 - i % R2) : (R1 / R2 - i / R2) * R2 + (R2 - 1 - i % R2);
}

template <typename T, int H>
__device__ __forceinline__ void zfwd_line(cplx<T> (&v)[Line<T, H>::R1], int t, cplx<T>* sl, cplx<T>* dst,
                                          const cplx<T>* __restrict__ tw_h, const cplx<T>* __restrict__ tw_n2,
                                          long long bc_doff, long long bc_dext) {
  using L = Line<T, H>;
  using V = cplx<T>;
  auto sm = [sl](int pos) -> V& { return sl[pos]; };
  L::template run<-1>(v, t, sm, tw_h);
  // The split needs Z_k and Z_{H-k}: for t != 0 the partner is register
  // R1-1-i of thread P-t of the same line, exchanged by a shuffle; thread 0
  // holds its own partners (zfwd_partner0).  No shared memory, no barrier.
  const unsigned wb = threadIdx.x & ~31u;
  const unsigned mask = blockDim.x - wb >= 32 ? 0xffffffffu : ((1u << (blockDim.x - wb)) - 1u);
  const int src = (L::P - t) % L::P;
#pragma unroll
  for (int i = 0; i < L::R1; ++i) {
    V zm;
    if constexpr (L::P > 1) {
      const V send = v[L::R1 - 1 - i];
      zm.x = __shfl_sync(mask, send.x, src, L::P);
      zm.y = __shfl_sync(mask, send.y, src, L::P);
      if (t == 0) zm = v[zfwd_partner0<L::R1, L::R2>(i)];
    } else {
      zm = v[zfwd_partner0<L::R1, L::R2>(i)];
    }
    if (dst) {
      const int k = L::out_pos(t, i);
      const V zk = v[i];
      V s;
      if (k == 0) {
        s = mk2(zk.x + zk.y, zk.x - zk.y);
      } else {
        const V Pz = padd(zk, zm), Mz = psub(zk, zm);
        const V e = mk2((T)0.5 * Pz.x, (T)0.5 * Mz.y);
        const V d = mk2(Mz.x, Pz.y);  // zk - conj(zm)
        const V o = mk2((T)0.5 * d.y, (T)-0.5 * d.x);  // -i d / 2
        s = e + cmul(o, __ldg(&tw_n2[k]));
      }
      dst[GS_BCO(bc_doff, k, bc_dext, BC_ZFWD_DST)] = s;
    }
  }
}

template <typename T> struct ZfwdArgs {
  const T* src[2 * GS_MAXF];   // row source of each field (n0*n1 rows of n2)
  int square[2 * GS_MAXF];     // 1: transform src^2 (eta^2), 0: src
  const T* mul[2 * GS_MAXF];   // when set: transform src * mul (eta lam, adjoint)
  const T* src0;               // when set: field f at src0 + f * fstride (batches)
  long long fstride;
  int square0;
  cplx<T>* dst;            // [F][n0][n1][h]
  long long rows_per_field;
  long long nrows;         // F * rows_per_field
  int lpc;                 // lines per block
  const cplx<T>* tw_h;     // w_h^m
  const cplx<T>* tw_n2;    // w_n2^m
};

template <typename T, int H>
__global__ void k_zfwd(ZfwdArgs<T> a) {
  using L = Line<T, H>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int t = threadIdx.x % L::P, line = threadIdx.x / L::P;
  const long long row = (long long)blockIdx.x * a.lpc + line;
  const bool act = row < a.nrows;
  GS_BC_SMEM_GUARD((long long)(blockDim.x / L::P) * L::PAD, V, BC_ZFWD_SMEM)
  V* sl = smb + line * L::PAD;
  V v[L::R1];
  if (act) {
    const int f = (int)(row / a.rows_per_field);
    const long long rin = row - (long long)f * a.rows_per_field;
    const V* src = reinterpret_cast<const V*>(a.src0 ? a.src0 + f * a.fstride : a.src[f]) + rin * H;
    const int sq = a.src0 ? a.square0 : a.square[f];
    const T* mp = a.src0 ? nullptr : a.mul[f];
    // source extent in complex pairs: one field's rows, or all fields of src0
    GS_BC_DECL(const long long soff = (a.src0 ? f * (a.fstride / 2) : 0) + rin * H,
               sext = a.rows_per_field * H +
                      (a.src0 ? (a.nrows / a.rows_per_field - 1) * (a.fstride / 2) : 0))
#pragma unroll
    for (int r = 0; r < L::R1; ++r) {
      V x = src[GS_BCO(soff, L::in_pos(t, r), sext, BC_ZFWD_SRC)];
      if (sq) x = mk2(x.x * x.x, x.y * x.y);
      if (mp) {
        const V m =
            reinterpret_cast<const V*>(mp)[GS_BCI(rin * H + L::in_pos(t, r), a.rows_per_field * H, BC_ZFWD_SRC)];
        x = mk2(x.x * m.x, x.y * m.y);
      }
      v[r] = x;
    }
  } else {
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[r] = mk2((T)0, (T)0);
  }
  zfwd_line<T, H>(v, t, sl, act ? a.dst + row * H : nullptr, a.tw_h, a.tw_n2, GS_BCX(row * H), GS_BCX(a.nrows * H));
}

// ---------------------------------------------------------------------------
// y pass (forward or inverse) over columns of TZ consecutive kz slots.
// ---------------------------------------------------------------------------
template <typename T> struct YArgs {
  cplx<T>* spec;  // [F][n0][n1][h]
  int n0, n1, h, tz;
  const cplx<T>* tw;  // w_n1^m
};

// R1: the first-stage radix of the line plan (the default plan, or the
// alternative split the autotuner may pick)
template <typename T, int N1, int DIR, int R1 = Plan<N1>::R1>
__global__ void k_ypass(YArgs<T> a) {
  using L = Line<T, N1, R1>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int TZ = a.tz;
  const int c = threadIdx.x % TZ, t = threadIdx.x / TZ;
  const int kz0 = blockIdx.x * TZ, x = blockIdx.y, f = blockIdx.z;
  const int h = a.h;
  GS_BC_SMEM_GUARD((long long)TZ * L::PAD, V, BC_Y_SMEM)
  V* base = a.spec + ((long long)(f * a.n0 + x) * N1) * h + kz0 + c;
  // the spectrum's logical extent: gridDim.z fields of n0 x N1 x h
  GS_BC_DECL(const long long boff = ((long long)(f * a.n0 + x) * N1) * h + kz0 + c,
             bext = (long long)gridDim.z * a.n0 * N1 * h)
  auto sm = [smb, TZ, c](int pos) -> V& { return smb[pos * TZ + c]; };
  const bool special = (kz0 == 0);
  constexpr int HH = N1 / 2;
  V v[L::R1];
  if (DIR < 0 || !special) {
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[r] = base[GS_BCO(boff, (long long)L::in_pos(t, r) * h, bext, BC_Y_SPEC)];
  } else {
    // inverse, tile holding kz slot 0: rebuild U(ky) = A(ky) + i B(ky)
#pragma unroll
    for (int r = 0; r < L::R1; ++r) {
      const int p = L::in_pos(t, r);
      sm(p) = base[GS_BCO(boff, (long long)p * h, bext, BC_Y_SPEC)];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < L::R1; ++r) {
      const int ky = L::in_pos(t, r);
      if (c != 0) {
        v[r] = sm(ky);
      } else {
        V A, B;
        if (ky == 0) {
          A = mk2(sm(0).x, (T)0);
          B = mk2(sm(HH).x, (T)0);
        } else if (ky == HH) {
          A = mk2(sm(0).y, (T)0);
          B = mk2(sm(HH).y, (T)0);
        } else if (ky < HH) {
          A = sm(ky);
          B = sm(HH + ky);
        } else {
          A = conjg(sm(N1 - ky));
          B = conjg(sm(HH + N1 - ky));
        }
        v[r] = mk2(A.x - B.y, A.y + B.x);
      }
    }
    __syncthreads();
  }
  L::template run<DIR>(v, t, sm, a.tw);
  if (DIR > 0 || !special) {
#pragma unroll
    for (int i = 0; i < L::R1; ++i) base[GS_BCO(boff, (long long)L::out_pos(t, i) * h, bext, BC_Y_SPEC)] = v[i];
  } else {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < L::R1; ++i) sm(L::out_pos(t, i)) = v[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < L::R1; ++i) {
      const int s = L::out_pos(t, i);
      V o;
      if (c != 0) {
        o = sm(s);
      } else if (s == 0) {
        o = mk2(sm(0).x, sm(HH).x);
      } else if (s == HH) {
        o = mk2(sm(0).y, sm(HH).y);
      } else if (s < HH) {
        const V u = sm(s), w = sm(N1 - s);
        o = mk2((T)0.5 * (u.x + w.x), (T)0.5 * (u.y - w.y));
      } else {
        const int j = s - HH;
        const V u = sm(j), w = sm(N1 - j);
        const V d = mk2(u.x - w.x, u.y + w.y);  // u - conj(w)
        o = mk2((T)0.5 * d.y, (T)-0.5 * d.x);
      }
      base[GS_BCO(boff, (long long)s * h, bext, BC_Y_SPEC)] = o;
    }
  }
}

// ---------------------------------------------------------------------------
// x pass: forward x FFT of F fields -> B(n) contraction -> inverse x FFT of
// G fields.  One block per (kz tile, ky slot); one thread group per field,
// so the F line FFTs of a tile run side by side.  The spectra meet in
// shared memory for the contraction, which every thread of the block shares.
// ---------------------------------------------------------------------------
// Semi-implicit CH/AC update of the precipitate in k space
// (src/dynamics_precipitate.cu:197-206,234-248): inputs [c, mu, eta_0, g_0,
// eta_1, g_1, ...], outputs [c', eta'_0..V-1], with K(k) = sum of per-axis tables
// (|k|^2 of the 3.14 vector in refcompat, the seven-point symbol otherwise).
template <typename T> struct PrecipUpd {
  int V, mass_proj;
  T dtM, dtL, kc, ke;      // dt*M, dt*L, kappa_c, kappa_eta
  T scale;                 // 1/N of the unnormalised transforms
  const T* ktab[3];        // K contribution per canonical axis and index
};

template <typename T> struct XArgs {
  const cplx<T>* in;  // [F][n0][n1][h]
  cplx<T>* out;       // [G][n0][n1][h] (may alias in)
  int n0, n1, n2, h, tz, F, G, groups;
  const cplx<T>* tw;  // w_n0^m
  ElasticConst<T> ec;
  PrecipUpd<T> pu;
  const T* simscale;  // batched: contraction multiplier of sim blockIdx.z (null: 1)
  int nsim;           // batched simulations (grid z), 0 or 1 for one
  // octant table of B (TableOp): entry of |folded index| (mx, my, mz) at
  // btab + ((mx * bt_d1 + my) * bt_d2 + mz) * bt_stride
  const T* btab;
  int bt_d1, bt_d2, bt_stride;
  int tz_req;  // column tile asked by the autotuner (0 = default)
  // x-pencil of a slab-decomposed simulation: this array holds the kz slots
  // kz_off .. kz_off + h - 1 of a spectrum of hg slots (hg = 0: the whole
  // spectrum, kz_off = 0); the kz = 0 packed columns exist only where
  // kz_off = 0, and wave vectors use the global slot index
  int kz_off, hg;
};

// per-point operations of the x pass
struct ContractOp {
  template <typename T, int FM, int GM>
  __device__ __forceinline__ static void apply(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                               const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    contract_at<T, FM, GM>(a.ec, nn, ix, iy, iz, in, out, a.simscale ? a.simscale[blockIdx.z] : (T)1);
  }
};
// Upper triangle of a symmetric FM x FM matrix, row by row: slot of (i, j), i <= j.
template <int FM> __host__ __device__ constexpr int tri_slot(int i, int j) {
  return i <= j ? i * FM - i * (i - 1) / 2 + (j - i) : j * FM - j * (j - 1) / 2 + (i - j);
}
template <int FM> struct TriStride {  // entries per table point, rounded to an even count
  static constexpr int v = ((FM * (FM + 1) / 2) + 1) & ~1;
};

// B(k) read from the octant table (B even in every axis: see the table fill).
// The table point of kx is also that of n0 - kx, so the x pass loads it once
// for the pair (kx_pair).
struct TableOp {
  static constexpr bool kx_pair = true;
  template <typename T, int FM>
  __device__ __forceinline__ static void load(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                              T (&bv)[TriStride<FM>::v]) {
    constexpr int S = TriStride<FM>::v;
    const int rc = a.ec.refcompat;
    int mx = fold_idx(ix, nn[0], rc), my = fold_idx(iy, nn[1], rc), mz = fold_idx(iz, nn[2], rc);
    mx = mx < 0 ? -mx : mx;
    my = my < 0 ? -my : my;
    mz = mz < 0 ? -mz : mz;
    const T* pt = a.btab + GS_BCI((((long long)mx * a.bt_d1 + my) * a.bt_d2 + mz) * S,
                                  (long long)(a.n0 / 2 + 1) * a.bt_d1 * a.bt_d2 * S, BC_X_TAB);
    if constexpr (sizeof(T) == 4 && S % 4 == 0) {
      const float4* b4 = reinterpret_cast<const float4*>(pt);
#pragma unroll
      for (int i = 0; i < S / 4; ++i) {
        const float4 w = __ldg(b4 + i);
        bv[4 * i] = w.x;
        bv[4 * i + 1] = w.y;
        bv[4 * i + 2] = w.z;
        bv[4 * i + 3] = w.w;
      }
    } else {
      const cplx<T>* b2 = reinterpret_cast<const cplx<T>*>(pt);
#pragma unroll
      for (int i = 0; i < S / 2; ++i) {
        const cplx<T> w = __ldg(b2 + i);
        bv[2 * i] = w.x;
        bv[2 * i + 1] = w.y;
      }
    }
  }
  template <typename T, int FM, int GM, bool EX = false>
  __device__ __forceinline__ static void contract(const XArgs<T>& a, const T (&bv)[TriStride<FM>::v],
                                                  const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    static_assert(FM == GM, "square tables only");
    const T mult = a.simscale ? a.simscale[blockIdx.z] : (T)1;
#pragma unroll
    for (int g = 0; g < GM; ++g) {
      cplx<T> acc = mk2((T)0, (T)0);
#pragma unroll
      for (int f = 0; f < FM; ++f)
        if (EX || f < a.F) acc = acc + in[f] * bv[tri_slot<FM>(g, f)];
      out[g] = acc * mult;
    }
  }
  template <typename T, int FM, int GM>
  __device__ __forceinline__ static void apply(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                               const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    T bv[TriStride<FM>::v];
    load<T, FM>(a, nn, ix, iy, iz, bv);
    contract<T, FM, GM>(a, bv, in, out);
  }
};

template <class Op, class = void> struct KxPair {
  static constexpr bool v = false;
};
template <class Op> struct KxPair<Op, decltype(void(Op::kx_pair))> {
  static constexpr bool v = Op::kx_pair;
};

// Octant table of the scaled, Nyquist-averaged B(k) of a square contraction
// (F = G = V, B symmetric): one point per |folded index| triple, filled by
// contracting unit inputs with contract_at, so that it holds exactly the
// numbers the on-the-fly contraction forms.  Valid when B is even in each
// axis separately (checked on the host: no shear coupling of any axis with
// extent > 1 in the stresses or the modulus), which makes B(+-mx, +-my,
// +-mz) one value.
template <typename T, int FM>
__global__ void k_btab_fill(ElasticConst<T> ec, int n0, int n1, int n2, int d0, int d1, int d2, T* tab) {
  constexpr int S = TriStride<FM>::v;
  const long long npt = (long long)d0 * d1 * d2;
  const int nn[3] = {n0, n1, n2};
  const int V = ec.nb;
  for (long long pt = (long long)blockIdx.x * blockDim.x + threadIdx.x; pt < npt;
       pt += (long long)gridDim.x * blockDim.x) {
    const int mz = (int)(pt % d2), my = (int)((pt / d2) % d1), mx = (int)(pt / ((long long)d1 * d2));
    T* o = tab + pt * S;
#pragma unroll 1
    for (int i = 0; i < S; ++i) o[i] = (T)0;
#pragma unroll 1
    for (int f = 0; f < V; ++f) {
      cplx<T> in[FM], out[FM];
#pragma unroll
      for (int q = 0; q < FM; ++q) in[q] = mk2(q == f ? (T)1 : (T)0, (T)0);
      contract_at<T, FM, FM>(ec, nn, mx, my, mz, in, out);
#pragma unroll
      for (int g = 0; g < FM; ++g)
        if (g <= f) o[tri_slot<FM>(g, f)] = out[g].x;
    }
  }
}

// A semi-implicit symbol scale / den (den >= 1, far below 2^126): FP32
// through the hardware reciprocal (__fdividef, within 2 ulp), FP64 by the
// IEEE division.
__device__ __forceinline__ float sym_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double sym_div(double a, double b) { return a / b; }

struct PrecipOp {
  template <typename T, int FM, int GM>
  __device__ __forceinline__ static void apply(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                               const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    const PrecipUpd<T>& u = a.pu;
    // the per-axis tables hold n0, n1 and n2 entries
    const T K = u.ktab[0][GS_BCI(ix, a.n0, BC_X_KTAB)] + u.ktab[1][GS_BCI(iy, a.n1, BC_X_KTAB)] +
                u.ktab[2][GS_BCI(iz, a.n2, BC_X_KTAB)];
    const T ic = sym_div(u.scale, (T)1 + u.dtM * u.kc * K * K);
    const T ie = sym_div(u.scale, (T)1 + u.dtL * u.ke * K);
#pragma unroll
    for (int g = 0; g < GM; ++g) out[g] = mk2((T)0, (T)0);
    out[0] = (in[0] - in[1] * (u.dtM * K)) * ic;
    if (u.mass_proj && ix == 0 && iy == 0 && iz == 0) out[0] = mk2((T)0, (T)0);
    // inputs interleaved per variant: in[2 + 2p] = eta_p, in[3 + 2p] = g_p
#pragma unroll
    for (int p = 0; p < GM - 1; ++p)
      if (p < u.V && 3 + 2 * p < FM) out[1 + p] = (in[2 + 2 * p] - in[3 + 2 * p] * u.dtL) * ie;
  }
};

// The same update, one (field, force) pair per grid-z slice: slice 0 is
// (c, mu) -> c', slice 1 + p is (eta_p, g_p) -> eta_p' (the chain-2 fields
// are stored pair after pair, its outputs one after another, so the batched
// slice offsets of the x pass address them directly).  Lighter blocks than
// one block over all 2V + 2 fields.
struct PrecipPairOp {
  template <typename T, int FM, int GM>
  __device__ __forceinline__ static void apply(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                               const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    const PrecipUpd<T>& u = a.pu;
    // the per-axis tables hold n0, n1 and n2 entries
    const T K = u.ktab[0][GS_BCI(ix, a.n0, BC_X_KTAB)] + u.ktab[1][GS_BCI(iy, a.n1, BC_X_KTAB)] +
                u.ktab[2][GS_BCI(iz, a.n2, BC_X_KTAB)];
#pragma unroll
    for (int g = 0; g < GM; ++g) out[g] = mk2((T)0, (T)0);
    if (blockIdx.z == 0) {
      const T ic = sym_div(u.scale, (T)1 + u.dtM * u.kc * K * K);
      out[0] = (in[0] - in[1] * (u.dtM * K)) * ic;
      if (u.mass_proj && ix == 0 && iy == 0 && iz == 0) out[0] = mk2((T)0, (T)0);
    } else {
      const T ie = sym_div(u.scale, (T)1 + u.dtL * u.ke * K);
      out[0] = (in[0] - in[1] * u.dtL) * ie;
    }
  }
};

// The Allen-Cahn half of the same update when the real-space sweep already
// formed u_p = eta_p - dt L g_p: one field per grid-z slice, eta_p' = D u_p
// with D = 1/(1 + dt L kappa_eta K).
struct PrecipEtaOp {
  template <typename T, int FM, int GM>
  __device__ __forceinline__ static void apply(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                               const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    const PrecipUpd<T>& u = a.pu;
    // the per-axis tables hold n0, n1 and n2 entries
    const T K = u.ktab[0][GS_BCI(ix, a.n0, BC_X_KTAB)] + u.ktab[1][GS_BCI(iy, a.n1, BC_X_KTAB)] +
                u.ktab[2][GS_BCI(iz, a.n2, BC_X_KTAB)];
#pragma unroll
    for (int g = 0; g < GM; ++g) out[g] = mk2((T)0, (T)0);
    out[0] = in[0] * sym_div(u.scale, (T)1 + u.dtL * u.ke * K);
  }
};

// The transposed precipitate update, one pair per grid-z slice: inputs
// (lambda', state') of c (slice 0) or eta_p (slice 1 + p); outputs
// D lambda', K D lambda', K^a D state' with D = 1/(1 + dt M kappa_c K^2),
// a = 2 for c, D = 1/(1 + dt L kappa_eta K), a = 1 for eta.  The symbols
// are real and even: each is its own transpose.
struct PrecipAdjOp {
  template <typename T, int FM, int GM>
  __device__ __forceinline__ static void apply(const XArgs<T>& a, const int (&nn)[3], int ix, int iy, int iz,
                                               const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
    const PrecipUpd<T>& u = a.pu;
    // the per-axis tables hold n0, n1 and n2 entries
    const T K = u.ktab[0][GS_BCI(ix, a.n0, BC_X_KTAB)] + u.ktab[1][GS_BCI(iy, a.n1, BC_X_KTAB)] +
                u.ktab[2][GS_BCI(iz, a.n2, BC_X_KTAB)];
#pragma unroll
    for (int g = 0; g < GM; ++g) out[g] = mk2((T)0, (T)0);
    if (blockIdx.z == 0) {
      const T d = sym_div(u.scale, (T)1 + u.dtM * u.kc * K * K);
      out[0] = in[0] * d;
      out[1] = in[0] * (K * d);
      out[2] = in[1] * (K * K * d);
    } else {
      const T d = sym_div(u.scale, (T)1 + u.dtL * u.ke * K);
      out[0] = in[0] * d;
      out[1] = in[0] * (K * d);
      out[2] = in[1] * (K * d);
    }
  }
};

// threads per block of the x pass for a field-count class (FM, GM)
template <int FM, int GM> struct XBounds {
  static constexpr int G = FM > GM ? FM : GM;
  static constexpr int v = G <= 3 ? 768 : (G <= 10 ? 640 : 576);
};

// One (ky, kz tile) column set of the x pass after its inputs are in
// registers (v, in_pos order, group grp = field grp): forward FFT along x,
// per-point operation, inverse FFT, store.  smb: the groups' line regions
// (region = PAD * TZ values each), part: GM x N0 values for the packed
// columns.  Shared by the plain and the TMA-fed kernels.
template <typename T, int N0, int FM, int GM, class Op, bool TWS = false, bool EX = false>
__device__ __forceinline__ void xpass_tile(const XArgs<T>& a, cplx<T>* smb, cplx<T>* part, int TZ, int grp, int c,
                                           int t, int kz0, int ky, cplx<T>* out_base,
                                           cplx<T> (&v)[Line<T, N0>::R1], const cplx<T>* tw) {
  using L = Line<T, N0>;
  using V = cplx<T>;
  const int h = a.h, n1 = a.n1, HH = n1 / 2;
  const long long fstride = (long long)a.n0 * n1 * h;
  const int rstride = n1 * h;
  const int region = L::PAD * TZ;
  V* rg = smb + grp * region + c;
  auto sm = [rg, TZ](int pos) -> V& { return rg[pos * TZ]; };
  const int Fn = EX ? FM : a.F, Gn = EX ? GM : a.G;  // EX: exactly FM inputs and GM outputs
  const bool fw = grp < Fn;
  const int kzg0 = kz0 + a.kz_off;       // global slot of the tile's first column
  const int hg = a.hg ? a.hg : h;        // global slot count (Nyquist index of z)
  const bool special_blk = kzg0 == 0 && (n1 == 1 || ky == 0 || ky == HH);
  const int nn[3] = {a.n0, a.n1, a.n2};
  // with a paired operator one item is kx and N0 - kx (kx <= N0 / 2)
  constexpr bool PAIR = KxPair<Op>::v;
  constexpr int NKX = PAIR ? N0 / 2 + 1 : N0;
  constexpr int S = TriStride<FM>::v;
  // the first PF items of a thread have their B-table points loaded before
  // the forward FFT, so that the loads (L2 round trips) overlap it (three
  // fields: 0.163 -> 0.156 ms at 256^3; five fields measured no gain)
  constexpr int PF = PAIR && S <= 8 ? 3 : 0;
  auto coords = [&](int idx, int& cc, int& kx, int& kyA, int& kzA, int& kyB, int& kzB) {
    cc = idx % TZ;
    kx = idx / TZ;
    const int kz = kzg0 + cc;
    kyA = ky; kzA = kz; kyB = 0; kzB = 0;
    if (kz == 0) {
      if (n1 == 1) {
        kyA = 0; kzA = 0; kyB = 0; kzB = hg;
      } else if (ky == 0) {
        kyA = 0; kzA = 0; kyB = HH; kzB = 0;
      } else if (ky == HH) {
        kyA = 0; kzA = hg; kyB = HH; kzB = hg;
      } else if (ky > HH) {
        kyA = ky - HH; kzA = hg;
      }
    }
  };
  T pre[PF > 0 ? PF : 1][S];
#pragma unroll
  for (int j = 0; j < PF; ++j) {
    const int idx = threadIdx.x + j * blockDim.x;
    int cc, kx, kyA, kzA, kyB, kzB;
    coords(idx, cc, kx, kyA, kzA, kyB, kzB);
    if (idx < NKX * TZ && !(special_blk && cc == 0)) {
      if constexpr (PAIR) Op::template load<T, FM>(a, nn, kx, kyA, kzA, pre[j]);
    }
  }
  L::template run<-1, TWS>(v, t, sm, tw);
  __syncthreads();
  if (fw) {
#pragma unroll
    for (int i = 0; i < L::R1; ++i) sm(L::out_pos(t, i)) = v[i];
  }
  __syncthreads();
  // contraction over all (kx, column) points of the tile; bvp: the item's
  // prefetched table point, or null
  auto point = [&](int idx, const T* bvp) {
    int cc, kx, kyA, kzA, kyB, kzB;
    coords(idx, cc, kx, kyA, kzA, kyB, kzB);
    if (!(special_blk && cc == 0)) {
      if constexpr (PAIR) {
        T bv[S];
        if (bvp) {
#pragma unroll
          for (int i = 0; i < S; ++i) bv[i] = bvp[i];
        } else {
          Op::template load<T, FM>(a, nn, kx, kyA, kzA, bv);
        }
        const int kx2 = (N0 - kx) % N0;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          if (side == 1 && kx2 == kx) break;
          const int px = side ? kx2 : kx;
          V* pt = smb + px * TZ + cc;
          V in[FM], out[GM];
#pragma unroll
          for (int f = 0; f < FM; ++f) in[f] = f < Fn ? pt[f * region] : mk2((T)0, (T)0);
          Op::template contract<T, FM, GM, EX>(a, bv, in, out);
#pragma unroll
          for (int g = 0; g < GM; ++g)
            if (g < Gn) pt[g * region] = out[g];
        }
      } else {
        V* pt = smb + kx * TZ + cc;
        V in[FM], out[GM];
#pragma unroll
        for (int f = 0; f < FM; ++f) in[f] = f < Fn ? pt[f * region] : mk2((T)0, (T)0);
        Op::template apply<T, FM, GM>(a, nn, kx, kyA, kzA, in, out);
#pragma unroll
        for (int g = 0; g < GM; ++g)
          if (g < Gn) pt[g * region] = out[g];
      }
    } else {
      // two real sequences packed in one column: A = (W(k) + conj W(-k))/2,
      // B = -i (W(k) - conj W(-k))/2, each contracted with its own k
#pragma unroll 1
      for (int side = 0; side < (PAIR ? 2 : 1); ++side) {
        const int kxa = side ? (N0 - kx) % N0 : kx;
        if (side == 1 && kxa == kx) break;
        const int kxb = (N0 - kxa) % N0;
        V res[2][GM];
#pragma unroll 1
        for (int half = 0; half < 2; ++half) {
          V in[FM];
#pragma unroll
          for (int f = 0; f < FM; ++f) {
            const V wa = f < Fn ? smb[f * region + kxa * TZ] : mk2((T)0, (T)0);
            const V wb = f < Fn ? smb[f * region + kxb * TZ] : mk2((T)0, (T)0);
            if (half == 0) {
              in[f] = mk2((T)0.5 * (wa.x + wb.x), (T)0.5 * (wa.y - wb.y));
            } else {
              in[f] = mk2((T)0.5 * (wa.y + wb.y), (T)-0.5 * (wa.x - wb.x));
            }
          }
          V out[GM];
          Op::template apply<T, FM, GM>(a, nn, kxa, half ? kyB : kyA, half ? kzB : kzA, in, out);
#pragma unroll
          for (int g = 0; g < GM; ++g) res[half][g] = out[g];
        }
#pragma unroll
        for (int g = 0; g < GM; ++g)
          if (g < Gn) part[g * N0 + kxa] = mk2(res[0][g].x - res[1][g].y, res[0][g].y + res[1][g].x);
      }
    }
  };
#pragma unroll
  for (int j = 0; j < PF; ++j) {
    const int idx = threadIdx.x + j * blockDim.x;
    if (idx < NKX * TZ) point(idx, pre[j]);
  }
#pragma unroll 1
  for (int idx = threadIdx.x + PF * blockDim.x; idx < NKX * TZ; idx += blockDim.x) point(idx, nullptr);
  __syncthreads();
  if (special_blk) {
    for (int idx = threadIdx.x; idx < Gn * N0; idx += blockDim.x) {
      const int g = idx / N0, kx = idx - g * N0;
      smb[g * region + kx * TZ] = part[g * N0 + kx];
    }
    __syncthreads();
  }
  // inverse FFT, group grp takes output field grp
  const bool iv = grp < Gn;
#pragma unroll
  for (int r = 0; r < L::R1; ++r) v[r] = iv ? sm(L::in_pos(t, r)) : mk2((T)0, (T)0);
  __syncthreads();
  L::template run<1, TWS>(v, t, sm, tw);
  if (iv) {
    V* dst = out_base + grp * fstride + (long long)ky * h + kz0 + c;
    GS_BC_DECL(const long long ooff = (out_base - a.out) + grp * fstride + (long long)ky * h + kz0 + c,
               oext = (long long)(a.nsim > 1 ? a.nsim : 1) * a.G * fstride)
#pragma unroll
    for (int i = 0; i < L::R1; ++i) dst[GS_BCO(ooff, (long long)L::out_pos(t, i) * rstride, oext, BC_X_OUT)] = v[i];
  }
}


template <typename T, int N0, int FM, int GM, int TZC, class Op, bool EX = false>
__global__ void __launch_bounds__(XBounds<FM, GM>::v) k_xpass(XArgs<T> a) {
  using L = Line<T, N0>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int TZ = TZC ? TZC : a.tz;  // compile-time tile width when TZC > 0
  const int gsz = TZ * L::P;
  const int grp = threadIdx.x / gsz, l = threadIdx.x - grp * gsz;
  const int c = l % TZ, t = l / TZ;
  const int kz0 = blockIdx.x * TZ, ky = blockIdx.y;
  const int h = a.h, n1 = a.n1;
  const long long fstride = (long long)a.n0 * n1 * h;
  const int rstride = n1 * h;
  // line regions of the groups, the packed-column results, the twiddles
  GS_BC_SMEM_GUARD((long long)a.groups * L::PAD * TZ + (long long)(GM + 1) * N0, V, BC_X_SMEM)
  // batched simulations: one sim per blockIdx.z, fields stored sim after sim
  const V* in_base = a.in + (long long)blockIdx.z * a.F * fstride;
  V* out_base = a.out + (long long)blockIdx.z * a.G * fstride;
  V* part = smb + a.groups * (L::PAD * TZ);  // GM x N0 results of the packed column
  // the x twiddles in shared memory (read 30 times per thread and tile); the
  // FFT's first barrier comes before their first use
  V* tws = part + GM * N0;
  for (int i = threadIdx.x; i < N0; i += blockDim.x) tws[i] = a.tw[i];
  V v[L::R1];
  // forward FFT input, group grp takes field grp
  const bool fw = grp < a.F;
  {
    const V* src = in_base + (fw ? grp : 0) * fstride + (long long)ky * h + kz0 + c + (long long)t * rstride;
    GS_BC_DECL(const long long ioff = (long long)blockIdx.z * a.F * fstride + (fw ? grp : 0) * fstride +
                                      (long long)ky * h + kz0 + c + (long long)t * rstride,
               iext = (long long)(a.nsim > 1 ? a.nsim : 1) * a.F * fstride)
#pragma unroll
    for (int r = 0; r < L::R1; ++r)
      v[r] = fw ? src[GS_BCO(ioff, (long long)r * (L::P * rstride), iext, BC_X_IN)] : mk2((T)0, (T)0);
  }
  xpass_tile<T, N0, FM, GM, Op, true, EX>(a, smb, part, TZ, grp, c, t, kz0, ky, out_base, v, tws);
}

// ---------------------------------------------------------------------------
// z inverse of a packed row into registers.  Loads each value S_k of the
// row with its partner S_{h-k} (no shared-memory round trip, no barrier),
// rebuilds Z'_k = (S_k + conj S_{h-k}) + i (S_k - conj S_{h-k}) w^-k and runs
// the inverse length-h FFT; every read of the row is done before the FFT's
// first barrier.  On return v[i] holds
// (r[2m], r[2m+1]) for m = out_pos(t, i).  All threads of the block call it.
// ---------------------------------------------------------------------------
template <typename T, int H>
__device__ __forceinline__ void zinv_row(const cplx<T>* __restrict__ srow, bool act, int t, cplx<T>* sl,
                                         const cplx<T>* __restrict__ tw_h, const cplx<T>* __restrict__ tw_n2,
                                         cplx<T> (&v)[Line<T, H>::R1], long long bc_soff,
                                         long long bc_sext) {
  using L = Line<T, H>;
  using V = cplx<T>;
  // each value and its partner H - k straight from the row (the partner is
  // another thread's own value of the same warp: an L1 hit)
#pragma unroll
  for (int r = 0; r < L::R1; ++r) {
    const int k = L::in_pos(t, r);
    V z;
    if (!act) {
      z = mk2((T)0, (T)0);
    } else if (k == 0) {
      const V s0 = srow[GS_BCO(bc_soff, 0, bc_sext, BC_ZINV_SPEC)];
      z = mk2(s0.x + s0.y, s0.x - s0.y);
    } else {
      const V sk = srow[GS_BCO(bc_soff, k, bc_sext, BC_ZINV_SPEC)];
      const V sm_ = srow[GS_BCO(bc_soff, H - k, bc_sext, BC_ZINV_SPEC)];
      const V Ps = padd(sk, sm_), Ms = psub(sk, sm_);
      const V A = mk2(Ps.x, Ms.y);   // sk + conj(sm)
      const V D = mk2(Ms.x, Ps.y);   // sk - conj(sm)
      const V w = __ldg(&tw_n2[k]);
      const V Bv = cmulc(D, w);                      // D * w^-k
      z = mk2(A.x - Bv.y, A.y + Bv.x);               // A + i Bv
    }
    v[r] = z;
  }
  auto sm = [sl](int pos) -> V& { return sl[pos]; };
  L::template run<1>(v, t, sm, tw_h);
}

// ---------------------------------------------------------------------------
// z inverse to real rows: spectra [F][rows][h] -> dst[f] rows of n2 reals.
// One field may get an FP64 offset added before rounding (the mass
// projection of the concentration).
// ---------------------------------------------------------------------------
template <typename T> struct ZinvArgs {
  const cplx<T>* spec;
  T* dst[GS_MAXG + 1];
  long long rows_per_field, nrows;  // nrows = F * rows_per_field
  int lpc;
  const cplx<T>* tw_h;
  const cplx<T>* tw_n2;
  int offset_field;  // -1: none
  double offset;
};

template <typename T, int H>
__global__ void k_zinv(ZinvArgs<T> a) {
  using L = Line<T, H>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int t = threadIdx.x % L::P, line = threadIdx.x / L::P;
  const long long row = (long long)blockIdx.x * a.lpc + line;
  const bool act = row < a.nrows;
  GS_BC_SMEM_GUARD((long long)(blockDim.x / L::P) * L::PAD, V, BC_ZFWD_SMEM)
  V* sl = smb + line * L::PAD;
  V r[L::R1];
  zinv_row<T, H>(a.spec + (act ? row : 0) * H, act, t, sl, a.tw_h, a.tw_n2, r, GS_BCX((act ? row : 0) * H),
                 GS_BCX(a.nrows * H));
  if (!act) return;
  const int f = (int)(row / a.rows_per_field);
  const long long rin = row - (long long)f * a.rows_per_field;
  V* dst = reinterpret_cast<V*>(a.dst[f]) + rin * H;
  const bool off = f == a.offset_field;
#pragma unroll
  for (int i = 0; i < L::R1; ++i) {
    V x = r[i];
    if (off) x = mk2((T)((double)x.x + a.offset), (T)((double)x.y + a.offset));
    dst[GS_BCO(rin * H, L::out_pos(t, i), a.rows_per_field * H, BC_ZINV_DST)] = x;
  }
}

}  // namespace gs
