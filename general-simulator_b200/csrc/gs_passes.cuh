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

// out[g] += w * sum_f B_gf(k) in[f], with B_gf = C:ea_g:eb_f - (n sigma_g)
// Omega (sigma_f n) evaluated inside the sum.  k is in the original axes.
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
  T m[9];
#pragma unroll
  for (int ij = 0; ij < 9; ++ij) {
    T sacc = 0;
#pragma unroll
    for (int q = 0; q < 6; ++q) sacc += ec.q[ij][q] * nn[q];
    m[ij] = sacc;
  }
  const T det = -m[2] * m[4] * m[6] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7] - m[0] * m[5] * m[7] -
                m[1] * m[3] * m[8] + m[0] * m[4] * m[8];
  T om[9];
  const bool ok = ec.refcompat ? (det >= (T)1e-8 || det <= (T)-1e-8) : (det != (T)0);
  if (ok) {
    const T id = gs_rcp(det);
    om[0] = (-m[5] * m[7] + m[4] * m[8]) * id;
    om[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    om[2] = (-m[2] * m[4] + m[1] * m[5]) * id;
    om[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    om[4] = (-m[2] * m[6] + m[0] * m[8]) * id;
    om[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    om[6] = (-m[4] * m[6] + m[3] * m[7]) * id;
    om[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    om[8] = (-m[1] * m[3] + m[0] * m[4]) * id;
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) om[i] = 0;
  }
  T wb[FM][3];
#pragma unroll
  for (int f = 0; f < FM; ++f) {
#pragma unroll
    for (int i = 0; i < 3; ++i) wb[f][i] = ec.sb[f][i][0] * n[0] + ec.sb[f][i][1] * n[1] + ec.sb[f][i][2] * n[2];
  }
#pragma unroll
  for (int g = 0; g < GM; ++g) {
    if (g < ec.na) {
      T va[3], ova[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) va[j] = n[0] * ec.sa[g][0][j] + n[1] * ec.sa[g][1][j] + n[2] * ec.sa[g][2][j];
#pragma unroll
      for (int c = 0; c < 3; ++c) ova[c] = va[0] * om[0 * 3 + c] + va[1] * om[1 * 3 + c] + va[2] * om[2 * 3 + c];
      cplx<T> acc = mk2((T)0, (T)0);
#pragma unroll
      for (int f = 0; f < FM; ++f) {
        if (f < ec.nb) {
          const T b = ec.a0[g][f] - (ova[0] * wb[f][0] + ova[1] * wb[f][1] + ova[2] * wb[f][2]);
          acc = acc + in[f] * b;
        }
      }
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
__device__ __forceinline__ void contract_at(const ElasticConst<T>& ec, const int (&perm)[3], const int (&nn)[3],
                                            int ix, int iy, int iz, const cplx<T> (&in)[FM], cplx<T> (&out)[GM]) {
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
  T k[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) k[perm[c]] = ec.kscale[c] * (T)m[c];
  if (!nyq) {
    contract_k<T, FM, GM>(ec, k, in, out, ec.scale);
    return;
  }
  contract_k<T, FM, GM>(ec, k, in, out, (T)0.5 * ec.scale);
#pragma unroll
  for (int c = 0; c < 3; ++c) k[perm[c]] = ec.kscale[c] * (T)(isnyq[c] ? -m[c] : m[c]);
  contract_k<T, FM, GM>(ec, k, in, out, (T)0.5 * ec.scale);
}

// ---------------------------------------------------------------------------
// z forward: real rows -> packed half spectrum, with a fused prologue.
// ---------------------------------------------------------------------------
template <typename T> struct ZfwdArgs {
  const T* src[GS_MAXF];   // row source of each field (n0*n1 rows of n2)
  int square[GS_MAXF];     // 1: transform src^2 (eta^2), 0: src
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
  V* sl = smb + line * L::PAD;
  auto sm = [sl](int pos) -> V& { return sl[pos]; };
  V v[L::R1];
  if (act) {
    const int f = (int)(row / a.rows_per_field);
    const long long rin = row - (long long)f * a.rows_per_field;
    const V* src = reinterpret_cast<const V*>(a.src[f]) + rin * H;
    const int sq = a.square[f];
#pragma unroll
    for (int r = 0; r < L::R1; ++r) {
      V x = src[L::in_pos(t, r)];
      if (sq) x = mk2(x.x * x.x, x.y * x.y);
      v[r] = x;
    }
  } else {
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[r] = mk2((T)0, (T)0);
  }
  L::template run<-1>(v, t, sm, a.tw_h);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < L::R1; ++i) sl[L::out_pos(t, i)] = v[i];
  __syncthreads();
  if (act) {
    V* dst = a.dst + row * H;
#pragma unroll
    for (int i = 0; i < L::R1; ++i) {
      const int k = L::out_pos(t, i);
      const V zk = sl[k];
      V s;
      if (k == 0) {
        s = mk2(zk.x + zk.y, zk.x - zk.y);
      } else {
        const V zm = sl[H - k];
        const V e = mk2((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
        const V d = mk2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
        const V o = mk2((T)0.5 * d.y, (T)-0.5 * d.x);  // -i d / 2
        s = e + cmul(o, __ldg(&a.tw_n2[k]));
      }
      dst[k] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// y pass (forward or inverse) over columns of TZ consecutive kz slots.
// ---------------------------------------------------------------------------
template <typename T> struct YArgs {
  cplx<T>* spec;  // [F][n0][n1][h]
  int n0, n1, h, tz;
  const cplx<T>* tw;  // w_n1^m
};

template <typename T, int N1, int DIR>
__global__ void k_ypass(YArgs<T> a) {
  using L = Line<T, N1>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int TZ = a.tz;
  const int c = threadIdx.x % TZ, t = threadIdx.x / TZ;
  const int kz0 = blockIdx.x * TZ, x = blockIdx.y, f = blockIdx.z;
  const int h = a.h;
  V* base = a.spec + ((long long)(f * a.n0 + x) * N1) * h + kz0 + c;
  auto sm = [smb, TZ, c](int pos) -> V& { return smb[pos * TZ + c]; };
  const bool special = (kz0 == 0);
  constexpr int HH = N1 / 2;
  V v[L::R1];
  if (DIR < 0 || !special) {
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[r] = base[(long long)L::in_pos(t, r) * h];
  } else {
    // inverse, tile holding kz slot 0: rebuild U(ky) = A(ky) + i B(ky)
#pragma unroll
    for (int r = 0; r < L::R1; ++r) {
      const int p = L::in_pos(t, r);
      sm(p) = base[(long long)p * h];
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
    for (int i = 0; i < L::R1; ++i) base[(long long)L::out_pos(t, i) * h] = v[i];
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
      base[(long long)s * h] = o;
    }
  }
}

// ---------------------------------------------------------------------------
// x pass: forward x FFT of F fields -> B(n) contraction -> inverse x FFT of
// G fields.  One block per (kz tile, ky slot).
// ---------------------------------------------------------------------------
template <typename T> struct XArgs {
  const cplx<T>* in;  // [F][n0][n1][h]
  cplx<T>* out;       // [G][n0][n1][h] (may alias in when G <= F)
  int n0, n1, n2, h, tz, F, G;
  int perm[3];
  const cplx<T>* tw;  // w_n0^m
  ElasticConst<T> ec;
};

template <typename T, int N0, int FM, int GM>
__global__ void k_xcontract(XArgs<T> a) {
  using L = Line<T, N0>;
  using V = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int TZ = a.tz;
  const int c = threadIdx.x % TZ, t = threadIdx.x / TZ;
  const int kz0 = blockIdx.x * TZ, ky = blockIdx.y;
  const int h = a.h, n1 = a.n1;
  const long long fstride = (long long)a.n0 * n1 * h;
  const long long colbase = (long long)ky * h + kz0;
  const int region = L::PAD * TZ;
  // forward FFT of each input field into its own shared region
  for (int f = 0; f < a.F; ++f) {
    V* rg = smb + f * region;
    auto sm = [rg, TZ, c](int pos) -> V& { return rg[pos * TZ + c]; };
    const V* col = a.in + f * fstride + colbase + c;
    V v[L::R1];
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[r] = col[(long long)L::in_pos(t, r) * n1 * h];
    L::template run<-1>(v, t, sm, a.tw);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < L::R1; ++i) sm(L::out_pos(t, i)) = v[i];
  }
  __syncthreads();
  // contraction over Hermitian pairs (kx, n0 - kx)
  {
    constexpr int npair = N0 / 2 + 1;
    const int HH = n1 / 2;
    const int nn[3] = {a.n0, a.n1, a.n2};
    for (int idx = threadIdx.x; idx < npair * TZ; idx += blockDim.x) {
      const int cc = idx % TZ, p = idx / TZ;
      const int kxa = p % N0, kxb = (N0 - p) % N0;
      const int kz = kz0 + cc;
      bool special = false;
      int kyA = ky, kzA = kz, kyB = 0, kzB = 0;
      if (kz == 0) {
        if (n1 == 1) {
          special = true;
          kyA = 0; kzA = 0; kyB = 0; kzB = h;
        } else if (ky == 0) {
          special = true;
          kyA = 0; kzA = 0; kyB = HH; kzB = 0;
        } else if (ky == HH) {
          special = true;
          kyA = 0; kzA = h; kyB = HH; kzB = h;
        } else if (ky > HH) {
          kyA = ky - HH; kzA = h;
        }
      }
      V wa[FM], wb[FM];
#pragma unroll
      for (int f = 0; f < FM; ++f) {
        wa[f] = f < a.F ? smb[f * region + kxa * TZ + cc] : mk2((T)0, (T)0);
        wb[f] = f < a.F ? smb[f * region + kxb * TZ + cc] : mk2((T)0, (T)0);
      }
      if (!special) {
        V oa[GM];
        contract_at<T, FM, GM>(a.ec, a.perm, nn, kxa, kyA, kzA, wa, oa);
#pragma unroll
        for (int g = 0; g < GM; ++g)
          if (g < a.G) smb[g * region + kxa * TZ + cc] = oa[g];
        if (kxb != kxa) {
          contract_at<T, FM, GM>(a.ec, a.perm, nn, kxb, kyA, kzA, wb, oa);
#pragma unroll
          for (int g = 0; g < GM; ++g)
            if (g < a.G) smb[g * region + kxb * TZ + cc] = oa[g];
        }
      } else {
        // two real sequences packed in one column: A = (W(k) + conj W(-k))/2,
        // B = -i (W(k) - conj W(-k))/2, contracted with their own k
        V Af[FM], Bf[FM];
#pragma unroll
        for (int f = 0; f < FM; ++f) {
          Af[f] = mk2((T)0.5 * (wa[f].x + wb[f].x), (T)0.5 * (wa[f].y - wb[f].y));
          const V d = mk2(wa[f].x - wb[f].x, wa[f].y + wb[f].y);
          Bf[f] = mk2((T)0.5 * d.y, (T)-0.5 * d.x);
        }
        V ra[GM], rb[GM];
        contract_at<T, FM, GM>(a.ec, a.perm, nn, kxa, kyA, kzA, Af, ra);
        contract_at<T, FM, GM>(a.ec, a.perm, nn, kxa, kyB, kzB, Bf, rb);
#pragma unroll
        for (int g = 0; g < GM; ++g) {
          if (g < a.G) {
            smb[g * region + kxa * TZ + cc] = mk2(ra[g].x - rb[g].y, ra[g].y + rb[g].x);
            if (kxb != kxa) smb[g * region + kxb * TZ + cc] = mk2(ra[g].x + rb[g].y, -ra[g].y + rb[g].x);
          }
        }
      }
    }
  }
  __syncthreads();
  // inverse FFT of each output field
  for (int g = 0; g < a.G; ++g) {
    V* rg = smb + g * region;
    auto sm = [rg, TZ, c](int pos) -> V& { return rg[pos * TZ + c]; };
    V v[L::R1];
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[r] = sm(L::in_pos(t, r));
    __syncthreads();
    L::template run<1>(v, t, sm, a.tw);
    V* col = a.out + g * fstride + colbase + c;
#pragma unroll
    for (int i = 0; i < L::R1; ++i) col[(long long)L::out_pos(t, i) * n1 * h] = v[i];
  }
}

// ---------------------------------------------------------------------------
// x pass with every field held in registers.  For a square plan (R1 == R2,
// or one stage) the forward FFT leaves X[out_pos(t,i)] with out_pos == in_pos,
// so the contraction runs on registers and its result is directly the input
// of the inverse FFT: shared memory carries only the FFT exchange (and, in the
// blocks holding the two packed columns, the Hermitian partners).
// ---------------------------------------------------------------------------
template <typename T, int N0, int F>
__global__ void __launch_bounds__(256) k_xreg(XArgs<T> a) {
  using L = Line<T, N0>;
  using V = cplx<T>;
  static_assert(L::R2 == 1 || L::R1 == L::R2, "square plan");
  extern __shared__ __align__(16) unsigned char smraw[];
  V* smb = reinterpret_cast<V*>(smraw);
  const int TZ = a.tz;
  const int c = threadIdx.x % TZ, t = threadIdx.x / TZ;
  const int kz0 = blockIdx.x * TZ, ky = blockIdx.y;
  const int h = a.h, n1 = a.n1, HH = n1 / 2;
  const long long fstride = (long long)a.n0 * n1 * h;
  const long long colbase = (long long)ky * h + kz0 + c;
  const long long rstride = (long long)n1 * h;
  auto sm = [smb, TZ, c](int pos) -> V& { return smb[pos * TZ + c]; };
  V v[F][L::R1];
#pragma unroll
  for (int f = 0; f < F; ++f)
#pragma unroll
    for (int r = 0; r < L::R1; ++r) v[f][r] = a.in[f * fstride + colbase + L::in_pos(t, r) * rstride];
#pragma unroll
  for (int f = 0; f < F; ++f) {
    if (f > 0) __syncthreads();
    L::template run<-1>(v[f], t, sm, a.tw);
  }
  // packed columns (kz slot 0 with ky slot 0 or n1/2, or n1 == 1) need W(-kx)
  const bool special_blk = kz0 == 0 && (n1 == 1 || ky == 0 || ky == HH);
  V* part = smb + L::PAD * TZ;  // F x N0 partner buffer after the exchange area
  if (special_blk) {
    __syncthreads();
    if (c == 0) {
#pragma unroll
      for (int f = 0; f < F; ++f)
#pragma unroll
        for (int i = 0; i < L::R1; ++i) part[f * N0 + L::out_pos(t, i)] = v[f][i];
    }
    __syncthreads();
  }
  const int nn[3] = {a.n0, a.n1, a.n2};
  const int kz = kz0 + c;
  int kyA = ky, kzA = kz, kyB = 0, kzB = 0;
  const bool special = special_blk && c == 0;
  if (kz == 0) {
    if (n1 == 1) {
      kyA = 0; kzA = 0; kyB = 0; kzB = h;
    } else if (ky == 0) {
      kyA = 0; kzA = 0; kyB = HH; kzB = 0;
    } else if (ky == HH) {
      kyA = 0; kzA = h; kyB = HH; kzB = h;
    } else if (ky > HH) {
      kyA = ky - HH; kzA = h;
    }
  }
#pragma unroll
  for (int i = 0; i < L::R1; ++i) {
    const int kx = L::out_pos(t, i);
    V in[F], out[F];
#pragma unroll
    for (int f = 0; f < F; ++f) in[f] = v[f][i];
    if (!special) {
      contract_at<T, F, F>(a.ec, a.perm, nn, kx, kyA, kzA, in, out);
#pragma unroll
      for (int f = 0; f < F; ++f) v[f][i] = out[f];
    } else {
      const int kxb = (N0 - kx) % N0;
      V Af[F], Bf[F], ra[F], rb[F];
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const V wb = part[f * N0 + kxb];
        Af[f] = mk2((T)0.5 * (in[f].x + wb.x), (T)0.5 * (in[f].y - wb.y));
        const V d = mk2(in[f].x - wb.x, in[f].y + wb.y);
        Bf[f] = mk2((T)0.5 * d.y, (T)-0.5 * d.x);
      }
      contract_at<T, F, F>(a.ec, a.perm, nn, kx, kyA, kzA, Af, ra);
      contract_at<T, F, F>(a.ec, a.perm, nn, kx, kyB, kzB, Bf, rb);
#pragma unroll
      for (int f = 0; f < F; ++f) v[f][i] = mk2(ra[f].x - rb[f].y, ra[f].y + rb[f].x);
    }
  }
#pragma unroll
  for (int f = 0; f < F; ++f) {
    __syncthreads();
    L::template run<1>(v[f], t, sm, a.tw);
    V* col = a.out + f * fstride + colbase;
#pragma unroll
    for (int i = 0; i < L::R1; ++i) col[L::out_pos(t, i) * rstride] = v[f][i];
  }
}

// ---------------------------------------------------------------------------
// z inverse of a packed row into registers.  Loads the row into the line's
// shared buffer, rebuilds Z'_k = (S_k + conj S_{h-k}) + i (S_k - conj
// S_{h-k}) w^-k and runs the inverse length-h FFT.  On return v[i] holds
// (r[2m], r[2m+1]) for m = out_pos(t, i).  All threads of the block call it.
// ---------------------------------------------------------------------------
template <typename T, int H>
__device__ __forceinline__ void zinv_row(const cplx<T>* __restrict__ srow, bool act, int t, cplx<T>* sl,
                                         const cplx<T>* __restrict__ tw_h, const cplx<T>* __restrict__ tw_n2,
                                         cplx<T> (&v)[Line<T, H>::R1]) {
  using L = Line<T, H>;
  using V = cplx<T>;
  if (act) {
#pragma unroll
    for (int r = 0; r < L::R1; ++r) {
      const int k = L::in_pos(t, r);
      sl[k] = srow[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < L::R1; ++r) {
    const int k = L::in_pos(t, r);
    V z;
    if (!act) {
      z = mk2((T)0, (T)0);
    } else if (k == 0) {
      const V s0 = sl[0];
      z = mk2(s0.x + s0.y, s0.x - s0.y);
    } else {
      const V sk = sl[k], sm_ = sl[H - k];
      const V A = mk2(sk.x + sm_.x, sk.y - sm_.y);   // sk + conj(sm)
      const V D = mk2(sk.x - sm_.x, sk.y + sm_.y);   // sk - conj(sm)
      const V w = __ldg(&tw_n2[k]);
      const V Bv = cmulc(D, w);                      // D * w^-k
      z = mk2(A.x - Bv.y, A.y + Bv.x);               // A + i Bv
    }
    v[r] = z;
  }
  __syncthreads();
  auto sm = [sl](int pos) -> V& { return sl[pos]; };
  L::template run<1>(v, t, sm, tw_h);
}

}  // namespace gs
