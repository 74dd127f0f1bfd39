// gs_fft.cuh -- register-resident DFT kernels and the two-stage line FFT.
//
// A line of N complex values is split N = R1 * R2 (R2 divides R1).  P = R2
// threads share a line.  Stage 1: thread t holds x[t + r*P], r < R1, and does
// one radix-R1 DFT in registers.  The stage outputs go through shared memory
// once; stage 2 does R1/R2 radix-R2 DFTs per thread after the twiddle
// w_N^(r*j) and leaves X[j + r*R1], j = t + P*b, in registers.  This is the
// Stockham self-sorting order of Govindaraju et al. (SC'08) with only two
// stages, so a line costs one shared-memory round trip.
#pragma once
#include "gs_common.cuh"

namespace gs {

// cos(2 pi k / 48), k = 0..12.
__host__ __device__ constexpr double c48_tab(int k) {
  return k == 0   ? 1.0
         : k == 1 ? 0.9914448613738104111446
         : k == 2 ? 0.9659258262890682867497
         : k == 3 ? 0.9238795325112867561282
         : k == 4 ? 0.8660254037844386467637
         : k == 5 ? 0.7933533402912351645798
         : k == 6 ? 0.7071067811865475244008
         : k == 7 ? 0.6087614290087206394161
         : k == 8 ? 0.5
         : k == 9 ? 0.3826834323650897717285
         : k == 10 ? 0.2588190451025207623489
         : k == 11 ? 0.1305261922200515915484
                   : 0.0;
}
__host__ __device__ constexpr double cos48(int k) {
  return (k = ((k % 48) + 48) % 48, k = (k > 24 ? 48 - k : k), k <= 12 ? c48_tab(k) : -c48_tab(24 - k));
}
__host__ __device__ constexpr double sin48(int k) { return cos48(k - 12); }

// cos(2 pi k / 64), k = 0..16 (the radix-32 and radix-64 register DFTs)
__host__ __device__ constexpr double c64_tab(int k) {
  return k == 0   ? 1.0
         : k == 1 ? 0.9951847266721968862448
         : k == 2 ? 0.9807852804032304491262
         : k == 3 ? 0.9569403357322088649357
         : k == 4 ? 0.9238795325112867561282
         : k == 5 ? 0.8819212643483550297128
         : k == 6 ? 0.8314696123025452370788
         : k == 7 ? 0.7730104533627369608109
         : k == 8 ? 0.7071067811865475244008
         : k == 9 ? 0.6343932841636454982151
         : k == 10 ? 0.5555702330196022247428
         : k == 11 ? 0.4713967368259976485564
         : k == 12 ? 0.3826834323650897717285
         : k == 13 ? 0.2902846772544623676362
         : k == 14 ? 0.1950903220161282678483
         : k == 15 ? 0.0980171403295606019942
                   : 0.0;
}
__host__ __device__ constexpr double cos64(int k) {
  return (k = ((k % 64) + 64) % 64, k = (k > 32 ? 64 - k : k), k <= 16 ? c64_tab(k) : -c64_tab(32 - k));
}
__host__ __device__ constexpr double sin64(int k) { return cos64(k - 16); }

// cos and sin of 2 pi m / R for the radices the plans use (R | 48 or R | 64)
template <int R> __host__ __device__ constexpr double cos_r(int m) {
  return 48 % R == 0 ? cos48(m * (48 / R)) : cos64(m * (64 / R));
}
template <int R> __host__ __device__ constexpr double sin_r(int m) {
  return 48 % R == 0 ? sin48(m * (48 / R)) : sin64(m * (64 / R));
}

// a * exp(DIR * 2 pi i m / R), m a compile-time value after unrolling.
template <int R, int DIR, typename V>
__device__ __forceinline__ V twmul(V a, int m) {
  static_assert(48 % R == 0 || 64 % R == 0, "radix without a twiddle table");
  m = ((m % R) + R) % R;
  if (m == 0) return a;
  if (2 * m == R) return mk2(-a.x, -a.y);
  if (4 * m == R) return DIR > 0 ? mk2(-a.y, a.x) : mk2(a.y, -a.x);
  if (4 * m == 3 * R) return DIR > 0 ? mk2(a.y, -a.x) : mk2(-a.y, a.x);
  using T = decltype(a.x);
  const T c = (T)cos_r<R>(m);
  const T s = (T)(DIR * sin_r<R>(m));
  return mk2(a.x * c - a.y * s, a.x * s + a.y * c);
}

template <int R> struct FirstFactor {
  static constexpr int v = (R % 4 == 0 && R != 4) ? 4 : (R % 2 == 0 && R != 2) ? 2 : 3;
};

template <int R, int DIR> struct Dft {
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    constexpr int Ra = FirstFactor<R>::v, Rb = R / Ra;
    V u[R];
#pragma unroll
    for (int j2 = 0; j2 < Rb; ++j2) {
      V t[Ra];
#pragma unroll
      for (int j1 = 0; j1 < Ra; ++j1) t[j1] = v[j2 + Rb * j1];
      Dft<Ra, DIR>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < Ra; ++k1) u[j2 * Ra + k1] = twmul<R, DIR>(t[k1], j2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < Ra; ++k1) {
      V t[Rb];
#pragma unroll
      for (int j2 = 0; j2 < Rb; ++j2) t[j2] = u[j2 * Ra + k1];
      Dft<Rb, DIR>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < Rb; ++k2) v[k1 + Ra * k2] = t[k2];
    }
  }
};
template <int DIR> struct Dft<1, DIR> {
  template <typename V> __device__ __forceinline__ static void run(V*) {}
};
template <int DIR> struct Dft<2, DIR> {
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    V a = v[0], b = v[1];
    v[0] = padd(a, b);
    v[1] = psub(a, b);
  }
};
template <int DIR> struct Dft<3, DIR> {
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    using T = decltype(v[0].x);
    const T h = (T)0.8660254037844386467637;  // sqrt(3)/2
    V t = v[1] + v[2], u = v[1] - v[2];
    V m = mk2(v[0].x - (T)0.5 * t.x, v[0].y - (T)0.5 * t.y);
    v[0] = v[0] + t;
    // w = -1/2 + DIR i sqrt(3)/2: X1 = m + DIR i h u, X2 = m - DIR i h u
    V s = mk2(-u.y * h * (T)DIR, u.x * h * (T)DIR);
    v[1] = m + s;
    v[2] = m - s;
  }
};
template <int DIR> struct Dft<4, DIR> {
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    V t0 = padd(v[0], v[2]), t1 = psub(v[0], v[2]), t2 = padd(v[1], v[3]), t3 = psub(v[1], v[3]);
    // w = DIR * i (the swapped lanes stay scalar)
    V w3 = DIR > 0 ? mk2(-t3.y, t3.x) : mk2(t3.y, -t3.x);
    v[0] = padd(t0, t2);
    v[2] = psub(t0, t2);
    v[1] = t1 + w3;
    v[3] = t1 - w3;
  }
};

// Two-stage plans: N = R1 * R2, R2 | R1, P = R2 threads per line.
template <int N> struct Plan;
#define GS_PLAN(N_, R1_, R2_)                 \
  template <> struct Plan<N_> {               \
    static constexpr int R1 = R1_, R2 = R2_;  \
  };
GS_PLAN(1, 1, 1)
GS_PLAN(2, 2, 1)
GS_PLAN(4, 4, 1)
GS_PLAN(6, 6, 1)
GS_PLAN(8, 8, 1)
GS_PLAN(12, 12, 1)
GS_PLAN(16, 16, 1)
GS_PLAN(24, 12, 2)
GS_PLAN(32, 8, 4)
GS_PLAN(48, 12, 4)
GS_PLAN(64, 8, 8)
GS_PLAN(96, 24, 4)
GS_PLAN(128, 16, 8)
GS_PLAN(256, 16, 16)
#undef GS_PLAN

// Line<T, N>: the default plan of length N; Line<T, N, R1>: another split
// N = R1 * (N / R1) (the y pass's alternative plans, chosen by the autotuner)
template <typename T, int N, int R1_ = Plan<N>::R1> struct Line {
  using V = cplx<T>;
  static constexpr int R1 = R1_, R2 = N / R1_;
  static constexpr int P = R2;        // threads per line
  static constexpr int NB = R1 / R2;  // stage-2 butterflies per thread
  static constexpr int PAD = N + N / R1;  // padded shared-memory line length
  static_assert(R1 * R2 == N, "plan");
  static_assert(R1 % R2 == 0, "plan");

  // padded position of element pos in a line buffer
  __device__ __forceinline__ static int spos(int pos) { return pos + pos / R1; }

  // Stage-1 input position of register r of thread t.
  __device__ __forceinline__ static int in_pos(int t, int r) { return t + r * P; }
  // Output position of register i (= b*R2 + r) of thread t.
  __device__ __forceinline__ static int out_pos(int t, int i) { return (t + P * (i / R2)) + (i % R2) * R1; }

  // Run the FFT of one line.  v: registers, in_pos order on entry, out_pos
  // order on exit.  sm(pos) returns a reference to the line's shared element
  // at padded position pos.  tw: w_N^m = exp(-2 pi i m / N), m < N.
  // Every thread of the block must call this (it synchronises the block).
  // TWS: tw is in shared memory (plain loads) instead of global memory.
  template <int DIR, bool TWS = false, class SM>
  __device__ __forceinline__ static void run(V (&v)[R1], int t, SM sm, const V* __restrict__ tw) {
    Dft<R1, DIR>::run(v);
    if constexpr (R2 == 1) {
      return;
    } else {
#pragma unroll
    for (int r = 0; r < R1; ++r) sm(spos(t * R1 + r)) = v[r];
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + P * b;
      V u[R2];
#pragma unroll
      for (int r = 0; r < R2; ++r) {
        V x = sm(spos(j + r * R1));
        if (r > 0) {
          V w = TWS ? tw[r * j] : __ldg(&tw[r * j]);
          if (DIR > 0) w.y = -w.y;
          x = cmul(x, w);
        }
        u[r] = x;
      }
      Dft<R2, DIR>::run(u);
#pragma unroll
      for (int r = 0; r < R2; ++r) v[b * R2 + r] = u[r];
    }
    }
  }
};

}  // namespace gs
