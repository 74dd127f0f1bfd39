// gs_common.cuh -- shared types of the sm_100a phase-field kernels.
//
// Fields are stored [F][n0][n1][n2] with n2 fastest (the reference's
// [V][nx][ny][nz], include/datamain.th:72-76, with unit axes dropped so that
// n2 is the last axis of extent > 1).  Spectra use the packed half-complex
// layout described in gs_passes.cuh: [F][n0][n1][n2/2] complex, the same
// bytes as the real field.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gs_bc.cuh"

#define GS_MAXF 9    // elastic fields: up to 8 variants + concentration
#define GS_MAXG 9    // contraction outputs (6 stress components or F)

namespace gs {

template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename T> using cplx = typename C2<T>::type;

__host__ __device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }

__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// Lane-wise add / subtract of two complex values: one packed FP32x2
// instruction for float2 (the same IEEE round-to-nearest result per lane as
// the scalar operations), two scalar ones for double2.
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ double2 padd(double2 a, double2 b) { return a + b; }
__device__ __forceinline__ double2 psub(double2 a, double2 b) { return a - b; }

template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
  return mk2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
  return mk2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename V> __host__ __device__ __forceinline__ V conjg(V a) { return mk2(a.x, -a.y); }
// i * a
template <typename V> __host__ __device__ __forceinline__ V muli(V a) { return mk2(-a.y, a.x); }

// Derived constants of one simulation, passed by value to every pass.
template <typename T> struct ElasticConst {
  int na, nb;           // rows (outputs) and columns (inputs) of B
  int refcompat;        // B(0) = C:ea:eb and |k| <= 5e-7 test (reference rule)
  T qs[6][6];           // Omega^-1_e = sum_{a<=b} qs[e][ab] n_a n_b, e = 00 01 02 11 12 22
  T sa[GS_MAXG][3][3];  // sigma of the output set, C:ea
  T sb[GS_MAXF][3][3];  // sigma of the input set, C:eb
  T a0[GS_MAXG][GS_MAXF];  // C:ea:eb
  T kscale[3];          // k_axis = kscale * folded index
  T scale;              // multiplier of the contraction (1/N and field scales)
};

// Division by a runtime constant d with one multiply-high and a shift
// (Granlund & Montgomery, PLDI'94, round-up variant); valid for n < 2^31.
struct FastDiv {
  uint32_t d = 1, m = 1, s = 0;
  FastDiv() = default;
  explicit FastDiv(uint32_t dv) : d(dv) {
    uint32_t l = 0;
    while ((1ull << l) < dv) ++l;
    m = (uint32_t)(((1ull << 32) * ((1ull << l) - dv)) / dv + 1);
    s = l;
  }
  __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi(n, m) + n) >> s; }
};

struct Geo {
  int n0, n1, n2, h;  // canonical extents, h = n2/2
  long long N;        // n0*n1*n2
};

}  // namespace gs
