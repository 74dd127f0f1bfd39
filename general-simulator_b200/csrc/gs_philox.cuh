// gs_philox.cuh -- counter-based Philox4x32-10 noise, generated in registers.
//
// Replaces the reference's cuRAND XORWOW field (src/random.cu:79-82,
// curandGenerateNormal into a V*N buffer each step).  Philox4x32-10 follows
// Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3"
// (SC'11): ten rounds of two 32x32->64 multiplies with the Weyl key bump.
//
// Counter layout of the phase-field noise: ctr = (cell >> 2, step, sim_id,
// slot), key = (seed lo, seed hi), where cell is the flat [nx][ny][nz] index
// and slot the variant (or V for the concentration).  One block serves four
// consecutive cells: Box-Muller of words (0,1) gives cells 0 (cos) and 1
// (sin), words (2,3) give cells 2 and 3.  Uniforms keep 24 bits,
// u = (x>>8 + 0.5)/2^24, exact in FP32 and FP64, so the CPU oracle sees the
// same bits.
#pragma once
#include <stdint.h>

namespace gs {

struct Philox4 {
  uint32_t x[4];
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    // one widening multiply per product (both halves from one instruction)
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  Philox4 o;
  o.x[0] = c0;
  o.x[1] = c1;
  o.x[2] = c2;
  o.x[3] = c3;
  return o;
}

// Box & Muller (1958) on two 24-bit uniforms: (r cos, r sin).
// FP32: the angle 2 pi u2 is shifted to [-pi, pi), where the hardware
// sine / cosine approximations have an absolute error below 2^-21.4; with
// sin(t) = -sin(t - pi) and cos(t) = -cos(t - pi).
__device__ __forceinline__ float2 box_muller(uint32_t a, uint32_t b, float) {
  const float u1 = ((float)(a >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float u2 = ((float)(b >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float r = sqrtf(-2.0f * logf(u1));
  float s, c;
  __sincosf(6.283185307179586f * u2 - 3.141592653589793f, &s, &c);
  return make_float2(-r * c, -r * s);
}
__device__ __forceinline__ double2 box_muller(uint32_t a, uint32_t b, double) {
  const double u1 = ((double)(a >> 8) + 0.5) * (1.0 / 16777216.0);
  const double u2 = ((double)(b >> 8) + 0.5) * (1.0 / 16777216.0);
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  return make_double2(r * c, r * s);
}

// N(0,1) noise of the four cells 4q..4q+3 of quad q for one slot.
template <typename T>
__device__ __forceinline__ void normal_quad(uint32_t quad, uint32_t step, uint32_t sim, uint32_t slot, uint32_t k0,
                                            uint32_t k1, T (&z)[4]) {
  const Philox4 o = philox4x32_10(quad, step, sim, slot, k0, k1);
  const auto a = box_muller(o.x[0], o.x[1], (T)0);
  const auto b = box_muller(o.x[2], o.x[3], (T)0);
  z[0] = a.x;
  z[1] = a.y;
  z[2] = b.x;
  z[3] = b.y;
}

}  // namespace gs
