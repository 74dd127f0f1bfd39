// gs_k_xreg.cu -- FP32 instances of the register-resident x pass (square
// FFT plans, F = G fields).
#include "gs_launch.h"
#include "gs_passes.cuh"

namespace gs {

template <int N0, int F> static cudaError_t xr_n(XArgs<float>& a, cudaStream_t s) {
  using L = Line<float, N0>;
  int tz = pick_tz(a.h);
  size_t smem = (size_t)tz * L::PAD * sizeof(float2) + (size_t)F * N0 * sizeof(float2);
  a.tz = tz;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_xreg<float, N0, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid(a.h / tz, a.n1);
  k_xreg<float, N0, F><<<grid, tz * L::P, smem, s>>>(a);
  return cudaGetLastError();
}

template <int N0> static cudaError_t xr_f(XArgs<float>& a, cudaStream_t s, bool* done) {
  *done = true;
  switch (a.F) {
    case 1: return xr_n<N0, 1>(a, s);
    case 2: return xr_n<N0, 2>(a, s);
    case 3: return xr_n<N0, 3>(a, s);
    case 4: return xr_n<N0, 4>(a, s);
    default: *done = false; return cudaSuccess;
  }
}

cudaError_t launch_xreg_f32(XArgs<float>& a, cudaStream_t s, bool* done) {
  *done = false;
  if (a.F != a.G) return cudaSuccess;
  switch (a.n0) {
    case 1: return xr_f<1>(a, s, done);
    case 2: return xr_f<2>(a, s, done);
    case 4: return xr_f<4>(a, s, done);
    case 6: return xr_f<6>(a, s, done);
    case 8: return xr_f<8>(a, s, done);
    case 12: return xr_f<12>(a, s, done);
    case 16: return xr_f<16>(a, s, done);
    case 64: return xr_f<64>(a, s, done);
    case 256: return xr_f<256>(a, s, done);
    default: return cudaSuccess;
  }
}

}  // namespace gs
