// gs_k_x_impl.cuh -- launcher template of the x pass for one field-count
// class (FM inputs, GM outputs at most); instantiated per class in its own
// translation unit so the classes compile in parallel.
#pragma once
#include "gs_launch.h"
#include "gs_passes.cuh"

namespace gs {

template <typename T, int N0, int FM, int GM> static cudaError_t xc_n(XArgs<T>& a, cudaStream_t s) {
  using L = Line<T, N0>;
  const int nreg = a.F > a.G ? a.F : a.G;
  int tz = pick_tz(a.h);
  size_t smem = (size_t)nreg * tz * L::PAD * sizeof(cplx<T>);
  while (tz > 1 && smem > 200 * 1024) {
    tz >>= 1;
    smem = (size_t)nreg * tz * L::PAD * sizeof(cplx<T>);
  }
  a.tz = tz;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_xcontract<T, N0, FM, GM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid(a.h / tz, a.n1);
  k_xcontract<T, N0, FM, GM><<<grid, tz * L::P, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T, int FM, int GM> cudaError_t launch_x_class(XArgs<T>& a, cudaStream_t s) {
  switch (a.n0) {
#define GS_C(N_) \
  case N_:       \
    return xc_n<T, N_, FM, GM>(a, s);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace gs
