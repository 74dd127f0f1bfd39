// gs_k_zy_impl.cuh -- launcher templates of the z-forward and y passes
// (instantiated per dtype in its own translation unit).
#pragma once
#include "gs_launch.h"
#include "gs_passes.cuh"

namespace gs {


// the launch-range check of a z-forward pass (F fields of rows_per_field rows of 2H values)
template <typename T, int H> static cudaError_t zfwd_ranges(const ZfwdArgs<T>& a) {
  const long long F = a.nrows / a.rows_per_field, per = a.rows_per_field * 2 * H;
  if (a.src0) {
    GS_RANGE(a.src0, (F - 1) * a.fstride + per, T, sizeof(cplx<T>), "z forward", "source fields");
  } else {
    for (long long f = 0; f < F; ++f) {
      GS_RANGE(a.src[f], per, T, sizeof(cplx<T>), "z forward", "source field");
      if (a.mul[f]) GS_RANGE(a.mul[f], per, T, sizeof(cplx<T>), "z forward", "multiplier field");
    }
  }
  GS_RANGE(a.dst, a.nrows * H, cplx<T>, sizeof(cplx<T>), "z forward", "spectrum");
  return cudaSuccess;
}

template <typename T, int H> static cudaError_t zfwd_n(ZfwdArgs<T>& a, cudaStream_t s, int lines_req) {
  using L = Line<T, H>;
  if (bounds_check_on()) {
    const cudaError_t e = zfwd_ranges<T, H>(a);
    if (e != cudaSuccess) return e;
  }
  long long lpc = 256 / L::P;
  // a requested line count (autotuner) when the block stays within 1024
  // threads and the shared-memory opt-in
  if (lines_req > 0 && (long long)lines_req * L::P <= max_block_threads<k_zfwd<T, H>>() &&
      (size_t)lines_req * L::PAD * sizeof(cplx<T>) <= 200 * 1024)
    lpc = lines_req;
  if (lpc < 1) lpc = 1;
  if (lpc > a.nrows) lpc = a.nrows;
  a.lpc = (int)lpc;
  const size_t smem = (size_t)lpc * L::PAD * sizeof(cplx<T>);
  allow_max_smem<k_zfwd<T, H>>();
  const long long grid = (a.nrows + lpc - 1) / lpc;
  k_zfwd<T, H><<<(unsigned)grid, (unsigned)(L::P * lpc), smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T> cudaError_t launch_zfwd(ZfwdArgs<T>& a, int H, cudaStream_t s, int lines_req) {
  switch (H) {
#define GS_C(N_) \
  case N_:       \
    return zfwd_n<T, N_>(a, s, lines_req);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T, int N1, int DIR, int R1 = Plan<N1>::R1>
static cudaError_t ypass_n(YArgs<T>& a, int F, cudaStream_t s, int cols_req) {
  using L = Line<T, N1, R1>;
  // a requested column count (autotuner): a power of two dividing h that the
  // kernel can launch with and whose tile fits the shared-memory opt-in
  if (cols_req > 0 && (cols_req & (cols_req - 1)) == 0 && a.h % cols_req == 0 &&
      (long long)cols_req * L::P <= max_block_threads<k_ypass<T, N1, DIR, R1>>() &&
      (size_t)cols_req * L::PAD * sizeof(cplx<T>) <= 200 * 1024)
    a.tz = cols_req;
  const size_t smem = (size_t)a.tz * L::PAD * sizeof(cplx<T>);
  GS_RANGE(a.spec, (long long)F * a.n0 * N1 * a.h, cplx<T>, sizeof(cplx<T>), "y pass", "spectrum");
  allow_max_smem<k_ypass<T, N1, DIR, R1>>();
  dim3 grid(a.h / a.tz, a.n0, F);
  k_ypass<T, N1, DIR, R1><<<grid, a.tz * L::P, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T, int N1, int DIR>
static cudaError_t ypass_plan(YArgs<T>& a, int F, cudaStream_t s, int cols_req, int radix) {
  if constexpr (N1 == 64 || N1 == 128 || N1 == 256) {
    constexpr int ALT = N1 == 64 ? 16 : 32;
    if (radix == ALT) return ypass_n<T, N1, DIR, ALT>(a, F, s, cols_req);
  }
  return ypass_n<T, N1, DIR>(a, F, s, cols_req);
}

template <typename T>
cudaError_t launch_ypass(YArgs<T>& a, int n1, int F, int dir, cudaStream_t s, int cols_req, int radix) {
  if (n1 == 1) return cudaSuccess;
  a.tz = pick_tz(a.h);
  // FP32 columns of 8 on lines of 256: y forward 0.076 against 0.087 ms for 16
  // at 256^3 x 3 (at 128^3, 16 stays faster)
  if (sizeof(T) == 4 && n1 >= 256 && a.tz > 8) a.tz = 8;
  switch (n1) {
#define GS_C(N_) \
  case N_:       \
    return dir < 0 ? ypass_plan<T, N_, -1>(a, F, s, cols_req, radix) : ypass_plan<T, N_, 1>(a, F, s, cols_req, radix);
    GS_SIZE_CASES(GS_C)
#undef GS_C
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace gs
