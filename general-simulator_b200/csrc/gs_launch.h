// gs_launch.h -- host launchers of the pass kernels (one translation unit
// per kernel family, dispatching the runtime line length to the compiled
// template instance).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include "gs_common.cuh"

namespace gs {

template <typename T> struct ZfwdArgs;
template <typename T> struct YArgs;
template <typename T> struct XArgs;
template <typename T> struct MartArgs;
template <typename T> struct ZinvArgs;
template <typename T> struct PrecipLocalArgs;
template <typename T> struct PrecipStatsArgs;

// line lengths with a compiled plan
bool size_supported(int n);
// columns per block of the y and x passes
int pick_tz(int h);

// lines_req / cols_req: tile sizes asked by the autotuner (0 = the default
// choice; values the launch cannot take fall back to it)
template <typename T> cudaError_t launch_zfwd(ZfwdArgs<T>& a, int H, cudaStream_t s, int lines_req = 0);
// radix: the first-stage radix of the y lines (0: the default plan;
// ypass_alt_radix(n1): the alternative split, for lines of 64, 128 and 256)
template <typename T>
cudaError_t launch_ypass(YArgs<T>& a, int n1, int F, int dir, cudaStream_t s, int cols_req = 0, int radix = 0);
inline int ypass_alt_radix(int n1) { return n1 == 256 ? 32 : n1 == 128 ? 32 : n1 == 64 ? 16 : 0; }
template <typename T> cudaError_t launch_xcontract(XArgs<T>& a, cudaStream_t s);
// TMA-fed x pass (gs_k_xtma.cu): cudaErrorNotSupported when the case is not
// covered (the caller then runs the plain pass)
cudaError_t launch_xtma(XArgs<float>& a, cudaStream_t s);
void set_x_prefetch(bool on);
bool x_prefetch();
unsigned int x_wait_timeouts();
template <typename T> cudaError_t launch_xprecip(XArgs<T>& a, cudaStream_t s);
// eta_p' = D u_p, one field per grid-z slice (F = G = 1)
template <typename T> cudaError_t launch_xprecip_eta(XArgs<T>& a, cudaStream_t s);
// the transposed precipitate update (F = 2, G = 3 per grid-z slice)
template <typename T> cudaError_t launch_xprecip_adjoint(XArgs<T>& a, cudaStream_t s);
// field-count class (3, 5 or 9) of the B octant table of V variants
inline int btab_class(int V) { return V <= 3 ? 3 : (V <= 5 ? 5 : 9); }
inline int btab_stride(int V) {
  const int c = btab_class(V);
  return ((c * (c + 1) / 2) + 1) & ~1;
}
template <typename T> struct ElasticConst;
template <typename T>
cudaError_t launch_btab_fill(const ElasticConst<T>& ec, int n0, int n1, int n2, T* tab, cudaStream_t s);
template <typename T> cudaError_t launch_zinv(ZinvArgs<T>& a, int H, cudaStream_t s);
template <typename T> cudaError_t launch_precip_local(PrecipLocalArgs<T>& a, cudaStream_t s);
template <typename T> struct PrecipMidArgs;
template <typename T> struct PrecipZArgs;
// returns cudaErrorInvalidConfiguration when a row's lines exceed one block
template <typename T> cudaError_t launch_precip_zinv_fwd(PrecipZArgs<T>& a, int H, cudaStream_t s);
// returns cudaErrorInvalidConfiguration when a row's lines exceed one block
template <typename T> cudaError_t launch_precip_mid(PrecipMidArgs<T>& a, int H, cudaStream_t s);
template <typename T> cudaError_t launch_defect(const T* eta, T* defect, long long N, int V, cudaStream_t s);
template <typename T> cudaError_t launch_precip_stats(PrecipStatsArgs<T>& a, cudaStream_t s, int* nblocks);
// returns the number of blocks through nblocks (statistics partial rows)
// nsim > 0: nsim batched simulations with constants in a.mcs
template <typename T>
cudaError_t launch_mart_update(MartArgs<T>& a, int H, bool stats, cudaStream_t s, int* nblocks, int nsim = 0);
template <typename T> struct MartConst;
template <typename T> cudaError_t launch_bump_step(MartConst<T>* mcs, int n, cudaStream_t s);

// the current device, and a bound on the devices the per-device caches below track
constexpr int kMaxDevices = 64;
inline int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    d = 0;
  }
  return d;
}

// opt a kernel in to the largest dynamic shared memory once per device (the
// attribute belongs to the current device; the launch still asks only for
// what it needs); no attribute calls during capture once a device has been
// used (one flag array per kernel: the template is instantiated per function)
template <auto Kernel> inline void allow_max_smem() {
  static std::atomic<bool> done[kMaxDevices];
  const int d = current_device();
  if (d < 0 || d >= kMaxDevices) {
    cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    return;
  }
  if (!done[d].load(std::memory_order_acquire)) {
    // setting the same value twice from two threads is harmless
    cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    done[d].store(true, std::memory_order_release);
  }
}
cudaError_t launch_reduce(const double* partials, int nb, int n, double* out, cudaStream_t s);

// the largest block a kernel can be launched with (its register use), once
template <auto Kernel> inline int max_block_threads() {
  static std::atomic<int> v{0};
  int r = v.load(std::memory_order_relaxed);
  if (!r) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, Kernel) == cudaSuccess) {
      r = fa.maxThreadsPerBlock;
    } else {
      cudaGetLastError();
      r = 256;
    }
    v.store(r, std::memory_order_relaxed);
  }
  return r;
}

// Bounds checks (gs_bounds.cu).  check_range: does [p, p + elems * elem_bytes)
// lie in one device allocation, with p aligned to `align` (cudaErrorInvalidValue
// and a message for bounds_message() otherwise; cudaSuccess while the check is
// off).  bc_after: the bounds-check build's end of a step entry (wait, then
// GS_EBOUNDS after an index violation); rc itself in a normal build.
bool bounds_check_on();
void set_bounds_check(bool on);
const char* bounds_message();
void clear_bounds_message();
cudaError_t check_range(const void* p, long long elems, size_t elem_bytes, size_t align, const char* kernel,
                        const char* what);
int bc_after(int rc, cudaStream_t st);
// in a launcher: refuse the launch when a buffer range does not fit
#define GS_RANGE(p, n, E, align, kernel, what)                                                            \
  do {                                                                                                    \
    if (::gs::bounds_check_on()) {                                                                        \
      const cudaError_t e__ = ::gs::check_range((p), (long long)(n), sizeof(E), (align), (kernel), (what)); \
      if (e__ != cudaSuccess) return e__;                                                                 \
    }                                                                                                     \
  } while (0)

#define GS_SIZE_CASES(M) \
  M(1) M(2) M(4) M(6) M(8) M(12) M(16) M(24) M(32) M(48) M(64) M(96) M(128) M(256)

}  // namespace gs
