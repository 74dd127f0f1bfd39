// gs_bounds.cu -- the bounds checks of the pass kernels.
//
// Two halves, both off in a normal run:
//
// (1) The launch-range check (every build).  With GS_BOUNDS_CHECK=1 in the
// environment (read once), after gs_set_bounds_check(1), or always in the
// bounds-check build, every pass launcher first checks, for each buffer its
// kernel reads or writes, that the byte range the launch's logical extent
// covers lies inside one device allocation (the driver's
// cuMemGetAddressRange) and starts on the alignment of the kernel's vector
// accesses.  A range that does not fit refuses the launch with
// cudaErrorInvalidValue and a message naming the kernel and the buffer; no
// kernel runs on a bad range.  Memory the driver cannot place (a module's
// static array) is checked for alignment only.
//
// (2) The index asserts (the bounds-check build, -DGS_BOUNDS_CHECK):
// GS_BCI in the kernels (gs_bc.cuh) checks each index against that logical
// extent, records the first violation per module and keeps the access inside
// the buffer.  This file gathers the modules' records.
//
// The range check costs a driver query per buffer per launch and the index
// asserts a compare per access: debugging aids, not for timing runs.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "gs_launch.h"
#include "../../include/gs_capi.h"

int gs_set_error(int code, const char* fmt, ...);
int gs_cuda_check(cudaError_t e, const char* what);

namespace gs {

namespace {
#ifdef GS_BOUNDS_CHECK
constexpr int kDefaultOn = 1;
#else
constexpr int kDefaultOn = 0;
#endif
std::atomic<int> g_on{-1};  // -1: not read from the environment yet
thread_local char g_msg[320] = "";

PFN_cuMemGetAddressRange_v3020 range_fn() {
  static const PFN_cuMemGetAddressRange_v3020 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuMemGetAddressRange_v3020>(p);
    cudaGetLastError();
    return static_cast<PFN_cuMemGetAddressRange_v3020>(nullptr);
  }();
  return fn;
}

const char* const kSiteNames[BC_COUNT] = {
    "none",           "selftest",        "zfwd source",       "zfwd spectrum",    "zfwd shared line",
    "y spectrum",     "y shared tile",   "x input spectrum",  "x output spectrum", "x B table",
    "x K table",      "x shared tile",   "update spectrum",   "update eta",        "update eta out",
    "update aux field", "update halo",   "update next spectrum", "update partials", "update shared rows",
    "zinv spectrum",  "zinv field",      "precip mid source", "precip mid spectrum", "precip mid shared",
    "precip z spectrum", "precip z field", "precip z shared", "precip local field", "x tma output"};

#ifdef GS_BOUNDS_CHECK
std::vector<BcReader>& readers() {
  static std::vector<BcReader> v;
  return v;
}
std::mutex& readers_mutex() {
  static std::mutex m;
  return m;
}
#endif
}  // namespace

#ifdef GS_BOUNDS_CHECK
void bc_register(BcReader r) {
  std::lock_guard<std::mutex> g(readers_mutex());
  readers().push_back(r);
}
#endif

bool bounds_check_on() {
  int v = g_on.load(std::memory_order_relaxed);
  if (v < 0) {
    const char* e = getenv("GS_BOUNDS_CHECK");
    v = (e && *e) ? (strcmp(e, "0") != 0 ? 1 : 0) : kDefaultOn;
    int expected = -1;
    g_on.compare_exchange_strong(expected, v);
    v = g_on.load();
  }
  return v == 1;
}

void set_bounds_check(bool on) { g_on.store(on ? 1 : 0); }

const char* bounds_message() { return g_msg; }
void clear_bounds_message() { g_msg[0] = 0; }

cudaError_t check_range(const void* p, long long elems, size_t elem_bytes, size_t align, const char* kernel,
                        const char* what) {
  if (!bounds_check_on() || elems <= 0) return cudaSuccess;
  if (!p) {
    snprintf(g_msg, sizeof(g_msg), "bounds check: %s: %s is null but %lld elements are reached", kernel, what,
             elems);
    return cudaErrorInvalidValue;
  }
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const size_t bytes = (size_t)elems * elem_bytes;
  if (align > 1 && (a % align) != 0) {
    snprintf(g_msg, sizeof(g_msg), "bounds check: %s: %s at %p is not %zu-byte aligned", kernel, what, p, align);
    return cudaErrorInvalidValue;
  }
  const auto fn = range_fn();
  if (!fn) return cudaSuccess;
  CUdeviceptr base = 0;
  size_t size = 0;
  if (fn(&base, &size, (CUdeviceptr)a) != CUDA_SUCCESS) return cudaSuccess;  // not a driver allocation
  const uintptr_t end = (uintptr_t)base + size;
  if (a < (uintptr_t)base || bytes > end - a) {
    snprintf(g_msg, sizeof(g_msg),
             "bounds check: %s: %s reaches %zu bytes from %p, its allocation ends %zu bytes after that address",
             kernel, what, bytes, p, (size_t)(a < end ? end - a : 0));
    return cudaErrorInvalidValue;
  }
  return cudaSuccess;
}

#ifdef GS_BOUNDS_CHECK
namespace {
__global__ void k_bc_selftest(int* buf, int cap, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    buf[GS_BCI(i, cap, BC_SELFTEST)] = i;
}

// sums the modules' records of the current device; the first nonzero record gives the site
cudaError_t bc_gather(long long out[kBcWords], bool clear) {
  for (int w = 0; w < kBcWords; ++w) out[w] = 0;
  std::lock_guard<std::mutex> g(readers_mutex());
  for (BcReader r : readers()) {
    unsigned long long rec[kBcWords];
    const cudaError_t e = r(rec, clear);
    if (e != cudaSuccess) return e;
    if (rec[0] && !out[0])
      for (int w = 1; w < kBcWords; ++w) out[w] = (long long)rec[w];
    out[0] += (long long)rec[0];
  }
  return cudaSuccess;
}
}  // namespace

// after a step entry: wait for its kernels (unless its stream is being
// captured) and turn recorded violations into GS_EBOUNDS
int bc_after(int rc, cudaStream_t st) {
  if (rc != GS_OK) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return rc;
  }
  const int r = gs_cuda_check(cudaDeviceSynchronize(), "bounds check: synchronize");
  if (r != GS_OK) return r;
  long long rec[kBcWords];
  const int r2 = gs_cuda_check(bc_gather(rec, false), "bounds check: read the records");
  if (r2 != GS_OK) return r2;
  if (rec[0] == 0) return GS_OK;
  const int site = (rec[1] >= 0 && rec[1] < BC_COUNT) ? (int)rec[1] : 0;
  return gs_set_error(GS_EBOUNDS, "bounds check: %lld index violation(s), first at %s: index %lld of %lld",
                      rec[0], kSiteNames[site], rec[2], rec[3]);
}
#else
int bc_after(int rc, cudaStream_t) { return rc; }
#endif

}  // namespace gs

extern "C" void gs_set_bounds_check(int on) { gs::set_bounds_check(on != 0); }
extern "C" int gs_bounds_check_enabled(void) { return gs::bounds_check_on() ? 1 : 0; }

extern "C" int gs_bounds_check_build(void) {
#ifdef GS_BOUNDS_CHECK
  return 1;
#else
  return 0;
#endif
}

extern "C" const char* gs_bounds_site_name(int site) {
  return (site >= 0 && site < gs::BC_COUNT) ? gs::kSiteNames[site] : "unknown";
}

extern "C" int gs_bounds_check_read(long long* out, int clear) {
  if (!out) return gs_set_error(GS_EINVAL, "gs_bounds_check_read: null output");
#ifdef GS_BOUNDS_CHECK
  const int r = gs_cuda_check(cudaDeviceSynchronize(), "gs_bounds_check_read: synchronize");
  if (r != GS_OK) return r;
  return gs_cuda_check(gs::bc_gather(out, clear != 0), "gs_bounds_check_read");
#else
  (void)clear;
  for (int w = 0; w < gs::kBcWords; ++w) out[w] = 0;
  return gs_set_error(GS_ENOTSUP, "gs_bounds_check_read: this library is not the bounds-check build");
#endif
}

extern "C" int gs_bounds_selftest(int* buf, int cap, int n, void* stream) {
  if (!buf || cap < 1 || n < 0) return gs_set_error(GS_EINVAL, "gs_bounds_selftest: bad arguments");
#ifdef GS_BOUNDS_CHECK
  const int r = gs_cuda_check(gs::check_range(buf, cap, sizeof(int), 4, "selftest", "buffer"), "gs_bounds_selftest");
  if (r != GS_OK) return gs_set_error(r, "%s", gs::bounds_message());
  const int grid = n > 0 ? (n + 255) / 256 : 1;
  gs::k_bc_selftest<<<grid < 1184 ? grid : 1184, 256, 0, static_cast<cudaStream_t>(stream)>>>(buf, cap, n);
  return gs_cuda_check(cudaGetLastError(), "gs_bounds_selftest");
#else
  (void)stream;
  // the unchecked kernel would write beyond cap: refused
  return gs_set_error(GS_ENOTSUP, "gs_bounds_selftest: this library is not the bounds-check build");
#endif
}
