// gs_k_xtma.cu -- launcher of the TMA-fed x pass (gs_xtma.cuh): tensor map of
// the input spectra, persistent grid of two blocks per SM.
#include <cudaTypedefs.h>

#include "gs_launch.h"
#include "gs_xtma.cuh"

namespace gs {

// off by default: at 256^3 x 3 the pass measured 0.167 ms against 0.163 ms
// for the one-tile-per-block pass, whose second resident block already hides
// the loads
static std::atomic<bool> g_x_prefetch{false};

void set_x_prefetch(bool on) { g_x_prefetch.store(on); }
bool x_prefetch() { return g_x_prefetch.load(); }

unsigned int x_wait_timeouts() {
  unsigned int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_x_wait_timeouts, sizeof(v)) != cudaSuccess) return ~0u;
  return v;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not offer it.
static PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  // a function-local static initialiser runs once, thread-safely
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
    return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
  }();
  return fn;
}

static int sm_count() {
  const int dev = current_device();
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = 148;
  }
  return n;
}

template <int N0, int FM, int TZ> static cudaError_t xtma_n(XArgs<float>& a, cudaStream_t s) {
  using Sh = XTmaShape<N0, FM, TZ>;
  const auto encode = encode_tiled();
  if (!encode) return cudaErrorNotSupported;
  const size_t vb = sizeof(cplx<float>);
  CUtensorMap map;
  const cuuint64_t dims[4] = {(cuuint64_t)a.h, (cuuint64_t)a.n1, (cuuint64_t)a.n0, (cuuint64_t)a.F};
  const cuuint64_t strides[3] = {(cuuint64_t)a.h * vb, (cuuint64_t)a.n1 * a.h * vb,
                                 (cuuint64_t)a.n0 * a.n1 * a.h * vb};
  const cuuint32_t box[4] = {(cuuint32_t)TZ, 1, (cuuint32_t)N0, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<cplx<float>*>(a.in), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorNotSupported;
  if (a.F != FM) return cudaErrorNotSupported;
  a.tz = TZ;
  a.groups = a.F;
  const size_t smem = 2 * (size_t)FM * Sh::region_bytes + (size_t)(FM + 1) * N0 * vb + 2 * sizeof(uint64_t);
  // two blocks per SM need the largest shared-memory carve-out; the grid is
  // what the occupancy calculator says fits at once
  // (attributes and occupancy belong to the current device: one entry per device)
  static std::atomic<int> per_sm_dev[kMaxDevices];
  const int dev = current_device();
  int per_sm = dev >= 0 && dev < kMaxDevices ? per_sm_dev[dev].load(std::memory_order_acquire) : 0;
  if (!per_sm) {
    const auto k = k_xpass_tma<N0, FM, TZ, TableOp>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, Sh::threads, smem) != cudaSuccess || per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    if (dev >= 0 && dev < kMaxDevices) per_sm_dev[dev].store(per_sm, std::memory_order_release);
  }
  const int ntiles = (a.h / TZ) * a.n1;
  int grid = per_sm * sm_count();
  if (grid > ntiles) grid = ntiles;
  k_xpass_tma<N0, FM, TZ, TableOp><<<grid, Sh::threads, smem, s>>>(a, map, ntiles);
  return cudaGetLastError();
}

// The TMA-fed pass covers the square table contraction of three or five
// fields of one FP32 simulation on n0 = 128 or 256 (8-column tiles, so
// h % 8 == 0); cudaErrorNotSupported sends the caller to the plain pass.
cudaError_t launch_xtma(XArgs<float>& a, cudaStream_t s) {
  if (!g_x_prefetch || !a.btab || a.F != a.G || a.nsim > 1 || a.simscale || a.kz_off || a.hg)
    return cudaErrorNotSupported;
  if (a.h % 8 != 0 || (reinterpret_cast<uintptr_t>(a.in) & 15) != 0) return cudaErrorNotSupported;
  if (a.F == 3) {
    if (a.n0 == 256) return xtma_n<256, 3, 8>(a, s);
    if (a.n0 == 128) return xtma_n<128, 3, 8>(a, s);
  } else if (a.F == 5) {  // precipitate: 4 variants + concentration
    if (a.n0 == 256) return xtma_n<256, 5, 8>(a, s);
    if (a.n0 == 128) return xtma_n<128, 5, 8>(a, s);
  }
  return cudaErrorNotSupported;
}

}  // namespace gs
