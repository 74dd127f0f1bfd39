// gs_bc.cuh -- index asserts of the bounds-check build.
//
// GS_BCI(i, n, site) names the element index i of a buffer of n elements
// (GS_BCO: index i from a pointer at element off of the buffer; GS_BCR: the
// w elements of a vector access from i).  In the normal build each is i
// itself and costs nothing.  In the bounds-check
// build (-DGS_BOUNDS_CHECK, libgsb200_bc.so) it checks 0 <= i < n; an index
// outside records the first violation of this module (site, index, extent,
// block, thread), counts every violation, and yields 0, so that the access
// lands on the buffer's first element: nothing outside the buffer is read or
// written, no thread traps, and every barrier is still reached.  A step that
// met a violation has void results; the library's step entries report it as
// GS_EBOUNDS, and gs_bounds_check_read returns the record.
//
// The extents n are the launch's logical extents, formed from the kernel's
// arguments (rows, lines, fields).  The host half of the check
// (gs_bounds.cu, check_range in the launchers) shows each logical extent to
// lie inside its allocation, so the two together bound every access.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gs {

// the checked access sites (the host names them in messages)
enum BcSite : int {
  BC_NONE = 0,
  BC_SELFTEST,
  BC_ZFWD_SRC,
  BC_ZFWD_DST,
  BC_ZFWD_SMEM,
  BC_Y_SPEC,
  BC_Y_SMEM,
  BC_X_IN,
  BC_X_OUT,
  BC_X_TAB,
  BC_X_KTAB,
  BC_X_SMEM,
  BC_UPD_SPEC,
  BC_UPD_ETA,
  BC_UPD_ETA_OUT,
  BC_UPD_AUX,
  BC_UPD_HALO,
  BC_UPD_NEXT,
  BC_UPD_PARTIALS,
  BC_UPD_SMEM,
  BC_ZINV_SPEC,
  BC_ZINV_DST,
  BC_PMID_SRC,
  BC_PMID_DST,
  BC_PMID_SMEM,
  BC_PZF_SPEC,
  BC_PZF_FIELD,
  BC_PZF_SMEM,
  BC_PLOCAL,
  BC_XTMA_OUT,
  BC_COUNT
};

// number of words of one module's record: violations, site, index, extent, block, thread
constexpr int kBcWords = 6;

#ifdef GS_BOUNDS_CHECK
// host side (gs_bounds.cu): every module registers the reader of its own record
using BcReader = cudaError_t (*)(unsigned long long* rec, bool clear);
void bc_register(BcReader r);

// internal linkage (static, no anonymous namespace, which nvcc's kernel
// registration cannot tell apart from a unit's own): one record per module
static __device__ unsigned long long bc_rec[kBcWords];

static __device__ __noinline__ void bc_note(int site, long long i, long long n) {
  if (atomicAdd(&bc_rec[0], 1ull) == 0ull) {
    bc_rec[1] = (unsigned long long)site;
    bc_rec[2] = (unsigned long long)i;
    bc_rec[3] = (unsigned long long)n;
    bc_rec[4] = (unsigned long long)blockIdx.x | ((unsigned long long)blockIdx.y << 32);
    bc_rec[5] = (unsigned long long)threadIdx.x;
  }
}

static __device__ __forceinline__ long long bc_idx(long long i, long long n, int site) {
  if ((unsigned long long)i < (unsigned long long)n) return i;
  bc_note(site, i, n);
  return 0;
}

// index i relative to a pointer at element off of the buffer: i itself when
// off + i lies in [0, n), else -off (the buffer's first element)
static __device__ __forceinline__ long long bc_off(long long off, long long i, long long n, int site) {
  if ((unsigned long long)(off + i) < (unsigned long long)n) return i;
  bc_note(site, off + i, n);
  return -off;
}

// the same for the w elements i .. i + w - 1 of a vector access
static __device__ __forceinline__ long long bc_range(long long off, long long i, long long w, long long n, int site) {
  if (off + i >= 0 && off + i + w <= n) return i;
  bc_note(site, off + i < 0 ? off + i : off + i + w - 1, n);
  return -off;
}

static __device__ __forceinline__ unsigned dyn_smem_bytes() {
  unsigned r;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
  return r;
}

// does a block's shared-memory layout of `need` elements of `bytes` each fit
// the dynamic shared memory it was launched with
static __device__ __forceinline__ bool bc_smem_fits(long long need, unsigned bytes, int site) {
  const long long have = (long long)(dyn_smem_bytes() / bytes);
  if (need <= have) return true;
  if (threadIdx.x == 0) bc_note(site, need - 1, have);
  return false;
}

static cudaError_t bc_read_module(unsigned long long* rec, bool clear) {
  cudaError_t e = cudaMemcpyFromSymbol(rec, bc_rec, sizeof(unsigned long long) * kBcWords);
  if (e == cudaSuccess && clear) {
    const unsigned long long z[kBcWords] = {0, 0, 0, 0, 0, 0};
    e = cudaMemcpyToSymbol(bc_rec, z, sizeof(z));
  }
  return e;
}

static const bool bc_module_registered = (bc_register(&bc_read_module), true);

#define GS_BCI(i, n, site) (::gs::bc_idx((long long)(i), (long long)(n), (site)))
#define GS_BCO(off, i, n, site) (::gs::bc_off((long long)(off), (long long)(i), (long long)(n), (site)))
#define GS_BCR(off, i, w, n, site) \
  (::gs::bc_range((long long)(off), (long long)(i), (long long)(w), (long long)(n), (site)))
// a statement only the check build compiles (extents and offsets of the checks),
// and an argument that is 0 in the normal build
#define GS_BC_DECL(...) __VA_ARGS__;
#define GS_BCX(...) (__VA_ARGS__)
// at a kernel's start: the whole block returns when its shared-memory layout
// (need elements of type E; the same for every thread) exceeds what it was
// launched with, before any thread touches shared memory or a barrier
#define GS_BC_SMEM_GUARD(need, E, site) \
  if (!::gs::bc_smem_fits((long long)(need), (unsigned)sizeof(E), (site))) return;
#else
// the index exactly as written at the use (no parentheses added), so the
// normal build compiles the same expressions as without the checks
#define GS_BCI(i, n, site) i
#define GS_BCO(off, i, n, site) i
#define GS_BCR(off, i, w, n, site) i
#define GS_BC_DECL(...)
#define GS_BCX(...) 0
#define GS_BC_SMEM_GUARD(need, E, site)
#endif

}  // namespace gs
