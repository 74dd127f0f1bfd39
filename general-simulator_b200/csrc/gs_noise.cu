// gs_noise.cu -- the noise stream of the step kernels, exposed for checking.
//
// The step kernels draw their Langevin noise in registers (gs_philox.cuh:
// Philox4x32-10 on the counter (quad, step, sim, slot), key = the 64-bit
// seed, Box-Muller on 24-bit uniforms); the reference draws it from cuRAND
// into a field (src/random.cu:79-82).  gs_noise_block evaluates exactly the
// device functions the kernels inline -- philox4x32_10 and normal_quad<T> --
// for a range of quads, so that a caller can compare the raw 32-bit words
// with any other Philox4x32-10 implementation bit for bit, and the normals
// with its own Box-Muller.
#include <cuda_runtime.h>

#include "../../include/gs_capi.h"
#include "gs_philox.cuh"
#include "gs_sim.h"

namespace {

template <typename T>
__global__ void k_noise_block(uint32_t k0, uint32_t k1, uint32_t step, uint32_t sim, uint32_t slot, uint32_t quad0,
                              int nquads, uint32_t* words, T* normals) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nquads) return;
  const uint32_t quad = quad0 + (uint32_t)q;  // wraps modulo 2^32 like the counter word
  const gs::Philox4 o = gs::philox4x32_10(quad, step, sim, slot, k0, k1);
  if (words) {
    uint4 w;
    w.x = o.x[0];
    w.y = o.x[1];
    w.z = o.x[2];
    w.w = o.x[3];
    reinterpret_cast<uint4*>(words)[q] = w;
  }
  if (normals) {
    T z[4];
    gs::normal_quad<T>(quad, step, sim, slot, k0, k1, z);
#pragma unroll
    for (int i = 0; i < 4; ++i) normals[4 * (long long)q + i] = z[i];
  }
}

template <typename T>
int noise_block(uint64_t seed, uint32_t step, uint32_t sim, uint32_t slot, uint32_t quad0, int nquads,
                uint32_t* words_host, void* normals_host) {
  uint32_t* dw = nullptr;
  T* dn = nullptr;
  auto done = [&](int rc) {
    if (dw) cudaFree(dw);
    if (dn) cudaFree(dn);
    return rc;
  };
  const size_t nw = 4 * (size_t)nquads;
  int rc;
  if (words_host && (rc = gs_cuda_check(cudaMalloc(&dw, nw * sizeof(uint32_t)), "cudaMalloc words")) != GS_OK)
    return done(rc);
  if (normals_host && (rc = gs_cuda_check(cudaMalloc(&dn, nw * sizeof(T)), "cudaMalloc normals")) != GS_OK)
    return done(rc);
  const int threads = 256;
  const int blocks = (nquads + threads - 1) / threads;
  k_noise_block<T><<<blocks, threads>>>((uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32), step, sim, slot,
                                        quad0, nquads, dw, dn);
  if ((rc = gs_cuda_check(cudaGetLastError(), "noise kernel")) != GS_OK) return done(rc);
  if (dw && (rc = gs_cuda_check(cudaMemcpy(words_host, dw, nw * sizeof(uint32_t), cudaMemcpyDeviceToHost),
                                "download words")) != GS_OK)
    return done(rc);
  if (dn && (rc = gs_cuda_check(cudaMemcpy(normals_host, dn, nw * sizeof(T), cudaMemcpyDeviceToHost),
                                "download normals")) != GS_OK)
    return done(rc);
  return done(GS_OK);
}

}  // namespace

extern "C" int gs_noise_block(uint64_t seed, uint32_t step, uint32_t sim, uint32_t slot, uint32_t quad0,
                              int nquads, int dtype, uint32_t* words, void* normals) {
  if (nquads < 0 || nquads > (1 << 24)) return gs_set_error(GS_EINVAL, "gs_noise_block: %d quads", nquads);
  if (dtype != GS_DTYPE_F32 && dtype != GS_DTYPE_F64) return gs_set_error(GS_EINVAL, "gs_noise_block: dtype %d", dtype);
  if (nquads == 0 || (!words && !normals)) return GS_OK;
  return dtype == GS_DTYPE_F64 ? noise_block<double>(seed, step, sim, slot, quad0, nquads, words, normals)
                               : noise_block<float>(seed, step, sim, slot, quad0, nquads, words, normals);
}
