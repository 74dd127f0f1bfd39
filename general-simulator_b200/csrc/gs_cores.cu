// gs_cores.cu -- nuclei of the precipitate chain painted on the device.
//
// Replaces the host triple loops of Dynamics_cores (src/dynamics_cores.cu:
// 55-186): every grid point is tested against every nucleus on the device.
// A point belongs to a nucleus at (ox, oy, oz) of radius r when one of seven
// images of its offset -- the offset itself and the offset shifted by +-n
// along one axis at a time, the reference's periodic rule -- has
// dx^2 + dy^2 + dz^2 <= r^2 (r^2 formed in double from the float radius, as
// pow(0.0f + Radius, 2) does there).  Inside a nucleus the concentration is
// c_core and eta of the nucleus's variant is 1; a point inside nuclei of
// several variants has each of them at 1; elsewhere c_matrix and 0.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/gs_capi.h"
#include "gs_sim.h"

namespace {

__device__ __forceinline__ bool in_core(int i, int j, int k, int ox, int oy, int oz, int nx, int ny, int nz, double r2) {
  const long long dx = i - ox, dy = j - oy, dz = k - oz;
  auto inside = [r2](long long a, long long b, long long c) { return (double)(a * a + b * b + c * c) <= r2; };
  return inside(dx, dy, dz) || inside(dx + nx, dy, dz) || inside(dx - nx, dy, dz) || inside(dx, dy + ny, dz) ||
         inside(dx, dy - ny, dz) || inside(dx, dy, dz + nz) || inside(dx, dy, dz - nz);
}

__global__ void k_cores(const int4* cores, int ncores, int nx, int ny, int nz, int V, double r2, float c_matrix,
                        float c_core, float* eta, float* conc) {
  const long long N = (long long)nx * ny * nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((long long)ny * nz));
    unsigned mask = 0;
    for (int q = 0; q < ncores; ++q) {
      const int4 o = cores[q];
      if (in_core(i, j, k, o.x, o.y, o.z, nx, ny, nz, r2)) mask |= 1u << o.w;
    }
    conc[c] = mask ? c_core : c_matrix;
    for (int v = 0; v < V; ++v) eta[(long long)v * N + c] = (mask >> v) & 1u ? 1.0f : 0.0f;
  }
}

}  // namespace

extern "C" int gs_cores_paint(int nx, int ny, int nz, int nvariants, int ncores, const int* centers,
                              const int* variant, double radius, double c_matrix, double c_core, float* eta_host,
                              float* conc_host) {
  if (nx < 1 || ny < 1 || nz < 1) return gs_set_error(GS_EINVAL, "gs_cores_paint: grid %d %d %d", nx, ny, nz);
  if (nvariants < 1 || nvariants > 32) return gs_set_error(GS_EINVAL, "gs_cores_paint: %d variants", nvariants);
  if (ncores < 0 || (ncores > 0 && (!centers || !variant)) || !eta_host || !conc_host)
    return gs_set_error(GS_EINVAL, "gs_cores_paint: bad arguments");
  std::vector<int4> hc(ncores > 0 ? ncores : 1);
  for (int q = 0; q < ncores; ++q) {
    if (variant[q] < 0 || variant[q] >= nvariants)
      return gs_set_error(GS_EINVAL, "gs_cores_paint: nucleus %d has variant %d of %d", q, variant[q], nvariants);
    hc[q] = make_int4(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2], variant[q]);
  }
  const long long N = (long long)nx * ny * nz;
  int4* dc = nullptr;
  float* de = nullptr;
  float* dcn = nullptr;
  auto done = [&](int rc) {
    cudaFree(dc);
    cudaFree(de);
    cudaFree(dcn);
    return rc;
  };
  int rc;
  if ((rc = gs_cuda_check(cudaMalloc(&dc, sizeof(int4) * hc.size()), "cudaMalloc nuclei")) != GS_OK) return done(rc);
  if ((rc = gs_cuda_check(cudaMalloc(&de, sizeof(float) * N * nvariants), "cudaMalloc eta")) != GS_OK) return done(rc);
  if ((rc = gs_cuda_check(cudaMalloc(&dcn, sizeof(float) * N), "cudaMalloc concentration")) != GS_OK) return done(rc);
  if ((rc = gs_cuda_check(cudaMemcpy(dc, hc.data(), sizeof(int4) * hc.size(), cudaMemcpyHostToDevice), "upload")) !=
      GS_OK)
    return done(rc);
  const double r = (double)(float)radius;
  long long nb = (N + 255) / 256;
  if (nb > 148 * 16) nb = 148 * 16;
  k_cores<<<(unsigned)nb, 256>>>(dc, ncores, nx, ny, nz, nvariants, r * r, (float)c_matrix, (float)c_core, de, dcn);
  if ((rc = gs_cuda_check(cudaGetLastError(), "nuclei kernel")) != GS_OK) return done(rc);
  if ((rc = gs_cuda_check(cudaMemcpy(eta_host, de, sizeof(float) * N * nvariants, cudaMemcpyDeviceToHost),
                          "download eta")) != GS_OK)
    return done(rc);
  if ((rc = gs_cuda_check(cudaMemcpy(conc_host, dcn, sizeof(float) * N, cudaMemcpyDeviceToHost),
                          "download concentration")) != GS_OK)
    return done(rc);
  return done(GS_OK);
}
