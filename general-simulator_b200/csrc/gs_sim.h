// gs_sim.h -- internal state of one simulation handle (gs_sim).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/gs_capi.h"

struct gs_plain_state;  // comparator in the reference's structure (gs_plain.cu)
struct gs_cufft_state;  // cuFFT R2C/C2R comparator (gs_cufft.cu)
struct gs_snaps;        // asynchronous field copies in flight (gs_capi.cu)

struct gs_sim {
  gs_params p;
  // canonical grid: unit axes moved to the front, n2 = last axis of extent > 1
  int n0 = 1, n1 = 1, n2 = 2, h = 1;
  long long N = 0;
  int perm[3] = {0, 1, 2};  // canonical axis -> original axis
  double dcan[3] = {1, 1, 1};
  cudaStream_t own_stream = nullptr;
  void* eta[2] = {nullptr, nullptr};  // ping-pong field set [V][N]
  int cur = 0;
  void* spec = nullptr;   // packed spectra [F][n0][n1][h]
  void* spec2 = nullptr;  // second spectral buffer (stress output, CH chain)
  void* defect = nullptr; // [N]
  void* K = nullptr;      // dislocation coupling sigma(x):eps_p, [V][N]
  void* conc = nullptr;   // concentration [N]
  void* rbuf = nullptr;   // elastic potentials R_a [F][N] (precipitate)
  void* mubuf = nullptr;  // mu_c and g_p [1 + V][N] (precipitate)
  void* stressbuf = nullptr;  // stress components [6][N] (stress model)
  void* ktab = nullptr;   // K(k) per canonical axis (precipitate)
  size_t ktab_off[3] = {0, 0, 0};
  double mass0 = 0;       // FP64 sum of the initial concentration
  void* tw = nullptr;     // twiddle tables
  size_t tw_off[4] = {0, 0, 0, 0};  // n2, h, n1, n0
  double* partials = nullptr;
  size_t partials_cap = 0;
  double* red = nullptr;
  int64_t step = 0;
  int64_t launches = 0;
  int use_graph = 0;
  gs_plain_state* plain = nullptr;
  gs_cufft_state* cufft = nullptr;
  // octant table of B(k) of the martensite contraction: state 1 = valid,
  // 0 = to build, -1 = never (handles that must not allocate), -2 = B is not
  // even in every axis (the contraction is formed on the fly)
  // tile schedule of the passes (0 = each launcher's default); set by the
  // autotuner or the caller
  gs_schedule sched = {0, 0, 0, 0, 0};
  bool trial = false;  // steps that leave the state as it was (autotuner timing)
  // the martensite update also writes the next step's z spectra (fused z
  // forward); spec_ready says the spectrum buffer holds those of eta[spec_cur]
  bool fuse = true;
  bool spec_ready = false;
  int spec_cur = -1;
  void* btab = nullptr;
  size_t btab_bytes = 0;
  int btab_state = 0;
  int btab_fields = 0;  // square size of the tabled contraction
  // batched group: nb simulations of one shape with their own coefficients,
  // fields stored sim after sim; per-sim constants live on the device
  int nb = 1;
  std::vector<gs_params> bp;
  std::vector<int64_t> bstep;
  void* d_mcs = nullptr;
  void* d_simscale = nullptr;
  // gs_sim_use_graph: a captured graph of two steps of a one-simulation group
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gexec_stream = nullptr;
  int gexec_cur = 0;
  // per-pass event marks of gs_sim_profile_step
  static constexpr int kMaxMarks = 32;
  cudaEvent_t marks[kMaxMarks] = {};
  const char* mark_names[kMaxMarks] = {};  // the pass that ends at each mark
  int nmarks = 0;
  bool profiling = false;
  gs_snaps* snaps = nullptr;  // created by the first gs_sim_copy_field_async
  // gs_sim_stage_field_async: the next field set, copied into `stage` on the
  // upload stream while the GPU steps; the next gs_sim_step swaps it in
  void* stage = nullptr;
  cudaStream_t up_stream = nullptr;
  cudaEvent_t up_done = nullptr;     // the staged copy has landed
  cudaEvent_t stage_free = nullptr;  // the buffer now in `stage` is no longer read
  bool staged = false;               // a staged field set waits for the next step
};

// record a pass boundary when gs_sim_profile_step (or GS_TIMING) is active;
// name: the pass that ends here
inline void gs_mark(gs_sim* s, cudaStream_t st, const char* name = nullptr) {
  if (s->profiling && s->nmarks < gs_sim::kMaxMarks) {
    s->mark_names[s->nmarks] = name;
    cudaEventRecord(s->marks[s->nmarks++], st);
  }
}

int gs_set_error(int code, const char* fmt, ...);
int gs_cuda_check(cudaError_t e, const char* what);
void gs_plain_free(gs_sim* s);
void gs_cufft_free(gs_sim* s);
void gs_cufft_invalidate(gs_sim* s);
