/*
 * gs_capi.h -- C ABI of the B200-native phase-field step of General-Simulator.
 *
 * The reference drives its physics through the C++ plugin class
 * GS_NS::Dynamics (src/dynamics.h:9-25): Initialize / Calculate / RunFunc /
 * Fix / Get, with parameters read from the string map Vars and fields from
 * the Data<Real> map Datas.  The plugins that carry the hot path are
 * Dynamics_mart (src/dynamics_mart.cu), Dynamics_precipitate
 * (src/dynamics_precipitate.cu) and Dynamics_stress (src/dynamics_stress.cu).
 *
 * This header replaces what those plugins do on the device with plain C entry
 * points: POD structs, host pointers and sizes, an int status, no exceptions
 * and no C++ or torch types.  The C++ front end (the gsi script interpreter,
 * host/ in this package) keeps the reference's Dynamics interface and calls
 * these functions from Initialize / Calculate / Get.
 *
 * Field layout everywhere: [V][nx][ny][nz], z fastest (include/datamain.th:
 * 72-76 in the reference).  Status codes 0 / -1 / -2 / -3 / -4 / -5 keep the
 * meaning of the reference's Code_* constants (src/pub.h:17-22); the codes
 * below -5 are new.
 */
#ifndef GS_CAPI_H
#define GS_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_CAPI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define GS_OK 0             /* Code_NORMAL */
#define GS_ERR (-1)         /* Code_ERR */
#define GS_EINVAL (-10)     /* bad argument, size or field name */
#define GS_ENOMEM (-11)     /* device allocation failed */
#define GS_ECUDA (-12)      /* a CUDA call or launch failed */
#define GS_ETIMEOUT (-13)   /* a bounded device wait gave up */
#define GS_ENOTSUP (-14)    /* configuration not supported by the kernels */
#define GS_ENODEV (-15)     /* no CUDA device visible */
#define GS_EBOUNDS (-16)    /* the bounds-check build saw an index outside its buffer */

/* ---- enums ------------------------------------------------------------- */
#define GS_MODEL_MART 1        /* Dynamics_mart: TDGL of V variants + FFT elasticity */
#define GS_MODEL_PRECIPITATE 2 /* Dynamics_precipitate: CH(c) + AC(eta_p), semi-implicit */
#define GS_MODEL_STRESS 3      /* Dynamics_stress: stress field of an eta configuration */

/* GS_MODE_BASELINE: the discretisation written for this project (2-4-6
 * Landau, kappa/dx^2 seven-point Laplacian, B(0)=0, k = 2*pi*m/(n*d)).
 * GS_MODE_REFCOMPAT: the reference's own formulas (HEAD side): Laplacian
 * divided by (2d)*3, the square-root Landau form of ChemiFor_Mart_Kernel,
 * k = 2*3.14*d*m/n, B(0) = C:eps:eps, elastic force without the factor 2. */
#define GS_MODE_BASELINE 0
#define GS_MODE_REFCOMPAT 1

#define GS_DTYPE_F32 0
#define GS_DTYPE_F64 1

#define GS_MAX_V 8

/* ---- parameters -------------------------------------------------------- */
typedef struct gs_params {
  int model;     /* GS_MODEL_* */
  int mode;      /* GS_MODE_* */
  int dtype;     /* GS_DTYPE_*: storage and arithmetic type of the fields */
  int nvariants; /* V, 1..GS_MAX_V */
  int nx, ny, nz;
  double dx, dy, dz;
  double dt;

  /* elasticity (all models): eigenstrain of each variant, C_ijkl, the
   * applied (uniform) stress and a multiplier of the elastic driving force */
  double eigenstrain[GS_MAX_V][3][3];
  double cijkl[3][3][3][3];
  double applied_stress[3][3];
  double weight_elastic;

  /* martensite, baseline: f = A2/2 S eta^2 - A4/4 S eta^4 + A6/6 (S eta^2)^3
   * + Ac S_{p<q} eta_p^2 eta_q^2; d eta/dt = -L (df/deta - kappa lap eta +
   * dE_el/deta - 2 sigma_a:eps_p eta_p) + noise */
  double landau[4]; /* A2 A4 A6 Ac */
  double kappa;
  double mobility;

  /* martensite, refcompat (src/dynamics_mart.cu:20-27,40,207-250) */
  double weight_gradient, weight_chemical, weight_dislocation;
  double lpc[4]; /* lpc[2], lpc[3]: a2, a3; a1 = 0.02 (T - T_tr) */
  double transition_temperature;
  double temperature;

  /* noise: baseline adds noise_amp * xi to eta every step; refcompat adds
   * dt * noise_amp * xi (weightnoise).  xi ~ N(0,1) from Philox4x32-10 with
   * key (seed lo, seed hi) and counter (cell, step, sim_id, block). */
  double noise_amp;
  uint64_t seed;
  uint32_t sim_id;
  uint32_t pad0;

  /* precipitate (src/dynamics_precipitate.cu:20-29,118-248): the local
   * free-energy derivatives use coef[1..7] exactly as the reference's
   * LocalCon/LocalEtaFreeEnergy kernels; baseline configs map onto them. */
  double coef[8];
  double c1, c2;          /* Concentration1, Concentration2 */
  double kappa_c;         /* beta: gradient coefficient of c */
  double kappa_eta;       /* arfi: gradient coefficient of eta */
  double mobility_c;      /* meta */
  double mobility_eta;    /* lpp */
  double xi;              /* elastic scale Xi (precipitate and stress) */
  double misfit_c;        /* dilatational eigenstrain per unit c (baseline) */
  int c_elastic;          /* 1: c couples to elasticity through misfit_c */
  int mass_projection;    /* 1: hold sum(c) at its FP64 initial value */
} gs_params;

/* FP64 statistics of the current state (compensated sums on the device). */
typedef struct gs_stats {
  double mass;            /* sum of c (precipitate) or of all eta (mart) */
  double eta_mean;        /* mean of eta over V*N (reference "eta" key) */
  double eta2[GS_MAX_V];  /* mean of eta_p^2 */
  double vf[GS_MAX_V];    /* fraction of cells with |eta_p| > 0.5 */
  double e_el;            /* elastic energy, dV/2 S_x S_p S_p R_p */
  double e_chem;          /* local (Landau / chemical) energy */
  double e_grad;          /* gradient energy */
  double e_appl;          /* applied / dislocation stress energy */
  double e_tot;
  /* reference "info" keys (means of the force fields, src/dynamics_mart.cu:443-456) */
  double gradient_mean, chemical_mean, elastic_mean, dislocation_mean;
  double c_mean;
  int64_t step;
} gs_stats;

typedef struct gs_sim gs_sim;

/* ---- library ----------------------------------------------------------- */
int gs_version(void);
/* sizeof(gs_params) / sizeof(gs_stats) as compiled, for FFI layout checks. */
size_t gs_sizeof_params(void);
size_t gs_sizeof_stats(void);
/* Copy the calling thread's last error message into buf. */
int gs_last_error(char* buf, size_t len);
/* Select the CUDA device of the calling thread (the script command
 * `device N` and `gsi script N`, src/input.cu:244-251, src/main.cu:23-28). */
int gs_set_device(int device);
/* Fill p with the defaults of model/mode (the reference's defaults for
 * GS_MODE_REFCOMPAT, src/dynamics_mart.cu:20-27,80-89 and
 * src/dynamics_precipitate.cu:21-29,55; the BASELINE configs otherwise). */
int gs_params_default(gs_params* p, int model, int mode);

/* ---- one simulation (replaces Dynamics_*::Initialize/Calculate/Get) ---- */
/* Dynamics_*::Initialize: allocate device state for the grid; builds the
 * per-direction B(n) constants (replaces GTensorB::InitB, src/gtensorb.cu:55-108). */
int gs_sim_create(const gs_params* p, gs_sim** out);
int gs_sim_destroy(gs_sim* s);
/* Upload a host field.  Names: "eta" [V][nx][ny][nz]; "concentration"
 * [nx][ny][nz]; "defect" [nx][ny][nz]; "dislocationstress" [6][nx][ny][nz]
 * (xx xy xz yy yz zz, src/dynamics_mart.cu:128-150).  dtype is the type of
 * the host buffer; count is its number of elements. */
int gs_sim_set_field(gs_sim* s, const char* name, const void* host, size_t count, int dtype);
/* Download a field: "eta", "concentration", "stress" [6][N], "defect",
 * "elastic_potential" (R of the current state: [V][N] for the martensite,
 * [F][N] for the precipitate, R of eta_p^2 then of c). */
int gs_sim_get_field(gs_sim* s, const char* name, void* host, size_t count, int dtype);
/* Per-step scalars read by Calculate: "temperature" (refcompat a1). */
int gs_sim_set_scalar(gs_sim* s, const char* name, double value);
/* Dynamics_*::Calculate, nsteps times, on stream (a cudaStream_t, NULL =
 * the library's own stream).  Replaces src/dynamics_mart.cu:348-417,
 * src/dynamics_precipitate.cu:278-289 and src/dynamics_stress.cu:179-194. */
int gs_sim_step(gs_sim* s, int nsteps, void* stream);
/* Dynamics_*::Get statistics of the current state, FP64. */
int gs_sim_stats(gs_sim* s, gs_stats* out, void* stream);
/* Device pointer of a resident field, for callers that keep data on the GPU:
 * "eta", "spectrum", and "btable" (the octant table of B(k) when the
 * martensite contraction reads one, else NULL and 0 bytes). */
int gs_sim_device_field(gs_sim* s, const char* name, void** dptr, size_t* bytes);

/* A field copy that overlaps the steps after it (the `dump` of a running
 * script; the reference dumps synchronously, GS::Run src/gs.cu:168-212 with
 * Data::Dump).  gs_sim_copy_field_async takes a device-side snapshot of the
 * field ("eta", "concentration", "stress", "defect") on `stream` (NULL: the
 * simulation's own), after the steps already issued there, and starts its
 * copy to the host on a copy stream; later steps may be issued at once.  The
 * copy goes to library-owned page-locked memory, or, when pinned_dst is not
 * NULL, straight into that caller-owned page-locked buffer of the
 * simulation's dtype (which must hold the whole field).
 * gs_sim_copy_field_wait(ticket) waits for the copy and, for a library-owned
 * one, writes `count` values of dtype to `host` (for a direct one host may be
 * NULL); it may run on another host thread than the stepping one.  Two copies
 * per simulation can be in flight; a third call waits up to two minutes for
 * a slot (GS_ETIMEOUT).  Every ticket must be waited for once.
 * gs_sim_set_field_async uploads "eta" in the simulation's dtype on `stream`
 * without waiting (page-locked `host` overlaps the copy with other work;
 * `host` must stay unchanged until the stream has passed it). */
int gs_sim_copy_field_async(gs_sim* s, const char* name, void* stream, void* pinned_dst, int* ticket);
int gs_sim_copy_field_wait(gs_sim* s, int ticket, void* host, size_t count, int dtype);
int gs_sim_set_field_async(gs_sim* s, const char* name, const void* host, size_t count, int dtype, void* stream);
/* The next step's field set ("eta", the simulation's dtype), copied from
 * `host` (page-locked for the copy to overlap) into a staging buffer on the
 * simulation's upload stream, so the copy runs while the GPU steps and
 * while an earlier download runs the other way; the next gs_sim_step waits
 * for it and swaps it in as the current field set.  gs_sim_set_field(_async)
 * of "eta" in between drops the staged set.  One staged set at a time
 * (GS_EINVAL otherwise); martensite simulations.  The caller keeps `host`
 * unchanged until that step has started on the GPU. */
int gs_sim_stage_field_async(gs_sim* s, const char* name, const void* host, size_t count, int dtype);
/* Run one step with a CUDA event between consecutive passes on the step's
 * stream; pass_ms[i] receives the device time of pass i (in launch order:
 * z forward, y forward, x contraction, y inverse, update for the
 * martensite step; y passes are absent when the middle axis is 1). */
int gs_sim_profile_step(gs_sim* s, void* stream, double* pass_ms, int max_pass, int* npass);
/* The name of pass i of the last gs_sim_profile_step (or GS_TIMING step):
 * "z_forward", "y_forward", "x_contraction", "y_inverse", "update",
 * "precip_mid", "x_kspace_update", ...; NULL past the last pass.  The string
 * is static. */
const char* gs_sim_pass_name(const gs_sim* s, int i);
/* Hand a field from one simulation to another on the device, replacing the
 * reference's file hand-off between stages (dump stress/defect, then read
 * dislocationstress/defect: scripts/in.precipitate.sh; remap on the host,
 * src/dynamics_mart.cu:128-154,305-321).  Pairs (dst <- src):
 * "dislocationstress" <- "stress" (stress model into martensite: K_p = sigma:eps_p
 * formed on the device), "defect" <- "defect", "eta" <- "eta".  Same grid. */
int gs_sim_take_field(gs_sim* dst, const char* dst_name, gs_sim* src, const char* src_name);
/* Number of kernel launches issued by the last gs_sim_step call. */
int64_t gs_sim_launch_count(const gs_sim* s);
/* Make gs_sim_step replay a captured CUDA graph of two steps (1) or launch
 * the passes directly (0, default).  Martensite only; the step constants
 * (noise counter, temperature) then live in device memory and are refreshed
 * at every gs_sim_step call, so results equal the direct launches bit for
 * bit.  Setting a field, a schedule or autotuning drops the captured graph. */
int gs_sim_use_graph(gs_sim* s, int on);

/* ---- nuclei for the precipitate chain ----------------------------------- */
/* Dynamics_cores::Calculate painting step (src/dynamics_cores.cu:55-186) on the
 * device: ncores nuclei at centers[3q..3q+2] of variant[q], radius `radius`
 * (used as a float, as the reference's Real), with the reference's periodic
 * rule (the offset and its shifts by +-n along one axis at a time).  Writes
 * eta [V][nx][ny][nz] (1 in a nucleus of that variant, else 0) and the
 * concentration [nx][ny][nz] (c_core in any nucleus, else c_matrix) to host
 * buffers.  The placement (random draws, marks) stays with the caller. */
int gs_cores_paint(int nx, int ny, int nz, int nvariants, int ncores, const int* centers, const int* variant,
                   double radius, double c_matrix, double c_core, float* eta_host, float* conc_host);

/* ---- tile schedule and autotuner ---------------------------------------- */
/* Tile sizes of the passes: z lines per block, y and x columns per block,
 * update rows per block (the martensite update, the precipitate's middle
 * sweep) (0 = the launcher's default; sizes a launch cannot take fall back
 * to it).  The reference has no counterpart (cuFFT plans internally).
 * gs_sim_autotune (martensite and precipitate simulations) times candidates
 * with CUDA events over `reps` trial steps that leave the simulation's state
 * and step counter as they were (coordinate descent, two sweeps) and keeps
 * the fastest; gs_batch_autotune
 * does so per group and drops a captured graph so the next step recaptures. */
typedef struct gs_schedule {
  int z_lines, y_cols, x_cols, update_rows;
  /* radix split of the y lines: 0 = the default two-stage plan (16 x 16 for
   * 256, 16 x 8 for 128, 8 x 8 for 64), or the alternative first-stage radix
   * (32, 32, 16); other lengths have one plan.  The plans round differently,
   * within the step's accuracy bar. */
  int y_radix;
} gs_schedule;
int gs_sim_set_schedule(gs_sim* s, const gs_schedule* sc);
int gs_sim_get_schedule(const gs_sim* s, gs_schedule* sc);
int gs_sim_autotune(gs_sim* s, int reps, void* stream, gs_schedule* chosen);

/* gs_set_x_prefetch(1): x passes launched after the call, for three-field
 * FP32 simulations with n0 = 128 or 256 and an octant B table, run as a
 * persistent kernel that has the TMA unit fetch its next column tile while
 * it transforms the current one (the same bits as the one-tile-per-block x
 * pass; captured graphs keep the kernel they captured).  Off by default: it
 * measured no faster.  gs_x_prefetch_timeouts counts waits for a fetched
 * tile that gave up after about a second (the block then ends early); it
 * stays 0 on a healthy GPU.  No counterpart in the reference. */
void gs_set_x_prefetch(int on);
unsigned int gs_x_prefetch_timeouts(void);

/* ---- a martensite step that allocates nothing -------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they step: a host whose pool allocator owns all of the GPU's
 * memory, a loop that must never enter the allocator, a plugin in a process
 * whose device memory belongs to someone else.  One martensite step (the
 * same passes as gs_sim_step) from eta_in to eta_out, both caller-owned
 * device buffers of [V][nx][ny][nz] elements of p->dtype on the current
 * device, not overlapping, each starting on a 16-byte boundary (the kernels
 * move fields in 16-byte vectors; other addresses get GS_EINVAL); `step` is the global step index that the noise
 * counter uses (gs_sim_step's k-th step from a fresh simulation has step
 * k).  Defect and dislocation-stress inputs are not taken.  The spectra and
 * twiddle tables live in one static device array of
 * gs_mart_step_noalloc_max_bytes() bytes (16 MiB) that every GPU loading the
 * library keeps until exit; a grid needing more (V*N*element size plus
 * about 4 KB) is rejected with GS_EINVAL.  No device memory is allocated or
 * freed.  The first call on a device looks up the array's device address,
 * so make it before any stream capture.  The call returns once the step has
 * finished on `stream` (NULL = the legacy default stream).  All calls share
 * the array and nothing in it has to start at zero; calls that overlap on
 * the GPU (from several host threads) race on it. */
int gs_mart_step_noalloc(const gs_params* p, const void* eta_in, void* eta_out, int64_t step, void* stream);
size_t gs_mart_step_noalloc_max_bytes(void);

/* ---- adjoint of the martensite run ------------------------------------ */
/* The reference has no adjoint; this is the transpose of its explicit step
 * (Dynamics_mart::Calculate, src/dynamics_mart.cu:348-417) in baseline mode,
 * noise included (it is additive) and defect/dislocation inputs excluded.
 * A handle holds a fixed grid and step count: gs_adjoint_forward runs eta_0
 * -> eta_T keeping every checkpoint_every-th state, gs_adjoint_backward
 * recomputes each segment from its checkpoint and sweeps the adjoint back to
 * eta_0.  Loss mode (gs_adjoint_set_loss, seed == NULL):
 *   J = sum (eta_T - target)^2 + lam_el (E_el(T) - e_target)^2;
 * seed mode: J = <seed, eta_T> + seed_e E_el(T) (a vector-Jacobian product).
 * grads[6] = dJ/d(kappa, A2, A4, A6, Ac, s), s the eigenstrain scale
 * (eps_p -> s eps_p at s = 1); grad_eta0 = dJ/deta_0 ([V][N], may be NULL);
 * loss[3] = (J, field term, E_el(T)) (NULL allowed). */
typedef struct gs_adjoint gs_adjoint;
int gs_adjoint_create(const gs_params* p, int nsteps, int checkpoint_every, gs_adjoint** out);
int gs_adjoint_destroy(gs_adjoint* a);
/* New coefficients for the next forward run (grid, V and dtype fixed). */
int gs_adjoint_set_params(gs_adjoint* a, const gs_params* p);
int gs_adjoint_set_loss(gs_adjoint* a, const void* target, int dtype, double lam_el, double e_target);
int gs_adjoint_forward(gs_adjoint* a, const void* eta0, int dtype, void* eta_final, double* e_el_final,
                       void* stream);
int gs_adjoint_backward(gs_adjoint* a, const void* seed, int seed_dtype, double seed_e, double* loss,
                        double* grads, void* grad_eta0, int grad_dtype, void* stream);
/* Replay the forward steps and the reverse sweep as CUDA graphs captured
 * after a first direct run (1, default) or always launch directly (0).
 * Results are the same either way; new parameters drop the graphs. */
int gs_adjoint_use_graph(gs_adjoint* a, int on);
/* Device bytes held by the handle (checkpoints, segment, adjoint fields). */
size_t gs_adjoint_device_bytes(const gs_adjoint* a);
/* Kernel launches issued by the last forward or backward call. */
int64_t gs_adjoint_launch_count(const gs_adjoint* a);

/* ---- adjoint of the precipitate run -------------------------------------- */
/* The transpose of the semi-implicit precipitate step (Dynamics_precipitate::
 * Calculate, src/dynamics_precipitate.cu:118-289) in baseline mode: the
 * Cahn-Hilliard and Allen-Cahn factors 1/(1 + dt M kappa_c K^2), 1/(1 + dt L
 * kappa_eta K) and the operator K are real even symbols, hence their own
 * transposes; the local terms' Jacobians are applied pointwise and the
 * elastic coupling through the same B convolution.  The noise is additive
 * and drops out; the mass projection only corrects rounding and is not
 * differentiated.  The forward keeps the state every checkpoint_every = K
 * steps and the states of the last segment; the backward recomputes each
 * earlier segment from its checkpoint (with the forward's own step
 * counters, so the states are the same bits) before sweeping it back, so
 * the device holds (ceil(nsteps/K) + K + 1) (V+1) N state values (K = 1:
 * every state, no recomputation).  After a first direct run the reverse
 * sweep (recomputes included) is replayed as one captured CUDA graph
 * (gs_precip_adjoint_use_graph(a, 0) launches directly; a new initial
 * concentration mass or stream recaptures).  gs_precip_adjoint_backward
 * returns, for J = <seed_c, c_T>
 * + <seed_eta, eta_T>, grads[9] = dJ/d(kappa_c, kappa_eta, coef[1..7]) and
 * dJ/dc0, dJ/deta0 (host buffers of dtype, NULL to skip).  NULL seeds reuse
 * the ones last given (gs_precip_adjoint_set_seed, kept on the device); NULL
 * c0 and eta0 rerun the forward from the previous initial state. */
typedef struct gs_padjoint gs_padjoint;
int gs_precip_adjoint_create(const gs_params* p, int nsteps, int checkpoint_every, gs_padjoint** out);
int gs_precip_adjoint_destroy(gs_padjoint* a);
int gs_precip_adjoint_use_graph(gs_padjoint* a, int on);
int gs_precip_adjoint_forward(gs_padjoint* a, const void* c0, const void* eta0, int dtype, void* c_final,
                              void* eta_final, void* stream);
int gs_precip_adjoint_set_seed(gs_padjoint* a, const void* seed_c, const void* seed_eta, int dtype);
int gs_precip_adjoint_backward(gs_padjoint* a, const void* seed_c, const void* seed_eta, int dtype, double* grads,
                               void* grad_c0, void* grad_eta0, void* stream);
/* Device bytes of the handle: checkpoints, segment, adjoint work arrays and
 * the simulation's own buffers. */
size_t gs_precip_adjoint_device_bytes(const gs_padjoint* a);

/* ---- batched ensembles ------------------------------------------------- */
/* Many independent martensite simulations advanced together.  Simulations
 * of one grid, variant count, modulus and eigenstrain direction form a group
 * and share every launch (one per pass per group); each keeps its own
 * Landau coefficients, kappa, mobility, eigenstrain magnitude, applied
 * stress, noise amplitude and seed.  With gs_batch_use_graph(b, 1) the step
 * is captured once as a CUDA graph of two steps and replayed. */
typedef struct gs_batch gs_batch;
int gs_batch_create(const gs_params* params, int nsims, gs_batch** out);
int gs_batch_destroy(gs_batch* b);
int gs_batch_set_field(gs_batch* b, int sim, const char* name, const void* host, size_t count, int dtype);
int gs_batch_get_field(gs_batch* b, int sim, const char* name, void* host, size_t count, int dtype);
int gs_batch_step(gs_batch* b, int nsteps, void* stream);
int gs_batch_stats(gs_batch* b, int sim, gs_stats* out, void* stream);
int gs_batch_use_graph(gs_batch* b, int on);
int gs_batch_groups(const gs_batch* b);
/* 1 (default): every shape group steps on a branch stream of its own, forked
 * from and joined to the caller's stream (parallel branches in the captured
 * graph), so the groups' passes overlap; 0: one group after the other on the
 * caller's stream.  The results are the same bits either way. */
int gs_batch_set_concurrent(gs_batch* b, int on);
int gs_batch_autotune(gs_batch* b, int reps, void* stream);
int gs_batch_get_schedule(const gs_batch* b, int group, gs_schedule* sc);
int64_t gs_batch_launch_count(const gs_batch* b);

/* ---- a simulation split into slabs across devices -------------------------- */
/* The reference keeps a whole grid on one device (one cuFFT plan over it,
 * src/dynamics_mart.cu:113-117); a grid too large for one GPU is split here
 * into R slabs of nx/R x-planes, one per rank (martensite, 3D grids, nx and
 * nz/2 multiples of R).  A step is three local phases; between them the
 * caller exchanges buffers it owns (device memory of `a2a_bytes` and
 * `halo_bytes`, 16-byte aligned):
 *   gs_slab_begin(send, halo_send): spectra along z and y of this slab,
 *     packed by destination rank into send = [R][V][nx/R][ny][h/R] complex
 *     (h = nz/2), and the slab's first and last x-plane into halo_send =
 *     [2][V][ny][nz];
 *   all-to-all of send into recv (equal pieces of a2a_bytes / R), and the
 *   halo: this rank's halo_recv[0] = halo_send[1] of rank - 1, halo_recv[1]
 *   = halo_send[0] of rank + 1 (periodic);
 *   gs_slab_xpass(recv, send): the x transforms and the B contraction of this
 *     rank's kz slots h/R rank .. h/R (rank + 1) - 1, packed back by
 *     destination x range;
 *   all-to-all again;
 *   gs_slab_end(recv, halo_recv): y inverse, the update (its x neighbours
 *     across the slab faces from halo_recv; the noise counter on global cell
 *     indices) and the next step's z forward.
 * The arithmetic of every line, table point and cell is that of gs_sim_step,
 * so the slabs reproduce a one-device run bit for bit.  Defect and
 * dislocation-stress fields and statistics are not taken on this path. */
typedef struct gs_slab gs_slab;
typedef struct gs_slab_geometry {
  int rank, nranks;
  int x0, nx_local;    /* the x-planes this rank owns */
  int kz0, nkz_local;  /* the kz slots of its x pass */
  size_t a2a_bytes;    /* bytes of the send and receive buffers (R equal pieces) */
  size_t halo_bytes;   /* bytes of halo_send and halo_recv */
  int64_t step;
} gs_slab_geometry;
int gs_slab_create(const gs_params* p, int rank, int nranks, gs_slab** out);
int gs_slab_destroy(gs_slab* sl);
int gs_slab_info(const gs_slab* sl, gs_slab_geometry* out);
/* "eta" of this slab: [V][nx/R][ny][nz] host values of dtype */
int gs_slab_set_field(gs_slab* sl, const char* name, const void* host, size_t count, int dtype);
int gs_slab_get_field(gs_slab* sl, const char* name, void* host, size_t count, int dtype);
int gs_slab_set_step(gs_slab* sl, int64_t step);
int gs_slab_begin(gs_slab* sl, void* send, void* halo_send, void* stream);
int gs_slab_xpass(gs_slab* sl, const void* recv, void* send, void* stream);
int gs_slab_end(gs_slab* sl, const void* recv, const void* halo_recv, void* stream);

/* ---- the noise stream ---------------------------------------------------- */
/* Replaces the reference's cuRAND normal field (Random::NewNormal_device,
 * src/random.cu:79-82), which the step kernels no longer store: they draw
 * Philox4x32-10 in registers on the counter (quad, step, sim, slot) with key
 * (seed & 0xffffffff, seed >> 32), quad = cell >> 2, slot = the variant (V
 * for the concentration), and turn words (0,1) and (2,3) into the normals of
 * cells 4 quad .. 4 quad + 3 by Box-Muller on 24-bit uniforms.  This call
 * evaluates those same device functions for quads quad0 .. quad0 + nquads - 1
 * (the quad word wraps modulo 2^32) and writes the raw words [nquads][4] to
 * `words` and the normals [nquads][4] of `dtype` to `normals` (host buffers;
 * either may be NULL), so that the stream can be checked against another
 * Philox4x32-10 implementation bit for bit. */
int gs_noise_block(uint64_t seed, uint32_t step, uint32_t sim, uint32_t slot, uint32_t quad0, int nquads,
                   int dtype, uint32_t* words, void* normals);

/* ---- comparator: the same step with cuFFT C2C and unfused sweeps ------ */
/* The plain GPU step in the reference's structure (cufftPlanMany C2C batch
 * V, B streamed from a [V][V][N] array, one sweep per term); used only as a
 * timed comparison, never on the product path. */
int gs_plain_create(const gs_params* p, gs_sim** out);
int gs_plain_step(gs_sim* s, int nsteps, void* stream);

/* The cuFFT comparator of the hand-written FFT passes: the same martensite
 * step with cufftExecR2C / cufftExecC2R batched over the variants (planned
 * once), one contraction sweep over the half spectrum (the octant B table,
 * or B formed per k), and the product's fused update kernel without its z
 * transforms as the single pointwise sweep (it also writes eta'^2 for the
 * next forward transform).  The reference's own convolution is the C2C one
 * of gs_plain_* (src/dynamics_mart.cu:113-117,281-303).  Timing only; the
 * handle otherwise behaves as gs_sim_create's (fields, stats, destroy). */
int gs_cufft_create(const gs_params* p, gs_sim** out);
int gs_cufft_step(gs_sim* s, int nsteps, void* stream);

/* ---- bounds checks (debugging; no counterpart in the reference, whose
 * kernels check nothing, src/dynamics_mart.cu:113-117) ------------------- */
/* The launch-range check, in every build: on != 0 makes each pass launcher
 * check, before it launches, that every buffer range its kernel reaches lies
 * inside one device allocation and is aligned for its vector accesses; a
 * range that does not fit refuses the launch (the step returns GS_ECUDA with
 * a message naming the kernel and the buffer).  Off by default; on when the
 * environment has GS_BOUNDS_CHECK=1 or in the bounds-check build. */
void gs_set_bounds_check(int on);
int gs_bounds_check_enabled(void);
/* 1 when this library is the bounds-check build (libgsb200_bc.so): its
 * kernels check every index against the launch's extents, record the first
 * violation and keep the access inside the buffer (no trap); gs_sim_step,
 * gs_batch_step, gs_mart_step_noalloc, gs_cufft_step, the adjoint and slab
 * entries then wait for their kernels and return GS_EBOUNDS after a
 * violation (not while their stream is being captured). */
int gs_bounds_check_build(void);
/* The bounds-check build's record on the current device, summed over the
 * library's modules: out[0] violations, out[1] site of the first one
 * (gs_bounds_site_name), out[2] its index, out[3] the extent it broke,
 * out[4] its block (x | y << 32), out[5] its thread.  clear != 0 zeroes the
 * records.  Synchronises the device.  GS_ENOTSUP in a normal build. */
int gs_bounds_check_read(long long out[6], int clear);
const char* gs_bounds_site_name(int site);
/* Self-test of the index asserts: a kernel stores i into buf[i] for i < n
 * through a checked index against cap elements.  The bounds-check build
 * records n - cap violations (n > cap) and writes nothing beyond buf[cap-1];
 * a normal build refuses it (GS_ENOTSUP), since its kernel would. */
int gs_bounds_selftest(int* buf, int cap, int n, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GS_CAPI_H */
