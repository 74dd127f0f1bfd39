/*
 * gs_oracle.h -- FP64 CPU restatement of the phase-field step.
 *
 * TEST INFRASTRUCTURE.  Only the tests, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this library, and only as
 * the checker or the timed CPU baseline.  The product path (libgsb200.so)
 * never links or calls it.
 *
 * It follows the reference's algorithm directly: full complex 3D DFTs
 * (the reference's cufftPlanMany C2C, src/dynamics_mart.cu:113-117), the
 * real part of the unnormalised inverse, B(n) built per k point
 * (src/gtensorb.cu:110-182), the update formulas of src/dynamics_mart.cu:
 * 181-417, src/dynamics_precipitate.cu:118-289 and src/dynamics_stress.cu:
 * 122-194 (GS_MODE_REFCOMPAT) and the project's baseline discretisation
 * (GS_MODE_BASELINE).  Everything is double precision.
 */
#ifndef GS_ORACLE_H
#define GS_ORACLE_H
#include <stdint.h>
#include "../include/gs_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), one block. */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Four N(0,1) samples of counter (cell, step, sim, block), key = seed. */
void or_normals4(uint64_t seed, uint32_t cell, uint32_t step, uint32_t sim, uint32_t block, double z[4]);

/* In-place unnormalised complex DFT of a [n0][n1][n2] array of interleaved
 * (re, im) doubles; sign -1 forward, +1 inverse. */
void or_fft3(double* data, int n0, int n1, int n2, int sign);

/* B matrix at wave vector k (index triple m folded by the model's rule).
 * which = 0: variants x variants (mart); 1: 6 unit strains x variants
 * (stress); 2: precipitate fields (eta_p^2 then c) x the same. */
int or_bmat_at(const gs_params* p, int which, int mx, int my, int mz, double* B, int* na, int* nb);

/* Martensite: advance eta ([V][N], in/out) nsteps from global step step0.
 * defect (N) and dstress (6 x N, xx xy xz yy yz zz) may be NULL. */
int or_mart_run(const gs_params* p, double* eta, const double* defect, const double* dstress,
                int nsteps, int64_t step0);
int or_mart_stats(const gs_params* p, const double* eta, const double* defect,
                  const double* dstress, gs_stats* st);
/* Elastic potential R_p = Re IFFT((1/N) sum_q B_pq FFT(eta_q^2)) of a state. */
int or_mart_potential(const gs_params* p, const double* eta, double* R);

/* Adjoint of the baseline martensite run from eta0 over nsteps.  Loss
 * J = sum (eta_T - target)^2 + lam_el (E_el(T) - e_target)^2, or, when seed
 * is given, J = <seed, eta_T> + seed_e E_el(T).  grads[6]: dJ/d kappa, A2,
 * A4, A6, Ac, eigenstrain scale s (eps -> s eps at s = 1); grad_eta0 = dJ/d
 * eta0 ([V][N], may be NULL); loss_out[3] = (J, field term, E_el(T)). */
int or_mart_adjoint(const gs_params* p, const double* eta0, int nsteps, const double* target, double lam_el,
                    double e_target, const double* seed, double seed_e, double* grads, double* grad_eta0,
                    double* loss_out);

/* Adjoint of the precipitate run (baseline mode): J = <seed_c, c_T> +
 * <seed_eta, eta_T>; grad_c0, grad_eta0 (may be NULL) and grads[9] =
 * dJ/d(kappa_c, kappa_eta, coef[1..7]). */
int or_precip_adjoint(const gs_params* p, const double* c0, const double* eta0, int nsteps, const double* seed_c,
                      const double* seed_eta, double* grad_c0, double* grad_eta0, double* grads);

/* Precipitate: advance c (N) and eta ([V][N]) nsteps. */
int or_precip_run(const gs_params* p, double* c, double* eta, int nsteps, int64_t step0);
int or_precip_stats(const gs_params* p, const double* c, const double* eta, gs_stats* st);

/* Stress: stress [6][N] and defect [N] of an eta configuration. */
int or_stress(const gs_params* p, const double* eta, double* stress, double* defect);

/* Nuclei of the precipitate chain (src/dynamics_cores.cu:55-186): paint
 * eta [V][N] and the concentration [N] (float, as the reference's Real);
 * or_cores_marked says whether (i, j, k) lies in one of the first ncores. */
int or_cores_paint(int nx, int ny, int nz, int V, int ncores, const int* centers, const int* variant, double radius,
                   double c_matrix, double c_core, float* eta, float* conc);
int or_cores_marked(int nx, int ny, int nz, int ncores, const int* centers, double radius, int i, int j, int k);

/* Set the number of OpenMP threads used by the oracle (0 = default). */
void or_set_threads(int n);
int or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
