/*
 * sphdem_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (plain C, FP64, one loop per reference kernel) of the
 * SOPHIA_gpu ISPH-DEM step SOPHIA_single_ISPH (ISPH_Calc_seperate.cuh:13-503)
 * and its host loop (ISPH_Calc_seperate.cuh:905-975).  It is the checker
 * for the CUDA engine: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it.  The product path never calls it.
 *
 * Parity pin: tests/golden/ holds outputs of the unmodified reference
 * kernels (built by oracle/Makefile into oracle/_ref/ and run on a B200)
 * for small seeded beds; tests/test_oracle_golden.py checks this file
 * against them.
 */
#ifndef SPHDEM_ORACLE_H
#define SPHDEM_ORACLE_H

#include "../include/sphdem.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleState OracleState;

OracleState* oracle_create(const SphdemParams* p, int n_sph, int n_dem);
void oracle_destroy(OracleState* s);

/* which: 0 SPH, 1 DEM.  Real fields take n doubles, int fields n int32,
 * in input order (before commit) or current sorted order (after). */
int oracle_set_field(OracleState* s, int which, int field, const void* src, int n);
int oracle_get_field(OracleState* s, int which, int field, void* dst, int n);

/* Bounding box, grid, buffer tags: ISPH.cuh:104-113, NNPS:60-200.
 * bbox_* are computed over the concatenation SPH-then-DEM of the input
 * rows unless the caller fixes them first with oracle_set_domain. */
int oracle_commit(OracleState* s);
/* Per-bed open-boundary rows {y, inlet_uz, inlet_temp, L1, L2, L3, L4} of
 * 2-D beds in planes y = const (the engine's sphdem_set_beds), before
 * commit: a particle takes the row of the nearest plane. */
int oracle_set_beds(OracleState* s, int nbeds, const double* rows7);
int oracle_set_domain(OracleState* s, const double* mins, const double* maxs,
                      double h0);

/* Advance nsteps full reference steps. */
int oracle_step(OracleState* s, int nsteps);

/* Neighbour list (kappa*h_i, self included) of the SPH set built at the
 * start of the last step, in the reference visit order. */
int oracle_get_neighbors(OracleState* s, int* counts, int* dst, int cap);

/* Grid and time bookkeeping. */
int oracle_get_grid(OracleState* s, int* nijk, double* bbox6, double* dcell);
int oracle_get_time(OracleState* s, double* time, int* count);

/* Contact history of the DEM set (16 slots): ids as double, del_s x3. */
int oracle_get_history(OracleState* s, double* ct_idx, double* del_s, int n);
int oracle_set_history(OracleState* s, const double* ct_idx, const double* del_s, int n);

/* Smoothing kernel of functions_KNL.cuh:2-144 for analytic checks:
 * returns W (deriv=0) or dW/dr (deriv=1) at distance r, 3-D. */
double oracle_kernel(int kernel_type, int dim, double h, double r, int deriv);

/* Iterations, relative residual and status (0 converged, 1 iteration
 * cap, 2 breakdown) of the last PPE solve in the Krylov modes. */
int oracle_get_ppe(OracleState* s, int* iters, double* rel_res, int* status);

/* Number of OpenMP threads used by the step loops (1 = serial). */
int oracle_set_threads(OracleState* s, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
