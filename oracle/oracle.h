/*
 * oracle.h -- CPU checker for the device solver. TEST INFRASTRUCTURE ONLY.
 *
 * A line-by-line C++ restatement of NuPPN's FP64 per-zone path (file:line citations in oracle.cpp)
 * that calls the reference's own SuperLU 5.0 (built from the reference tree into oracle/_ref by
 * oracle/Makefile and loaded at run time) for every sparse LU, exactly as the reference does:
 * slu_solve for the implicit-Euler Newton solve (linalg.F90:115) and c_fortran_dgssv_ for
 * Bader-Deuflhard (bader_deuflhard.F90:435-464).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm may load it, and
 * only as the checker: the product path never links or calls it.
 *
 * Parity status: the SuperLU part is pinned (it is the reference's code, and its 20x20 smoke system
 * of slu_f90/matrixtest.f90 is checked). The Fortran parts cannot be compiled here (no Fortran
 * compiler), so their restatement is pinned by review against the cited lines and by invariants;
 * see the test suite.
 */
#ifndef NUPPN_ORACLE_H
#define NUPPN_ORACLE_H
#include <stdint.h>
#include "../include/nuppn.h"

#ifdef __cplusplus
extern "C" {
#endif

/* dlopen the reference SuperLU (oracle/_ref/libslu_ref.so). 0 on success. */
int oracle_load_superlu(const char *path);

void *oracle_net_create(const nuppn_net_desc *desc, const nuppn_knobs *knobs);
void oracle_net_destroy(void *net);
int oracle_nnz(void *net);
int oracle_jac_pattern(void *net, int32_t *row, int32_t *col, int32_t *dns2csr_map);

int oracle_eval_rates(void *net, double t9, double rho, double ye, const double *X, double *v);
int oracle_dxdt(void *net, const double *v, const double *X, double *dxdt);
int oracle_jacobian(void *net, const double *v, const double *X, double dt, double *jac,
                    uint8_t *entry_set, uint8_t *mask);
/* reduced solve of newton_iteration through slu_solve; returns slu ierr */
int oracle_solve_reduced(void *net, const double *jac, const uint8_t *entry_set,
                         const uint8_t *mask, double dt, const double *b, double *x);

/* integrate_network for nz zones on nthreads host threads (zone-major X, stride ldx). bd_state is
 * the per-zone Bader-Deuflhard (kopt, first-call) state, may be NULL (fresh zones). */
int oracle_integrate(void *net, int32_t nz, double *X, int32_t ldx, const double *t9_0,
                     const double *t9_1, const double *rho_0, const double *rho_1, double *ye,
                     const double *dtwant, int32_t *ierr, nuppn_zone_stats *stats,
                     int32_t *bd_state, int32_t nthreads);

/* Ye from composition, calculate_ye (utils.F90:537-553) */
double oracle_calculate_ye(void *net, const double *X);
// tppnp's trajectory loop (tppnp.F90:131-168) per zone over npts points ([nz][npts] arrays).
int oracle_integrate_trajectories(void *net, int32_t nz, int32_t npts, double *X, int32_t ldx, const double *time,
                                  const double *t9, const double *rho, double *ye, int32_t *ierr, int32_t *fail,
                                  nuppn_zone_stats *stats, int32_t nthreads);
// compute_nse (nse_swj.F90:272-384) per zone from a fresh state: X[z*ldx + i], chemical potentials,
// Newton iterations and the outcome code. Returns -1 if the network has no protons or no Ni56.
int oracle_nse(void *net, int32_t nz, const double *t9, const double *rho, const double *ye, double *X,
               int32_t ldx, double *mu_p, double *mu_n, int32_t *iters, int32_t *ierr);
/* sortedsum (utils.F90:481-501) with the NR heapsort indexx (sort.F90:73-127) */
double oracle_sortedsum(const double *a, int32_t n);
/* the reference's VITAL formula for slot 1-9, 14-17 or 73 at T9 (clipped to 10), rho, X(p); 0 otherwise */
double oracle_vital_reference(int32_t slot, double t9, double rho, double xprot);

#ifdef __cplusplus
}
#endif
#endif
