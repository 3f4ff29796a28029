/*
 * polymer_scf.h -- C ABI of the SCF iteration kernels in libpolymer_fock.so:
 * the device side of one batched closed-shell SCF iteration around the Fock
 * build (Fock assembly and energy, commutator DIIS, SP2 density projection,
 * density bookkeeping).  The reference performs these steps on the host
 * (FOCK_BUILD src/pfock.f90:185-337, DIIS src/pdensitymatrix.f90:253-339,
 * ENERGY_CALC, the density update of src/pselfconsistentfield.f90); here they
 * run on the device, so that an iteration can be one CUDA graph replay.
 *
 * Every function works on a batch of `nb` real symmetric n x n matrices stored
 * one after another (n*n doubles each; symmetric, so row- and column-major
 * agree).  All pointers are device pointers; `stream` is a cudaStream_t.
 * Per-molecule flags are bytes (0/1), per-molecule scalars doubles.  `work`
 * is caller-provided scratch of at least pfe_scf_workspace(nb, n, ndiis)
 * doubles.  No function allocates, synchronises or reads back: each is one
 * to three kernel launches on `stream` (capturable into a CUDA graph).
 * Return 0 or a negative PFE_E* code; the message is available from
 * pfe_last_error.  The dense products (orthogonal-basis transforms, F P,
 * X X) are the caller's GEMMs.
 */
#ifndef POLYMER_SCF_H
#define POLYMER_SCF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Doubles of scratch the functions below need for nb matrices of order n with
 * ndiis history slots (ndiis <= 16). */
int64_t pfe_scf_workspace(int32_t nb, int32_t n, int32_t ndiis);

/* Density of the next build.  P = P_new where take[b], P_nuc where restart[b]
 * (P_nuc may be NULL: no restarts; a restart also clears valid[b][*]), else
 * unchanged; then dP = (P - incr[b] P_ref) live[b]. */
int32_t pfe_scf_next_density(int32_t nb, int32_t n, int32_t ndiis, double *p, const double *p_new,
                             const double *p_nuc, const uint8_t *take, const uint8_t *restart, const double *incr,
                             const double *live, const double *p_ref, double *dp, uint8_t *valid, void *stream);

/* Fock assembly after a (possibly incremental) build of J = d_c, K = d_x:
 * C = d_c + incr[b] C_ref, X = d_x + incr[b] X_ref (C_ref, X_ref and P_ref
 * take C, X and P), F = (G + G^T)/2 with G = H + C - hfx[b]/2 X, and
 * energy[b] = sum_ij P (H + C/2 - hfx[b]/4 X) + e_nuc[b] (fixed summation
 * order). */
int32_t pfe_scf_fock_assemble(int32_t nb, int32_t n, const double *h, const double *d_c, const double *d_x,
                              double *c_ref, double *x_ref, const double *p, double *p_ref, const double *incr,
                              const double *hfx, const double *e_nuc, double *f, double *energy, double *work,
                              void *stream);

/* The DIIS error of the orthogonal-basis F_o, P_o from the caller's product
 * A = F_o P_o: E = A - A^T (= F_o P_o - P_o F_o) is stored into history slot
 * *slot of hist_e [nb][ndiis][n][n], F_o into the same slot of hist_f,
 * valid[b][*slot] = 1, err_max[b] = max |E|. */
int32_t pfe_scf_commutator(int32_t nb, int32_t n, int32_t ndiis, const double *a, const double *f_o,
                           const int64_t *slot, double *hist_e, double *hist_f, uint8_t *valid, double *err_max,
                           double *work, void *stream);

/* Pulay extrapolation.  Refreshes row and column *slot of the Gram matrices
 * gram [nb][ndiis][ndiis] of the history (kept between calls; zero before the
 * first), solves G c = 1 over the valid slots with G scaled by its largest
 * valid diagonal and 1e-12 added to that diagonal (Cholesky), normalises
 * sum c = 1, and falls back to the newest slot alone when the solve fails;
 * coef [nb][ndiis] receives c and f_x = sum_d c_d hist_f[d]. */
int32_t pfe_scf_diis(int32_t nb, int32_t n, int32_t ndiis, const double *hist_e, const double *hist_f,
                     const uint8_t *valid, const int64_t *slot, double *gram, double *coef, double *f_x, double *work,
                     void *stream);

/* SP2 start: X = (hi I - F)/(hi - lo) with [lo, hi] the Gershgorin bounds of
 * F over the rows not marked in pad [nb][n] (hi raised to lo + 1e-8 at
 * least); rows and columns marked in pad are zero. */
int32_t pfe_scf_sp2_init(int32_t nb, int32_t n, const double *f, const uint8_t *pad, double *x, void *stream);

/* One SP2 step after the caller's product X2 = X X: with t1 = tr X and
 * t2 = tr X2, defect[b] = |t1 - t2|; X takes X2 where
 * |t2 - nocc| < |2 t1 - t2 - nocc|, else 2X - X2. */
int32_t pfe_scf_sp2_step(int32_t nb, int32_t n, int32_t nocc, double *x, const double *x2, double *defect,
                         double *work, void *stream);

/* The projected density and the statistics of the iteration: P_new = scale Q
 * (Q the caller's back-transformed projector), and stats [nb][4] rows
 * (energy[b], err_max[b], sqrt(sum (P_new - P)^2 / n^2), defect[b]). */
int32_t pfe_scf_finish(int32_t nb, int32_t n, double scale, const double *q, const double *p, double *p_new,
                       const double *energy, const double *err_max, const double *defect, double *stats,
                       double *work, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* POLYMER_SCF_H */
