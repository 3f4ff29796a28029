/*
 * polymer_guess.h -- C ABI of the learned initial guess kernels in
 * libpolymer_fock.so.  No counterpart in the reference (whose guess is the
 * nuclear-charge diagonal, src/pdensitymatrix.f90:83-127): a small MLP that
 * predicts density blocks for the first SCF iteration, trained and evaluated
 * on the GPU.  All pointers are device pointers; `stream` is a cudaStream_t.
 * Matrices are row-major with their row length as stride.  Return 0 or a
 * negative PFE_E* code; the message is available from pfe_last_error.
 */
#ifndef POLYMER_GUESS_H
#define POLYMER_GUESS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[m,n] (+)= op(A)[m,k] op(B)[k,n] on the tensor cores: A, B BF16 (A is m x k,
 * or k x m when trans_a; B is k x n, or n x k when trans_b), C FP32, FP32
 * accumulation; accumulate != 0 adds to C.  m, n, k: multiples of 64. */
int32_t pfe_mlp_gemm(const void *a, const void *b, float *c, int32_t m, int32_t n, int32_t k, int32_t trans_a,
                     int32_t trans_b, int32_t accumulate, void *stream);

/* z[m,n] += bias[n]; h = act(z) (act 1: SiLU, 0: identity); h_bf16 (may be
 * NULL) receives h in BF16. */
int32_t pfe_mlp_bias_act(float *z, const float *bias, float *h, void *h_bf16, int32_t m, int32_t n, int32_t act,
                         void *stream);

/* dz = dh * act'(z), in FP32 and BF16. */
int32_t pfe_mlp_act_grad(const float *dh, const float *z, float *dz, void *dz_bf16, int64_t n, int32_t act,
                         void *stream);

/* db[n] = column sums of dz[m,n]. */
int32_t pfe_mlp_colsum(const float *dz, float *db, int32_t m, int32_t n, void *stream);

/* Weighted mean-square error: *loss += sum w (y - t)^2 * inv_wsum,
 * dy = 2 w (y - t) inv_wsum. */
int32_t pfe_mlp_mse(const float *y, const float *t, const float *w, float inv_wsum, float *dy, float *loss, int64_t n,
                    void *stream);

/* One Adam step (bias-corrected for `step` >= 1, L2 decay) on FP32 weights; the
 * BF16 copy w_bf16 (may be NULL) is refreshed. */
int32_t pfe_mlp_adam(float *w, void *w_bf16, const float *g, float *m, float *v, int64_t n, float lr, float beta1,
                     float beta2, float eps, int32_t step, float decay, void *stream);

/* y = BF16(x). */
int32_t pfe_mlp_to_bf16(const float *x, void *y, int64_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* POLYMER_GUESS_H */
