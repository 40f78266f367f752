/* tensorsvm_testing.h - test hooks of libtensorsvm_b200 (not part of the training API).
 *
 * Each hook runs one internal device routine on caller-owned DEVICE buffers and synchronises,
 * so the parity tests can check a kernel in isolation against the CPU oracle.  The routines
 * they expose stand in for the reference's calls noted below; they have no counterpart of
 * their own in the reference's (non-existent) library API.
 */
#ifndef TENSORSVM_TESTING_H
#define TENSORSVM_TESTING_H

#include "tensorsvm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* glibc rand() stream from the default seed (count values): the generator behind
 * gaussrand() (tensorsvm-train.cu:2629-2630). */
tsvm_status tsvm_test_rand_stream(tsvm_context *ctx, int64_t count, uint32_t *out);
/* The reference's gaussrand() stream (tensorsvm-train.cu:2621-2643), count floats. */
tsvm_status tsvm_test_sketch(tsvm_context *ctx, int64_t count, float *out);
/* count values of the Philox4x32-10 Box-Muller sketch with this seed (TSVM_SKETCH_PHILOX). */
tsvm_status tsvm_test_sketch_philox(tsvm_context *ctx, uint64_t seed, int64_t count, float *out);
/* W (n x kp) = (Y K Y) A (n x kp) with the given precision (kermatmul, T:2476-2567); for the
 * tensor-core precisions split = 0 (one product), 1 (the kernel block as hi + lo) or 2 (A as
 * hi + lo). */
tsvm_status tsvm_test_kermatmul(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                int32_t d, double gamma, const float *A, int32_t kp, float *W,
                                int32_t precision, int32_t split);
/* The half product of a symmetric projection on the tensor cores: R (n x kp) = Y (K o H) Y A with
 * H_ij = 1 (j > i), 1/2 (j == i), 0 (j < i), and sym (kp + 1 doubles) = [s, A^T y] such that
 * A^T (Y K Y) A = A^T R + R^T A + s (A^T y)(A^T y)^T (s: the kernel-mean shift, or 0).  split 0
 * or 2 (A as hi + lo) as tsvm_test_kermatmul. */
tsvm_status tsvm_test_kermatmul_half(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                     int32_t d, double gamma, const float *A, int32_t kp,
                                     float *R, double *sym, int32_t precision, int32_t split);
/* The two products above when only the first kw columns of A may be nonzero (the rest zero):
 * above 256 columns, kw rounded up to 16 at most 416 runs the product as one launch over kw
 * columns (the other columns of the output written as zeros), otherwise in 256-column slabs. */
tsvm_status tsvm_test_kermatmul_cols(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                     int32_t d, double gamma, const float *A, int32_t kp,
                                     int32_t kw, float *W, int32_t precision, int32_t split);
tsvm_status tsvm_test_kermatmul_half_cols(tsvm_context *ctx, const float *X, const float *y,
                                          int64_t n, int32_t d, double gamma, const float *A,
                                          int32_t kp, int32_t kw, float *R, double *sym,
                                          int32_t precision, int32_t split);
/* out (na x nu, FP64) = sum_j w_ij exp(-gamma ||a_i - b_j||^2) U[j][:], w = 1 or (deriv)
 * -||a_i - b_j||^2, by the hypergradient's SIMT products or (tensor_cores) the tcgen05 form. */
tsvm_status tsvm_test_kprod(tsvm_context *ctx, const float *A, int64_t na, const float *B,
                            int64_t nb, int32_t d, double gamma, const double *U, int32_t nu,
                            double *out, int32_t deriv, int32_t tensor_cores);
/* In-place lower Cholesky of A (n x n row-major); *info_host = 0 or failing column (T:1709). */
tsvm_status tsvm_test_chol(tsvm_context *ctx, double *A, int32_t n, int32_t *info_host);
/* Solve L L^T X = B, B holds nrhs rows of length ldb (T:1834). */
tsvm_status tsvm_test_potrs(tsvm_context *ctx, const double *L, int32_t n, double *B,
                            int32_t nrhs, int32_t ldb);
/* Eigen-decomposition of the symmetric A (n x n); w eigenvalues, V eigenvectors as columns
 * (T:2191). */
tsvm_status tsvm_test_eig(tsvm_context *ctx, double *A, int32_t n, double *w, double *V,
                          int32_t *sweeps_host);
/* `count` symmetric n x n eigenproblems at once (the batched factor's eigensolver, the
 * reference's dsyevd, T:2191): A (count x n x n, row-major, overwritten), w (count x n), V
 * (count x n x n, eigenvectors in columns); *max_sweeps_host = the most sweeps any needed. */
tsvm_status tsvm_test_eig_batched(tsvm_context *ctx, double *A, int32_t n, int32_t count,
                                  double *w, double *V, int32_t *max_sweeps_host);
/* G (ka x kb) = A^T diag(s) B over n rows with FP64 accumulation; s may be NULL. */
tsvm_status tsvm_test_gram(tsvm_context *ctx, const float *A, int64_t lda, const float *B,
                           int64_t ldb, int64_t n, int32_t ka, int32_t kb, int32_t symmetric,
                           const double *s, double *G);

/* M (k x k fp64) = I + Z^T diag(dinv) Z by the mixed-precision path of the IPM: rows with
 * dinv <= tau through the tensor-core SYRK of a `ways`-term (2 or 3) BF16 split, the others
 * exactly in FP64; *exact_rows receives their count.  k <= 256. */
tsvm_status tsvm_test_syrk_mixed(tsvm_context *ctx, const float *Z, int32_t ldz, int64_t n,
                                 int32_t k, const double *dinv, double tau, int32_t ways,
                                 double *M, int32_t *exact_rows);

/* Allocation-failure injection: after `after` more device allocations of ctx's scratch (0: the
 * next one), growing a scratch buffer returns TSVM_ERR_OUT_OF_MEMORY instead of calling
 * cudaMalloc; -1 switches the hook off.  The context stays usable. */
tsvm_status tsvm_test_fail_alloc(tsvm_context *ctx, int32_t after);

/* One cooperative launch of `blocks` blocks (<= the SM count) meeting once at the grid barrier of
 * the cooperative eigensolver, which expects `arrivals` blocks and polls at most `max_spins`
 * (<= 2^24) times.  *released_blocks: how many were released.  Returns TSVM_ERR_TIMEOUT when the
 * wait ran out (arrivals > blocks: an arrival that never comes), the context staying usable. */
tsvm_status tsvm_test_grid_barrier(tsvm_context *ctx, int32_t blocks, int32_t arrivals,
                                   int64_t max_spins, int32_t *released_blocks);

#ifdef __cplusplus
}
#endif
#endif /* TENSORSVM_TESTING_H */
