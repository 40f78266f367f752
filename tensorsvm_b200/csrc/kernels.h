// Internal (non-ABI) entry points shared between the .cu files of the library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "context.h"
#include "tensorsvm.h"

namespace tsvm {

// ---- sketch.cu -------------------------------------------------------------------------
// The reference's gaussrand() stream (count floats, contiguous) into Q.
tsvm_status sketch_glibc(tsvm_context *ctx, int64_t count, float *Q);
// count N(0, 1) values of the counter-based Philox4x32-10 + Box-Muller sketch (Q 16-byte aligned)
tsvm_status sketch_philox(tsvm_context *ctx, uint64_t seed, int64_t count, float *Q);
// Raw glibc rand() stream (count values) into out (device).
tsvm_status glibc_rand_stream(tsvm_context *ctx, int64_t count, uint32_t *out);

// ---- features.cu -----------------------------------------------------------------------
// Centre X (n x d row-major) by its column means into Xc (n x d), write row norms ||xc||^2.
tsvm_status centre_features(tsvm_context *ctx, const float *X, int64_t n, int d, float *Xc,
                            float *norms);
// XJc, XIc = XJ, XI less the column means of XJ (one centre for both point sets).
tsvm_status centre_pair(tsvm_context *ctx, const float *XJ, int64_t nj, const float *XI,
                        int64_t ni, int d, float *XJc, float *XIc);
// Copy src (n x k, leading dim lds) into dst (n x ldd), zero columns k..ldd-1.
tsvm_status pad_rows(tsvm_context *ctx, const float *src, int64_t lds, int64_t n, int k,
                     float *dst, int64_t ldd);
// Z = diag(y) X padded to ldz columns (linear kernel, tensorsvm-train.cu:909-914).
// Linear model bias (writemodel's rule) from device X (n x d), labels and alpha; b_host host.
tsvm_status linear_bias(tsvm_context *ctx, const float *X, const float *y, const double *alpha,
                        int64_t n, int d, double C, double *b_host);
tsvm_status label_rows(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                       float *Z, int64_t ldz);

// ---- kermatmul_simt.cu -----------------------------------------------------------------
// W (n x kp) = (Y K Y) A (n x kp), K_ij = exp(-gamma ||xc_i - xc_j||^2); FP32 SIMT.
// kp must be a multiple of 64; d <= 64.  With a row range, W holds only the rows
// [row0, row0 + nr) of the product (nr rows), still summed over all n rows of A.
tsvm_status kermatmul_fp32(tsvm_context *ctx, const float *Xc, const float *norms,
                           const float *y, int64_t n, int d, double gamma, const float *A,
                           int kp, float *W, int64_t row0 = 0, int64_t nr = -1);

// ---- kermatmul_tc.cu -------------------------------------------------------------------
bool kermatmul_tc_supported(int d, int kp);
// Tensor-core (tcgen05) version; precision TSVM_PREC_FP16 or TSVM_PREC_BF16 for P and A.
// round_back (may be A itself, or null) receives A rounded to the 16-bit operand type.
// split: 0 one product; 1 the kernel block P as hi + lo (two products); 2 the operand A as
// hi + lo (two products).  kw (0: kp): the columns of A that may be nonzero (the rest are zero);
// above 256 columns, when kw rounded up to 16 is at most 416 the product runs as one launch
// (else in column slabs of 256 that each recompute the kernel block).
tsvm_status kermatmul_tc(tsvm_context *ctx, const float *Xc, const float *norms, const float *y,
                         int64_t n, int d, double gamma, const float *A, int kp, float *W,
                         int precision, float *kernel_ms, float *round_back = nullptr,
                         int split = 0, int64_t row0 = 0, int64_t nr = -1, int kw = 0);

// W (ni x kp) = Y_I K(X_I, X_J) Y_J A on the tensor cores, I rows XI (ni x d) and J rows XJ
// (nj x d; A nj x kp), both centred by the same vector; null labels mean all ones; XI may be XJ.
// split: 0..2 as kermatmul_tc, 3 = both the kernel block and A as hi + lo (about FP32 accuracy);
// deriv (split 3, FP16 only): the entries are -gamma log2(e) ||x_i - x_j||^2 K_ij.
tsvm_status kermatmul_tc_core(tsvm_context *ctx, const float *XI, const float *yI, int64_t ni,
                              const float *XJ, const float *yJ, int64_t nj, int d, double gamma,
                              const float *A, int kp, float *W, int precision, float *kernel_ms,
                              float *round_back, int split, bool deriv, double *sym = nullptr,
                              bool reuse_gram = false, int kw = 0);

// Half product for a symmetric projection (same rows on both sides): R = Y (K o H) Y A with
// H_ij = 1 (j > i), 1/2 (j == i), 0 (j < i), so that A^T (Y K Y) A = A^T R + R^T A + s u u^T with
// sym[0] = s (the kernel-mean shift the tensor-core form took off) and sym[1..kp] = u = A^T y
// (kp + 1 doubles, written by this call).  About half the tiles of kermatmul_tc.  reuse_gram:
// the call just before on this context was a kermatmul_tc over the same rows Xc with the same
// gamma, so its Gram operands are reused instead of rebuilt.
tsvm_status kermatmul_tc_half(tsvm_context *ctx, const float *Xc, const float *y, int64_t n, int d,
                              double gamma, const float *A, int kp, float *R, int precision,
                              float *kernel_ms, float *round_back, int split, double *sym,
                              bool reuse_gram = false, int kw = 0);

// Kernel-vector products of the hypergradient (hypergrad.cu): out (na x nu, FP64) =
// [K or K' = -||a - b||^2 K](A, B) U with U nb x nu FP64, on the SIMT kernel or the tensor cores.
tsvm_status kprod_any(tsvm_context *ctx, const float *A, int64_t na, const float *B, int64_t nb,
                      int d, double gamma, const double *U, int nu, double *out, bool deriv,
                      bool tc);

// Precision classes of tsvm_precision.
inline bool precision_valid(int p) { return p >= TSVM_PREC_FP32 && p <= TSVM_PREC_FP16_FAST; }
inline bool precision_is_bf16(int p) { return p == TSVM_PREC_BF16 || p == TSVM_PREC_BF16_FAST; }
// the tensor-core forms that split the accuracy-setting operand of each factor pass
inline bool precision_is_split(int p) { return p == TSVM_PREC_BF16 || p == TSVM_PREC_FP16; }

// A unit of batched work: rows [row0, row0 + rows) of problem p; goff is the index of the
// unit's first row in the problems' concatenated per-row vectors.
struct WorkUnit {
  int32_t p, rows;
  int64_t row0, goff;
};

// ---- tallskinny.cu ---------------------------------------------------------------------
// G (ka x kb, row-major fp64, ldg = kb) = A^T B over n rows; A n x lda fp32, B n x ldb fp32.
// If symmetric (A == B, ka == kb) only the lower triangle is accumulated and G is mirrored.
// rowscale (n doubles, may be null) weights row i: G = A^T diag(rowscale) B.
tsvm_status gram_fp64(tsvm_context *ctx, const float *A, int64_t lda, const float *B,
                      int64_t ldb, int64_t n, int ka, int kb, bool symmetric, double *G,
                      const double *rowscale = nullptr);
// G (k x k, fp64) = sum over the rows listed in rowidx[0 .. *count_dev) of rowscale[i] a_i a_i^T
// (count read on the device, at most n_max rows).
tsvm_status gram_fp64_rows(tsvm_context *ctx, const float *A, int64_t lda, int64_t n_max, int k,
                           const int64_t *rowidx, const int *count_dev, const double *rowscale,
                           double *G);
// Per-unit partial Gram matrices of a batch: part[u] (k x k, lower 64 x 64 tiles filled) =
// sum over the unit's rows j of rowscale[goff + j] z_j z_j^T with z_j rows of Zs[p] (lda);
// units of problems with active[p] == 0 are skipped.  With rowidx and counts, only the
// counts[u] rows rowidx[goff + i] (indices within the unit) of each unit are summed, the list
// cut into `parts` pieces of whole 32-row slabs, piece j into part[u * parts + j]; a piece past
// the end of the list writes nothing (gram_units_piece_rows says which pieces hold rows).
tsvm_status gram_fp64_units(tsvm_context *ctx, const float *const *Zs, int64_t lda, int k,
                            const WorkUnit *units, int nunits, const int *active,
                            const double *rowscale, double *part, const int64_t *rowidx = nullptr,
                            const int *counts = nullptr, int parts = 1);
// Whether piece j of `parts` of a list of cnt rows holds any (the cut of gram_fp64_units).
__host__ __device__ inline bool gram_units_piece_rows(int cnt, int parts, int j) {
  const int per = ((cnt + parts - 1) / parts + 31) / 32 * 32;
  return j * per < cnt;
}
// Out (n x kp) = A (n x kp) * R (kp x kp, fp32 row-major). Out may alias A.
tsvm_status apply_right_fp32(tsvm_context *ctx, const float *A, int64_t n, int kp,
                             const float *R, float *Out);

// ---- dense.cu (small k x k FP64, single device) ----------------------------------------
// In-place lower Cholesky of the n x n row-major matrix A (lda, n <= 864); *info_dev receives 0
// or the 1-based failing column.  Dinv (ceil(n/32) blocks of 32 x 32 doubles) receives the
// inverses of the diagonal 32 x 32 blocks of L, used by potrs_fp64 and trinv_lower_fp64.
// The upper triangle is left untouched.
tsvm_status chol_fp64(tsvm_context *ctx, double *A, int n, int lda, int *info_dev, double *Dinv,
                      cudaStream_t stream = nullptr);
// SMs one chol_fp64 of order n occupies (a cluster of 8 CTAs up to n = 256, else one CTA).
int chol_fp64_sms(int n);
// Dinv of an existing lower factor L (as chol_fp64 writes it).
tsvm_status tri_diag_inverse(tsvm_context *ctx, const double *L, int n, int lda, double *Dinv);
// Solve (L L^T) X = B for nrhs (<= 4) right-hand sides stored as rows of B (nrhs x ldb).
tsvm_status potrs_fp64(tsvm_context *ctx, const double *L, int n, int lda, const double *Dinv,
                       double *B, int nrhs, int ldb);
// Batched forms: `count` independent n x n problems at A + b * strideA (Dinv + b * strideD,
// info_dev[b], B + b * strideB), problems with active[b] == 0 skipped; one CTA per problem.
// The factorisations of `count` problems (stride strideA / strideD, info_dev[p]) with the same
// arithmetic per problem as chol_fp64: one launch of one CTA per problem (those with
// active[p] != 0) when n <= 128, else chol_fp64 for each problem in `pending`.
tsvm_status chol_fp64_same(tsvm_context *ctx, double *A, int n, int lda, int64_t strideA,
                           int *info_dev, double *Dinv, int64_t strideD, int count,
                           const int *active, const std::vector<int> &pending);
tsvm_status chol_fp64_batched(tsvm_context *ctx, double *A, int n, int lda, int64_t strideA,
                              int *info_dev, double *Dinv, int64_t strideD, int count,
                              const int *active);
tsvm_status potrs_fp64_batched(tsvm_context *ctx, const double *L, int n, int lda,
                               int64_t strideA, const double *Dinv, int64_t strideD, double *B,
                               int nrhs, int ldb, int64_t strideB, int count, const int *active);
// Lower-triangular inverse: Linv = L^-1 (both n x n row-major, lda).
tsvm_status trinv_lower_fp64(tsvm_context *ctx, const double *L, int n, int lda,
                             const double *Dinv, double *Linv);
// Symmetric eigen-decomposition by cyclic Jacobi: A (n x n, lda) is overwritten; w (n) gets
// the eigenvalues, V (n x n row-major) the eigenvectors as COLUMNS.
tsvm_status eig_jacobi_fp64(tsvm_context *ctx, double *A, int n, int lda, double *w, double *V,
                            int *sweeps_out);
// count problems (A count x n x n, w count x n, V count x n x n, contiguous) in one launch when
// n <= 128 (one CTA each); *max_sweeps_out = the most sweeps any problem took.
tsvm_status eig_jacobi_fp64_batched(tsvm_context *ctx, double *A, int n, int count, double *w,
                                    double *V, int *max_sweeps_out);
// Elementwise helpers on small matrices (device kernels, defined in dense.cu).
tsvm_status small_add_diag(tsvm_context *ctx, double *A, int n, int lda, double shift);
tsvm_status small_symmetrize(tsvm_context *ctx, double *A, int n, int lda);

// ---- syrk_tc.cu ------------------------------------------------------------------------
bool syrk_tc_supported(int k);
// idx[0 .. *count_dev) = the rows with dinv > tau, in increasing order.
tsvm_status big_rows(tsvm_context *ctx, const double *dinv, int64_t n, double tau, int64_t *idx,
                     int *count_dev);
// M (k x k, fp64, full) = I + G64 + sum over rows with dinv <= tau of dinv_j z_j z_j^T, the
// latter from a `ways`-term BF16 split on the tensor cores with FP32 accumulation.  G64 may be
// null.  A timed-out tensor-core launch leaves NaN in M (the Cholesky then reports failure).
// The batched form for k <= 256 (one window, 2-way split, ldz <= 256): per work unit u, the
// rows with dinv <= taus[p] through the fused tensor-core SYRK into FP32 part_tc[u] (KP x KP,
// KP = 128 for k <= 128 else 256), and the others listed in index order (rowidx[goff + i],
// counts[u]) and summed exactly into FP64 part64[u] (k x k).  big_rows_units only lists.
tsvm_status big_rows_units(tsvm_context *ctx, const double *dinv, const WorkUnit *units,
                           int nunits, const int *active, const double *taus, int64_t *rowidx,
                           int *counts);
tsvm_status syrk_units_tc(tsvm_context *ctx, const float *const *Zs, int64_t ldz, int k,
                          const WorkUnit *units, int nunits, const int *active,
                          const double *dinv, const double *taus, float *part_tc, int *err);
int syrk_units_kp(int k);
tsvm_status syrk_capacitance_tc(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k,
                                const double *dinv, double tau, int ways, const double *G64,
                                double *M);

// ---- ipm.cu ----------------------------------------------------------------------------
tsvm_status ipm_solve(tsvm_context *ctx, const float *Z, int ldz, const float *y, int64_t n,
                      int k, double C, const tsvm_ipm_options &opt, double *alpha_out,
                      double *xi_out, double *s_out, double *ymult_out, tsvm_ipm_stats *stats);
// KKT adjoint at a converged dual solution: lambda solves [Q + D, a; a^T, 0][lambda; nu] =
// [c; 0] with Q = Z Z^T and D = s/x + xi/(C - x) of the final iterate, through SMW.
// out (kz doubles) = Z^T v and out (n doubles) = Z g through the streaming passes.
tsvm_status zt_vec(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k, const double *v,
                   double *out);
tsvm_status zw_vec(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k, const double *g,
                   double *out);
tsvm_status kkt_adjoint(tsvm_context *ctx, const float *Z, int ldz, const float *y, int64_t n,
                        int k, double C, const double *alpha, const double *xi, const double *s,
                        const double *c, double *lambda);
// out = Z (Z^T Z)^-1 Z^T v, the projection onto the range of the factor.
tsvm_status project_range(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k,
                          const double *v, double *out);
tsvm_status ipm_solve_batched(tsvm_context *ctx, const tsvm_ipm_problem *problems, int count,
                              int k, int ldz, const tsvm_ipm_options &opt, tsvm_ipm_stats *stats,
                              tsvm_batch_info *info);
tsvm_status bias_rbf(tsvm_context *ctx, const float *Z, int ldz, const float *y,
                     const double *alpha, int64_t n, int k, double C, double *b, double *bstd,
                     int32_t *nsv, int32_t *nfree);

// ---- factor.cu -------------------------------------------------------------------------
// What the hypergradient keeps of a factorisation: the sketch Omega (n x kp copy), the combined
// CholeskyQR factor R (k x k upper, pass-1 output B = W R; the buffer holds 2 k x k doubles) and
// a copy of the orthonormal basis W (n x kp) taken before the second pass rounds W in place to
// the tensor-core operand type (B = W R holds for the copy, not for the rounded W).
struct FactorKeep {
  float *omega;
  double *R;
  float *W;
};
// With a row range (row0, nr) the rows [row0, row0 + nr) of Z are computed (Z holds nr rows)
// against all n rows of X, across the ranks of ctx's communicator (keep must be null).
tsvm_status factor_rbf(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                       double gamma, int k, int precision, int sketch, const float *Q_user,
                       float *Z, int ldz, tsvm_factor_info *info, FactorKeep *keep = nullptr,
                       int64_t row0 = 0, int64_t nr = -1, double *C_out = nullptr);
// With C_out set, factor_rbf stops after the projection: C_out (k x k FP64) holds the symmetrised
// C = W^T (K W) and Z (ldz = kp) the orthonormal basis W; factor_finish then forms
// Z = W V diag(sqrt(max(w, 0))) in place from C's eigen-decomposition (V k x k row-major, w k).
// factor_rbf keeping the hypergradient's factor state in the context (SLOT_HG_OMEGA / _R / _W /
// _Z, ctx->kept); Z (ldz) receives the factor as from factor_rbf.
tsvm_status factor_rbf_keep(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                            double gamma, int k, int precision, float *Z, int ldz,
                            tsvm_factor_info *info);
tsvm_status factor_finish(tsvm_context *ctx, float *Z, int64_t n, int k, const double *V,
                          const double *w, tsvm_factor_info *info);
// Factors of `count` independent problems (shared d, k, precision): every problem through the
// projection, one batched eigensolver launch, then every Z.  ms_eig: the eigensolver launch.
tsvm_status factor_rbf_batched(tsvm_context *ctx, const tsvm_factor_problem *pr, int count, int d,
                               int k, int precision, int sketch, int ldz,
                               tsvm_factor_info *infos, double *ms_eig);

// ---- predict.cu ---------------------------------------------------------------------------
// Decision values of m rows under a model (device arrays); asynchronous on ctx->stream.
tsvm_status decision_values(tsvm_context *ctx, const tsvm_model_view *mv, const float *X,
                            int64_t m, double *f);
// out2 (host): ||K~||_F, ||K~ - Z Z^T||_F in FP64; synchronises.
tsvm_status kernel_residual(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                            double gamma, const float *Z, int64_t ldz, int k, double *out2);

}  // namespace tsvm
