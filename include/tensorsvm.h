/* tensorsvm.h - C ABI of the B200-native TensorSVM training path.
 *
 * The reference trainer (robbwu/tensorsvm, tensorsvm-train.cu) has no library API: its seams
 * are two C++ functions that pass state through globals,
 *     double LRA(float *Z, int ldz, double *U, int ldu, long n, long k)      tensorsvm-train.cu:1941
 *     void   mpc(double *Z, double *a, double C, double *X, double *Xi, int N, int d)
 *                                                                          tensorsvm-train.cu:1507
 * plus the bias computation inside writemodel (tensorsvm-train.cu:355-376) and the driver in
 * main (tensorsvm-train.cu:858-1059).  Each entry point below names the one it replaces.
 *
 * Conventions (all entry points):
 *   - every call returns a tsvm_status; none calls exit();
 *   - pointers documented as "device" are caller-owned CUDA device buffers on the context's
 *     device; "host" buffers are caller-owned host memory;
 *   - the library owns its device scratch inside the context (grown on demand, freed by
 *     tsvm_destroy);
 *   - one context per host thread; all work is issued on the context's stream, and every
 *     call returns after that stream is synchronised unless noted otherwise.
 */
#ifndef TENSORSVM_H
#define TENSORSVM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tsvm_status {
  TSVM_OK = 0,
  TSVM_ERR_INVALID_ARGUMENT = 1,
  TSVM_ERR_CUDA = 2,
  TSVM_ERR_OUT_OF_MEMORY = 3,
  /* capacitance matrix I + Z^T D^-1 Z is not positive definite; the reference prints
   * "Cholesky fact info error" and returns early (tensorsvm-train.cu:1709-1714) */
  TSVM_ERR_NOT_SPD = 4,
  TSVM_ERR_UNSUPPORTED = 5,
  TSVM_ERR_NO_DEVICE = 6,
  /* a bounded device-side wait gave up; the context stays usable */
  TSVM_ERR_TIMEOUT = 7,
  /* IPM stopped because max(D)/min(D) > 1e18 (tensorsvm-train.cu:1653-1658); results valid */
  TSVM_WARN_ILL_CONDITIONED = 8,
  /* IPM stopped at the iteration cap (MAX_MPC_ITER, tensorsvm-train.cu:62); results valid */
  TSVM_WARN_MAX_ITER = 9,
  /* the Gaussian sketch stream ran short of accepted pairs (retry limit reached) */
  TSVM_ERR_SKETCH = 10,
  TSVM_ERR_IO = 11,
  /* a collective of the row-sharded path (tsvm_comm.allreduce) reported a failure */
  TSVM_ERR_COMM = 12
} tsvm_status;

/* -t kernel_type values accepted by the reference (tensorsvm-train.cu:1112-1118) */
typedef enum tsvm_kernel { TSVM_KERNEL_LINEAR = 0, TSVM_KERNEL_RBF = 2 } tsvm_kernel;

/* Arithmetic of the two contractions (kernel-block product and Z^T D^-1 Z).
 * FP32: SIMT FP32 (the "plain" form, what the reference computes without -tensorcore).
 * BF16/FP16: tcgen05 tensor cores with FP32 accumulation (the "-tensorcore" form).  In each
 *   factor pass the operand whose rounding sets the factor's accuracy is carried as a 16-bit
 *   hi + lo pair, contracted by two MMAs into the same FP32 accumulator: the kernel block in
 *   the range-finder pass W = K Q, the orthonormal basis in the projection pass K W.
 * BF16_FAST/FP16_FAST: one 16-bit product per pass (about 1.7x faster factor); the basis of
 *   the projection pass is rounded in place.  The factor's weak eigen-directions then move by
 *   the 16-bit rounding, and with them the solution along the dual's flat optimal face. */
typedef enum tsvm_precision {
  TSVM_PREC_FP32 = 0,
  TSVM_PREC_BF16 = 1,
  TSVM_PREC_FP16 = 2,
  TSVM_PREC_BF16_FAST = 3,
  TSVM_PREC_FP16_FAST = 4
} tsvm_precision;

/* Sketch source.  GLIBC reproduces the reference's gaussrand() stream exactly (glibc rand()
 * from its default seed, Marsaglia polar method, tensorsvm-train.cu:2621-2643) on the GPU: the
 * parity mode.  USER takes a caller-provided n x k row-major float matrix.  PHILOX draws the
 * entries from the counter-based Philox4x32-10 generator (Salmon et al., SC 2011) keyed by the
 * context's seed (tsvm_set_sketch_seed), two Box-Muller pairs per 128-bit block: the same
 * matrix for the same seed on any launch shape, with no sequential stream. */
typedef enum tsvm_sketch {
  TSVM_SKETCH_GLIBC = 0,
  TSVM_SKETCH_USER = 1,
  TSVM_SKETCH_PHILOX = 2
} tsvm_sketch;

typedef struct tsvm_context tsvm_context;

typedef struct tsvm_factor_info {
  int64_t n;
  int32_t d, k, k_padded;
  int32_t realk;                 /* eigenvalues of C kept (> 0), tensorsvm-train.cu:2197-2211 */
  int32_t precision;
  double eig_max, eig_min;       /* largest / smallest eigenvalue of C (the "[LRA]" print) */
  double ms_sketch, ms_pass1, ms_ortho, ms_pass2, ms_project, ms_total;
  double ms_kermatmul_kernel;    /* device time of the two fused kernel-block launches */
  double flops_kermatmul;        /* algorithmic flops: 2 passes x (2 n^2 k + 2 n^2 d) */
} tsvm_factor_info;

typedef struct tsvm_ipm_options {
  int32_t max_iter;       /* iteration cap, default 100 (tensorsvm-train.cu:62) */
  double tol;             /* reference stop: mu, ||rd||, |rp| all < tol; default 1e-7 (T:1647) */
  double rel_gap_tol;     /* additional stop when rel_gap = (pobj-dobj)/max(1,|pobj|) <= tol
                             and ||rd||/(1+sqrt n), |rp|/(1+sqrt n) <= tol; <= 0 disables */
  int32_t precision;      /* capacitance matrix M = I + Z^T D^-1 Z: TSVM_PREC_FP32 sums it
                             exactly in FP64 (the reference's DSYRK); TSVM_PREC_BF16 or _FP16
                             uses the tensor-core SYRK of a BF16 hi+lo split (FP32 accumulate)
                             for the rows with small weight, FP64 for the rest (k <= 256) */
  int32_t refine_sweeps;  /* mixed precision: refinement sweeps of every capacitance solve
                             against the exact operator (1..2; 0 means 1) */
  int32_t kernel;         /* initialisation rule: TSVM_KERNEL_RBF (T:1535) or _LINEAR (T:1553) */
  int32_t verbose;        /* print the reference's "iter %d, mu=..." lines every 5 iterations */
} tsvm_ipm_options;

typedef struct tsvm_ipm_stats {
  int32_t iters;
  int32_t status;         /* tsvm_status of the solve */
  double mu, norm_rd, norm_rp, cond_d, pobj, dobj, rel_gap;
  double ms_total, ms_syrk, ms_factor, ms_streams;
  double t_rel_gap_1e6_ms; /* wall time at the first iterate with rel_gap <= 1e-6 (or -1) */
  /* Mixed-precision capacitance matrix (precision BF16/FP16): 1 if used; iterations redone
   * with more rows summed exactly; rows summed exactly in FP64 per iteration (max, mean); the
   * largest relative residual of an unrefined capacitance solve. */
  int32_t mixed_syrk, syrk_retries, exact_rows_max;
  double exact_rows_mean, refine_res_max;
} tsvm_ipm_stats;

/* One problem of a batched interior-point solve (all problems share k and ldz). */
typedef struct tsvm_ipm_problem {
  const float *Z;      /* device, n x ldz row-major factor (columns k..ldz-1 ignored) */
  const float *y;      /* device, n labels in {+1, -1} */
  int64_t n;
  double C;
  double *alpha_out;   /* device, n */
  double *xi_out;      /* device, n, or NULL */
} tsvm_ipm_problem;

/* How a batched solve ran. */
typedef struct tsvm_batch_info {
  int32_t units;       /* work units of the streaming passes (a unit is a row range of one problem) */
  int32_t unit_rows;   /* rows per unit chosen by the autotuner */
  int32_t graph_used;  /* 1 if the iterations were replayed from a captured CUDA graph */
  int32_t iters_max;   /* iterations of the slowest problem */
  double ms_total, ms_autotune;
} tsvm_batch_info;

/* Human-readable status. */
const char *tsvm_status_string(tsvm_status s);

/* Create a context on CUDA device `device` with its own stream.  Replaces the per-call
 * cublasCreate/cudaStreamCreate/cusolverDnCreate of LRA and mpc (T:1509-1514, T:1945-1961). */
tsvm_status tsvm_create(tsvm_context **ctx, int device);
tsvm_status tsvm_destroy(tsvm_context *ctx);

/* Issue the context's work on a caller-owned CUDA stream (cudaStream_t passed as void*);
 * NULL restores the context's own stream.  The library never destroys a caller's stream. */
tsvm_status tsvm_set_stream(tsvm_context *ctx, void *stream);

/* Row-sharded training over several GPUs, one process (and context) per GPU.  Each rank owns a
 * contiguous range of the n training rows (its rows of X, y, Z, alpha, s and xi); the ranks
 * exchange only k x k matrices, k-vectors and scalars in the interior-point solver, and the
 * factor's basis once per factor (the projection pass needs every row of it).  The reference
 * has no multi-GPU path (one process, one GPU, host chunk loops, tensorsvm-train.cu:1999-2063
 * and 1674-1697); this communicator is how the caller's collective library (NCCL over
 * NVLink, or any other) is plugged in.
 *   allreduce: in-place all-reduce over the ranks of `count` values at the DEVICE pointer
 *     `buf`, ordered on the CUDA stream `stream` (cudaStream_t as void*): the library's later
 *     work on that stream must see the result.  dtype 0 = double, 1 = float; op 0 = sum,
 *     1 = min.  Returns 0 on success; anything else makes the calling entry point return
 *     TSVM_ERR_COMM.  Every rank makes the same calls in the same order (the control flow of
 *     the sharded solve depends only on reduced values), so a rank that fails or leaves shows
 *     up as a failing collective on the others. */
typedef struct tsvm_comm {
  int32_t rank, world;
  int (*allreduce)(void *user, void *buf, int64_t count, int32_t dtype, int32_t op,
                   void *stream);
  void *user;
} tsvm_comm;

/* Attach a communicator to the context (copied; NULL detaches).  While one is attached,
 * tsvm_ipm and tsvm_bias work on this rank's rows of a row-sharded problem: their Z, y, alpha,
 * xi, s are the rank's rows, n is the rank's row count, and every reduction (k-vectors,
 * scalars, the capacitance matrix I + Z^T D^-1 Z, the bias's free-SV terms) is completed
 * across the ranks; the statistics are global.  tsvm_factor_rows uses it for the factor. */
tsvm_status tsvm_set_comm(tsvm_context *ctx, const tsvm_comm *comm);

/* Seed of the TSVM_SKETCH_PHILOX sketch of this context's factors (default 0).  The
 * reference's sketch has no seed: glibc rand() is never seeded (tensorsvm-train.cu:1966). */
tsvm_status tsvm_set_sketch_seed(tsvm_context *ctx, uint64_t seed);

/* With keep = 1, every tsvm_factor of this context with the glibc sketch keeps what the
 * hypergradient needs of it in the context (the sketch, the CholeskyQR factor, the basis before
 * its 16-bit rounding and Z: about 3 n k_padded floats), and tsvm_hypergrad on the same X, y, n, d,
 * gamma, k and precision reuses them instead of recomputing the factor.  Off (0) by default: when
 * memory is tight the hypergradient recomputes the factor.  The kept factor's orthonormalisation
 * uses exact FP64 Gram matrices (as the recomputation does). */
tsvm_status tsvm_set_factor_keep(tsvm_context *ctx, int32_t keep);

/* Fill `opt` with the reference's defaults (max_iter 100, tol 1e-7, FP32, RBF init). */
void tsvm_ipm_default_options(tsvm_ipm_options *opt);

/* Kernel factor (replaces LRA, tensorsvm-train.cu:1941-2374).
 * Computes Z (n x k, row-major, leading dimension ldz >= k) with Z Z^T ~= Y K Y, K the RBF
 * kernel exp(-gamma ||x_i - x_j||^2) of X: sketch Q, W = Y K Y Q, W = orth(W), Q = Y K Y W,
 * C = W^T Q, C = V diag(w) V^T, Z = W V diag(sqrt(max(w, 0))).  Columns k..ldz-1 of Z are 0.
 *   X      device, n x d row-major float
 *   y      device, n labels in {+1, -1}
 *   Q_user device, n x k row-major float when sketch == TSVM_SKETCH_USER, else NULL
 *   Z      device, n x ldz row-major float (output)
 *   info   host, may be NULL */
tsvm_status tsvm_factor(tsvm_context *ctx, const float *X, const float *y, int64_t n, int32_t d,
                        double gamma, int32_t k, int32_t precision, int32_t sketch,
                        const float *Q_user, float *Z, int32_t ldz, tsvm_factor_info *info);

/* Kernel factor of a row-sharded problem (replaces LRA, tensorsvm-train.cu:1941-2374, across
 * the ranks of the attached communicator): X (n_global x d) and y (n_global) are the whole
 * training set on every rank (small: 72 MB at n = 1M, d = 18); this rank computes the rows
 * [row0, row0 + n_rows) of Z (n_rows x ldz, device).  Every rank draws the whole sketch (or
 * reads Q_user, n_global x k), computes its rows of W = Y K Y Q against all rows, and the
 * CholeskyQR Gram matrices and C = W^T (K W) are all-reduced; the basis W is all-gathered
 * (as an all-reduce of the zero-padded rows) once for the projection pass.  With no
 * communicator attached, row0 = 0 and n_rows = n_global, it is tsvm_factor. */
tsvm_status tsvm_factor_rows(tsvm_context *ctx, const float *X, const float *y, int64_t n_global,
                             int32_t d, int64_t row0, int64_t n_rows, double gamma, int32_t k,
                             int32_t precision, int32_t sketch, const float *Q_user, float *Z,
                             int32_t ldz, tsvm_factor_info *info);

/* One problem of a batched factorisation. */
typedef struct tsvm_factor_problem {
  const float *X;      /* device, n x d row-major */
  const float *y;      /* device, n labels in {+1, -1} */
  int64_t n;
  double gamma;
  float *Z;            /* device, n x ldz output (ldz = k rounded up to 64) */
} tsvm_factor_problem;

/* Kernel factors of `count` independent problems of the same d, k and precision (replaces
 * running LRA, tensorsvm-train.cu:1941-2374, once per problem; the reference trains one problem
 * per process).  Each problem runs its sketch, kernel-block passes, CholeskyQR and projection
 * C = W^T (K W); then the eigen-decompositions of all the C's are one launch (one CTA per
 * problem for k <= 128, side by side on their own SMs), and every Z = W V diag(sqrt(w+)) is
 * formed in place.  infos[count] (may be NULL) receive each problem's factor statistics. */
tsvm_status tsvm_factor_batched(tsvm_context *ctx, const tsvm_factor_problem *problems,
                                int32_t count, int32_t d, int32_t k, int32_t precision,
                                int32_t sketch, int32_t ldz, tsvm_factor_info *infos);

/* Linear "factor": Z = diag(y) X, k = d (tensorsvm-train.cu:909-914).  Device buffers. */
tsvm_status tsvm_linear_factor(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                               int32_t d, float *Z, int32_t ldz);

/* Interior-point solve of  min 1/2 a^T Q a - e^T a,  y^T a = 0,  0 <= a <= C,  Q = Z Z^T
 * (replaces mpc, tensorsvm-train.cu:1507-1785, with NewtonStep 1794-1822 and SMWSolve
 * 1824-1840).  Newton steps go through M = I + Z^T D^-1 Z (FP64 Cholesky on the device).
 *   Z          device, n x ldz row-major float (columns beyond k ignored)
 *   y          device, n labels in {+1, -1}
 *   alpha_out  device, n doubles (the dual variables "X" of the reference)
 *   xi_out     device, n doubles or NULL
 *   s_out      device, n doubles or NULL: the multipliers of alpha >= 0 at the final iterate
 *              (with xi, ymult and alpha what tsvm_hypergrad needs)
 *   ymult_out  host, the equality multiplier (the reference's local "y"), or NULL
 *   opt        host, NULL for defaults;  stats host, may be NULL
 * Returns TSVM_OK on convergence, TSVM_WARN_ILL_CONDITIONED / TSVM_WARN_MAX_ITER when the
 * reference's other stopping rules fired (outputs valid), TSVM_ERR_NOT_SPD on a failed
 * Cholesky (outputs hold the last iterate, as the reference leaves X). */
tsvm_status tsvm_ipm(tsvm_context *ctx, const float *Z, int32_t ldz, const float *y, int64_t n,
                     int32_t k, double C, const tsvm_ipm_options *opt, double *alpha_out,
                     double *xi_out, double *s_out, double *ymult_out,
                     tsvm_ipm_stats *stats);

/* Batched interior-point solve (replaces running mpc, T:1507-1840, once per problem): `count`
 * independent SVM duals of uneven n -- one-vs-rest classes, a (C, gamma) grid, folds -- solved
 * together.  Every streaming pass is one launch over work units (row ranges of one problem)
 * of all unconverged problems, the k x k Cholesky and solves are one launch with a CTA per
 * problem, the host synchronises once per iteration for all stopping rules, and from the second
 * iteration on the iteration's launches are replayed from a captured CUDA graph.  The unit
 * size is autotuned on the first pass.  opt->precision TSVM_PREC_FP32 sums the capacitance
 * matrices in FP64 (the reference's DSYRK numerics); the 16-bit precisions (k <= 256, ldz <=
 * 256) build them as tsvm_ipm does -- per work unit the tensor-core SYRK of the rows with weight
 * <= tau and the other rows exactly in FP64, every solve refined once against the exact
 * operator, tau adapted per problem on the device, a failed step retried with more rows exact.
 * stats[count] receives each
 * problem's statistics (status in stats[i].status); the call returns TSVM_OK when every
 * problem ended with a usable alpha (OK, WARN_*), else the first failing status. */
tsvm_status tsvm_ipm_batched(tsvm_context *ctx, const tsvm_ipm_problem *problems, int32_t count,
                             int32_t k, int32_t ldz, const tsvm_ipm_options *opt,
                             tsvm_ipm_stats *stats, tsvm_batch_info *info);

/* Result of tsvm_hypergrad. */
typedef struct tsvm_hypergrad_result {
  double loss;               /* (1/m) sum_v max(0, 1 - y_v f(x_v))^2 on the validation set */
  double dloss_dlog_gamma;   /* through the dual solution, the bias and the validation kernel */
  double dloss_dlog_C;
  int32_t n_free_bias;       /* free SVs the bias was averaged over (<= 50) */
  double ms;
  int32_t factor_reused;     /* 1: the factor kept by tsvm_factor was reused, 0: recomputed */
} tsvm_hypergrad_result;

/* Hypergradient of the validation squared-hinge loss of a trained RBF SVM (no counterpart in
 * the reference; extends LRA T:1941-2374, mpc T:1507-1840 and the bias T:355-376).  Given the
 * training set (X n x d, labels y), gamma, C, k and the factor precision used for training,
 * the solution of tsvm_ipm (alpha, xi, s, the equality multiplier ymult) and the bias b of
 * tsvm_bias, the model is f(x) = sum_i alpha_i y_i exp(-gamma ||x_i - x||^2) + b.  The factor
 * is reused when tsvm_factor kept it (tsvm_set_factor_keep) for the same inputs, else recomputed
 * (same sketch, same Z as training), the KKT system of the dual is differentiated
 * implicitly with one adjoint solve through I + Z^T D^-1 Z (SMW, as the IPM's Newton step),
 * and the gamma derivative goes through the range finder with the sketch held fixed.  dXv
 * (device, nv x d, may be NULL) receives dL/dXv.  All arrays are device pointers; d <= 64. */
tsvm_status tsvm_hypergrad(tsvm_context *ctx, const float *X, const float *y, int64_t n, int32_t d,
                           const float *Xv, const float *yv, int64_t nv, double gamma, double C,
                           int32_t k, int32_t precision, const double *alpha, const double *xi,
                           const double *s, double ymult, double b,
                           tsvm_hypergrad_result *result, float *dXv);

/* Bias of the RBF model (replaces tensorsvm-train.cu:355-376): the mean over the first <= 50
 * free SVs j (1e-6 < alpha_j < C - 1e-6, in index order) of y_j - sum_{i in SV} alpha_i y_j
 * (Z_i . Z_j).  b is NaN when there is no free SV (as the reference's 0/0).
 *   Z, y, alpha device;  b_out, b_std_out, n_sv, n_free host (any may be NULL) */
tsvm_status tsvm_bias(tsvm_context *ctx, const float *Z, int32_t ldz, const float *y,
                      const double *alpha, int64_t n, int32_t k, double C, double *b_out,
                      double *b_std_out, int32_t *n_sv, int32_t *n_free);

/* Allocation-free variant of tsvm_bias, for callers that must not let a library allocate
 * device memory (a serving process whose HBM is pre-partitioned by its own pool, a host
 * framework that forbids plug-in allocations, or a process that has already committed all
 * device memory).  It has no counterpart in the reference, whose bias loop runs on the host.
 * It needs no tsvm_context and calls no allocator: its scratch is a fixed ~2.4 MB static
 * device array (resident on each device that loads the library until exit).
 *   Z, y, alpha  device inputs as for tsvm_bias, on the current device
 *   out          device, 4 doubles: b, b_std, number of SVs, number of free SVs
 *   stream       cudaStream_t (void*), NULL for the legacy default stream; the call is
 *                asynchronous on it
 * Limits: k <= 1024, otherwise TSVM_ERR_INVALID_ARGUMENT.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress) with that device current; make
 * it before any stream capture.  All calls share the array: calls that overlap on the GPU
 * race and must be ordered by the caller. */
tsvm_status tsvm_bias_noalloc(const float *Z, int32_t ldz, const float *y, const double *alpha,
                              int64_t n, int32_t k, double C, double *out, void *stream);

/* End-to-end training from HOST buffers (the path main() drives, tensorsvm-train.cu:907-1024):
 * copies X and y to the device, factors (RBF) or labels (linear), solves, computes the bias
 * and copies alpha back.  For the linear kernel `gamma` and `k` are ignored and w is not
 * formed here (the caller forms it from alpha, as writemodel does).
 *   X host n x d row-major; y host labels +-1; alpha_out host n doubles; b_out host. */
tsvm_status tsvm_train(tsvm_context *ctx, const float *X, const float *y, int64_t n, int32_t d,
                       int32_t kernel, double gamma, double C, int32_t k, int32_t precision,
                       const tsvm_ipm_options *opt, double *alpha_out, double *b_out,
                       tsvm_factor_info *finfo, tsvm_ipm_stats *istats);

/* A trained binary model as the model file holds it (writemodel, tensorsvm-train.cu:340-349
 * LIBLINEAR, 384-406 RBF):
 *   RBF:    f(x) = sum_i coef_i exp(-gamma ||sv_i - x||^2) - rho, coef_i = y_i alpha_i over the
 *           nsv support vectors (rows of sv, nsv x d row-major), rho = -b;
 *   LINEAR: f(x) = w . x - rho with w = sv (d floats), coef and gamma unused, rho = -b.
 * The predicted label is the model's first label (+1 side) when f(x) > 0, else the second. */
typedef struct tsvm_model_view {
  int32_t kernel;        /* TSVM_KERNEL_RBF or TSVM_KERNEL_LINEAR */
  int32_t d;             /* features */
  int64_t nsv;           /* support vectors (RBF) */
  const float *sv;       /* RBF: nsv x d; LINEAR: w, d floats */
  const double *coef;    /* RBF: nsv coefficients */
  double rho;
  double gamma;
} tsvm_model_view;

/* Decision values f(x_v) of m rows (no counterpart in the reference, which leaves prediction
 * to ThunderSVM, README.md:27-31; its own predict T:166-270 is never called).  The model's
 * arrays, X (m x d row-major) and f (m doubles) are device pointers. */
tsvm_status tsvm_decision_values(tsvm_context *ctx, const tsvm_model_view *model, const float *X,
                                 int64_t m, double *f);

/* tsvm_decision_values on HOST buffers (the model's arrays, X and f): copies in, computes,
 * copies f back. */
tsvm_status tsvm_predict(tsvm_context *ctx, const tsvm_model_view *model, const float *X,
                         int64_t m, double *f);

/* Frobenius norms ||K~||_F and ||K~ - Z Z^T||_F, K~_ij = y_i y_j exp(-gamma ||x_i - x_j||^2),
 * in FP64 (replaces rbf_fnorm_res, tensorsvm-train.cu:2388-2467, run by -analysis).
 * X (n x d), y (n), Z (n x ldz, first k columns used) device; fnorm, fnorm_res host. */
tsvm_status tsvm_kernel_residual(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                 int32_t d, double gamma, const float *Z, int32_t ldz, int32_t k,
                                 double *fnorm, double *fnorm_res);

/* tsvm_kernel_residual of the last RBF tsvm_train on this context (its device copies of X and
 * y and its factor), as the reference's -analysis follows its LRA.  TSVM_ERR_INVALID_ARGUMENT
 * when the context has not trained an RBF model, or a later call reused that memory. */
tsvm_status tsvm_train_residual(tsvm_context *ctx, double *fnorm, double *fnorm_res);

/* ---- Host I/O (no device work, no context) ------------------------------------------------ */

/* LIBSVM text reader (replaces libsvmread, tensorsvm-train.cu:1162-1278), parsed by `threads`
 * host threads (0: one per core).  *labels (n floats) and *X (n x d row-major, dense) are
 * allocated here: release them with tsvm_free.  Indices are shifted by the smallest index seen
 * (1 for 1-based files); d is the largest index (+1 for a 0-based file).  scale256 divides every
 * value by 256 (-scale256).  A malformed or empty line returns TSVM_ERR_IO with *bad_line set to
 * its 1-based number (the reference prints a message and keeps what it read). */
tsvm_status tsvm_read_libsvm(const char *path, int32_t scale256, int32_t threads, float **labels,
                             float **X, int64_t *n, int64_t *d, int64_t *nnz, int64_t *bad_line);
void tsvm_free(void *p);

/* Model file writer (replaces writemodel, tensorsvm-train.cu:273-417), byte-identical text:
 * RBF: LIBSVM c_svc header and one "y_j alpha_j idx:val ..." line per SV (alpha_j > 1e-6),
 * values "%7f", zero features omitted, nr_sv = (free, bounded), rho = -b;  LINEAR: LIBLINEAR
 * header, w = sum_SV alpha_j y_j x_j (%.16f per line) and b.  X, y (+-1), alpha host; the SV
 * lines are formatted by `threads` threads (0: one per core).  n_sv, n_free may be NULL. */
tsvm_status tsvm_write_model(const char *path, int32_t kernel, const float *X, const float *y,
                             const double *alpha, int64_t n, int32_t d, double C, double gamma,
                             double b, int32_t pos, int32_t neg, int32_t threads, int64_t *n_sv,
                             int64_t *n_free);

/* Model file reader (either format above; LIBSVM RBF files written by other tools too): fills
 * *model with host arrays allocated here (release with tsvm_free_model) and the two labels
 * (f > 0 predicts label_pos).  For RBF models d is the largest feature index in the SV
 * section; pad rows and SVs to a common d before predicting. */
tsvm_status tsvm_read_model(const char *path, tsvm_model_view *model, int32_t *label_pos,
                            int32_t *label_neg);
void tsvm_free_model(tsvm_model_view *model);

/* Number of tensorsvm kernels this library launched since the context was created. */
int64_t tsvm_kernel_launches(const tsvm_context *ctx);

#ifdef __cplusplus
}
#endif
#endif /* TENSORSVM_H */
