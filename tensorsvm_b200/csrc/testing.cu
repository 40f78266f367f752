// Test hooks (include/tensorsvm_testing.h): thin wrappers that run one internal routine and
// synchronise, so parity tests can check kernels in isolation.
#include "common.cuh"
#include "context.h"
#include "kernels.h"
#include "tensorsvm_testing.h"

#include <vector>

using namespace tsvm;

namespace {

// Every block arrives once at a grid barrier that expects `arrivals` blocks and records whether
// it was released.  With arrivals > gridDim.x the last arrival never comes: each block gives up
// after max_spins polls, sets the barrier's error flag and returns (the bounded wait of the
// cooperative eigensolver, made to run out).
__global__ void barrier_probe(GridBarrier *gb, unsigned int arrivals, long long max_spins,
                              int *released) {
  const bool ok = grid_sync(gb, arrivals, max_spins);
  if (threadIdx.x == 0) released[blockIdx.x] = ok ? 1 : 0;
}

}  // namespace

extern "C" {

tsvm_status tsvm_test_rand_stream(tsvm_context *ctx, int64_t count, uint32_t *out) {
  if (!ctx || !out || count < 0) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_TRY(glibc_rand_stream(ctx, count, out));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_sketch(tsvm_context *ctx, int64_t count, float *out) {
  if (!ctx || !out || count < 0) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_TRY(sketch_glibc(ctx, count, out));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_sketch_philox(tsvm_context *ctx, uint64_t seed, int64_t count, float *out) {
  if (!ctx || !out || count < 0) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_TRY(sketch_philox(ctx, seed, count, out));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_kprod(tsvm_context *ctx, const float *A, int64_t na, const float *B,
                            int64_t nb, int32_t d, double gamma, const double *U, int32_t nu,
                            double *out, int32_t deriv, int32_t tensor_cores) {
  if (!ctx || !A || !B || !U || !out || na < 1 || nb < 1 || d < 1 || nu < 1 || nu > 64)
    return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_TRY(kprod_any(ctx, A, na, B, nb, d, gamma, U, nu, out, deriv != 0, tensor_cores != 0));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_kermatmul(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                int32_t d, double gamma, const float *A, int32_t kp, float *W,
                                int32_t precision, int32_t split) {
  return tsvm_test_kermatmul_cols(ctx, X, y, n, d, gamma, A, kp, 0, W, precision, split);
}

tsvm_status tsvm_test_kermatmul_cols(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                     int32_t d, double gamma, const float *A, int32_t kp,
                                     int32_t kw, float *W, int32_t precision, int32_t split) {
  if (!ctx || !X || !y || !A || !W || n < 1 || d < 1 || kp < 1) return TSVM_ERR_INVALID_ARGUMENT;
  if (kw < 0 || kw > kp) return TSVM_ERR_INVALID_ARGUMENT;
  if (!precision_valid(precision) || split < 0 || split > 2) return TSVM_ERR_INVALID_ARGUMENT;
  float *Xc = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_XC, (size_t)n * d + (size_t)n + 64, &Xc));
  float *norms = Xc + (size_t)n * d;
  TSVM_TRY(centre_features(ctx, X, n, d, Xc, norms));
  float ms = 0.f;
  if (precision == TSVM_PREC_FP32) {
    TSVM_TRY(kermatmul_fp32(ctx, Xc, norms, y, n, d, gamma, A, kp, W));
  } else {
    if (!kermatmul_tc_supported(d, kp)) return TSVM_ERR_UNSUPPORTED;
    TSVM_TRY(kermatmul_tc(ctx, Xc, norms, y, n, d, gamma, A, kp, W, precision, &ms, nullptr,
                          split, 0, -1, kw));
  }
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_kermatmul_half(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                     int32_t d, double gamma, const float *A, int32_t kp,
                                     float *R, double *sym, int32_t precision, int32_t split) {
  return tsvm_test_kermatmul_half_cols(ctx, X, y, n, d, gamma, A, kp, 0, R, sym, precision,
                                       split);
}

tsvm_status tsvm_test_kermatmul_half_cols(tsvm_context *ctx, const float *X, const float *y,
                                          int64_t n, int32_t d, double gamma, const float *A,
                                          int32_t kp, int32_t kw, float *R, double *sym,
                                          int32_t precision, int32_t split) {
  if (!ctx || !X || !y || !A || !R || !sym || n < 1 || d < 1 || kp < 1 || kw < 0 || kw > kp)
    return TSVM_ERR_INVALID_ARGUMENT;
  if (!precision_valid(precision) || precision == TSVM_PREC_FP32 || split < 0 || split > 2)
    return TSVM_ERR_INVALID_ARGUMENT;
  if (!kermatmul_tc_supported(d, kp)) return TSVM_ERR_UNSUPPORTED;
  float *Xc = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_XC, (size_t)n * d + (size_t)n + 64, &Xc));
  float *norms = Xc + (size_t)n * d;
  TSVM_TRY(centre_features(ctx, X, n, d, Xc, norms));
  float ms = 0.f;
  TSVM_TRY(kermatmul_tc_half(ctx, Xc, y, n, d, gamma, A, kp, R, precision, &ms, nullptr, split,
                             sym, false, kw));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_chol(tsvm_context *ctx, double *A, int32_t n, int32_t *info_host) {
  if (!ctx || !A || n < 1) return TSVM_ERR_INVALID_ARGUMENT;
  int *info = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, 16, &info));
  double *Dinv = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL2, (size_t)ceil_div(n, 32) * 1024, &Dinv));
  TSVM_TRY(chol_fp64(ctx, A, n, n, info, Dinv));
  int h = 0;
  TSVM_CUDA(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (info_host) *info_host = h;
  return TSVM_OK;
}

tsvm_status tsvm_test_potrs(tsvm_context *ctx, const double *L, int32_t n, double *B,
                            int32_t nrhs, int32_t ldb) {
  if (!ctx || !L || !B || n < 1 || ldb < n) return TSVM_ERR_INVALID_ARGUMENT;
  double *Dinv = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL2, (size_t)ceil_div(n, 32) * 1024, &Dinv));
  TSVM_TRY(tri_diag_inverse(ctx, L, n, n, Dinv));
  TSVM_TRY(potrs_fp64(ctx, L, n, n, Dinv, B, nrhs, ldb));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_eig(tsvm_context *ctx, double *A, int32_t n, double *w, double *V,
                          int32_t *sweeps_host) {
  if (!ctx || !A || !w || !V || n < 1) return TSVM_ERR_INVALID_ARGUMENT;
  int sweeps = 0;
  tsvm_status st = eig_jacobi_fp64(ctx, A, n, n, w, V, &sweeps);
  if (sweeps_host) *sweeps_host = sweeps;
  return st;
}

tsvm_status tsvm_test_eig_batched(tsvm_context *ctx, double *A, int32_t n, int32_t count,
                                  double *w, double *V, int32_t *max_sweeps_host) {
  if (!ctx || !A || !w || !V || n < 1 || count < 1) return TSVM_ERR_INVALID_ARGUMENT;
  int sweeps = 0;
  tsvm_status st = eig_jacobi_fp64_batched(ctx, A, n, count, w, V, &sweeps);
  if (max_sweeps_host) *max_sweeps_host = sweeps;
  return st;
}

tsvm_status tsvm_test_gram(tsvm_context *ctx, const float *A, int64_t lda, const float *B,
                           int64_t ldb, int64_t n, int32_t ka, int32_t kb, int32_t symmetric,
                           const double *s, double *G) {
  if (!ctx || !A || !B || !G || n < 1) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_TRY(gram_fp64(ctx, A, lda, B, ldb, n, ka, kb, symmetric != 0, G, s));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_test_syrk_mixed(tsvm_context *ctx, const float *Z, int32_t ldz, int64_t n,
                                 int32_t k, const double *dinv, double tau, int32_t ways,
                                 double *M, int32_t *exact_rows) {
  if (!ctx || !Z || !dinv || !M || n < 1 || k < 1 || ldz < k) return TSVM_ERR_INVALID_ARGUMENT;
  int64_t *idx = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_IDX, (size_t)n + 8, &idx));
  int *cnt = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, 16, &cnt));
  double *G64 = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, (size_t)k * k, &G64));
  TSVM_TRY(big_rows(ctx, dinv, n, tau, idx, cnt));
  TSVM_TRY(gram_fp64_rows(ctx, Z, ldz, n, k, idx, cnt, dinv, G64));
  TSVM_TRY(syrk_capacitance_tc(ctx, Z, ldz, n, k, dinv, tau, ways, G64, M));
  int h = 0;
  TSVM_CUDA(cudaMemcpyAsync(&h, cnt, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (exact_rows) *exact_rows = h;
  return TSVM_OK;
}

tsvm_status tsvm_test_fail_alloc(tsvm_context *ctx, int32_t after) {
  if (!ctx || after < -1) return TSVM_ERR_INVALID_ARGUMENT;
  ctx->alloc_fail_after = after;
  return TSVM_OK;
}

tsvm_status tsvm_test_grid_barrier(tsvm_context *ctx, int32_t blocks, int32_t arrivals,
                                   int64_t max_spins, int32_t *released_blocks) {
  if (!ctx || blocks < 1 || blocks > ctx->num_sms || arrivals < 1 || max_spins < 1 ||
      max_spins > (1ll << 24))
    return TSVM_ERR_INVALID_ARGUMENT;
  int *buf = nullptr;   // GridBarrier (4 ints) | released[blocks]
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, (size_t)blocks + 4, &buf));
  TSVM_CUDA(cudaMemsetAsync(buf, 0, sizeof(int) * ((size_t)blocks + 4), ctx->stream));
  GridBarrier *gb = reinterpret_cast<GridBarrier *>(buf);
  int *released = buf + 4;
  unsigned int arr = (unsigned int)arrivals;
  long long spins = max_spins;
  void *args[] = {&gb, &arr, &spins, &released};
  TSVM_CUDA(cudaLaunchCooperativeKernel((const void *)barrier_probe, dim3((unsigned)blocks),
                                        dim3(64), args, 0, ctx->stream));
  TSVM_LAUNCHED(ctx);
  std::vector<int> h((size_t)blocks + 4);
  TSVM_CUDA(cudaMemcpyAsync(h.data(), buf, sizeof(int) * h.size(), cudaMemcpyDeviceToHost,
                            ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  int n = 0;
  for (int b = 0; b < blocks; ++b) n += h[4 + b];
  if (released_blocks) *released_blocks = n;
  return h[2] ? TSVM_ERR_TIMEOUT : TSVM_OK;   // GridBarrier::error
}

}  // extern "C"
