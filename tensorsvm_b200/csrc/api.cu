// C ABI of the library (include/tensorsvm.h): context management, argument checking and the
// end-to-end train call.  All compute lives in the other .cu files.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"
#include "trace.h"

namespace tsvm {

tsvm_status cuda_status(cudaError_t e, const char *what, const char *file, int line) {
  if (getenv("TSVM_DEBUG"))
    fprintf(stderr, "tensorsvm: CUDA error %s (%s) at %s:%d\n", cudaGetErrorString(e), what, file,
            line);
  if (e == cudaErrorMemoryAllocation) return TSVM_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) return TSVM_ERR_NO_DEVICE;
  return TSVM_ERR_CUDA;
}

tsvm_status timeout_status(const char *where) {
  if (getenv("TSVM_DEBUG")) fprintf(stderr, "tensorsvm: bounded device wait timed out in %s\n", where);
  return TSVM_ERR_TIMEOUT;
}

tsvm_status scratch(tsvm_context *ctx, Slot s, size_t bytes, void **out) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (bytes == 0) bytes = 256;
  if (ctx->bytes[s] < bytes) {
    if (ctx->buf[s]) {
      TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
      TSVM_CUDA(cudaFree(ctx->buf[s]));
      ctx->buf[s] = nullptr;
      ctx->bytes[s] = 0;
    }
    // test hook (tsvm_test_fail_alloc): the allocation after the next `alloc_fail_after` fails
    if (ctx->alloc_fail_after >= 0 && ctx->alloc_fail_after-- == 0) return TSVM_ERR_OUT_OF_MEMORY;
    void *p = nullptr;
    TSVM_CUDA(cudaMalloc(&p, bytes));
    ctx->buf[s] = p;
    ctx->bytes[s] = bytes;
  }
  *out = ctx->buf[s];
  return TSVM_OK;
}

tsvm_status comm_allreduce(tsvm_context *ctx, void *buf, int64_t count, int dtype, int op) {
  if (!ctx->has_comm || ctx->comm.world <= 1 || count <= 0) return TSVM_OK;
  const int rc = ctx->comm.allreduce(ctx->comm.user, buf, count, dtype, op, ctx->stream);
  return rc == 0 ? TSVM_OK : TSVM_ERR_COMM;
}

tsvm_status comm_sum_host(tsvm_context *ctx, double *value) {
  if (!sharded(ctx)) return TSVM_OK;
  double *d = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_COMM, 8, &d));
  TSVM_CUDA(cudaMemcpyAsync(d, value, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  TSVM_TRY(comm_allreduce(ctx, d, 1, 0, COMM_SUM));
  TSVM_CUDA(cudaMemcpyAsync(value, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

float event_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}
}  // namespace tsvm

using namespace tsvm;

extern "C" {

const char *tsvm_status_string(tsvm_status s) {
  switch (s) {
    case TSVM_OK: return "ok";
    case TSVM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TSVM_ERR_CUDA: return "CUDA error";
    case TSVM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case TSVM_ERR_NOT_SPD: return "capacitance matrix not positive definite (Cholesky failed)";
    case TSVM_ERR_UNSUPPORTED: return "unsupported shape or precision";
    case TSVM_ERR_NO_DEVICE: return "no CUDA device";
    case TSVM_ERR_TIMEOUT: return "bounded device wait timed out";
    case TSVM_WARN_ILL_CONDITIONED: return "stopped: max/min(D) > 1e18";
    case TSVM_WARN_MAX_ITER: return "stopped: iteration limit reached";
    case TSVM_ERR_SKETCH: return "sketch stream exhausted";
    case TSVM_ERR_IO: return "I/O error";
    case TSVM_ERR_COMM: return "collective of the row-sharded path failed";
  }
  return "unknown status";
}

tsvm_status tsvm_create(tsvm_context **out, int device) {
  if (!out) return TSVM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return TSVM_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(device));
  tsvm_context *ctx = new tsvm_context();
  ctx->device = device;
  cudaError_t e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  ctx->stream = ctx->own_stream;
  for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = cudaEventCreate(&ctx->ev[i]);
  if (e == cudaSuccess) {
    int lo = 0, hi = 0;
    e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, hi);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->host_scalars, 4096);
  if (e != cudaSuccess) {
    tsvm_destroy(ctx);
    return cuda_status(e, "tsvm_create", __FILE__, __LINE__);
  }
  *out = ctx;
  return TSVM_OK;
}

tsvm_status tsvm_destroy(tsvm_context *ctx) {
  if (!ctx) return TSVM_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->side_stream) cudaStreamSynchronize(ctx->side_stream);
  for (int i = 0; i < SLOT_COUNT_; ++i)
    if (ctx->buf[i]) cudaFree(ctx->buf[i]);
  for (int i = 0; i < 8; ++i)
    if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->host_scalars) cudaFreeHost(ctx->host_scalars);
  if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return TSVM_OK;
}

tsvm_status tsvm_set_stream(tsvm_context *ctx, void *stream) {
  if (!ctx) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return TSVM_OK;
}

tsvm_status tsvm_set_comm(tsvm_context *ctx, const tsvm_comm *comm) {
  if (!ctx) return TSVM_ERR_INVALID_ARGUMENT;
  if (!comm) {
    ctx->has_comm = false;
    ctx->comm = tsvm_comm{};
    return TSVM_OK;
  }
  if (comm->world < 1 || comm->rank < 0 || comm->rank >= comm->world ||
      (comm->world > 1 && !comm->allreduce))
    return TSVM_ERR_INVALID_ARGUMENT;
  ctx->comm = *comm;
  ctx->has_comm = true;
  return TSVM_OK;
}

tsvm_status tsvm_set_factor_keep(tsvm_context *ctx, int32_t keep) {
  if (!ctx || keep < 0 || keep > 1) return TSVM_ERR_INVALID_ARGUMENT;
  ctx->keep_factor = keep;
  return TSVM_OK;
}

tsvm_status tsvm_set_sketch_seed(tsvm_context *ctx, uint64_t seed) {
  if (!ctx) return TSVM_ERR_INVALID_ARGUMENT;
  ctx->sketch_seed = seed;
  return TSVM_OK;
}

void tsvm_ipm_default_options(tsvm_ipm_options *opt) {
  if (!opt) return;
  opt->max_iter = 100;
  opt->tol = 1e-7;
  opt->rel_gap_tol = 0.0;
  opt->precision = TSVM_PREC_FP32;
  opt->refine_sweeps = 1;
  opt->kernel = TSVM_KERNEL_RBF;
  opt->verbose = 0;
}

int64_t tsvm_kernel_launches(const tsvm_context *ctx) { return ctx ? ctx->launches : 0; }

tsvm_status tsvm_factor(tsvm_context *ctx, const float *X, const float *y, int64_t n, int32_t d,
                        double gamma, int32_t k, int32_t precision, int32_t sketch,
                        const float *Q_user, float *Z, int32_t ldz, tsvm_factor_info *info) {
  if (!ctx || !X || !y || !Z) return TSVM_ERR_INVALID_ARGUMENT;
  if (!precision_valid(precision)) return TSVM_ERR_INVALID_ARGUMENT;
  if (sharded(ctx)) return TSVM_ERR_UNSUPPORTED;   // row-sharded: tsvm_factor_rows
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_factor");
  if (ctx->keep_factor && sketch == TSVM_SKETCH_GLIBC && k >= 1 && n >= 2 && ldz >= k)
    return factor_rbf_keep(ctx, X, y, n, d, gamma, k, precision, Z, ldz, info);
  return factor_rbf(ctx, X, y, n, d, gamma, k, precision, sketch, Q_user, Z, ldz, info);
}

tsvm_status tsvm_factor_rows(tsvm_context *ctx, const float *X, const float *y, int64_t n_global,
                             int32_t d, int64_t row0, int64_t n_rows, double gamma, int32_t k,
                             int32_t precision, int32_t sketch, const float *Q_user, float *Z,
                             int32_t ldz, tsvm_factor_info *info) {
  if (!ctx || !X || !y || !Z) return TSVM_ERR_INVALID_ARGUMENT;
  if (!precision_valid(precision)) return TSVM_ERR_INVALID_ARGUMENT;
  if (row0 < 0 || n_rows < 1 || row0 + n_rows > n_global) return TSVM_ERR_INVALID_ARGUMENT;
  if ((row0 != 0 || n_rows != n_global) && !sharded(ctx)) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_factor_rows");
  return factor_rbf(ctx, X, y, n_global, d, gamma, k, precision, sketch, Q_user, Z, ldz, info,
                    nullptr, row0, n_rows);
}

tsvm_status tsvm_factor_batched(tsvm_context *ctx, const tsvm_factor_problem *problems,
                                int32_t count, int32_t d, int32_t k, int32_t precision,
                                int32_t sketch, int32_t ldz, tsvm_factor_info *infos) {
  if (!ctx || !problems || count < 1 || d < 1 || k < 1) return TSVM_ERR_INVALID_ARGUMENT;
  if (!precision_valid(precision) || (sketch != TSVM_SKETCH_GLIBC && sketch != TSVM_SKETCH_PHILOX))
    return TSVM_ERR_INVALID_ARGUMENT;
  for (int p = 0; p < count; ++p)
    if (!problems[p].X || !problems[p].y || !problems[p].Z || problems[p].n < 2)
      return TSVM_ERR_INVALID_ARGUMENT;
  if (sharded(ctx)) return TSVM_ERR_UNSUPPORTED;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_factor_batched");
  return factor_rbf_batched(ctx, problems, count, d, k, precision, sketch, ldz, infos, nullptr);
}

tsvm_status tsvm_linear_factor(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                               int32_t d, float *Z, int32_t ldz) {
  if (!ctx || !X || !y || !Z || n < 1 || d < 1 || ldz < d) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TSVM_TRY(label_rows(ctx, X, y, n, d, Z, ldz));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_ipm(tsvm_context *ctx, const float *Z, int32_t ldz, const float *y, int64_t n,
                     int32_t k, double C, const tsvm_ipm_options *opt, double *alpha_out,
                     double *xi_out, double *s_out, double *ymult_out,
                     tsvm_ipm_stats *stats) {
  if (!ctx || !Z || !y || !alpha_out || n < 2 || k < 1 || ldz < k || !(C > 0))
    return TSVM_ERR_INVALID_ARGUMENT;
  if ((ldz % 4) != 0 || (reinterpret_cast<uintptr_t>(Z) & 15) != 0) return TSVM_ERR_INVALID_ARGUMENT;
  tsvm_ipm_options o;
  tsvm_ipm_default_options(&o);
  if (opt) o = *opt;
  if (o.max_iter < 0 || !(o.tol > 0)) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_ipm");
  return ipm_solve(ctx, Z, ldz, y, n, k, C, o, alpha_out, xi_out, s_out, ymult_out, stats);
}

tsvm_status tsvm_ipm_batched(tsvm_context *ctx, const tsvm_ipm_problem *problems, int32_t count,
                             int32_t k, int32_t ldz, const tsvm_ipm_options *opt,
                             tsvm_ipm_stats *stats, tsvm_batch_info *info) {
  if (!ctx || !problems || count < 1 || k < 1 || ldz < k || (ldz % 4) != 0)
    return TSVM_ERR_INVALID_ARGUMENT;
  if (sharded(ctx)) return TSVM_ERR_UNSUPPORTED;   // problems are partitioned, not sharded
  for (int32_t p = 0; p < count; ++p) {
    const tsvm_ipm_problem &q = problems[p];
    if (!q.Z || !q.y || !q.alpha_out || q.n < 2 || !(q.C > 0) ||
        (reinterpret_cast<uintptr_t>(q.Z) & 15) != 0)
      return TSVM_ERR_INVALID_ARGUMENT;
  }
  tsvm_ipm_options o;
  tsvm_ipm_default_options(&o);
  if (opt) o = *opt;
  if (o.max_iter < 0 || !(o.tol > 0)) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_ipm_batched");
  return ipm_solve_batched(ctx, problems, count, k, ldz, o, stats, info);
}

tsvm_status tsvm_bias(tsvm_context *ctx, const float *Z, int32_t ldz, const float *y,
                      const double *alpha, int64_t n, int32_t k, double C, double *b_out,
                      double *b_std_out, int32_t *n_sv, int32_t *n_free) {
  if (!ctx || !Z || !y || !alpha || n < 1 || k < 1 || ldz < k) return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_bias");
  return bias_rbf(ctx, Z, ldz, y, alpha, n, k, C, b_out, b_std_out, n_sv, n_free);
}

tsvm_status tsvm_train(tsvm_context *ctx, const float *X, const float *y, int64_t n, int32_t d,
                       int32_t kernel, double gamma, double C, int32_t k, int32_t precision,
                       const tsvm_ipm_options *opt, double *alpha_out, double *b_out,
                       tsvm_factor_info *finfo, tsvm_ipm_stats *istats) {
  if (ctx && sharded(ctx)) return TSVM_ERR_UNSUPPORTED;   // row-sharded: factor_rows + ipm
  if (!ctx || !X || !y || !alpha_out || n < 2 || d < 1) return TSVM_ERR_INVALID_ARGUMENT;
  if (kernel != TSVM_KERNEL_LINEAR && kernel != TSVM_KERNEL_RBF) return TSVM_ERR_UNSUPPORTED;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_train");
  tsvm_ipm_options o;
  tsvm_ipm_default_options(&o);
  if (opt) o = *opt;
  o.kernel = kernel;
  float *dX = nullptr, *dZ = nullptr;
  double *dalpha = nullptr;
  ctx->last_train.valid = false;
  TSVM_TRY(scratch_t(ctx, SLOT_DEV_IN, (size_t)n * d + (size_t)n + 64, &dX));
  float *dy = dX + (size_t)n * d;
  TSVM_CUDA(cudaMemcpyAsync(dX, X, sizeof(float) * n * d, cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  TSVM_TRY(scratch_t(ctx, SLOT_DEV_OUT, (size_t)n, &dalpha));
  tsvm_status st;
  if (kernel == TSVM_KERNEL_RBF) {
    const int kp = (int)round_up(k, 64);
    TSVM_TRY(scratch_t(ctx, SLOT_DEV_Z, (size_t)n * kp, &dZ));
    TSVM_TRY(factor_rbf(ctx, dX, dy, n, d, gamma, k, precision, TSVM_SKETCH_GLIBC, nullptr, dZ, kp,
                        finfo));
    st = ipm_solve(ctx, dZ, kp, dy, n, k, C, o, dalpha, nullptr, nullptr, nullptr, istats);
    if (st != TSVM_OK && st != TSVM_WARN_ILL_CONDITIONED && st != TSVM_WARN_MAX_ITER &&
        st != TSVM_ERR_NOT_SPD)
      return st;
    double b = 0.0;
    TSVM_TRY(bias_rbf(ctx, dZ, kp, dy, dalpha, n, k, C, &b, nullptr, nullptr, nullptr));
    ctx->last_train.valid = true;
    ctx->last_train.n = n;
    ctx->last_train.d = d;
    ctx->last_train.k = k;
    ctx->last_train.ldz = kp;
    ctx->last_train.gamma = gamma;
    if (b_out) *b_out = b;
    TSVM_CUDA(cudaMemcpyAsync(alpha_out, dalpha, sizeof(double) * n, cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  } else {
    const int ldz = (int)round_up(d, 4);
    TSVM_TRY(scratch_t(ctx, SLOT_DEV_Z, (size_t)n * ldz, &dZ));
    TSVM_TRY(label_rows(ctx, dX, dy, n, d, dZ, ldz));
    st = ipm_solve(ctx, dZ, ldz, dy, n, d, C, o, dalpha, nullptr, nullptr, nullptr, istats);
    if (st != TSVM_OK && st != TSVM_WARN_ILL_CONDITIONED && st != TSVM_WARN_MAX_ITER &&
        st != TSVM_ERR_NOT_SPD)
      return st;
    if (b_out) TSVM_TRY(linear_bias(ctx, dX, dy, dalpha, n, d, C, b_out));
    TSVM_CUDA(cudaMemcpyAsync(alpha_out, dalpha, sizeof(double) * n, cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return st;
}

tsvm_status tsvm_decision_values(tsvm_context *ctx, const tsvm_model_view *model, const float *X,
                                 int64_t m, double *f) {
  if (!ctx || !model || !X || !f || m < 0 || model->d < 1 || !model->sv)
    return TSVM_ERR_INVALID_ARGUMENT;
  if (model->kernel != TSVM_KERNEL_RBF && model->kernel != TSVM_KERNEL_LINEAR)
    return TSVM_ERR_UNSUPPORTED;
  if (model->kernel == TSVM_KERNEL_RBF && (model->nsv < 0 || (model->nsv > 0 && !model->coef)))
    return TSVM_ERR_INVALID_ARGUMENT;
  if (m == 0) return TSVM_OK;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange tr("tsvm_decision_values");
  TSVM_TRY(decision_values(ctx, model, X, m, f));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_predict(tsvm_context *ctx, const tsvm_model_view *model, const float *X,
                         int64_t m, double *f) {
  if (!ctx || !model || !X || !f || m < 0 || model->d < 1 || !model->sv)
    return TSVM_ERR_INVALID_ARGUMENT;
  if (model->kernel != TSVM_KERNEL_RBF && model->kernel != TSVM_KERNEL_LINEAR)
    return TSVM_ERR_UNSUPPORTED;
  const bool rbf = model->kernel == TSVM_KERNEL_RBF;
  if (rbf && (model->nsv < 0 || (model->nsv > 0 && !model->coef))) return TSVM_ERR_INVALID_ARGUMENT;
  if (m == 0) return TSVM_OK;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  const int64_t d = model->d;
  const int64_t nsv = rbf ? model->nsv : 0;
  const size_t sv_floats = rbf ? (size_t)(nsv * d) : (size_t)d;
  // layout: coef (nsv doubles) | sv floats | X floats, each 256-byte aligned
  const size_t o_sv = round_up((int64_t)nsv * 8, 256);
  const size_t o_x = o_sv + round_up((int64_t)sv_floats * 4, 256);
  const size_t bytes = o_x + (size_t)m * d * 4 + 256;
  uint8_t *buf = nullptr;
  double *df = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_PRED_IN, bytes, &buf));
  TSVM_TRY(scratch_t(ctx, SLOT_PRED_OUT, (size_t)m, &df));
  double *dcoef = reinterpret_cast<double *>(buf);
  float *dsv = reinterpret_cast<float *>(buf + o_sv);
  float *dX = reinterpret_cast<float *>(buf + o_x);
  if (nsv > 0)
    TSVM_CUDA(cudaMemcpyAsync(dcoef, model->coef, sizeof(double) * nsv, cudaMemcpyHostToDevice,
                              ctx->stream));
  if (sv_floats > 0)
    TSVM_CUDA(cudaMemcpyAsync(dsv, model->sv, sizeof(float) * sv_floats, cudaMemcpyHostToDevice,
                              ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(dX, X, sizeof(float) * m * d, cudaMemcpyHostToDevice, ctx->stream));
  tsvm_model_view dv = *model;
  dv.sv = dsv;
  dv.coef = rbf ? dcoef : nullptr;
  dv.nsv = nsv;
  TSVM_TRY(decision_values(ctx, &dv, dX, m, df));
  TSVM_CUDA(cudaMemcpyAsync(f, df, sizeof(double) * m, cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

tsvm_status tsvm_kernel_residual(tsvm_context *ctx, const float *X, const float *y, int64_t n,
                                 int32_t d, double gamma, const float *Z, int32_t ldz, int32_t k,
                                 double *fnorm, double *fnorm_res) {
  if (!ctx || !X || !y || !Z || n < 1 || d < 1 || k < 1 || ldz < k || !(gamma > 0))
    return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  double out[2];
  TSVM_TRY(kernel_residual(ctx, X, y, n, d, gamma, Z, ldz, k, out));
  if (fnorm) *fnorm = out[0];
  if (fnorm_res) *fnorm_res = out[1];
  return TSVM_OK;
}

tsvm_status tsvm_train_residual(tsvm_context *ctx, double *fnorm, double *fnorm_res) {
  if (!ctx || !ctx->last_train.valid) return TSVM_ERR_INVALID_ARGUMENT;
  const auto &t = ctx->last_train;
  const float *dX = static_cast<const float *>(ctx->buf[SLOT_DEV_IN]);
  const float *dZ = static_cast<const float *>(ctx->buf[SLOT_DEV_Z]);
  if (!dX || !dZ) return TSVM_ERR_INVALID_ARGUMENT;
  return tsvm_kernel_residual(ctx, dX, dX + (size_t)t.n * t.d, t.n, t.d, t.gamma, dZ, t.ldz, t.k,
                              fnorm, fnorm_res);
}

}  // extern "C"
