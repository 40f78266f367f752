// Kernel factor Z with Z Z^T ~= Y K Y (replaces LRA, tensorsvm-train.cu:1941-2374).
//
// Same method as the reference, with every step on the device and every matrix resident:
//   sketch Q = gaussrand stream               (T:1966-1974)       sketch.cu
//   W = (Y K Y) Q                              (T:2067)            kermatmul_{simt,tc}.cu
//   W = orth(W)                                (T:2075, TSQR)      shifted CholeskyQR3 here
//   Q = (Y K Y) W                              (T:2085)
//   C = W^T Q, symmetrised                     (T:2122-2160)       gram_fp64 + symmetrize
//   C = V diag(w) V^T, X = V diag(sqrt(w+))   (T:2179-2211)       Jacobi eigensolver
//   Z = W X                                    (T:2213-2241)       apply_right_fp32
// The orthonormalisation is shifted CholeskyQR3 (Fukaya et al., SIAM J. Sci. Comput. 2020):
// G = W^T W accumulated exactly in FP64, G + s I with s = 11 (n k + k (k+1)) u ||W||_F^2,
// then two unshifted CholeskyQR steps.  Only range(W) matters for Z Z^T = W C+ W^T, so any
// orthonormal basis of the same range gives the reference's factor.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"
#include "trace.h"

namespace tsvm {
namespace {

// C <- C + C^T + s u u^T with s = sym[0], u = sym[1..k]: the projection W^T K W from the half
// product's C = W^T R (pairs i <= j, one thread each)
__global__ void half_projection_finish(double *C, int k, const double *__restrict__ sym) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)k * k) return;
  const int i = (int)(e / k), j = (int)(e % k);
  if (i > j) return;
  const double v = C[(int64_t)i * k + j] + C[(int64_t)j * k + i] + sym[0] * sym[1 + i] * sym[1 + j];
  C[(int64_t)i * k + j] = v;
  C[(int64_t)j * k + i] = v;
}

// G[i][i] += factor * trace(G)   (one block)
__global__ void shift_by_trace(double *G, int k, double factor) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < k; i += blockDim.x) s += G[(int64_t)i * k + i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    sh[0] = t;
  }
  __syncthreads();
  const double shift = factor * sh[0];
  for (int i = threadIdx.x; i < k; i += blockDim.x) G[(int64_t)i * k + i] += shift;
}

// R32 (kp x kp fp32) = Linv^T padded with zeros: W R32 = W L^-T.
__global__ void rinv_to_fp32(const double *__restrict__ Linv, int k, int kp,
                             float *__restrict__ R32) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)kp * kp) return;
  const int m = (int)(e / kp), c = (int)(e % kp);
  R32[e] = (m < k && c < k) ? (float)Linv[(int64_t)c * k + m] : 0.f;
}

// X32 (kp x kp fp32) = V diag(sqrt(max(w, 0))) padded with zeros (T:2199-2210).
__global__ void eigfactor_to_fp32(const double *__restrict__ V, const double *__restrict__ w,
                                  int k, int kp, float *__restrict__ X32) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)kp * kp) return;
  const int m = (int)(e / kp), c = (int)(e % kp);
  float v = 0.f;
  if (m < k && c < k) {
    const double wc = w[c];
    v = wc > 0.0 ? (float)(V[(int64_t)m * k + c] * sqrt(wc)) : 0.f;
  }
  X32[e] = v;
}

// Rout = L^T Rin for L lower (k x k, only its lower triangle read) and Rin upper: the combined
// CholeskyQR factor after one more step (W_new = W L^-T, so B = W_new (L^T R)).
__global__ void accumulate_r(const double *__restrict__ L, int k, const double *__restrict__ Rin,
                             double *__restrict__ Rout) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)k * k) return;
  const int i = (int)(e / k), j = (int)(e % k);
  double s = 0.0;
  for (int m = i; m <= j; ++m) s += L[(int64_t)m * k + i] * Rin[(int64_t)m * k + j];
  Rout[e] = s;
}

__global__ void fill_value(double *v, int64_t n, double value) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = value;
}

__global__ void set_scaled_identity(double *A, int k, double value) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (int64_t)k * k) A[e] = (e / k == e % k) ? value : 0.0;
}

__global__ void set_identity(double *R, int k) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (int64_t)k * k) R[e] = (e / k == e % k) ? 1.0 : 0.0;
}

struct Phase {
  tsvm_context *ctx;
  cudaEvent_t a, b;
};

}  // namespace

// round_back, split, row range: see kermatmul_tc (the FP32 form ignores round_back and split:
// its operand is not rounded).
static tsvm_status kermatmul(tsvm_context *ctx, const float *Xc, const float *norms,
                             const float *y, int64_t n, int d, double gamma, const float *A,
                             int kp, float *W, int precision, float *kernel_ms,
                             float *round_back, int split, int64_t row0, int64_t nr, int kw) {
  if (precision == TSVM_PREC_FP32)
    return kermatmul_fp32(ctx, Xc, norms, y, n, d, gamma, A, kp, W, row0, nr);
  if (!kermatmul_tc_supported(d, kp)) return TSVM_ERR_UNSUPPORTED;
  return kermatmul_tc(ctx, Xc, norms, y, n, d, gamma, A, kp, W, precision, kernel_ms, round_back,
                      split, row0, nr, kw);
}

// Rkeep (2 k x k doubles, may be null): the combined factor R with (input W) = (output W) R.
// tc_gram: steps 2 and 3 (W already near-orthonormal after the shifted first step) take their
// Gram matrix from the tensor-core SYRK with a 3-way BF16 split (about FP32 accuracy, the
// precision W is stored in) instead of the exact FP64 sum; the first, ill-conditioned step
// always uses the exact FP64 Gram.
// n_total: rows of the whole problem (this rank's W holds n of them when row-sharded: the Gram
// matrices are then all-reduced, and W's rows are updated locally).
static tsvm_status orthonormalise(tsvm_context *ctx, float *W, int64_t n, int k, int kp,
                                  double *Rkeep, bool tc_gram, int64_t n_total) {
  double *G = nullptr, *Linv = nullptr;
  float *R32 = nullptr;
  int *info = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL, (size_t)k * k + 8, &G));
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL2, (size_t)k * k + (size_t)ceil_div(k, 32) * 1024, &Linv));
  double *Dinv = Linv + (size_t)k * k;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)kp * kp, &R32));
  info = reinterpret_cast<int *>(G + (size_t)k * k);
  const double u = ldexp(1.0, -53);
  const unsigned gk = (unsigned)ceil_div((int64_t)k * k, 256);
  if (Rkeep) {
    set_identity<<<gk, 256, 0, ctx->stream>>>(Rkeep, k);
    TSVM_LAUNCHED(ctx);
  }
  for (int step = 0; step < 3; ++step) {
    double factor = step == 0 ? 11.0 * ((double)n_total * k + (double)k * (k + 1)) * u : 0.0;
    for (int attempt = 0; attempt < 4; ++attempt) {
      if (tc_gram && step > 0 && attempt == 0) {
        // M = I + sum_j 1 * w_j w_j^T (every row on the tensor cores) plus the exact -I
        double *ones = nullptr, *negI = nullptr;
        TSVM_TRY(scratch_t(ctx, SLOT_IPM_VEC, (size_t)n, &ones));
        TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, (size_t)k * k, &negI));
        fill_value<<<(unsigned)ceil_div(n, 256), 256, 0, ctx->stream>>>(ones, n, 1.0);
        TSVM_LAUNCHED(ctx);
        set_scaled_identity<<<gk, 256, 0, ctx->stream>>>(negI, k, -1.0);
        TSVM_LAUNCHED(ctx);
        TSVM_TRY(syrk_capacitance_tc(ctx, W, kp, n, k, ones, 2.0, 3, negI, G));
      } else {
        TSVM_TRY(gram_fp64(ctx, W, kp, W, kp, n, k, k, true, G));
      }
      TSVM_TRY(comm_allreduce(ctx, G, (int64_t)k * k, 0, COMM_SUM));   // row-sharded
      if (factor > 0) {
        shift_by_trace<<<1, 256, 0, ctx->stream>>>(G, k, factor);
        TSVM_LAUNCHED(ctx);
      }
      TSVM_TRY(chol_fp64(ctx, G, k, k, info, Dinv));
      int hinfo = 0;
      TSVM_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
      if (hinfo == 0) break;
      if (attempt == 3) return TSVM_ERR_NOT_SPD;
      factor = factor > 0 ? factor * 100.0
                          : 11.0 * ((double)n_total * k + (double)k * (k + 1)) * u;
    }
    if (Rkeep) {
      double *Rtmp = Rkeep + (size_t)k * k;
      accumulate_r<<<gk, 256, 0, ctx->stream>>>(G, k, Rkeep, Rtmp);
      TSVM_LAUNCHED(ctx);
      TSVM_CUDA(cudaMemcpyAsync(Rkeep, Rtmp, sizeof(double) * k * k, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    }
    TSVM_TRY(trinv_lower_fp64(ctx, G, k, k, Dinv, Linv));
    rinv_to_fp32<<<(unsigned)ceil_div((int64_t)kp * kp, 256), 256, 0, ctx->stream>>>(Linv, k, kp,
                                                                                      R32);
    TSVM_LAUNCHED(ctx);
    TSVM_TRY(apply_right_fp32(ctx, W, n, kp, R32, W));
  }
  return TSVM_OK;
}

tsvm_status factor_rbf(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                       double gamma, int k, int precision, int sketch, const float *Q_user,
                       float *Z, int ldz, tsvm_factor_info *info, FactorKeep *keep, int64_t row0,
                       int64_t nr, double *C_out) {
  if (n < 2 || d < 1 || k < 1 || k > 1000 || ldz < k || !(gamma > 0)) return TSVM_ERR_INVALID_ARGUMENT;
  if (k > n) return TSVM_ERR_INVALID_ARGUMENT;
  if (nr < 0) nr = n - row0;
  if (row0 < 0 || nr < 1 || row0 + nr > n) return TSVM_ERR_INVALID_ARGUMENT;
  // row-sharded: this rank computes Z's rows [row0, row0 + nr) (W, the pass outputs and Z hold
  // nr rows; X, y and the pass operands all n)
  const bool rows = row0 != 0 || nr != n;
  if (rows && keep) return TSVM_ERR_UNSUPPORTED;
  if (C_out && (rows || keep || ldz != (int)round_up(k, 64))) return TSVM_ERR_UNSUPPORTED;
  const int kp = (int)round_up(k, 64);
  cudaEvent_t *ev = ctx->ev;
  TracePhases phase;
  phase.next("factor: sketch");
  TSVM_CUDA(cudaEventRecord(ev[0], ctx->stream));
  float *Xc = nullptr, *Q = nullptr, *W = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_XC, (size_t)n * d + (size_t)n + 64, &Xc));
  float *norms = Xc + (size_t)n * d;
  TSVM_TRY(centre_features(ctx, X, n, d, Xc, norms));
  TSVM_TRY(scratch_t(ctx, SLOT_Q, (size_t)n * kp, &Q));
  TSVM_TRY(scratch_t(ctx, SLOT_W, (size_t)nr * kp, &W));
  if (sketch == TSVM_SKETCH_GLIBC) {
    // every rank draws the whole stream (stream order = row-major n x k): pass 1 needs all rows
    float *raw = W;
    if (rows) TSVM_TRY(scratch_t(ctx, SLOT_W2, (size_t)n * k, &raw));
    TSVM_TRY(sketch_glibc(ctx, n * (int64_t)k, raw));
    TSVM_TRY(pad_rows(ctx, raw, k, n, k, Q, kp));
  } else if (sketch == TSVM_SKETCH_PHILOX) {
    float *raw = W;
    if (rows) TSVM_TRY(scratch_t(ctx, SLOT_W2, (size_t)n * k, &raw));
    TSVM_TRY(sketch_philox(ctx, ctx->sketch_seed, n * (int64_t)k, raw));
    TSVM_TRY(pad_rows(ctx, raw, k, n, k, Q, kp));
  } else if (sketch == TSVM_SKETCH_USER) {
    if (!Q_user) return TSVM_ERR_INVALID_ARGUMENT;
    TSVM_TRY(pad_rows(ctx, Q_user, k, n, k, Q, kp));
  } else {
    return TSVM_ERR_INVALID_ARGUMENT;
  }
  if (keep)
    TSVM_CUDA(cudaMemcpyAsync(keep->omega, Q, sizeof(float) * n * kp, cudaMemcpyDeviceToDevice,
                              ctx->stream));
  TSVM_CUDA(cudaEventRecord(ev[1], ctx->stream));
  phase.next("factor: kernel-block pass 1");
  float km1 = 0.f, km2 = 0.f;
  // split forms: the kernel block as hi + lo in this pass (its rounding would perturb the
  // kernel whose range is found; rounding the sketch only draws another Gaussian sketch)
  const bool split = precision_is_split(precision);
  TSVM_TRY(kermatmul(ctx, Xc, norms, y, n, d, gamma, Q, kp, W, precision, &km1, nullptr,
                     split ? 1 : 0, row0, nr, k));
  TSVM_CUDA(cudaEventRecord(ev[2], ctx->stream));
  phase.next("factor: orthonormalise");
  const bool tc_gram = precision != TSVM_PREC_FP32 && keep == nullptr && syrk_tc_supported(k) &&
                       k >= 32;
  TSVM_TRY(orthonormalise(ctx, W, nr, k, kp, keep ? keep->R : nullptr, tc_gram, n));
  if (keep)
    TSVM_CUDA(cudaMemcpyAsync(keep->W, W, sizeof(float) * n * kp, cudaMemcpyDeviceToDevice,
                              ctx->stream));
  TSVM_CUDA(cudaEventRecord(ev[3], ctx->stream));
  phase.next("factor: kernel-block pass 2");
  // split forms: the basis W as hi + lo (rounding it would tilt the subspace K is projected
  // on).  One-product forms round W to the tensor-core operand type in place instead, so that
  // C = W^T (K W) and Z = W V diag(sqrt w) use the W the tensor cores contracted and the weak
  // eigen-directions of C do not pick up the rounding of one side only.
  // Row-sharded: the pass needs every row of W, gathered as an all-reduce of the zero-padded
  // rows (exact: each entry is one rank's value plus zeros).
  float *Wall = W;
  if (rows) {
    TSVM_TRY(scratch_t(ctx, SLOT_SHARD_A, (size_t)n * kp, &Wall));
    TSVM_CUDA(cudaMemsetAsync(Wall, 0, sizeof(float) * n * kp, ctx->stream));
    TSVM_CUDA(cudaMemcpyAsync(Wall + row0 * kp, W, sizeof(float) * nr * kp,
                              cudaMemcpyDeviceToDevice, ctx->stream));
    TSVM_TRY(comm_allreduce(ctx, Wall, n * (int64_t)kp, 1, COMM_SUM));
  }
  // The projection needs only C = W^T K W: on one device the tensor-core forms take the half
  // product R over the J blocks from the diagonal on (about half the tiles) and
  // C = W^T R + R^T W + s u u^T.
  double *Cm = nullptr, *V = nullptr, *w = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL, (size_t)k * k + 8 + (size_t)kp + 8, &Cm));
  double *sym = Cm + (size_t)k * k + 8;
  const bool half = precision != TSVM_PREC_FP32 && !rows;
  if (half) {
    // the range-finder pass above built the Gram operands of the same rows and gamma (nothing
    // in between touches them)
    TSVM_TRY(kermatmul_tc_half(ctx, Xc, y, n, d, gamma, W, kp, Q, precision, &km2,
                               split ? nullptr : W, split ? 2 : 0, sym, true, k));
  } else if (split) {
    TSVM_TRY(kermatmul(ctx, Xc, norms, y, n, d, gamma, Wall, kp, Q, precision, &km2, nullptr, 2,
                       row0, nr, k));
  } else {
    TSVM_TRY(kermatmul(ctx, Xc, norms, y, n, d, gamma, Wall, kp, Q, precision, &km2, Wall, 0,
                       row0, nr, k));
    if (rows && precision != TSVM_PREC_FP32)   // this rank's rows as the tensor cores saw them
      TSVM_CUDA(cudaMemcpyAsync(W, Wall + row0 * kp, sizeof(float) * nr * kp,
                                cudaMemcpyDeviceToDevice, ctx->stream));
  }
  TSVM_CUDA(cudaEventRecord(ev[4], ctx->stream));
  phase.next("factor: projection and eigensolver");
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL2, (size_t)k * k + (size_t)k, &V));
  w = V + (size_t)k * k;
  TSVM_TRY(gram_fp64(ctx, W, kp, Q, kp, nr, k, k, false, Cm));
  if (half) {
    half_projection_finish<<<(unsigned)ceil_div((int64_t)k * k, 256), 256, 0, ctx->stream>>>(
        Cm, k, sym);
    TSVM_LAUNCHED(ctx);
  } else {
    TSVM_TRY(comm_allreduce(ctx, Cm, (int64_t)k * k, 0, COMM_SUM));   // row-sharded
    TSVM_TRY(small_symmetrize(ctx, Cm, k, k));
  }
  if (C_out) {   // stop here: the batched factor solves the eigenproblems of all problems at once
    TSVM_CUDA(cudaMemcpyAsync(C_out, Cm, sizeof(double) * k * k, cudaMemcpyDeviceToDevice,
                              ctx->stream));
    TSVM_CUDA(cudaMemcpyAsync(Z, W, sizeof(float) * n * kp, cudaMemcpyDeviceToDevice,
                              ctx->stream));
    TSVM_CUDA(cudaEventRecord(ev[5], ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (info) {
      info->n = n;
      info->d = d;
      info->k = k;
      info->k_padded = kp;
      info->precision = precision;
      info->ms_sketch = event_ms(ev[0], ev[1]);
      info->ms_pass1 = event_ms(ev[1], ev[2]);
      info->ms_ortho = event_ms(ev[2], ev[3]);
      info->ms_pass2 = event_ms(ev[3], ev[4]);
      info->ms_project = event_ms(ev[4], ev[5]);
      info->ms_total = event_ms(ev[0], ev[5]);
      info->ms_kermatmul_kernel =
          precision == TSVM_PREC_FP32 ? info->ms_pass1 + info->ms_pass2 : (double)km1 + km2;
      info->flops_kermatmul = 2.0 * (2.0 * (double)n * n * k + 2.0 * (double)n * n * d);
    }
    return TSVM_OK;
  }
  int sweeps = 0;
  TSVM_TRY(eig_jacobi_fp64(ctx, Cm, k, k, w, V, &sweeps));
  float *X32 = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)kp * kp, &X32));
  eigfactor_to_fp32<<<(unsigned)ceil_div((int64_t)kp * kp, 256), 256, 0, ctx->stream>>>(V, w, k,
                                                                                         kp, X32);
  TSVM_LAUNCHED(ctx);
  if (ldz == kp) {
    TSVM_TRY(apply_right_fp32(ctx, W, nr, kp, X32, Z));
  } else {
    TSVM_TRY(apply_right_fp32(ctx, W, nr, kp, X32, Q));  // Q is free again
    TSVM_TRY(pad_rows(ctx, Q, kp, nr, k, Z, ldz));
  }
  TSVM_CUDA(cudaEventRecord(ev[5], ctx->stream));
  std::vector<double> hw(k);
  TSVM_CUDA(cudaMemcpyAsync(hw.data(), w, sizeof(double) * k, cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (info) {
    info->n = n;
    info->d = d;
    info->k = k;
    info->k_padded = kp;
    info->precision = precision;
    int realk = 0;
    double wmax = -INFINITY, wmin = INFINITY;
    for (int i = 0; i < k; ++i) {
      realk += hw[i] > 0.0;
      wmax = fmax(wmax, hw[i]);
      wmin = fmin(wmin, hw[i]);
    }
    info->realk = realk;
    info->eig_max = wmax;
    info->eig_min = wmin;
    info->ms_sketch = event_ms(ev[0], ev[1]);
    info->ms_pass1 = event_ms(ev[1], ev[2]);
    info->ms_ortho = event_ms(ev[2], ev[3]);
    info->ms_pass2 = event_ms(ev[3], ev[4]);
    info->ms_project = event_ms(ev[4], ev[5]);
    info->ms_total = event_ms(ev[0], ev[5]);
    info->ms_kermatmul_kernel =
        precision == TSVM_PREC_FP32 ? info->ms_pass1 + info->ms_pass2 : (double)km1 + km2;
    info->flops_kermatmul = 2.0 * (2.0 * (double)n * n * k + 2.0 * (double)n * n * d);
  }
  return TSVM_OK;
}

tsvm_status factor_finish(tsvm_context *ctx, float *Z, int64_t n, int k, const double *V,
                          const double *w, tsvm_factor_info *info) {
  const int kp = (int)round_up(k, 64);
  float *X32 = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)kp * kp, &X32));
  eigfactor_to_fp32<<<(unsigned)ceil_div((int64_t)kp * kp, 256), 256, 0, ctx->stream>>>(V, w, k,
                                                                                         kp, X32);
  TSVM_LAUNCHED(ctx);
  // in place: every block reads all of its 128 rows before it writes them
  TSVM_TRY(apply_right_fp32(ctx, Z, n, kp, X32, Z));
  if (info) {
    std::vector<double> hw(k);
    TSVM_CUDA(cudaMemcpyAsync(hw.data(), w, sizeof(double) * k, cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    int realk = 0;
    double wmax = -INFINITY, wmin = INFINITY;
    for (int i = 0; i < k; ++i) {
      realk += hw[i] > 0.0;
      wmax = fmax(wmax, hw[i]);
      wmin = fmin(wmin, hw[i]);
    }
    info->realk = realk;
    info->eig_max = wmax;
    info->eig_min = wmin;
  }
  return TSVM_OK;
}

// Shifted CholeskyQR3 of the bases W_p = Zs[p] (ns[p] x kp) of `count` problems, stage by stage:
// each step forms every problem's Gram matrix (the same kernels as orthonormalise), factors them
// all in one launch (chol_fp64_same: the single-problem arithmetic), reads all statuses with one
// host synchronisation, retries the failed ones with a larger shift, then applies R^-1 problem
// by problem.  The result is that of orthonormalise for each problem.
static tsvm_status orthonormalise_batched(tsvm_context *ctx, float *const *Zs, const int64_t *ns,
                                          int count, int k, int kp, bool tc_gram) {
  const size_t kk = (size_t)k * k;
  const int64_t strideD = (int64_t)ceil_div(k, 32) * 1024;
  int64_t n_max = 0;
  for (int p = 0; p < count; ++p) n_max = std::max(n_max, ns[p]);
  double *Gall = nullptr, *Linv = nullptr;
  float *R32 = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_B_FACG, (kk + (size_t)strideD) * count + (size_t)count + 8, &Gall));
  double *Dall = Gall + kk * count;
  int *d_info = reinterpret_cast<int *>(Dall + (size_t)strideD * count);
  int *d_active = d_info + count;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL2, kk, &Linv));
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)kp * kp, &R32));
  double *ones = nullptr, *negI = nullptr;
  const unsigned gk = (unsigned)ceil_div((int64_t)k * k, 256);
  if (tc_gram) {
    TSVM_TRY(scratch_t(ctx, SLOT_IPM_VEC, (size_t)n_max, &ones));
    TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, kk, &negI));
    fill_value<<<(unsigned)ceil_div(n_max, 256), 256, 0, ctx->stream>>>(ones, n_max, 1.0);
    TSVM_LAUNCHED(ctx);
    set_scaled_identity<<<gk, 256, 0, ctx->stream>>>(negI, k, -1.0);
    TSVM_LAUNCHED(ctx);
  }
  const double u = ldexp(1.0, -53);
  std::vector<double> fac(count);
  std::vector<int> hinfo(count), act(count);
  for (int step = 0; step < 3; ++step) {
    std::vector<int> pending(count);
    for (int p = 0; p < count; ++p) {
      pending[p] = p;
      fac[p] = step == 0 ? 11.0 * ((double)ns[p] * k + (double)k * (k + 1)) * u : 0.0;
    }
    for (int attempt = 0; !pending.empty(); ++attempt) {
      for (int p : pending) {
        double *G = Gall + kk * p;
        if (tc_gram && step > 0 && attempt == 0)
          TSVM_TRY(syrk_capacitance_tc(ctx, Zs[p], kp, ns[p], k, ones, 2.0, 3, negI, G));
        else
          TSVM_TRY(gram_fp64(ctx, Zs[p], kp, Zs[p], kp, ns[p], k, k, true, G));
        if (fac[p] > 0) {
          shift_by_trace<<<1, 256, 0, ctx->stream>>>(G, k, fac[p]);
          TSVM_LAUNCHED(ctx);
        }
      }
      std::fill(act.begin(), act.end(), 0);
      for (int p : pending) act[p] = 1;
      TSVM_CUDA(cudaMemcpyAsync(d_active, act.data(), sizeof(int) * count, cudaMemcpyHostToDevice,
                                ctx->stream));
      TSVM_TRY(chol_fp64_same(ctx, Gall, k, k, (int64_t)kk, d_info, Dall, strideD, count,
                              d_active, pending));
      TSVM_CUDA(cudaMemcpyAsync(hinfo.data(), d_info, sizeof(int) * count, cudaMemcpyDeviceToHost,
                                ctx->stream));
      TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
      std::vector<int> failed;
      for (int p : pending)
        if (hinfo[p] != 0) failed.push_back(p);
      if (!failed.empty() && attempt == 3) return TSVM_ERR_NOT_SPD;
      for (int p : failed)
        fac[p] = fac[p] > 0 ? fac[p] * 100.0
                            : 11.0 * ((double)ns[p] * k + (double)k * (k + 1)) * u;
      pending.swap(failed);
    }
    for (int p = 0; p < count; ++p) {
      TSVM_TRY(trinv_lower_fp64(ctx, Gall + kk * p, k, k, Dall + (size_t)strideD * p, Linv));
      rinv_to_fp32<<<(unsigned)ceil_div((int64_t)kp * kp, 256), 256, 0, ctx->stream>>>(Linv, k,
                                                                                        kp, R32);
      TSVM_LAUNCHED(ctx);
      TSVM_TRY(apply_right_fp32(ctx, Zs[p], ns[p], kp, R32, Zs[p]));
    }
  }
  return TSVM_OK;
}

// The factors of `count` problems (tsvm_factor_batched), stage by stage so that the small k x k
// steps of all problems share launches and host synchronisations: one sketch (the glibc and
// Philox streams are prefixes of each other, so the first n_p rows of the longest problem's
// sketch are problem p's), every range-finder pass, one batched CholeskyQR3, every projection
// pass with C_p = W_p^T (K W_p), all eigenproblems in one launch, then Z_p = W_p V diag(sqrt w)
// in place.  Every kernel is the one factor_rbf runs for that problem, on the same data: the
// factors are those of tsvm_factor.
tsvm_status factor_rbf_batched(tsvm_context *ctx, const tsvm_factor_problem *pr, int count, int d,
                               int k, int precision, int sketch, int ldz,
                               tsvm_factor_info *infos, double *ms_eig) {
  const int kp = (int)round_up(k, 64);
  if (count < 1 || ldz != kp || d < 1 || k < 1 || k > 1000) return TSVM_ERR_INVALID_ARGUMENT;
  int64_t n_max = 0;
  std::vector<int64_t> ns(count), xo(count + 1, 0);
  std::vector<float *> Zs(count);
  for (int p = 0; p < count; ++p) {
    ns[p] = pr[p].n;
    if (ns[p] < 2 || k > ns[p] || !(pr[p].gamma > 0)) return TSVM_ERR_INVALID_ARGUMENT;
    n_max = std::max(n_max, ns[p]);
    Zs[p] = pr[p].Z;
    xo[p + 1] = xo[p] + round_up(ns[p] * (d + 1) + 64, 4);   // rows then norms, 16-byte aligned
  }
  TraceRange tr_b("factor batched");
  const size_t kk = (size_t)k * k;
  double *buf = nullptr;   // [count][k][k] C, then [count][k][k] V, then [count][k] w
  TSVM_TRY(scratch_t(ctx, SLOT_B_EIG, (2 * kk + (size_t)k) * count, &buf));
  double *Cb = buf, *Vb = buf + kk * count, *wb = Vb + kk * count;
  float *Xall = nullptr, *Q = nullptr, *raw = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_B_FXC, (size_t)xo[count], &Xall));
  TSVM_TRY(scratch_t(ctx, SLOT_Q, (size_t)n_max * kp, &Q));
  TSVM_TRY(scratch_t(ctx, SLOT_W2, (size_t)n_max * k, &raw));
  if (sketch == TSVM_SKETCH_GLIBC)
    TSVM_TRY(sketch_glibc(ctx, n_max * (int64_t)k, raw));
  else if (sketch == TSVM_SKETCH_PHILOX)
    TSVM_TRY(sketch_philox(ctx, ctx->sketch_seed, n_max * (int64_t)k, raw));
  else
    return TSVM_ERR_INVALID_ARGUMENT;
  TSVM_TRY(pad_rows(ctx, raw, k, n_max, k, Q, kp));
  const bool split = precision_is_split(precision);
  std::vector<float> km(count, 0.f);
  // range-finder passes: W_p = Y K Y Q_p into Z_p
  for (int p = 0; p < count; ++p) {
    float *Xc = Xall + xo[p], *norms = Xc + ns[p] * d;
    TSVM_TRY(centre_features(ctx, pr[p].X, ns[p], d, Xc, norms));
    float km1 = 0.f;
    TSVM_TRY(kermatmul(ctx, Xc, norms, pr[p].y, ns[p], d, pr[p].gamma, Q, kp, Zs[p], precision,
                       &km1, nullptr, split ? 1 : 0, 0, -1, k));
    km[p] += km1;
  }
  const bool tc_gram = precision != TSVM_PREC_FP32 && syrk_tc_supported(k) && k >= 32;
  TSVM_TRY(orthonormalise_batched(ctx, Zs.data(), ns.data(), count, k, kp, tc_gram));
  // projection passes and C_p (the sketch in Q is no longer needed: Q takes each pass's output)
  double *sym = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL, (size_t)kp + 8, &sym));
  const bool half = precision != TSVM_PREC_FP32;
  for (int p = 0; p < count; ++p) {
    float *Xc = Xall + xo[p], *norms = Xc + ns[p] * d, *W = Zs[p];
    double *Cm = Cb + kk * p;
    float km2 = 0.f;
    if (half)
      TSVM_TRY(kermatmul_tc_half(ctx, Xc, pr[p].y, ns[p], d, pr[p].gamma, W, kp, Q, precision,
                                 &km2, split ? nullptr : W, split ? 2 : 0, sym, false, k));
    else
      TSVM_TRY(kermatmul(ctx, Xc, norms, pr[p].y, ns[p], d, pr[p].gamma, W, kp, Q, precision,
                         &km2, W, 0, 0, -1, k));
    km[p] += km2;
    TSVM_TRY(gram_fp64(ctx, W, kp, Q, kp, ns[p], k, k, false, Cm));
    if (half) {
      half_projection_finish<<<(unsigned)ceil_div((int64_t)k * k, 256), 256, 0, ctx->stream>>>(
          Cm, k, sym);
      TSVM_LAUNCHED(ctx);
    } else {
      TSVM_TRY(small_symmetrize(ctx, Cm, k, k));
    }
  }
  cudaEvent_t e0 = ctx->ev[6], e1 = ctx->ev[7];
  TSVM_CUDA(cudaEventRecord(e0, ctx->stream));
  int sweeps = 0;
  TSVM_TRY(eig_jacobi_fp64_batched(ctx, Cb, k, count, wb, Vb, &sweeps));
  TSVM_CUDA(cudaEventRecord(e1, ctx->stream));
  for (int p = 0; p < count; ++p)
    TSVM_TRY(factor_finish(ctx, Zs[p], ns[p], k, Vb + kk * p, wb + (size_t)k * p, nullptr));
  std::vector<double> hw((size_t)k * count);
  TSVM_CUDA(cudaMemcpyAsync(hw.data(), wb, sizeof(double) * hw.size(), cudaMemcpyDeviceToHost,
                            ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ms_eig) *ms_eig = event_ms(e0, e1);
  if (infos) {
    for (int p = 0; p < count; ++p) {
      tsvm_factor_info &in = infos[p];
      memset(&in, 0, sizeof(in));
      in.n = ns[p];
      in.d = d;
      in.k = k;
      in.k_padded = kp;
      in.precision = precision;
      int realk = 0;
      double wmax = -INFINITY, wmin = INFINITY;
      for (int i = 0; i < k; ++i) {
        const double v = hw[(size_t)k * p + i];
        realk += v > 0.0;
        wmax = fmax(wmax, v);
        wmin = fmin(wmin, v);
      }
      in.realk = realk;
      in.eig_max = wmax;
      in.eig_min = wmin;
      in.ms_kermatmul_kernel = km[p];
      in.flops_kermatmul = 2.0 * (2.0 * (double)ns[p] * ns[p] * k + 2.0 * (double)ns[p] * ns[p] * d);
    }
  }
  return TSVM_OK;
}

tsvm_status factor_rbf_keep(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                            double gamma, int k, int precision, float *Z, int ldz,
                            tsvm_factor_info *info) {
  const int kp = (int)round_up(k, 64);
  float *Zk = nullptr, *Om = nullptr, *Wk = nullptr;
  double *Rbuf = nullptr;
  ctx->kept.valid = false;
  TSVM_TRY(scratch_t(ctx, SLOT_HG_Z, (size_t)n * kp, &Zk));
  TSVM_TRY(scratch_t(ctx, SLOT_HG_OMEGA, (size_t)n * kp, &Om));
  TSVM_TRY(scratch_t(ctx, SLOT_HG_R, (size_t)2 * k * k + 2 * (size_t)kp + 64, &Rbuf));
  TSVM_TRY(scratch_t(ctx, SLOT_HG_W, (size_t)n * kp, &Wk));
  FactorKeep keep{Om, Rbuf, Wk};
  TSVM_TRY(factor_rbf(ctx, X, y, n, d, gamma, k, precision, TSVM_SKETCH_GLIBC, nullptr, Zk, kp,
                      info, &keep));
  if (Z && Z != Zk)
    TSVM_CUDA(cudaMemcpy2DAsync(Z, sizeof(float) * ldz, Zk, sizeof(float) * kp,
                                sizeof(float) * (ldz < kp ? ldz : kp), n, cudaMemcpyDeviceToDevice,
                                ctx->stream));
  if (Z && ldz > kp)
    TSVM_CUDA(cudaMemset2DAsync(Z + kp, sizeof(float) * ldz, 0, sizeof(float) * (ldz - kp), n,
                                ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->kept.valid = true;
  ctx->kept.X = X;
  ctx->kept.y = y;
  ctx->kept.n = n;
  ctx->kept.d = d;
  ctx->kept.k = k;
  ctx->kept.precision = precision;
  ctx->kept.gamma = gamma;
  return TSVM_OK;
}

}  // namespace tsvm
