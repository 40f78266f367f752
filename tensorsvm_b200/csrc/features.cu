// Feature preparation for the kernel factor and the linear path.
//  * centre_features: the RBF kernel is translation invariant, so X is centred by its column
//    means (FP64 reduction) before the distance expansion ||xi||^2 + ||xj||^2 - 2 xi.xj; this
//    shrinks the cancellation the reference suffers in rbf_kergen (tensorsvm-train.cu:2608).
//    The squared row norms replace vecnorm (tensorsvm-train.cu:2569-2581), computed once per
//    dataset instead of once per block pair.
//  * label_rows: Z = diag(y) X for the linear kernel (tensorsvm-train.cu:909-914).
//  * pad_rows: copy with zero padding to an aligned leading dimension.
#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
namespace {

// grid.x = split over rows; each block writes d partial column sums.
__global__ void colsum_partial(const float *__restrict__ X, int64_t n, int d,
                               int64_t rows_per_block, double *__restrict__ part) {
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = min(n, r0 + rows_per_block);
  __shared__ double sh[256];
  for (int c = 0; c < d; ++c) {
    double s = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) s += X[r * d + c];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(int64_t)blockIdx.x * d + c] = sh[0];
    __syncthreads();
  }
}

__global__ void colmean_finish(const double *__restrict__ part, int nblocks, int d, int64_t n,
                               float *__restrict__ mean) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += part[(int64_t)b * d + c];
  mean[c] = (float)(s / (double)n);
}

__global__ void centre_rows(const float *__restrict__ X, int64_t n, int d,
                            const float *__restrict__ mean, float *__restrict__ Xc,
                            float *__restrict__ norms) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double s = 0.0;
  for (int c = 0; c < d; ++c) {
    const float v = X[r * d + c] - mean[c];
    Xc[r * d + c] = v;
    s += (double)v * (double)v;
  }
  norms[r] = (float)s;
}

__global__ void pad_rows_kernel(const float *__restrict__ src, int64_t lds, int64_t n, int k,
                                float *__restrict__ dst, int64_t ldd, const float *__restrict__ y) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * ldd) return;
  const int64_t r = e / ldd;
  const int c = (int)(e % ldd);
  float v = c < k ? src[r * lds + c] : 0.f;
  if (y) v *= y[r];
  dst[e] = v;
}

}  // namespace

tsvm_status centre_features(tsvm_context *ctx, const float *X, int64_t n, int d, float *Xc,
                            float *norms) {
  const int nb = (int)std::min<int64_t>(ctx->num_sms * 2, ceil_div(n, 256));
  const int64_t rpb = ceil_div(n, nb);
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, (size_t)nb * d + 2 * (size_t)d, &part));
  float *mean = reinterpret_cast<float *>(part + (size_t)nb * d);
  colsum_partial<<<nb, 256, 0, ctx->stream>>>(X, n, d, rpb, part);
  TSVM_LAUNCHED(ctx);
  colmean_finish<<<(unsigned)ceil_div(d, 64), 64, 0, ctx->stream>>>(part, nb, d, n, mean);
  TSVM_LAUNCHED(ctx);
  centre_rows<<<(unsigned)ceil_div(n, 256), 256, 0, ctx->stream>>>(X, n, d, mean, Xc, norms);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status pad_rows(tsvm_context *ctx, const float *src, int64_t lds, int64_t n, int k,
                     float *dst, int64_t ldd) {
  pad_rows_kernel<<<(unsigned)ceil_div(n * ldd, 256), 256, 0, ctx->stream>>>(src, lds, n, k, dst,
                                                                             ldd, nullptr);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status label_rows(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                       float *Z, int64_t ldz) {
  pad_rows_kernel<<<(unsigned)ceil_div(n * ldz, 256), 256, 0, ctx->stream>>>(X, d, n, d, Z, ldz,
                                                                             y);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

}  // namespace tsvm
