// Feature preparation for the kernel factor and the linear path.
//  * centre_features: the RBF kernel is translation invariant, so X is centred by its column
//    means (FP64 reduction) before the distance expansion ||xi||^2 + ||xj||^2 - 2 xi.xj; this
//    shrinks the cancellation the reference suffers in rbf_kergen (tensorsvm-train.cu:2608).
//    The squared row norms replace vecnorm (tensorsvm-train.cu:2569-2581), computed once per
//    dataset instead of once per block pair.
//  * label_rows: Z = diag(y) X for the linear kernel (tensorsvm-train.cu:909-914).
//  * linear_bias: w = sum over SVs (alpha > 1e-6) of alpha_j y_j x_j and b = the mean over the
//    first <= 5000 free SVs (1e-6 < alpha < C - 1e-6, index order) of y_j - w . x_j, the rule of
//    writemodel (tensorsvm-train.cu:301-332), with fixed-order FP64 reductions.
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
  if (norms) norms[r] = (float)s;
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

tsvm_status centre_pair(tsvm_context *ctx, const float *XJ, int64_t nj, const float *XI,
                        int64_t ni, int d, float *XJc, float *XIc) {
  const int nb = (int)std::min<int64_t>(ctx->num_sms * 2, ceil_div(nj, 256));
  const int64_t rpb = ceil_div(nj, nb);
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, (size_t)nb * d + 2 * (size_t)d, &part));
  float *mean = reinterpret_cast<float *>(part + (size_t)nb * d);
  colsum_partial<<<nb, 256, 0, ctx->stream>>>(XJ, nj, d, rpb, part);
  TSVM_LAUNCHED(ctx);
  colmean_finish<<<(unsigned)ceil_div(d, 64), 64, 0, ctx->stream>>>(part, nb, d, nj, mean);
  TSVM_LAUNCHED(ctx);
  centre_rows<<<(unsigned)ceil_div(nj, 256), 256, 0, ctx->stream>>>(XJ, nj, d, mean, XJc, nullptr);
  TSVM_LAUNCHED(ctx);
  centre_rows<<<(unsigned)ceil_div(ni, 256), 256, 0, ctx->stream>>>(XI, ni, d, mean, XIc, nullptr);
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

namespace {

constexpr int kLinFree = 5000;   // free SVs the linear bias averages over (writemodel)

// w partials: block (x, y) takes rows [x rpb, (x + 1) rpb) and columns [256 y, 256 y + 256); warp
// w takes rows w, w + 8, ...; lane l columns l + 32 j.  part[x][c] (FP64, fixed order).
__global__ void __launch_bounds__(256)
lin_w_partial(const float *__restrict__ X, const float *__restrict__ y,
              const double *__restrict__ alpha, int64_t n, int d, int64_t rpb,
              double *__restrict__ part) {
  __shared__ double red[8][257];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c0 = blockIdx.y * 256;
  const int64_t r0 = (int64_t)blockIdx.x * rpb, r1 = min(n, r0 + rpb);
  double acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.0;
  for (int64_t r = r0 + warp; r < r1; r += 8) {
    const double a = alpha[r];
    if (!(a > 1e-6)) continue;
    const double coef = a * (double)y[r];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = c0 + lane + 32 * j;
      if (c < d) acc[j] += coef * (double)X[r * d + c];
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) red[warp][lane + 32 * j] = acc[j];
  __syncthreads();
  const int c = c0 + threadIdx.x;
  if (c < d) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w][threadIdx.x];
    part[(int64_t)blockIdx.x * d + c] = t;
  }
}

__global__ void lin_w_reduce(const double *__restrict__ part, int nparts, int d,
                             double *__restrict__ w) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d) return;
  double t = 0.0;
  for (int x = 0; x < nparts; ++x) t += part[(int64_t)x * d + c];
  w[c] = t;
}

__device__ __forceinline__ bool lin_free(double a, double C) { return a > 1e-6 && a < C - 1e-6; }

// free SVs per block of rows (same row ranges as below)
__global__ void __launch_bounds__(256)
lin_free_count(const double *__restrict__ alpha, int64_t n, double C, int64_t rpb,
               int *__restrict__ counts) {
  __shared__ int wsum[8];
  const int64_t r0 = (int64_t)blockIdx.x * rpb, r1 = min(n, r0 + rpb);
  int c = 0;
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) c += lin_free(alpha[i], C) ? 1 : 0;
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += wsum[w];
    counts[blockIdx.x] = t;
  }
}

// sum of y_j - w . x_j over the free SVs of this block whose index-order rank is below 5000
__global__ void __launch_bounds__(256)
lin_bias_partial(const float *__restrict__ X, const float *__restrict__ y,
                 const double *__restrict__ alpha, int64_t n, int d, double C, int64_t rpb,
                 const int *__restrict__ counts, const double *__restrict__ w,
                 double *__restrict__ partb) {
  __shared__ int wcnt[8];
  __shared__ int base_sh;
  __shared__ double wsh[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t r0 = (int64_t)blockIdx.x * rpb, r1 = min(n, r0 + rpb);
  if (threadIdx.x == 0) {
    int t = 0;
    for (int b = 0; b < (int)blockIdx.x; ++b) t += counts[b];
    base_sh = t;
  }
  __syncthreads();
  int base = base_sh;
  double s = 0.0;
  for (int64_t b0 = r0; b0 < r1 && base < kLinFree; b0 += blockDim.x) {
    const int64_t i = b0 + threadIdx.x;
    const bool f = i < r1 && lin_free(alpha[i], C);
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int rank = base;
    for (int q = 0; q < warp; ++q) rank += wcnt[q];
    rank += __popc(bal & ((1u << lane) - 1u));
    if (f && rank < kLinFree) {
      double v = (double)y[i];
      for (int c = 0; c < d; ++c) v -= w[c] * (double)X[i * d + c];
      s += v;
    }
    int tot = 0;
    for (int q = 0; q < 8; ++q) tot += wcnt[q];
    __syncthreads();
    base += tot;
  }
  s = warp_sum(s);
  if (lane == 0) wsh[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < 8; ++q) t += wsh[q];
    partb[blockIdx.x] = t;
  }
}

__global__ void lin_bias_finish(const double *__restrict__ partb, const int *__restrict__ counts,
                                int nb, double *__restrict__ b) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  int64_t m = 0;
  for (int x = 0; x < nb; ++x) {
    s += partb[x];
    m += counts[x];
  }
  if (m > kLinFree) m = kLinFree;
  b[0] = m > 0 ? s / (double)m : 0.0;
}

}  // namespace

tsvm_status linear_bias(tsvm_context *ctx, const float *X, const float *y, const double *alpha,
                        int64_t n, int d, double C, double *b_host) {
  const int nb = ctx->num_sms * 2;
  const int64_t rpb = ceil_div(n, (int64_t)nb);
  const int nct = (int)ceil_div(d, 256);
  double *buf = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, (size_t)nb * d + d + nb + 8 + nb / 2 + 8, &buf));
  double *part = buf, *w = part + (size_t)nb * d, *partb = w + d, *bdev = partb + nb;
  int *counts = reinterpret_cast<int *>(bdev + 8);
  lin_w_partial<<<dim3(nb, nct), 256, 0, ctx->stream>>>(X, y, alpha, n, d, rpb, part);
  TSVM_LAUNCHED(ctx);
  lin_w_reduce<<<(unsigned)ceil_div(d, 256), 256, 0, ctx->stream>>>(part, nb, d, w);
  TSVM_LAUNCHED(ctx);
  lin_free_count<<<nb, 256, 0, ctx->stream>>>(alpha, n, C, rpb, counts);
  TSVM_LAUNCHED(ctx);
  lin_bias_partial<<<nb, 256, 0, ctx->stream>>>(X, y, alpha, n, d, C, rpb, counts, w, partb);
  TSVM_LAUNCHED(ctx);
  lin_bias_finish<<<1, 32, 0, ctx->stream>>>(partb, counts, nb, bdev);
  TSVM_LAUNCHED(ctx);
  TSVM_CUDA(cudaMemcpyAsync(b_host, bdev, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
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
