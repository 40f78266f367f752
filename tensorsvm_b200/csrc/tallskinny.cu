// Tall-skinny products over n rows:
//  * gram_fp64:  G = A^T B with every product formed exactly in FP64 (FP32 x FP32 fits) and
//    FP64 accumulation, split over row chunks with a fixed-order reduction.  Used for the
//    shifted-CholeskyQR Gram W^T W that replaces the reference's TSQR (ortho/CAQR,
//    tensorsvm-train.cu:707-856) and for C = W^T Q (tensorsvm-train.cu:2122-2160, where the
//    reference converts W and Q to FP64 on the host and calls cublasDgemm).
//  * apply_right_fp32:  Out = A R (n x kp times kp x kp) in FP32, for W <- W R^-1 and
//    U = W X (tensorsvm-train.cu:2226-2236, a chunked cublasSgemm there).
#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
namespace {

constexpr int kGT = 64;      // output tile edge
constexpr int kGRows = 32;   // rows staged per step

// grid: (tile index, split).  Each block accumulates a 64x64 tile over rows [r0, r1).
// Operands are converted to FP64 once, while staging 32-row slabs into shared memory (with the
// optional row weight folded into the A side), so the inner loop is pure DFMA: each thread owns
// a 4x4 block of the tile and reads 4 + 4 doubles per row.
__global__ void __launch_bounds__(256)
gram_partial_kernel(const float *__restrict__ A, int64_t lda, const float *__restrict__ B,
                    int64_t ldb, int64_t n, int ka, int kb, int tiles_b, int symmetric,
                    int64_t rows_per_split, const double *__restrict__ rowscale,
                    const int64_t *__restrict__ rowidx, const int *__restrict__ count,
                    const WorkUnit *__restrict__ units, const float *const *__restrict__ Zs,
                    const int *__restrict__ active, double *__restrict__ part) {
  __shared__ double As[kGRows][kGT];
  __shared__ double Bs[kGRows][kGT];
  int t = blockIdx.x, ta, tb;
  if (symmetric) {  // lower-triangle tile enumeration
    ta = 0;
    while ((ta + 1) * (ta + 2) / 2 <= t) ++ta;
    tb = t - ta * (ta + 1) / 2;
  } else {
    ta = t / tiles_b;
    tb = t % tiles_b;
  }
  const int a0 = ta * kGT, b0 = tb * kGT;
  if (units) {  // batched: this block sums the rows of one work unit (symmetric, A = B)
    const WorkUnit u = units[blockIdx.y];
    if (active && !active[u.p]) return;
    A = Zs[u.p] + u.row0 * lda;
    B = A;
    n = u.rows;
    rows_per_split = u.rows;
    rowscale += u.goff;
  }
  if (count) {  // row count on the device: split it evenly over gridDim.y
    n = *count;
    rows_per_split = (n + gridDim.y - 1) / gridDim.y;
    rows_per_split = (rows_per_split + kGRows - 1) / kGRows * kGRows;
  }
  const int64_t r0 = units ? 0 : (int64_t)blockIdx.y * rows_per_split;
  const int64_t r1 = min(n, r0 + rows_per_split);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int64_t r = r0; r < r1; r += kGRows) {
    __syncthreads();
    for (int e = threadIdx.x; e < kGRows * kGT; e += 256) {
      const int rr = e / kGT, c = e % kGT;
      const int64_t gr = r + rr;
      const bool in = gr < r1;
      const int64_t row = in ? (rowidx ? rowidx[gr] : gr) : 0;
      const double sc = in ? (rowscale ? rowscale[row] : 1.0) : 0.0;
      As[rr][c] = (in && a0 + c < ka) ? (double)A[row * lda + a0 + c] * sc : 0.0;
      Bs[rr][c] = (in && b0 + c < kb) ? (double)B[row * ldb + b0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < kGRows; ++rr) {
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[rr][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[rr][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
  }
  // partial layout: [split][ka][kb]
  double *P = part + (int64_t)blockIdx.y * ka * kb;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int ga = a0 + ty + 16 * i, gb = b0 + tx + 16 * j;
      if (ga < ka && gb < kb) P[(int64_t)ga * kb + gb] = acc[i][j];
    }
}

__global__ void gram_reduce_kernel(const double *__restrict__ part, int nsplit, int ka, int kb,
                                   int symmetric, double *__restrict__ G) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)ka * kb) return;
  const int a = (int)(e / kb), b = (int)(e % kb);
  if (symmetric && b > a) return;
  double s = 0.0;
  for (int sp = 0; sp < nsplit; ++sp) s += part[(int64_t)sp * ka * kb + e];
  G[(int64_t)a * kb + b] = s;
  if (symmetric && a != b) G[(int64_t)b * kb + a] = s;
}

// Out[I, 0:KP] = A[I, 0:kin] * R[0:kin, 0:KP]; CTA = 128 rows, KP (<= 256) output columns in
// registers (8 x KPT per thread).  kin is a multiple of 16; R has leading dimension ldr.
template <int KPT>
__global__ void __launch_bounds__(256, 1)
apply_right_kernel(const float *__restrict__ A, int64_t lda, int kin, int64_t n,
                   const float *__restrict__ R, int64_t ldr, float *Out, int64_t ldo) {
  constexpr int KP = KPT * 16;
  constexpr int TM = 16;
  __shared__ __align__(16) float As[TM][128 + 4];
  __shared__ __align__(16) float Rs[TM][KP];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t i0 = (int64_t)blockIdx.x * 128;
  float acc[8][KPT];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < KPT; ++c) acc[r][c] = 0.f;
  for (int m0 = 0; m0 < kin; m0 += TM) {
    __syncthreads();
    for (int e = tid; e < 128 * TM; e += 256) {
      const int r = e / TM, c = e % TM;
      const int64_t gi = i0 + r;
      As[c][r] = gi < n ? A[gi * lda + m0 + c] : 0.f;
    }
    for (int e = tid; e < TM * KP / 4; e += 256) {
      const int r = e / (KP / 4), c4 = e % (KP / 4);
      reinterpret_cast<float4 *>(&Rs[r][0])[c4] =
          reinterpret_cast<const float4 *>(R + (int64_t)(m0 + r) * ldr)[c4];
    }
    __syncthreads();
#pragma unroll 4
    for (int m = 0; m < TM; ++m) {
      float a[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) a[r] = As[m][ty * 8 + r];
#pragma unroll
      for (int q = 0; q < KPT / 4; ++q) {
        const float4 b = reinterpret_cast<const float4 *>(&Rs[m][q * 64])[tx];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          acc[r][4 * q + 0] = fmaf(a[r], b.x, acc[r][4 * q + 0]);
          acc[r][4 * q + 1] = fmaf(a[r], b.y, acc[r][4 * q + 1]);
          acc[r][4 * q + 2] = fmaf(a[r], b.z, acc[r][4 * q + 2]);
          acc[r][4 * q + 3] = fmaf(a[r], b.w, acc[r][4 * q + 3]);
        }
      }
    }
  }
  __syncthreads();  // all reads of this CTA's rows done before in-place writes
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t gi = i0 + ty * 8 + r;
    if (gi >= n) continue;
#pragma unroll
    for (int q = 0; q < KPT / 4; ++q)
      reinterpret_cast<float4 *>(Out + gi * ldo + q * 64)[tx] =
          make_float4(acc[r][4 * q], acc[r][4 * q + 1], acc[r][4 * q + 2], acc[r][4 * q + 3]);
  }
}

template <int KPT>
tsvm_status launch_apply(tsvm_context *ctx, const float *A, int64_t lda, int kin, int64_t n,
                         const float *R, int64_t ldr, float *Out, int64_t ldo) {
  apply_right_kernel<KPT><<<(unsigned)ceil_div(n, 128), 256, 0, ctx->stream>>>(
      A, lda, kin, n, R, ldr, Out, ldo);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status apply_slab(tsvm_context *ctx, const float *A, int64_t lda, int kin, int64_t n,
                       const float *R, int64_t ldr, int width, float *Out, int64_t ldo) {
  switch (width / 16) {
    case 4: return launch_apply<4>(ctx, A, lda, kin, n, R, ldr, Out, ldo);
    case 8: return launch_apply<8>(ctx, A, lda, kin, n, R, ldr, Out, ldo);
    case 12: return launch_apply<12>(ctx, A, lda, kin, n, R, ldr, Out, ldo);
    case 16: return launch_apply<16>(ctx, A, lda, kin, n, R, ldr, Out, ldo);
    default: return TSVM_ERR_UNSUPPORTED;
  }
}

}  // namespace

tsvm_status gram_fp64(tsvm_context *ctx, const float *A, int64_t lda, const float *B,
                      int64_t ldb, int64_t n, int ka, int kb, bool symmetric, double *G,
                      const double *rowscale) {
  const int tiles_a = (int)ceil_div(ka, kGT), tiles_b = (int)ceil_div(kb, kGT);
  const int ntiles = symmetric ? tiles_a * (tiles_a + 1) / 2 : tiles_a * tiles_b;
  const int target = ctx->num_sms * 4;
  int nsplit = (int)ceil_div(target, ntiles);
  const int64_t max_split = ceil_div(n, kGRows);
  if (nsplit > max_split) nsplit = (int)max_split;
  if (nsplit < 1) nsplit = 1;
  const int64_t rows_per_split = round_up(ceil_div(n, nsplit), kGRows);
  nsplit = (int)ceil_div(n, rows_per_split);
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_PART, (size_t)nsplit * ka * kb, &part));
  gram_partial_kernel<<<dim3(ntiles, nsplit), 256, 0, ctx->stream>>>(
      A, lda, B, ldb, n, ka, kb, tiles_b, symmetric ? 1 : 0, rows_per_split, rowscale, nullptr,
      nullptr, nullptr, nullptr, nullptr, part);
  TSVM_LAUNCHED(ctx);
  const int64_t tot = (int64_t)ka * kb;
  gram_reduce_kernel<<<(unsigned)ceil_div(tot, 256), 256, 0, ctx->stream>>>(
      part, nsplit, ka, kb, symmetric ? 1 : 0, G);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status gram_fp64_rows(tsvm_context *ctx, const float *A, int64_t lda, int64_t n_max, int k,
                           const int64_t *rowidx, const int *count_dev, const double *rowscale,
                           double *G) {
  const int tiles = (int)ceil_div(k, kGT);
  const int ntiles = tiles * (tiles + 1) / 2;
  int nsplit = (int)ceil_div(ctx->num_sms * 4, ntiles);
  const int64_t max_split = ceil_div(n_max, kGRows);
  if (nsplit > max_split) nsplit = (int)max_split;
  if (nsplit < 1) nsplit = 1;
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_PART, (size_t)nsplit * k * k, &part));
  gram_partial_kernel<<<dim3(ntiles, nsplit), 256, 0, ctx->stream>>>(
      A, lda, A, lda, n_max, k, k, tiles, 1, 0, rowscale, rowidx, count_dev, nullptr, nullptr,
      nullptr, part);
  TSVM_LAUNCHED(ctx);
  gram_reduce_kernel<<<(unsigned)ceil_div((int64_t)k * k, 256), 256, 0, ctx->stream>>>(
      part, nsplit, k, k, 1, G);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status gram_fp64_units(tsvm_context *ctx, const float *const *Zs, int64_t lda, int k,
                            const WorkUnit *units, int nunits, const int *active,
                            const double *rowscale, double *part) {
  if (nunits < 1 || nunits > 65535) return TSVM_ERR_UNSUPPORTED;
  const int tiles = (int)ceil_div(k, kGT);
  const int ntiles = tiles * (tiles + 1) / 2;
  gram_partial_kernel<<<dim3(ntiles, nunits), 256, 0, ctx->stream>>>(
      nullptr, lda, nullptr, lda, 0, k, k, tiles, 1, 0, rowscale, nullptr, nullptr, units, Zs,
      active, part);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status apply_right_fp32(tsvm_context *ctx, const float *A, int64_t n, int kp,
                             const float *R, float *Out) {
  if (kp % 64 != 0) return TSVM_ERR_UNSUPPORTED;
  if (kp <= 256) return apply_slab(ctx, A, kp, kp, n, R, kp, kp, Out, kp);
  // wider factors: 256-column output slabs; in-place needs a staging copy of A
  const float *src = A;
  if (Out == A) {
    float *tmp = nullptr;
    TSVM_TRY(scratch_t(ctx, SLOT_W2, (size_t)n * kp, &tmp));
    TSVM_CUDA(cudaMemcpyAsync(tmp, A, (size_t)n * kp * sizeof(float), cudaMemcpyDeviceToDevice,
                              ctx->stream));
    src = tmp;
  }
  for (int c0 = 0; c0 < kp; c0 += 256) {
    const int w = kp - c0 < 256 ? kp - c0 : 256;
    TSVM_TRY(apply_slab(ctx, src, kp, kp, n, R + c0, kp, w, Out + c0, kp));
  }
  return TSVM_OK;
}

}  // namespace tsvm
