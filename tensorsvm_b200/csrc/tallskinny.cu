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

// One staged slab into a thread's 4 x 4 block of the tile (rows ty + 16 i, columns tx + 16 j).
// DIAG (a diagonal tile of a symmetric product, of which only the lower triangle is used): the
// blocks i < j lie wholly above the diagonal and are skipped, 6 of the 16 products a row.
template <bool DIAG>
__device__ __forceinline__ void gram_slab(const double (*As)[kGT], const double (*Bs)[kGT], int tx,
                                          int ty, double (&acc)[4][4]) {
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
      for (int j = 0; j < 4; ++j)
        if (!DIAG || i >= j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
  }
}

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
  int64_t rows_beg = 0;
  if (units) {  // batched: this block sums the rows of one work unit (symmetric, A = B)
    const WorkUnit u = units[blockIdx.y];
    if (active && !active[u.p]) return;
    A = Zs[u.p] + u.row0 * lda;
    B = A;
    n = u.rows;
    rows_per_split = u.rows;
    rowscale += u.goff;
    if (count) {   // only the unit's listed rows (indices within the unit) at rowidx + goff,
                   // the list cut into gridDim.z parts of whole slabs; an empty part writes
                   // nothing (the reduction skips it)
      const int cnt = count[blockIdx.y], S = (int)gridDim.z;
      const int per = ((cnt + S - 1) / S + kGRows - 1) / kGRows * kGRows;
      const int b = (int)blockIdx.z * per;
      if (b >= cnt) return;
      rows_beg = b;
      n = min(cnt, b + per);
      rows_per_split = n - b;
      rowidx += u.goff;
    }
  } else if (count) {  // row count on the device: split it evenly over gridDim.y
    n = *count;
    rows_per_split = (n + gridDim.y - 1) / gridDim.y;
    rows_per_split = (rows_per_split + kGRows - 1) / kGRows * kGRows;
  }
  const int64_t r0 = units ? rows_beg : (int64_t)blockIdx.y * rows_per_split;
  const int64_t r1 = min(n, r0 + rows_per_split);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  // a tile on the diagonal of a symmetric product: only its lower triangle is read back
  const bool diag = symmetric && ta == tb;
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
    if (diag)
      gram_slab<true>(As, Bs, tx, ty, acc);
    else
      gram_slab<false>(As, Bs, tx, ty, acc);
  }
  // partial layout: [split][ka][kb] (batched: [unit][part][ka][kb])
  double *P = part + ((int64_t)blockIdx.y * gridDim.z + blockIdx.z) * ka * kb;
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

// Asynchronous 16-byte global -> shared copies (LDGSTS), grouped and waited on per stage.
__device__ __forceinline__ void cp_async16(float *dst, const float *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Out[I, 0:KP] = A[I, 0:kin] * R[0:kin, 0:KP]; CTA = 128 rows, KP (<= 256) output columns in
// registers (8 x KPT per thread).  kin is a multiple of 32; A's and R's rows start on 16-byte
// boundaries (lda, ldr multiples of 4).  32-deep K slabs of A (row-major, padded rows) and R
// are staged in two shared-memory stages by cp.async, the next slab in flight while the
// current one is multiplied.  Out may be A itself: a CTA writes its rows after it has read all
// of them, and no other CTA reads them.
constexpr int kApTM = 32;            // K slab
constexpr int kApAP = kApTM + 4;     // padded A row in shared memory (floats)
template <int KPT>
constexpr size_t apply_smem() {
  return sizeof(float) * 2 * ((size_t)128 * kApAP + (size_t)kApTM * KPT * 16);
}

template <int KPT>
__global__ void __launch_bounds__(256, 1)
apply_right_kernel(const float *__restrict__ A, int64_t lda, int kin, int64_t n,
                   const float *__restrict__ R, int64_t ldr, float *Out, int64_t ldo) {
  constexpr int KP = KPT * 16, TM = kApTM, AP = kApAP;
  extern __shared__ __align__(16) float apsm[];
  float *const As0 = apsm;                    // [2][128][AP]
  float *const Rs0 = apsm + 2 * 128 * AP;     // [2][TM][KP]
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t i0 = (int64_t)blockIdx.x * 128;
  auto load = [&](int stage, int m0) {
    float *As = As0 + stage * 128 * AP;
    float *Rs = Rs0 + stage * TM * KP;
    for (int e = tid; e < 128 * (TM / 4); e += 256) {
      const int r = e / (TM / 4), c4 = e % (TM / 4);
      const int64_t gi = i0 + r;
      float *dst = As + r * AP + 4 * c4;
      if (gi < n)
        cp_async16(dst, A + gi * lda + m0 + 4 * c4);
      else
        *reinterpret_cast<float4 *>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int e = tid; e < TM * (KP / 4); e += 256) {
      const int r = e / (KP / 4), c4 = e % (KP / 4);
      cp_async16(Rs + r * KP + 4 * c4, R + (int64_t)(m0 + r) * ldr + 4 * c4);
    }
    cp_async_commit();
  };
  float acc[8][KPT];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < KPT; ++c) acc[r][c] = 0.f;
  load(0, 0);
  for (int m0 = 0, st = 0; m0 < kin; m0 += TM, st ^= 1) {
    if (m0 + TM < kin) {
      load(st ^ 1, m0 + TM);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const float *As = As0 + st * 128 * AP;
    const float *Rs = Rs0 + st * TM * KP;
#pragma unroll 4
    for (int m = 0; m < TM; ++m) {
      float a[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) a[r] = As[(ty * 8 + r) * AP + m];
#pragma unroll
      for (int q = 0; q < KPT / 4; ++q) {
        const float4 b = reinterpret_cast<const float4 *>(Rs + m * KP + q * 64)[tx];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          acc[r][4 * q + 0] = fmaf(a[r], b.x, acc[r][4 * q + 0]);
          acc[r][4 * q + 1] = fmaf(a[r], b.y, acc[r][4 * q + 1]);
          acc[r][4 * q + 2] = fmaf(a[r], b.z, acc[r][4 * q + 2]);
          acc[r][4 * q + 3] = fmaf(a[r], b.w, acc[r][4 * q + 3]);
        }
      }
    }
    __syncthreads();   // this stage is read out before the next iteration refills it
  }
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
  if (kin % kApTM != 0 || lda % 4 != 0 || ldr % 4 != 0 ||
      (reinterpret_cast<uintptr_t>(A) & 15) != 0 || (reinterpret_cast<uintptr_t>(R) & 15) != 0)
    return TSVM_ERR_UNSUPPORTED;
  constexpr size_t smem = apply_smem<KPT>();
  TSVM_CUDA(cudaFuncSetAttribute(apply_right_kernel<KPT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  apply_right_kernel<KPT><<<(unsigned)ceil_div(n, 128), 256, smem, ctx->stream>>>(
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
                            const double *rowscale, double *part, const int64_t *rowidx,
                            const int *counts, int parts) {
  if (nunits < 1 || nunits > 65535) return TSVM_ERR_UNSUPPORTED;
  if ((rowidx == nullptr) != (counts == nullptr)) return TSVM_ERR_INVALID_ARGUMENT;
  if (parts < 1 || parts > 64 || (parts > 1 && !counts)) return TSVM_ERR_INVALID_ARGUMENT;
  const int tiles = (int)ceil_div(k, kGT);
  const int ntiles = tiles * (tiles + 1) / 2;
  gram_partial_kernel<<<dim3(ntiles, nunits, parts), 256, 0, ctx->stream>>>(
      nullptr, lda, nullptr, lda, 0, k, k, tiles, 1, 0, rowscale, rowidx, counts, units, Zs,
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
