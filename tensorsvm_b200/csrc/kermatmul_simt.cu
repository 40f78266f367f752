// FP32 SIMT fused kernel-block product: W = (Y K Y) A without materialising K.
//
// Replaces rbf_kermatmul + vecnorm + rbf_kergen + the XIJ and K*A cuBLAS SGEMMs
// (tensorsvm-train.cu:2476-2612) and the host chunk loop RBF_KERMATMUL (1999-2063).
// One CTA owns 128 rows I of W and all kp columns; it walks every 32-row tile J of X:
//   S_IJ = Xc_I Xc_J^T (d-long dot products), P = y_i y_j exp2(-gamma log2(e) (n_i + n_j - 2 S)),
//   W_I += P A_J        (8 x kp/16 register tile per thread).
// The kernel block P lives only in shared memory; X, y, A stay resident in HBM.
// This is the "plain FP32" form of the contraction; kermatmul_tc.cu is the tcgen05 form.
#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
namespace {

constexpr int kTI = 128;   // rows of W per CTA
constexpr int kTJ = 32;    // rows of X / A per inner tile
constexpr int kMaxD = 64;

// KPT = columns per thread (kp / 16); thread (ty, tx) owns rows ty*8..+8 and the column
// groups {tx*4 + 64*m + 0..3 : m < KPT/4}.
template <int KPT>
__global__ void __launch_bounds__(256, 1)
kermatmul_simt_kernel(const float *__restrict__ Xc, const float *__restrict__ norms,
                      const float *__restrict__ y, int64_t n, int d, float g2,
                      const float *__restrict__ A, float *__restrict__ W, int64_t i_begin,
                      int64_t i_end) {
  constexpr int KP = KPT * 16;
  extern __shared__ float4 smem4[];
  float *sm = reinterpret_cast<float *>(smem4);
  float *XI = sm;                       // [d][kTI]
  float *XJ = XI + kMaxD * kTI;         // [d][kTJ]
  float *P = XJ + kMaxD * kTJ;          // [kTJ][kTI]
  float *AJ = P + kTJ * kTI;            // [kTJ][KP]
  float *nI = AJ + kTJ * KP;            // [kTI]
  float *yI = nI + kTI;                 // [kTI]
  float *nJ = yI + kTI;                 // [kTJ]
  float *yJ = nJ + kTJ;                 // [kTJ]

  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  // rows I of this CTA: [i0, i0 + kTI) within [i_begin, i_end); J runs over all n rows
  const int64_t i0 = i_begin + (int64_t)blockIdx.x * kTI;

  for (int e = tid; e < kTI * d; e += 256) {
    const int r = e / d, c = e % d;
    const int64_t gi = i0 + r;
    XI[c * kTI + r] = gi < i_end ? Xc[gi * d + c] : 0.f;
  }
  for (int r = tid; r < kTI; r += 256) {
    const int64_t gi = i0 + r;
    nI[r] = gi < i_end ? norms[gi] : 0.f;
    yI[r] = gi < i_end ? y[gi] : 0.f;
  }

  float acc[8][KPT];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < KPT; ++c) acc[r][c] = 0.f;

  // P-phase assignment: thread computes rows pi and columns pj0..pj0+3 of the 128 x 32 block.
  const int pi = tid & 127;
  const int pj0 = (tid >> 7) * 16;

  for (int64_t j0 = 0; j0 < n; j0 += kTJ) {
    __syncthreads();  // previous tile fully consumed
    for (int e = tid; e < kTJ * d; e += 256) {
      const int r = e / d, c = e % d;
      const int64_t gj = j0 + r;
      XJ[c * kTJ + r] = gj < n ? Xc[gj * d + c] : 0.f;
    }
    if (tid < kTJ) {
      const int64_t gj = j0 + tid;
      nJ[tid] = gj < n ? norms[gj] : 0.f;
      yJ[tid] = gj < n ? y[gj] : 0.f;   // y = 0 beyond n zeroes the padded columns of P
    }
    for (int e = tid; e < kTJ * KP / 4; e += 256) {
      const int r = e / (KP / 4), c4 = e % (KP / 4);
      const int64_t gj = j0 + r;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (gj < n) v = reinterpret_cast<const float4 *>(A + gj * KP)[c4];
      reinterpret_cast<float4 *>(AJ + r * KP)[c4] = v;
    }
    __syncthreads();
    {
      float s[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) s[q] = 0.f;
      for (int c = 0; c < d; ++c) {
        const float xi = XI[c * kTI + pi];
#pragma unroll
        for (int q = 0; q < 16; ++q) s[q] = fmaf(xi, XJ[c * kTJ + pj0 + q], s[q]);
      }
      const float ni = nI[pi], yi = yI[pi];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float dist = fmaxf(ni + nJ[pj0 + q] - 2.f * s[q], 0.f);
        P[(pj0 + q) * kTI + pi] = yi * yJ[pj0 + q] * exp2f(g2 * dist);
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int j = 0; j < kTJ; ++j) {
      const float4 a0 = reinterpret_cast<const float4 *>(P + j * kTI + ty * 8)[0];
      const float4 a1 = reinterpret_cast<const float4 *>(P + j * kTI + ty * 8)[1];
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
      for (int m = 0; m < KPT / 4; ++m) {
        const float4 b = reinterpret_cast<const float4 *>(AJ + j * KP + m * 64)[tx];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          acc[r][4 * m + 0] = fmaf(a[r], b.x, acc[r][4 * m + 0]);
          acc[r][4 * m + 1] = fmaf(a[r], b.y, acc[r][4 * m + 1]);
          acc[r][4 * m + 2] = fmaf(a[r], b.z, acc[r][4 * m + 2]);
          acc[r][4 * m + 3] = fmaf(a[r], b.w, acc[r][4 * m + 3]);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t gi = i0 + ty * 8 + r;
    if (gi >= i_end) continue;
#pragma unroll
    for (int m = 0; m < KPT / 4; ++m)
      reinterpret_cast<float4 *>(W + (gi - i_begin) * KP + m * 64)[tx] =
          make_float4(acc[r][4 * m + 0], acc[r][4 * m + 1], acc[r][4 * m + 2], acc[r][4 * m + 3]);
  }
}

template <int KPT>
tsvm_status launch_simt(tsvm_context *ctx, const float *Xc, const float *norms, const float *y,
                        int64_t n, int d, float g2, const float *A, float *W, int64_t row0,
                        int64_t nr) {
  constexpr int KP = KPT * 16;
  const size_t smem = sizeof(float) * (size_t)(kMaxD * kTI + kMaxD * kTJ + kTJ * kTI + kTJ * KP +
                                               2 * kTI + 2 * kTJ);
  TSVM_CUDA(cudaFuncSetAttribute(kermatmul_simt_kernel<KPT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kermatmul_simt_kernel<KPT><<<(unsigned)ceil_div(nr, kTI), 256, smem, ctx->stream>>>(
      Xc, norms, y, n, d, g2, A, W, row0, row0 + nr);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

}  // namespace

tsvm_status kermatmul_fp32(tsvm_context *ctx, const float *Xc, const float *norms,
                           const float *y, int64_t n, int d, double gamma, const float *A,
                           int kp, float *W, int64_t row0, int64_t nr) {
  if (d < 1 || d > kMaxD || kp % 64 != 0 || kp <= 0) return TSVM_ERR_UNSUPPORTED;
  if (nr < 0) nr = n - row0;
  if (row0 < 0 || nr < 1 || row0 + nr > n) return TSVM_ERR_INVALID_ARGUMENT;
  const float g2 = (float)(-gamma * 1.4426950408889634);
  // Columns are processed in chunks of at most 256 (the register tile); each chunk is an
  // independent launch over a column slice of A and W with the same leading dimension kp.
  // Chunk slices need a matching leading dimension, so A and W are addressed with ld = kp by
  // launching on compact per-chunk copies when kp > 256.
  if (kp <= 256) {
    switch (kp / 16) {
      case 4: return launch_simt<4>(ctx, Xc, norms, y, n, d, g2, A, W, row0, nr);
      case 8: return launch_simt<8>(ctx, Xc, norms, y, n, d, g2, A, W, row0, nr);
      case 12: return launch_simt<12>(ctx, Xc, norms, y, n, d, g2, A, W, row0, nr);
      case 16: return launch_simt<16>(ctx, Xc, norms, y, n, d, g2, A, W, row0, nr);
      default: return TSVM_ERR_UNSUPPORTED;
    }
  }
  // kp > 256: split columns into 256-wide slabs (plus remainder) through compact buffers.
  float *Ac = nullptr, *Wc = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_W2, (size_t)(n + nr) * 256, &Ac));
  Wc = Ac + (size_t)n * 256;
  for (int c0 = 0; c0 < kp; c0 += 256) {
    const int w = kp - c0 < 256 ? kp - c0 : 256;
    TSVM_CUDA(cudaMemcpy2DAsync(Ac, (size_t)w * 4, A + c0, (size_t)kp * 4, (size_t)w * 4, n,
                                cudaMemcpyDeviceToDevice, ctx->stream));
    TSVM_TRY(kermatmul_fp32(ctx, Xc, norms, y, n, d, gamma, Ac, w, Wc, row0, nr));
    TSVM_CUDA(cudaMemcpy2DAsync(W + c0, (size_t)kp * 4, Wc, (size_t)w * 4, (size_t)w * 4, nr,
                                cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return TSVM_OK;
}

}  // namespace tsvm
