// Decision values of a trained model and the factor's Frobenius residual (-analysis).
//
// Decision values replace the external predictor the reference hands its model file to
// (ThunderSVM, README.md:27-31; the reference's own `predict`, tensorsvm-train.cu:166-270, is
// never called): f(x) = sum_i coef_i exp(-gamma ||sv_i - x||^2) - rho for the RBF model file
// (coef_i = y_i alpha_i, rho = -b, writemodel tensorsvm-train.cu:384-406), f(x) = w . x - rho
// for the LIBLINEAR one (tensorsvm-train.cu:340-349).  One thread per test row keeps the row in
// registers; support vectors stream through shared memory 64 at a time.  Distances come from
// differences (no ||x||^2 + ||y||^2 - 2 x.y cancellation), exp in FP32, each tile's 64 terms
// summed in FP32 and the tiles in FP64.
//
// The residual replaces rbf_fnorm_res (tensorsvm-train.cu:2388-2467, driven by -analysis,
// 2328-2360): ||K~||_F and ||K~ - Z Z^T||_F with K~_ij = y_i y_j exp(-gamma ||x_i - x_j||^2),
// all in FP64.  The reference builds each 8192 x 8192 block of K~ in memory and reduces it
// with two more passes; here one persistent kernel walks the 64 x 64 tiles of the lower
// triangle (off-diagonal tiles count twice), forms K~ and Z Z^T for a tile in registers and
// keeps only the two sums.
#include <math.h>

#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace tsvm {
namespace {

constexpr int kPR = 256;   // rows per block (one per thread)
constexpr int kPT = 64;    // support vectors per shared-memory tile

template <int DC>
__global__ void __launch_bounds__(kPR)
decision_rbf_kernel(const float *__restrict__ X, int64_t m, int d, const float *__restrict__ SV,
                    int64_t nsv, const double *__restrict__ coef, float gl2, double rho,
                    double *__restrict__ f) {
  __shared__ float S[kPT][DC + 1];
  __shared__ float cf[kPT];
  const int64_t v = (int64_t)blockIdx.x * kPR + threadIdx.x;
  float x[DC];
#pragma unroll
  for (int c = 0; c < DC; ++c) x[c] = (v < m && c < d) ? X[v * d + c] : 0.f;
  double acc = 0.0;
  for (int64_t i0 = 0; i0 < nsv; i0 += kPT) {
    __syncthreads();
    for (int e = threadIdx.x; e < kPT * DC; e += kPR) {
      const int r = e / DC, c = e % DC;
      const int64_t i = i0 + r;
      S[r][c] = (i < nsv && c < d) ? SV[i * d + c] : 0.f;
    }
    for (int r = threadIdx.x; r < kPT; r += kPR)
      cf[r] = i0 + r < nsv ? (float)coef[i0 + r] : 0.f;
    __syncthreads();
    const int rn = (int)(nsv - i0 < kPT ? nsv - i0 : kPT);
    float part = 0.f;
    for (int r = 0; r < rn; ++r) {
      float d2 = 0.f;
#pragma unroll
      for (int c = 0; c < DC; ++c) {
        const float t = x[c] - S[r][c];
        d2 = fmaf(t, t, d2);
      }
      float e;
      asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-gl2 * d2));
      part = fmaf(e, cf[r], part);
    }
    acc += (double)part;
  }
  if (v < m) f[v] = acc - rho;
}

// d > 64: the row is re-read in 32-feature chunks for every tile of 32 support vectors.
constexpr int kCT = 32;
__global__ void __launch_bounds__(kPR)
decision_rbf_wide_kernel(const float *__restrict__ X, int64_t m, int d,
                         const float *__restrict__ SV, int64_t nsv,
                         const double *__restrict__ coef, float gl2, double rho,
                         double *__restrict__ f) {
  __shared__ float S[kCT][kCT + 1];
  const int64_t v = (int64_t)blockIdx.x * kPR + threadIdx.x;
  const int64_t vr = v < m ? v : m - 1;
  double acc = 0.0;
  for (int64_t i0 = 0; i0 < nsv; i0 += kCT) {
    float d2[kCT];
#pragma unroll
    for (int r = 0; r < kCT; ++r) d2[r] = 0.f;
    for (int c0 = 0; c0 < d; c0 += kCT) {
      __syncthreads();
      for (int e = threadIdx.x; e < kCT * kCT; e += kPR) {
        const int r = e / kCT, c = e % kCT;
        const int64_t i = i0 + r;
        S[r][c] = (i < nsv && c0 + c < d) ? SV[i * d + c0 + c] : 0.f;
      }
      __syncthreads();
      float x[kCT];
#pragma unroll
      for (int c = 0; c < kCT; ++c) x[c] = c0 + c < d ? X[vr * d + c0 + c] : 0.f;
#pragma unroll
      for (int r = 0; r < kCT; ++r)
#pragma unroll
        for (int c = 0; c < kCT; ++c) {
          const float t = x[c] - S[r][c];
          d2[r] = fmaf(t, t, d2[r]);
        }
    }
    float part = 0.f;
#pragma unroll
    for (int r = 0; r < kCT; ++r) {
      if (i0 + r < nsv) {
        float e;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-gl2 * d2[r]));
        part = fmaf(e, (float)coef[i0 + r], part);
      }
    }
    acc += (double)part;
  }
  if (v < m) f[v] = acc - rho;
}

__global__ void decision_linear_kernel(const float *__restrict__ X, int64_t m, int d,
                                       const float *__restrict__ w, double rho,
                                       double *__restrict__ f) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m) return;
  double s = 0.0;
  for (int c = 0; c < d; ++c) s += (double)w[c] * (double)X[v * d + c];
  f[v] = s - rho;
}

// ---------------------------------------------------------------------------------------
// Frobenius residual
// ---------------------------------------------------------------------------------------
constexpr int kRT = 64;    // tile edge
constexpr int kRK = 16;    // columns (of Z or X) staged per step

// Tile t of the lower triangle (ti >= tj) in row-major order: t = ti (ti + 1) / 2 + tj.
__device__ __forceinline__ void tri_tile(int64_t t, int64_t &ti, int64_t &tj) {
  int64_t i = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > t) --i;
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  ti = i;
  tj = t - i * (i + 1) / 2;
}

// Block b takes the tiles b, b + G, ... and leaves (sum K~^2, sum (K~ - Z Z^T)^2) over them in
// part[2 b], part[2 b + 1]; each thread owns a 4 x 4 sub-block of the tile.
__global__ void __launch_bounds__(256)
residual_kernel(const float *__restrict__ X, const float *__restrict__ y, int64_t n, int d,
                const float *__restrict__ Z, int64_t ldz, int k, double gamma, int64_t ntiles,
                double *__restrict__ part) {
  __shared__ double Ai[kRK][kRT + 1];
  __shared__ double Aj[kRK][kRT + 1];
  __shared__ double sh[16];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double s_k = 0.0, s_r = 0.0;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int64_t ti, tj;
    tri_tile(t, ti, tj);
    const int64_t i0 = ti * kRT, j0 = tj * kRT;
    double G[4][4], D[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) G[a][b] = D[a][b] = 0.0;
    // Z Z^T over k, then squared distances over d (two operand kinds, one staging loop)
    for (int pass = 0; pass < 2; ++pass) {
      const float *A = pass == 0 ? Z : X;
      const int64_t lda = pass == 0 ? ldz : d;
      const int kk = pass == 0 ? k : d;
      for (int c0 = 0; c0 < kk; c0 += kRK) {
        __syncthreads();
        for (int e = threadIdx.x; e < kRK * kRT; e += 256) {
          const int r = e / kRK, c = e % kRK;
          const bool cin = c0 + c < kk;
          const int64_t gi = i0 + r, gj = j0 + r;
          Ai[c][r] = (cin && gi < n) ? (double)A[gi * lda + c0 + c] : 0.0;
          Aj[c][r] = (cin && gj < n) ? (double)A[gj * lda + c0 + c] : 0.0;
        }
        __syncthreads();
        const int cn = kk - c0 < kRK ? kk - c0 : kRK;
        for (int c = 0; c < cn; ++c) {
          double av[4], bv[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) av[a] = Ai[c][ty + 16 * a];
#pragma unroll
          for (int b = 0; b < 4; ++b) bv[b] = Aj[c][tx + 16 * b];
          if (pass == 0) {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int b = 0; b < 4; ++b) G[a][b] = fma(av[a], bv[b], G[a][b]);
          } else {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int b = 0; b < 4; ++b) {
                const double q = av[a] - bv[b];
                D[a][b] = fma(q, q, D[a][b]);
              }
          }
        }
      }
    }
    const double w = ti == tj ? 1.0 : 2.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int64_t gi = i0 + ty + 16 * a;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int64_t gj = j0 + tx + 16 * b;
        if (gi < n && gj < n) {
          const double kv = (double)y[gi] * (double)y[gj] * exp(-gamma * D[a][b]);
          const double r = kv - G[a][b];
          s_k += w * kv * kv;
          s_r += w * r * r;
        }
      }
    }
  }
  double v[2] = {s_k, s_r};
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = v[0];
    part[2 * blockIdx.x + 1] = v[1];
  }
}

__global__ void residual_finish(const double *__restrict__ part, int nb, double *__restrict__ out) {
  if (threadIdx.x != 0) return;
  double a = 0.0, b = 0.0;
  for (int i = 0; i < nb; ++i) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  out[0] = sqrt(a);
  out[1] = sqrt(b);
}

}  // namespace

tsvm_status decision_values(tsvm_context *ctx, const tsvm_model_view *mv, const float *X,
                            int64_t m, double *f) {
  const unsigned g = (unsigned)ceil_div(m, kPR);
  if (mv->kernel == TSVM_KERNEL_LINEAR) {
    decision_linear_kernel<<<g, kPR, 0, ctx->stream>>>(X, m, mv->d, mv->sv, mv->rho, f);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
  const float gl2 = (float)(mv->gamma * 1.4426950408889634);
  const int d = mv->d;
  if (d <= 16)
    decision_rbf_kernel<16><<<g, kPR, 0, ctx->stream>>>(X, m, d, mv->sv, mv->nsv, mv->coef, gl2,
                                                         mv->rho, f);
  else if (d <= 24)
    decision_rbf_kernel<24><<<g, kPR, 0, ctx->stream>>>(X, m, d, mv->sv, mv->nsv, mv->coef, gl2,
                                                         mv->rho, f);
  else if (d <= 32)
    decision_rbf_kernel<32><<<g, kPR, 0, ctx->stream>>>(X, m, d, mv->sv, mv->nsv, mv->coef, gl2,
                                                         mv->rho, f);
  else if (d <= 64)
    decision_rbf_kernel<64><<<g, kPR, 0, ctx->stream>>>(X, m, d, mv->sv, mv->nsv, mv->coef, gl2,
                                                         mv->rho, f);
  else
    decision_rbf_wide_kernel<<<g, kPR, 0, ctx->stream>>>(X, m, d, mv->sv, mv->nsv, mv->coef, gl2,
                                                         mv->rho, f);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status kernel_residual(tsvm_context *ctx, const float *X, const float *y, int64_t n, int d,
                            double gamma, const float *Z, int64_t ldz, int k, double *out2) {
  const int64_t nt = ceil_div(n, kRT);
  const int64_t ntiles = nt * (nt + 1) / 2;
  const int nb = (int)std::min<int64_t>(ntiles, (int64_t)ctx->num_sms * 4);
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, (size_t)2 * nb + 8, &part));
  double *res = part + 2 * nb;
  residual_kernel<<<nb, 256, 0, ctx->stream>>>(X, y, n, d, Z, ldz, k, gamma, ntiles, part);
  TSVM_LAUNCHED(ctx);
  residual_finish<<<1, 32, 0, ctx->stream>>>(part, nb, res);
  TSVM_LAUNCHED(ctx);
  TSVM_CUDA(cudaMemcpyAsync(out2, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  return TSVM_OK;
}

}  // namespace tsvm
