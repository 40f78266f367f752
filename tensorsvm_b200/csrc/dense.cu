// Small dense FP64 linear algebra on the device for the k x k matrices of the path
// (k <= 1024).  These replace host LAPACK calls of the reference:
//   LAPACKE_dpotrf (capacitance matrix, tensorsvm-train.cu:1709)   -> chol_fp64
//   LAPACKE_dpotrs (SMW solve, tensorsvm-train.cu:1834)             -> potrs_fp64
//   LAPACKE_dsyevd (C = V diag(w) V^T, tensorsvm-train.cu:2191)     -> eig_jacobi_fp64
// plus a triangular inverse used by the shifted CholeskyQR that replaces the TSQR.
// Matrices are row-major with leading dimension lda; only lower triangles are referenced
// where noted.
#include <math.h>

#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
namespace {

constexpr int kNB = 32;

// Left-looking blocked Cholesky in one CTA of 1024 threads.  For each 32-column block:
// (1) update the panel with the already factored columns (lanes = panel columns, one warp
// per row), (2) factor the diagonal block with one warp, (3) triangular solve of the panel
// rows below, one thread per row.
__global__ void __launch_bounds__(1024) chol_kernel(double *__restrict__ A, int n, int lda,
                                                    int *__restrict__ info) {
  extern __shared__ double sh[];
  __shared__ int fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  if (tid == 0) fail = 0;
  __syncthreads();
  for (int jb = 0; jb < n; jb += kNB) {
    const int nb = min(kNB, n - jb);
    const int ldp = jb + 1;  // padded row stride of the staged panel rows
    double *Lp = sh;         // [nb][jb] rows jb..jb+nb of L, columns 0..jb
    for (int e = tid; e < nb * jb; e += blockDim.x) {
      const int r = e / jb, c = e % jb;
      Lp[r * ldp + c] = A[(int64_t)(jb + r) * lda + c];
    }
    __syncthreads();
    // (1) A[i][jb+lane] -= sum_m L[i][m] L[jb+lane][m]  for i >= jb
    for (int i = jb + warp; i < n; i += nwarps) {
      if (lane < nb && jb + lane <= i) {
        const double *Li = A + (int64_t)i * lda;
        double s = 0.0;
        for (int m = 0; m < jb; ++m) s = fma(Li[m], Lp[lane * ldp + m], s);
        A[(int64_t)i * lda + jb + lane] -= s;
      }
    }
    __syncthreads();
    // (2) diagonal block, one warp, in shared memory
    double *Dg = sh;  // reuse: [nb][kNB + 1]
    for (int e = tid; e < nb * nb; e += blockDim.x) {
      const int r = e / nb, c = e % nb;
      Dg[r * (kNB + 1) + c] = (c <= r) ? A[(int64_t)(jb + r) * lda + jb + c] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      for (int c = 0; c < nb; ++c) {
        const double dcc = Dg[c * (kNB + 1) + c];
        if (!(dcc > 0.0)) {
          if (lane == 0 && !fail) fail = jb + c + 1;
          break;
        }
        const double dc = sqrt(dcc);
        __syncwarp();
        if (lane == c) Dg[c * (kNB + 1) + c] = dc;
        if (lane > c && lane < nb) Dg[lane * (kNB + 1) + c] /= dc;
        __syncwarp();
        if (lane > c && lane < nb) {
          const double lrc = Dg[lane * (kNB + 1) + c];
          for (int s2 = c + 1; s2 <= lane; ++s2)
            Dg[lane * (kNB + 1) + s2] -= lrc * Dg[s2 * (kNB + 1) + c];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (fail) break;
    for (int e = tid; e < nb * nb; e += blockDim.x) {
      const int r = e / nb, c = e % nb;
      if (c <= r) A[(int64_t)(jb + r) * lda + jb + c] = Dg[r * (kNB + 1) + c];
    }
    // (3) rows below: x L_d^T = a  ->  forward substitution per row
    for (int i = jb + nb + tid; i < n; i += blockDim.x) {
      double x[kNB];
      double *Ai = A + (int64_t)i * lda + jb;
#pragma unroll
      for (int c = 0; c < kNB; ++c) x[c] = c < nb ? Ai[c] : 0.0;
#pragma unroll
      for (int c = 0; c < kNB; ++c) {
        if (c < nb) {
          double v = x[c];
          for (int m = 0; m < c; ++m) v -= x[m] * Dg[c * (kNB + 1) + m];
          x[c] = v / Dg[c * (kNB + 1) + c];
        }
      }
#pragma unroll
      for (int c = 0; c < kNB; ++c)
        if (c < nb) Ai[c] = x[c];
    }
    __syncthreads();
  }
  if (tid == 0) *info = fail;
}

// Solve L L^T X = B for nrhs (<= 4) right-hand sides stored as rows of B.  One CTA.
__global__ void __launch_bounds__(512) potrs_kernel(const double *__restrict__ L, int n, int lda,
                                                    double *__restrict__ B, int nrhs, int ldb) {
  __shared__ double Dg[kNB][kNB + 1];
  __shared__ double yb[4][kNB];
  const int tid = threadIdx.x;
  // forward: L y = b
  for (int jb = 0; jb < n; jb += kNB) {
    const int nb = min(kNB, n - jb);
    for (int e = tid; e < nb * nb; e += blockDim.x) {
      const int r = e / nb, c = e % nb;
      Dg[r][c] = c <= r ? L[(int64_t)(jb + r) * lda + jb + c] : 0.0;
    }
    __syncthreads();
    if (tid < nrhs) {
      double *b = B + (int64_t)tid * ldb + jb;
      for (int c = 0; c < nb; ++c) {
        double v = b[c];
        for (int m = 0; m < c; ++m) v -= Dg[c][m] * yb[tid][m];
        yb[tid][c] = v / Dg[c][c];
        b[c] = yb[tid][c];
      }
    }
    __syncthreads();
    for (int e = tid; e < (n - jb - nb) * nrhs; e += blockDim.x) {
      const int i = jb + nb + e / nrhs, r = e % nrhs;
      const double *Li = L + (int64_t)i * lda + jb;
      double s = 0.0;
      for (int c = 0; c < nb; ++c) s = fma(Li[c], yb[r][c], s);
      B[(int64_t)r * ldb + i] -= s;
    }
    __syncthreads();
  }
  // backward: L^T x = y
  const int last = ((n - 1) / kNB) * kNB;
  for (int jb = last; jb >= 0; jb -= kNB) {
    const int nb = min(kNB, n - jb);
    for (int e = tid; e < nb * nb; e += blockDim.x) {
      const int r = e / nb, c = e % nb;
      Dg[r][c] = c <= r ? L[(int64_t)(jb + r) * lda + jb + c] : 0.0;
    }
    __syncthreads();
    if (tid < nrhs) {
      double *b = B + (int64_t)tid * ldb + jb;
      for (int c = nb - 1; c >= 0; --c) {
        double v = b[c];
        for (int m = c + 1; m < nb; ++m) v -= Dg[m][c] * yb[tid][m];
        yb[tid][c] = v / Dg[c][c];
        b[c] = yb[tid][c];
      }
    }
    __syncthreads();
    for (int e = tid; e < jb * nrhs; e += blockDim.x) {
      const int i = e / nrhs, r = e % nrhs;
      double s = 0.0;
      for (int m = 0; m < nb; ++m) s = fma(L[(int64_t)(jb + m) * lda + i], yb[r][m], s);
      B[(int64_t)r * ldb + i] -= s;
    }
    __syncthreads();
  }
}

// Column-parallel lower-triangular inverse: thread j produces column j of L^-1.
__global__ void trinv_kernel(const double *__restrict__ L, int n, int lda,
                             double *__restrict__ Linv) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int i = 0; i < j; ++i) Linv[(int64_t)i * lda + j] = 0.0;
  Linv[(int64_t)j * lda + j] = 1.0 / L[(int64_t)j * lda + j];
  for (int i = j + 1; i < n; ++i) {
    const double *Li = L + (int64_t)i * lda;
    double s = 0.0;
    for (int m = j; m < i; ++m) s = fma(Li[m], Linv[(int64_t)m * lda + j], s);
    Linv[(int64_t)i * lda + j] = -s / Li[i];
  }
}

__global__ void add_diag_kernel(double *A, int n, int lda, double shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(int64_t)i * lda + i] += shift;
}

__global__ void symmetrize_kernel(double *A, int n, int lda) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int r = (int)(e / n), c = (int)(e % n);
  if (c < r) {
    const double v = 0.5 * (A[(int64_t)r * lda + c] + A[(int64_t)c * lda + r]);
    A[(int64_t)r * lda + c] = v;
    A[(int64_t)c * lda + r] = v;
  }
}

// ---------------------------------------------------------------------------------------
// Cyclic Jacobi eigensolver (Golub & Van Loan, symmetric Schur 2x2 rotations) with the
// round-robin ("circle") ordering: each round applies ne/2 disjoint rotations at once.  A
// cooperative grid processes the rotation pairs of a round; rows p, q of the next iterate
// only need rows p, q of the current one and the table of all rotations, so one grid
// barrier per round suffices (ping-pong buffers).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int circle_player(int pos, int round, int ne) {
  if (pos == 0) return 0;
  return 1 + (pos - 1 + round) % (ne - 1);
}

__global__ void __launch_bounds__(256)
jacobi_kernel(double *__restrict__ A0, double *__restrict__ A1, double *__restrict__ Vt, int ne,
              int max_sweeps, double tol, GridBarrier *gb, double *__restrict__ acc,
              int *__restrict__ sweeps_out) {
  extern __shared__ double jsh[];
  double *cs = jsh;                                   // [ne] coefficient c for index i
  double *sn = cs + ne;                               // [ne] coefficient s (signed) for index i
  int *partner = reinterpret_cast<int *>(sn + ne);    // [ne]
  const unsigned G = gridDim.x;
  double *cur = A0, *nxt = A1;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    for (int round = 0; round < ne - 1; ++round) {
      // rotation table from the current iterate (every block computes all of it)
      for (int m = threadIdx.x; m < ne / 2; m += blockDim.x) {
        const int p = circle_player(m, round, ne), q = circle_player(ne - 1 - m, round, ne);
        // buffers are rewritten by other blocks between rounds: read through L2 only
        const double app = __ldcg(cur + (int64_t)p * ne + p), aqq = __ldcg(cur + (int64_t)q * ne + q);
        const double apq = __ldcg(cur + (int64_t)p * ne + q);
        double c = 1.0, s = 0.0;
        if (fabs(apq) > 1e-300) {
          const double tau = (aqq - app) / (2.0 * apq);
          double t;
          if (fabs(tau) > 1e150) t = 0.5 / tau;
          else t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        cs[p] = c; sn[p] = -s; partner[p] = q;
        cs[q] = c; sn[q] = s;  partner[q] = p;
      }
      __syncthreads();
      for (int m = blockIdx.x; m < ne / 2; m += G) {
        const int p = circle_player(m, round, ne), q = circle_player(ne - 1 - m, round, ne);
        const double c = cs[p], s = -sn[p];
        const double *Ap = cur + (int64_t)p * ne, *Aq = cur + (int64_t)q * ne;
        double *Np = nxt + (int64_t)p * ne, *Nq = nxt + (int64_t)q * ne;
        for (int col = threadIdx.x; col < ne; col += blockDim.x) {
          const int pc = partner[col];
          const double cc = cs[col], sc = sn[col];
          const double bp = cc * __ldcg(Ap + col) + sc * __ldcg(Ap + pc);
          const double bq = cc * __ldcg(Aq + col) + sc * __ldcg(Aq + pc);
          __stcg(Np + col, c * bp - s * bq);
          __stcg(Nq + col, s * bp + c * bq);
        }
        double *Vp = Vt + (int64_t)p * ne, *Vq = Vt + (int64_t)q * ne;
        for (int r = threadIdx.x; r < ne; r += blockDim.x) {
          const double vp = __ldcg(Vp + r), vq = __ldcg(Vq + r);
          __stcg(Vp + r, c * vp - s * vq);
          __stcg(Vq + r, s * vp + c * vq);
        }
      }
      if (!grid_sync(gb, G)) { if (blockIdx.x == 0 && threadIdx.x == 0) *sweeps_out = -1; return; }
      double *t = cur; cur = nxt; nxt = t;
    }
    // convergence: off-diagonal mass against the diagonal, accumulated per block
    double off = 0.0, dia = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)ne * ne;
         e += (int64_t)G * blockDim.x) {
      const int r = (int)(e / ne), c = (int)(e % ne);
      const double v = __ldcg(cur + e);
      if (r == c) dia += v * v; else off += v * v;
    }
    off = warp_sum(off);
    dia = warp_sum(dia);
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&acc[2 * (sweep & 1)], off);
      atomicAdd(&acc[2 * (sweep & 1) + 1], dia);
    }
    if (!grid_sync(gb, G)) { if (blockIdx.x == 0 && threadIdx.x == 0) *sweeps_out = -1; return; }
    const double o = __ldcg(acc + 2 * (sweep & 1)), dsum = __ldcg(acc + 2 * (sweep & 1) + 1);
    if (!grid_sync(gb, G)) { if (blockIdx.x == 0 && threadIdx.x == 0) *sweeps_out = -1; return; }
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // clear the other parity slot for the next sweep
      acc[2 * ((sweep + 1) & 1)] = 0.0;
      acc[2 * ((sweep + 1) & 1) + 1] = 0.0;
    }
    if (o <= tol * tol * (dsum + o)) { ++sweep; break; }
  }
  // results: the converged iterate is `cur`; copy into A0 if it lives in A1
  if (cur != A0) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)ne * ne;
         e += (int64_t)G * blockDim.x)
      A0[e] = __ldcg(cur + e);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *sweeps_out = sweep;
}

__global__ void eig_pack_in(const double *__restrict__ A, int n, int lda, int ne,
                            double *__restrict__ A0, double *__restrict__ Vt) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)ne * ne) return;
  const int r = (int)(e / ne), c = (int)(e % ne);
  A0[e] = (r < n && c < n) ? A[(int64_t)r * lda + c] : 0.0;
  Vt[e] = (r == c) ? 1.0 : 0.0;
}

__global__ void eig_pack_out(const double *__restrict__ A0, const double *__restrict__ Vt, int n,
                             int ne, double *__restrict__ w, double *__restrict__ V) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int r = (int)(e / n), c = (int)(e % n);
  V[e] = Vt[(int64_t)c * ne + r];  // column c of V = row c of Vt
  if (c == 0) w[r] = A0[(int64_t)r * ne + r];
}

}  // namespace

tsvm_status chol_fp64(tsvm_context *ctx, double *A, int n, int lda, int *info_dev) {
  if (n < 1 || n > 864) return TSVM_ERR_UNSUPPORTED;  // staged panel must fit shared memory
  const size_t smem = sizeof(double) * (size_t)kNB * (size_t)(n + 1 > kNB + 1 ? n + 1 : kNB + 1);
  TSVM_CUDA(cudaFuncSetAttribute(chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  chol_kernel<<<1, 1024, smem, ctx->stream>>>(A, n, lda, info_dev);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status potrs_fp64(tsvm_context *ctx, const double *L, int n, int lda, double *B, int nrhs,
                       int ldb) {
  if (nrhs < 1 || nrhs > 4) return TSVM_ERR_UNSUPPORTED;
  potrs_kernel<<<1, 512, 0, ctx->stream>>>(L, n, lda, B, nrhs, ldb);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status trinv_lower_fp64(tsvm_context *ctx, const double *L, int n, int lda, double *Linv) {
  trinv_kernel<<<(unsigned)ceil_div(n, 64), 64, 0, ctx->stream>>>(L, n, lda, Linv);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status small_add_diag(tsvm_context *ctx, double *A, int n, int lda, double shift) {
  add_diag_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, ctx->stream>>>(A, n, lda, shift);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status small_symmetrize(tsvm_context *ctx, double *A, int n, int lda) {
  symmetrize_kernel<<<(unsigned)ceil_div((int64_t)n * n, 256), 256, 0, ctx->stream>>>(A, n, lda);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status eig_jacobi_fp64(tsvm_context *ctx, double *A, int n, int lda, double *w, double *V,
                            int *sweeps_out) {
  if (n < 1 || n > 1024) return TSVM_ERR_UNSUPPORTED;
  int ne = n + (n & 1);
  if (ne < 2) ne = 2;
  double *buf = nullptr;
  const size_t need = (size_t)3 * ne * ne + 8 + 4;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, need, &buf));
  double *A0 = buf, *A1 = buf + (size_t)ne * ne, *Vt = buf + 2 * (size_t)ne * ne;
  double *acc = Vt + (size_t)ne * ne;
  GridBarrier *gb = reinterpret_cast<GridBarrier *>(acc + 4);
  int *sweeps_dev = reinterpret_cast<int *>(acc + 6);
  TSVM_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 12, ctx->stream));
  eig_pack_in<<<(unsigned)ceil_div((int64_t)ne * ne, 256), 256, 0, ctx->stream>>>(A, n, lda, ne,
                                                                                   A0, Vt);
  TSVM_LAUNCHED(ctx);
  const size_t smem = sizeof(double) * 2 * ne + sizeof(int) * ne;
  int per_sm = 0;
  TSVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_kernel, 256, smem));
  int grid = ne / 2;
  const int cap = per_sm * ctx->num_sms;
  if (grid > cap) grid = cap;
  if (grid < 1) return TSVM_ERR_UNSUPPORTED;
  int max_sweeps = 40;
  double tol = 1e-13;
  void *args[] = {&A0, &A1, &Vt, &ne, &max_sweeps, &tol, &gb, &acc, &sweeps_dev};
  TSVM_CUDA(cudaLaunchCooperativeKernel((const void *)jacobi_kernel, dim3(grid), dim3(256), args,
                                        smem, ctx->stream));
  TSVM_LAUNCHED(ctx);
  eig_pack_out<<<(unsigned)ceil_div((int64_t)n * n, 256), 256, 0, ctx->stream>>>(A0, Vt, n, ne, w,
                                                                                 V);
  TSVM_LAUNCHED(ctx);
  int sweeps = 0;
  TSVM_CUDA(cudaMemcpyAsync(&sweeps, sweeps_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (sweeps_out) *sweeps_out = sweeps;
  if (sweeps < 0) return TSVM_ERR_TIMEOUT;
  return TSVM_OK;
}

}  // namespace tsvm
