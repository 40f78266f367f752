// Small dense FP64 linear algebra on the device for the k x k matrices of the path
// (k <= 1024).  These replace host LAPACK calls of the reference:
//   LAPACKE_dpotrf (capacitance matrix, tensorsvm-train.cu:1709)   -> chol_fp64
//   LAPACKE_dpotrs (SMW solve, tensorsvm-train.cu:1834)             -> potrs_fp64
//   LAPACKE_dsyevd (C = V diag(w) V^T, tensorsvm-train.cu:2191)     -> eig_jacobi_fp64
// plus a triangular inverse used by the shifted CholeskyQR that replaces the TSQR.
// Matrices are row-major with leading dimension lda; only lower triangles are referenced
// where noted.
#include <cooperative_groups.h>
#include <math.h>

#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
namespace {

constexpr int kNB = 32;
constexpr int kDP = kNB + 1;   // padded shared-memory row of a 32 x 32 block
constexpr int kMaxDense = 864; // largest n: the Cholesky panel (32 x n doubles) in shared memory

// Inverse of the lower-triangular nb x nb block Dg into Di (both shared, stride kDP, Di lower
// with zeros above); rdiag[r] = 1 / Dg[r][r].  Column c by warp c % nwarps: Di[c][c] =
// rdiag[c] and, for r > c, Di[r][c] = -(sum_{m=c}^{r-1} Dg[r][m] Di[m][c]) rdiag[r] (the lanes
// split the sum).
__device__ void tri_inverse_block(const double *Dg, double *Di, int nb, const double *rdiag) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
    const int r = e / kNB, c = e % kNB;
    if (c > r || r >= nb) Di[r * kDP + c] = 0.0;
  }
  __syncthreads();
  for (int c = warp; c < nb; c += nwarps) {
    if (lane == 0) Di[c * kDP + c] = rdiag[c];
    __syncwarp();
    for (int r = c + 1; r < nb; ++r) {
      const int m = c + lane;
      double v = m < r ? Dg[r * kDP + m] * Di[m * kDP + c] : 0.0;
      v = warp_sum(v);
      if (lane == 0) Di[r * kDP + c] = -v * rdiag[r];
      __syncwarp();
    }
  }
  __syncthreads();
}

// Factor the nb x nb diagonal block held in Dg (lower part, zeros above the diagonal and past
// nb) in place by one warp, and form its inverse Di: lane r keeps row r in registers for the
// factorisation (each pivot broadcast by a shuffle, every lane taking the square root and
// reciprocal itself), then lane c forward-substitutes column c of the inverse,
// Di[r][c] = (delta_rc - sum_{m<r} L[r][m] Di[m][c]) / L[r][r], reading L's rows as shared-memory
// broadcasts.  No block barrier inside.  Returns 0, or 1 + the failing column.
__device__ int diag_block_warp(double *Dg, double *Di, int nb, double *rdiag) {
  const int lane = threadIdx.x & 31;
  double a[kNB];
#pragma unroll
  for (int c = 0; c < kNB; ++c) a[c] = Dg[lane * kDP + c];
  int bad = 0;
#pragma unroll
  for (int c = 0; c < kNB; ++c) {
    if (c < nb && bad == 0) {
      const double d = __shfl_sync(0xffffffffu, a[c], c);
      if (!(d > 0.0)) {
        bad = c + 1;
      } else {
        const double inv = rsqrt(d), sq = d * inv;   // one call on the pivot's chain
        const double l = lane > c ? a[c] * inv : (lane == c ? sq : a[c]);
        a[c] = l;
        if (lane == 0) rdiag[c] = inv;
#pragma unroll
        for (int s = c + 1; s < kNB; ++s) {
          const double ls = __shfl_sync(0xffffffffu, l, s);
          if (lane >= s) a[s] = fma(-l, ls, a[s]);
        }
      }
    }
  }
  if (bad) return bad;
#pragma unroll
  for (int c = 0; c < kNB; ++c) Dg[lane * kDP + c] = (lane < nb && c <= lane) ? a[c] : 0.0;
  __syncwarp();
  double x[kNB];
#pragma unroll
  for (int r = 0; r < kNB; ++r) {
    // four independent partial sums: the substitution's chain is then r / 4 FMAs long
    double t[4] = {r == lane ? 1.0 : 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < r; ++m) t[m & 3] = fma(-Dg[r * kDP + m], x[m], t[m & 3]);
    x[r] = (r < nb && lane < nb && r >= lane) ? ((t[0] + t[1]) + (t[2] + t[3])) * rdiag[r] : 0.0;
  }
#pragma unroll
  for (int r = 0; r < kNB; ++r) Di[r * kDP + lane] = x[r];
  return 0;
}

// Right-looking blocked Cholesky in one CTA, 32-column panels:
//  (a, b) one warp factors the diagonal block in registers and forms its inverse Di (stored in
//      Dinv, block jb/32, 32 x 32 row-major, for the triangular solves; diag_block_warp);
//  (c) the panel below becomes A_below Di^T (four rows per warp at a time, each row broadcast by
//      shuffles), kept transposed in shared memory;
//  (d) the trailing lower triangle is updated with the panel (4 x 4 register tiles per thread).
// Batched launches run one CTA per problem.
constexpr int kCholThreads = 512;   // 128 registers a thread: the diagonal block's rows fit
__global__ void __launch_bounds__(kCholThreads) chol_kernel(double *__restrict__ A, int n, int lda,
                                                    double *__restrict__ Dinv,
                                                    int *__restrict__ info, int64_t strideA,
                                                    int64_t strideD,
                                                    const int *__restrict__ active) {
  // batched launches: problem blockIdx.x
  if (active && !active[blockIdx.x]) return;
  A += blockIdx.x * strideA;
  Dinv += blockIdx.x * strideD;
  info += blockIdx.x;
  extern __shared__ double PT[];  // [kNB][ldp] panel, transposed: PT[c][i] = L[r0 + i][jb + c]
  __shared__ double Dg[kNB * kDP], Di[kNB * kDP];
  __shared__ double rdiag[kNB];
  __shared__ int fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ldp = n > kNB ? n - kNB : 1;
  if (tid == 0) fail = 0;
  __syncthreads();
  for (int jb = 0; jb < n; jb += kNB) {
    const int nb = min(kNB, n - jb), m = n - jb - nb, r0 = jb + nb;
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
      const int r = e >> 5, c = e & 31;
      Dg[r * kDP + c] = (r < nb && c <= r) ? A[(int64_t)(jb + r) * lda + jb + c] : 0.0;
    }
    __syncthreads();
    // (a) + (b): the diagonal block and its inverse, one warp
    if (warp == 0) {
      const int bad = diag_block_warp(Dg, Di, nb, rdiag);
      if (lane == 0 && bad) fail = jb + bad;
    }
    __syncthreads();
    if (fail) break;
    {
      double *Dblk = Dinv + (int64_t)(jb / kNB) * kNB * kNB;
      for (int e = tid; e < kNB * kNB; e += blockDim.x) {
        const int r = e >> 5, c = e & 31;
        Dblk[e] = Di[r * kDP + c];
        if (r < nb && c <= r) A[(int64_t)(jb + r) * lda + jb + c] = Dg[r * kDP + c];
      }
    }
    // (c) L[r0 + i][jb + c] = sum_{q <= c} A[r0 + i][jb + q] Di[c][q], four rows per warp at a
    // time (independent accumulation chains)
    const int nwarps = (int)(blockDim.x >> 5);
    for (int i0 = 4 * warp; i0 < m; i0 += 4 * nwarps) {
      double a4[4], v4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u;
        a4[u] = (lane < nb && i < m) ? A[(int64_t)(r0 + i) * lda + jb + lane] : 0.0;
        v4[u] = 0.0;
      }
#pragma unroll 8
      for (int q = 0; q < kNB; ++q) {
        const double dq = q <= lane ? Di[lane * kDP + q] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u) v4[u] = fma(__shfl_sync(0xffffffffu, a4[u], q), dq, v4[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u;
        if (lane < nb && i < m) {
          PT[lane * ldp + i] = v4[u];
          A[(int64_t)(r0 + i) * lda + jb + lane] = v4[u];
        }
      }
    }
    __syncthreads();
    // (d) A[r0 + i][r0 + j] -= sum_c L[r0 + i][jb + c] L[r0 + j][jb + c], j <= i
    const int nt = (m + 3) / 4;
    const int ntiles = nt * (nt + 1) / 2;
    for (int t = tid; t < ntiles; t += blockDim.x) {
      int ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
      while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
      while (ti * (ti + 1) / 2 > t) --ti;
      const int tj = t - ti * (ti + 1) / 2;
      double acc[4][4];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int z = 0; z < 4; ++z) acc[x][z] = 0.0;
      int ia[4], ja[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        ia[x] = min(4 * ti + x, m - 1);   // clamped: rows past m are computed but not stored
        ja[x] = min(4 * tj + x, m - 1);
      }
      for (int c = 0; c < nb; ++c) {
        const double *pc = PT + c * ldp;
        double av[4], bv[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          av[x] = pc[ia[x]];
          bv[x] = pc[ja[x]];
        }
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int z = 0; z < 4; ++z) acc[x][z] = fma(av[x], bv[z], acc[x][z]);
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int z = 0; z < 4; ++z) {
          const int i = 4 * ti + x, j = 4 * tj + z;
          if (i < m && j <= i) A[(int64_t)(r0 + i) * lda + r0 + j] -= acc[x][z];
        }
    }
    __syncthreads();
  }
  if (tid == 0) *info = fail;
}

// Trailing update of one 32 x 32 block (ti, tj) (relative to row r0) with the panel PT (nb columns),
// by one warp, lane = column: A[r][c] -= sum_q L[r][jb + q] L[c][jb + q].  The lane's panel row
// stays in registers; the block's rows are read four at a time as 16-byte broadcasts.  With Dout
// (the next diagonal block, its current entries staged in Dout by the caller) the result goes
// into Dout instead (lower part, zeros elsewhere).
__device__ __forceinline__ void la_update_block(double *__restrict__ A, int lda, int n,
                                                const double *__restrict__ PT, int ldp, int nb,
                                                int r0, int ti, int tj, double *Dout, int lane) {
  const int gi0 = r0 + ti * kNB, col = r0 + tj * kNB + lane;
  const bool colok = col < n;
  double bj[kNB];
#pragma unroll
  for (int c = 0; c < kNB; ++c) bj[c] = (c < nb && colok) ? PT[c * ldp + (col - r0)] : 0.0;
  // the block's current entries: from Dout (staged there by the caller) or from A, loaded one
  // 4-row step ahead so that the L2 round trip overlaps the step before
  auto load4 = [&](int i0, double *a) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int row = gi0 + i0 + u;
      a[u] = Dout ? Dout[(i0 + u) * kDP + lane]
                  : ((row < n && colok) ? A[(int64_t)row * lda + col] : 0.0);
    }
  };
  double an[4];
  load4(0, an);
#pragma unroll 1
  for (int i0 = 0; i0 < kNB; i0 += 4) {
    double a[4], acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = an[u];
    if (i0 + 4 < kNB) load4(i0 + 4, an);
    const double *pr = PT + (gi0 - r0) + i0;
#pragma unroll
    for (int c = 0; c < kNB; ++c) {
      if (c < nb) {
        const double2 v0 = *reinterpret_cast<const double2 *>(pr + c * ldp);
        const double2 v1 = *reinterpret_cast<const double2 *>(pr + c * ldp + 2);
        acc[0] = fma(v0.x, bj[c], acc[0]);
        acc[1] = fma(v0.y, bj[c], acc[1]);
        acc[2] = fma(v1.x, bj[c], acc[2]);
        acc[3] = fma(v1.y, bj[c], acc[3]);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = i0 + u, row = gi0 + r;
      const bool in = row < n && colok && (ti != tj || lane <= r);
      if (Dout) Dout[r * kDP + lane] = in ? a[u] - acc[u] : 0.0;
      else if (in) A[(int64_t)row * lda + col] = a[u] - acc[u];
    }
  }
}

// Right-looking blocked Cholesky in one CTA with a one-panel lookahead, 32-column panels.  Step j:
//  (1) warps 1..: the panel below diagonal block j, L_ij = A_ij Di_j^T (Di_j formed in the step
//      before), into A and, transposed, into shared memory (four rows per warp at a time), while
//      warp 0 loads the next diagonal block;
//  (2) warp 0 updates the next diagonal block with the panel, factors it and forms its inverse
//      (diag_block_warp) while the other warps update the rest of the trailing lower triangle,
//      one 32 x 32 block per warp at a time (la_update_block).
// So the chain of diagonal factorisations runs beside the trailing updates instead of between
// them.  Three barriers a step.
constexpr int kCholLAThreads = 512;
constexpr int kCholLAWarps = kCholLAThreads / 32;
__global__ void __launch_bounds__(kCholLAThreads, 1)
chol_la_kernel(double *__restrict__ A, int n, int lda, double *__restrict__ Dinv,
               int *__restrict__ info) {
  extern __shared__ __align__(16) double PTs[];   // [kNB][ldp] (+ slack): PT[c][i] = L[r0 + i][jb + c]
  __shared__ double Dg[kNB * kDP], Di[kNB * kDP];
  __shared__ double rdiag[kNB];
  __shared__ int fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ldp = ((n > kNB ? n - kNB : 1) + 1) & ~1;   // even: rows of 16-byte pairs
  const int nblk = (n + kNB - 1) / kNB;
  if (tid == 0) fail = 0;
  {
    const int nb = min(kNB, n);
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
      const int r = e >> 5, c = e & 31;
      Dg[r * kDP + c] = (r < nb && c <= r) ? A[(int64_t)r * lda + c] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      const int bad = diag_block_warp(Dg, Di, nb, rdiag);
      if (lane == 0 && bad) fail = bad;
    }
    __syncthreads();
  }
  for (int j = 0; j < nblk; ++j) {
    if (fail) break;
    const int jb = j * kNB, nb = min(kNB, n - jb), r0 = jb + nb, m = n - r0;
    {
      double *Dblk = Dinv + (int64_t)j * kNB * kNB;
      for (int e = tid; e < kNB * kNB; e += blockDim.x) {
        const int r = e >> 5, c = e & 31;
        Dblk[e] = Di[r * kDP + c];
        if (r < nb && c <= r) A[(int64_t)(jb + r) * lda + jb + c] = Dg[r * kDP + c];
      }
    }
    if (m <= 0) break;
    __syncthreads();   // Dg has been read: warp 0 stages the next diagonal block there
    if (warp == 0) {
      // the next diagonal block's entries (lane = column), loaded while the panel is formed
#pragma unroll
      for (int r = 0; r < kNB; ++r)
        Dg[r * kDP + lane] =
            (r < m && lane < m && lane <= r) ? A[(int64_t)(r0 + r) * lda + r0 + lane] : 0.0;
    }
    // (1) L[r0 + i][jb + c] = sum_{q <= c} A[r0 + i][jb + q] Di[c][q], warps 1..
    for (int i0 = 4 * (warp - 1); warp > 0 && i0 < m; i0 += 4 * (kCholLAWarps - 1)) {
      double a4[4], v4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u;
        a4[u] = (lane < nb && i < m) ? A[(int64_t)(r0 + i) * lda + jb + lane] : 0.0;
        v4[u] = 0.0;
      }
#pragma unroll 8
      for (int q = 0; q < kNB; ++q) {
        const double dq = q <= lane ? Di[lane * kDP + q] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u) v4[u] = fma(__shfl_sync(0xffffffffu, a4[u], q), dq, v4[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u;
        if (lane < nb && i < m) {
          PTs[lane * ldp + i] = v4[u];
          A[(int64_t)(r0 + i) * lda + jb + lane] = v4[u];
        }
      }
    }
    __syncthreads();
    // (2) the next diagonal block (warp 0) beside the rest of the trailing update
    const int nt = (m + kNB - 1) / kNB, ntot = nt * (nt + 1) / 2;
    if (warp == 0) {
      la_update_block(A, lda, n, PTs, ldp, nb, r0, 0, 0, Dg, lane);
      __syncwarp();
      const int bad = diag_block_warp(Dg, Di, min(kNB, m), rdiag);
      if (lane == 0 && bad) fail = r0 + bad;
    } else {
      for (int b = warp; b < ntot; b += kCholLAWarps - 1) {
        int ti = 0;
        while ((ti + 1) * (ti + 2) / 2 <= b) ++ti;
        la_update_block(A, lda, n, PTs, ldp, nb, r0, ti, b - ti * (ti + 1) / 2, nullptr, lane);
      }
    }
    __syncthreads();
  }
  if (tid == 0) *info = fail;
}

// Dinv blocks of an existing lower factor L: one CTA per 32 x 32 diagonal block.
__global__ void __launch_bounds__(1024) diag_inverse_kernel(const double *__restrict__ L, int n,
                                                            int lda, double *__restrict__ Dinv) {
  __shared__ double Dg[kNB * kDP], Di[kNB * kDP], rdiag[kNB];
  const int jb = blockIdx.x * kNB, nb = min(kNB, n - jb);
  for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
    const int r = e / kNB, c = e % kNB;
    Dg[r * kDP + c] = (r < nb && c <= r) ? L[(int64_t)(jb + r) * lda + jb + c] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x < nb) rdiag[threadIdx.x] = 1.0 / Dg[threadIdx.x * kDP + threadIdx.x];
  __syncthreads();
  tri_inverse_block(Dg, Di, nb, rdiag);
  for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x)
    Dinv[(int64_t)blockIdx.x * kNB * kNB + e] = Di[(e / kNB) * kDP + e % kNB];
}

// Cholesky of a matrix of at most 128 columns held entirely in shared memory (its lower
// triangle, rows padded to n + 1 doubles), one CTA: per 32-column panel one warp factors the
// diagonal block in registers and forms its inverse (diag_block_warp, the same as the general
// kernels), then all warps form the panel below, L_ij = A_ij Di^T, and update the trailing lower
// triangle (a warp a row, lane = column, the row's panel entries as broadcasts).  At this size
// the general kernels' round trips to L2 between the phases cost more than the arithmetic
// (148 against 187 us for chol_la_kernel at n = 128).  Writes L (lower part) and the Dinv blocks
// as chol_kernel does; strideA / strideD / active allow one CTA per problem: the batched
// factorisations (chol_fp64_same) run it, one CTA a problem; a single factorisation takes the
// cluster kernel below, whose per-entry arithmetic is the same (the same panel sums and the same
// four-chain trailing-update sums, in the same step order).
constexpr int kCholSmallN = 128;
constexpr int kCholSmallThreads = 512;
__global__ void __launch_bounds__(kCholSmallThreads, 1)
chol_small_kernel(double *__restrict__ A, int n, int lda, double *__restrict__ Dinv,
                  int *__restrict__ info, int64_t strideA, int64_t strideD,
                  const int *__restrict__ active) {
  if (active && !active[blockIdx.x]) return;
  A += blockIdx.x * strideA;
  Dinv += blockIdx.x * strideD;
  info += blockIdx.x;
  extern __shared__ __align__(16) double S[];   // [n][n + 1]
  __shared__ double Dg[kNB * kDP], Di[kNB * kDP], rdiag[kNB];
  __shared__ int fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = kCholSmallThreads / 32;
  const int ld = n + 1;
  if (tid == 0) fail = 0;
  for (int e = tid; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e % n;
    if (c <= r) S[r * ld + c] = A[(int64_t)r * lda + c];
  }
  __syncthreads();
  for (int jb = 0; jb < n; jb += kNB) {
    const int nb = min(kNB, n - jb), r0 = jb + nb, m = n - r0;
    if (warp == 0) {
#pragma unroll 4
      for (int c = 0; c < kNB; ++c)
        Dg[lane * kDP + c] = (lane < nb && c <= lane) ? S[(jb + lane) * ld + jb + c] : 0.0;
      __syncwarp();
      const int bad = diag_block_warp(Dg, Di, nb, rdiag);
      if (bad) {
        if (lane == 0) fail = jb + bad;
      } else {
        if (lane < nb)
          for (int c = 0; c <= lane; ++c) S[(jb + lane) * ld + jb + c] = Dg[lane * kDP + c];
        double *Dblk = Dinv + (int64_t)(jb / kNB) * kNB * kNB;
        for (int r = 0; r < kNB; ++r) Dblk[r * kNB + lane] = Di[r * kDP + lane];
      }
    }
    __syncthreads();
    if (fail || m <= 0) break;
    // the panel below: L[r0 + i][jb + c] = sum_{q <= c} A[r0 + i][jb + q] Di[c][q]
    constexpr int kPer = (kCholSmallN * kNB) / kCholSmallThreads;   // entries a thread, at most
    double v[kPer];
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int e = tid + t * kCholSmallThreads, i = r0 + e / kNB, c = e % kNB;
      double a = 0.0;
      if (e < m * kNB && c < nb)
        for (int q = 0; q <= c; ++q) a = fma(S[i * ld + jb + q], Di[c * kDP + q], a);
      v[t] = a;
    }
    __syncthreads();   // every panel entry read before any is overwritten
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int e = tid + t * kCholSmallThreads, i = r0 + e / kNB, c = e % kNB;
      if (e < m * kNB && c < nb) S[i * ld + jb + c] = v[t];
    }
    __syncthreads();
    // trailing lower triangle: A[i][j] -= sum_c L[i][jb + c] L[j][jb + c], r0 <= j <= i
    for (int i = r0 + warp; i < n; i += kWarps) {
      double li[kNB];
#pragma unroll
      for (int c = 0; c < kNB; ++c) li[c] = c < nb ? S[i * ld + jb + c] : 0.0;
      for (int j = r0 + lane; j <= i; j += 32) {
        const double *lj = S + j * ld + jb;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int c = 0; c < kNB; ++c)
          if (c < nb) acc[c & 3] = fma(li[c], lj[c], acc[c & 3]);
        S[i * ld + j] -= (acc[0] + acc[1]) + (acc[2] + acc[3]);
      }
    }
    __syncthreads();
  }
  if (!fail)
    for (int e = tid; e < n * n; e += blockDim.x) {
      const int r = e / n, c = e % n;
      if (c <= r) A[(int64_t)r * lda + c] = S[r * ld + c];
    }
  if (tid == 0) *info = fail;
}

size_t chol_small_smem(int n) { return sizeof(double) * (size_t)n * (n + 1); }

// Cholesky of at most 256 columns by a cluster of 8 CTAs, one 32-row block row each, held in the
// CTA's shared memory (its lower part, L written in place); the cluster's distributed shared
// memory carries the panels between the CTAs and its hardware barrier orders the steps.
// Block column j:
//  (a) CTA j (warp 0) factors its diagonal block, updated by the steps before, and forms its
//      inverse Di_j (diag_block_warp); L_jj and Di_j go to global memory;
//  (b) cluster barrier; every CTA reads CTA j's status (a failure ends all of them together);
//  (c) every CTA i > j copies Di_j from CTA j and forms L_ij = A_ij Di_j^T in place (and in A);
//  (d) cluster barrier;
//  (e) every CTA i > j copies L_cj (j < c <= i) from CTA c and updates its blocks
//      A_ic -= L_ij L_cj^T; CTA j + 1 goes straight on to (a) of the next column while the others
//      still update.
// A one-CTA factorisation waits on L2 round trips between its phases (0.36 ms at k = 256 alone,
// 0.5-0.6 ms beside a streaming pass); here the block rows stay on chip and the eight CTAs
// share the updates.  Writes L (lower part), the Dinv blocks and info as chol_la_kernel does.
constexpr int kClusterCTAs = 8;
constexpr int kClusterMaxN = kClusterCTAs * kNB;
constexpr int kClusterThreads = 256;
constexpr int kRS = kClusterMaxN + 2;   // row stride of a block row (doubles): rows on 16-byte
                                        // boundaries, 4 banks apart
constexpr int kPS = kNB + 2;            // row stride of a staged 32 x 32 block, likewise
struct ClusterSmem {
  double R[kNB * kRS];                     // this CTA's block row (columns 0 .. 32 (rank + 1))
  double P[(kClusterCTAs - 1) * kNB * kPS];   // staged L_cj blocks of the update
  double Dl[kNB * kDP];                    // staged Di_j of the panel
  double Dg[kNB * kDP], Di[kNB * kDP];     // this CTA's diagonal block: factor and inverse
  double rdiag[kNB];
  int status;                              // 0, or 1 + the failing column (global index)
};
__global__ void __cluster_dims__(kClusterCTAs, 1, 1) __launch_bounds__(kClusterThreads, 1)
chol_cluster_kernel(double *__restrict__ A, int n, int lda, double *__restrict__ Dinv,
                    int *__restrict__ info) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) uint8_t cl_raw[];
  ClusterSmem &sm = *reinterpret_cast<ClusterSmem *>(cl_raw);
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nblk = (n + kNB - 1) / kNB;
  const int row0 = rank * kNB;
  const bool mine = rank < nblk;   // CTAs past the last block row only keep the barriers
  // this CTA's block row: the lower part of rows row0 .. row0 + 31, zero past n (eight loads
  // in flight a thread)
#pragma unroll 8
  for (int m = 0; m < kNB * kClusterMaxN / kClusterThreads; ++m) {
    const int e = tid + m * kClusterThreads;
    const int r = e / kClusterMaxN, c = e % kClusterMaxN, gr = row0 + r;
    sm.R[r * kRS + c] = (mine && gr < n && c <= gr) ? A[(int64_t)gr * lda + c] : 0.0;
  }
  if (tid == 0) sm.status = 0;
  __syncthreads();
  // entries of a 32 x 32 block per thread: row tid / 8, columns tid % 8 + 8 u
  const int er = tid >> 3, ec = tid & 7;
  int fail = 0;
  for (int j = 0; j < nblk; ++j) {
    const int jb = j * kNB;
    if (rank == j && warp == 0) {   // (a)
      const int nb = min(kNB, n - jb);
#pragma unroll 4
      for (int c = 0; c < kNB; ++c)
        sm.Dg[lane * kDP + c] = (lane < nb && c <= lane) ? sm.R[lane * kRS + jb + c] : 0.0;
      __syncwarp();
      const int bad = diag_block_warp(sm.Dg, sm.Di, nb, sm.rdiag);
      if (bad) {
        if (lane == 0) sm.status = jb + bad;
      } else {
        double *Dblk = Dinv + (int64_t)j * kNB * kNB;
        for (int r = 0; r < kNB; ++r) {
          Dblk[r * kNB + lane] = sm.Di[r * kDP + lane];
          if (r < nb && lane <= r) {
            const double l = sm.Dg[r * kDP + lane];
            sm.R[r * kRS + jb + lane] = l;
            A[(int64_t)(jb + r) * lda + jb + lane] = l;
          }
        }
      }
    }
    cl.sync();   // (b)
    fail = *cl.map_shared_rank(&sm.status, j);
    if (fail) break;
    const bool below = mine && rank > j;
    if (below) {   // (c)
      const double *Dj = cl.map_shared_rank(sm.Di, j);
      double dv[kNB * kNB / kClusterThreads];   // every remote load issued before the stores
#pragma unroll
      for (int m = 0; m < kNB * kNB / kClusterThreads; ++m) {
        const int e = tid + m * kClusterThreads;
        dv[m] = Dj[(e >> 5) * kDP + (e & 31)];
      }
#pragma unroll
      for (int m = 0; m < kNB * kNB / kClusterThreads; ++m) {
        const int e = tid + m * kClusterThreads;
        sm.Dl[(e >> 5) * kDP + (e & 31)] = dv[m];
      }
      __syncthreads();
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int c = ec + 8 * u;
        double a = 0.0;
        for (int q = 0; q <= c; ++q) a = fma(sm.R[er * kRS + jb + q], sm.Dl[c * kDP + q], a);
        v[u] = a;
      }
      __syncthreads();   // the block read by every thread before any entry is replaced
      const int gr = row0 + er;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int c = ec + 8 * u;
        sm.R[er * kRS + jb + c] = v[u];
        if (gr < n) A[(int64_t)gr * lda + jb + c] = v[u];
      }
    }
    cl.sync();   // (d)
    if (below) {   // (e)
      const int nc = rank - j;   // blocks c = j + 1 .. rank
      // every remote 16-byte load of the step issued before the stores: thread tid moves
      // entries (r, 2 p) and (r, 2 p + 1) of each block, r = e / 16, p = e % 16, e = tid, tid + 256
      constexpr int kH = kNB * kNB / 2 / kClusterThreads;   // 16-byte pieces a thread per block
      double2 pv[kClusterCTAs - 1][kH];
#pragma unroll
      for (int t = 0; t < kClusterCTAs - 1; ++t)
        if (t < nc) {
          const double *Lc = cl.map_shared_rank(sm.R, j + 1 + t);
#pragma unroll
          for (int h = 0; h < kH; ++h) {
            const int e = tid + h * kClusterThreads;
            pv[t][h] = *reinterpret_cast<const double2 *>(Lc + (e >> 4) * kRS + jb + 2 * (e & 15));
          }
        }
#pragma unroll
      for (int t = 0; t < kClusterCTAs - 1; ++t)
        if (t < nc) {
          double *Pt = sm.P + (size_t)t * kNB * kPS;
#pragma unroll
          for (int h = 0; h < kH; ++h) {
            const int e = tid + h * kClusterThreads;
            *reinterpret_cast<double2 *>(Pt + (e >> 4) * kPS + 2 * (e & 15)) = pv[t][h];
          }
        }
      __syncthreads();
      double li[kNB];
#pragma unroll
      for (int q = 0; q < kNB; ++q) li[q] = sm.R[er * kRS + jb + q];
      for (int t = 0; t < nc; ++t) {
        const double *Pt = sm.P + (size_t)t * kNB * kPS;
        const int cb = (j + 1 + t) * kNB;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int s = ec + 8 * u;
          double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int q = 0; q < kNB; ++q) acc[q & 3] = fma(li[q], Pt[s * kPS + q], acc[q & 3]);
          sm.R[er * kRS + cb + s] -= (acc[0] + acc[1]) + (acc[2] + acc[3]);
        }
      }
      __syncthreads();
    }
  }
  cl.sync();   // no CTA leaves while another may still read its shared memory
  if (rank == 0 && tid == 0) *info = fail;
}

// Solve L L^T X = B for nrhs (<= 4) right-hand sides (rows of B) with the blocked forward and
// backward substitutions; the diagonal blocks are applied through their inverses (Dinv, staged
// in shared memory per block), so every step is a set of independent dot products.  One CTA of
// 1024 threads.
__global__ void __launch_bounds__(1024) potrs_kernel(const double *__restrict__ L, int n, int lda,
                                                    const double *__restrict__ Dinv,
                                                    double *__restrict__ B, int nrhs, int ldb,
                                                    int64_t strideA, int64_t strideD,
                                                    int64_t strideB,
                                                    const int *__restrict__ active) {
  // batched launches: problem blockIdx.x
  if (active && !active[blockIdx.x]) return;
  L += blockIdx.x * strideA;
  Dinv += blockIdx.x * strideD;
  B += blockIdx.x * strideB;
  extern __shared__ double y[];      // [nrhs][n], then the backward partials [32][4][kNB]
  double *part = y + (size_t)nrhs * n;
  __shared__ double t[4][kNB];
  __shared__ double Ds[kNB * kDP];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < nrhs * n; e += blockDim.x) y[e] = B[(int64_t)(e / n) * ldb + e % n];
  __syncthreads();
  // forward: L y = b
  for (int jb = 0; jb < n; jb += kNB) {
    const int nb = min(kNB, n - jb);
    Ds[(tid >> 5) * kDP + (tid & 31)] = Dinv[(int64_t)(jb / kNB) * kNB * kNB + tid];
    if (warp < nb) {
      const double *Lr = L + (int64_t)(jb + warp) * lda;
      double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
      for (int m = lane; m < jb; m += 32) {
        const double l = __ldcg(Lr + m);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q < nrhs) s[q] = fma(l, y[q * n + m], s[q]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (q < nrhs) {   // uniform over the warp
          const double v = warp_sum(s[q]);
          if (lane == 0) t[q][warp] = y[q * n + jb + warp] - v;
        }
      }
    }
    __syncthreads();
    if (tid < nrhs * nb) {
      // the 32-term product with the inverted diagonal block, unrolled into four independent
      // chains (the loads issue together; a serial chain of shared-memory loads and FMAs was
      // the longest step of each block)
      const int q = tid / nb, r = tid % nb;
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int c = 0; c < kNB; ++c)
        if (c <= r) v[c & 3] = fma(Ds[r * kDP + c], t[q][c], v[c & 3]);
      y[q * n + jb + r] = (v[0] + v[1]) + (v[2] + v[3]);
    }
    __syncthreads();
  }
  // backward: L^T x = y
  for (int jb = ((n - 1) / kNB) * kNB; jb >= 0; jb -= kNB) {
    const int nb = min(kNB, n - jb);
    Ds[(tid >> 5) * kDP + (tid & 31)] = Dinv[(int64_t)(jb / kNB) * kNB * kNB + tid];
    {
      double s[4] = {0.0, 0.0, 0.0, 0.0};
      if (lane < nb) {
#pragma unroll 4
        for (int m = jb + nb + warp; m < n; m += 32) {
          const double l = __ldcg(L + (int64_t)m * lda + jb + lane);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < nrhs) s[q] = fma(l, y[q * n + m], s[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) part[(warp * 4 + q) * kNB + lane] = s[q];
    }
    __syncthreads();
    if (tid < nrhs * nb) {
      const int q = tid / nb, r = tid % nb;
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int w = 0; w < 32; ++w) v[w & 3] += part[(w * 4 + q) * kNB + r];
      t[q][r] = y[q * n + jb + r] - ((v[0] + v[1]) + (v[2] + v[3]));
    }
    __syncthreads();
    if (tid < nrhs * nb) {
      const int q = tid / nb, r = tid % nb;
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int c = 0; c < kNB; ++c)
        if (c >= r && c < nb) v[c & 3] = fma(Ds[c * kDP + r], t[q][c], v[c & 3]);
      y[q * n + jb + r] = (v[0] + v[1]) + (v[2] + v[3]);
    }
    __syncthreads();
  }
  for (int e = tid; e < nrhs * n; e += blockDim.x) B[(int64_t)(e / n) * ldb + e % n] = y[e];
}

// L^-1 by 32-column blocks, one CTA per block column j: X_jj = Dinv_jj and, going down,
// X_ij = -Dinv_ii sum_{m=j}^{i-1} L_im X_mj.  X is written (and re-read) in global memory.
__global__ void __launch_bounds__(1024) trinv_kernel(const double *__restrict__ L, int n, int lda,
                                                    const double *__restrict__ Dinv,
                                                    double *__restrict__ X) {
  __shared__ double T[kNB][kDP];
  const int jb = blockIdx.x * kNB, nbj = min(kNB, n - jb);
  const int tid = threadIdx.x, r = tid / kNB, c = tid % kNB;
  for (int e = tid; e < jb * nbj; e += blockDim.x)
    X[(int64_t)(e / nbj) * lda + jb + e % nbj] = 0.0;
  if (r < nbj && c < nbj)
    X[(int64_t)(jb + r) * lda + jb + c] = Dinv[(int64_t)blockIdx.x * kNB * kNB + r * kNB + c];
  __syncthreads();
  for (int ib = jb + kNB; ib < n; ib += kNB) {
    const int nbi = min(kNB, n - ib);
    if (r < nbi && c < nbj) {
      const double *Lr = L + (int64_t)(ib + r) * lda;
      double v = 0.0;
      for (int m = jb; m < ib; ++m) v = fma(Lr[m], X[(int64_t)m * lda + jb + c], v);
      T[r][c] = v;
    }
    __syncthreads();
    if (r < nbi && c < nbj) {
      const double *Di = Dinv + (int64_t)(ib / kNB) * kNB * kNB + r * kNB;
      double v = 0.0;
      for (int q = 0; q <= r; ++q) v = fma(Di[q], T[q][c], v);
      X[(int64_t)(ib + r) * lda + jb + c] = -v;
    }
    __syncthreads();
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

// The same cyclic Jacobi in one CTA for ne <= 128 (the grid version pays a grid barrier per
// round, ~2000 of them at ne = 128): the lower triangle of A packed in shared memory
// (r (r + 1) / 2 + c) and Vt (row p = eigenvector p) beside it, 196 KB at ne = 128.  A round
// rotates ne / 2 disjoint pairs; with J_i the rotation of pair i, the 2 x 2 block of rows of
// pair i and columns of pair j becomes J_i^T A_ij J_j, one block per thread with no conflicts
// (blocks i > j are the transposes of i < j and are not stored), and rows p, q of Vt are rotated
// alongside.  Same rotation formulas, ordering, tolerance and sweep limit as jacobi_kernel.
// A round is bound by shared-memory wavefronts (at ne = 128: 2 x 2 block updates ~1450,
// Vt rows 2048); pair indices and packed offsets are computed, not loaded, (c, s) is one
// broadcast 16-byte load, and the rotations of round r + 1 (two warps, a chain of FP64
// divisions and square roots) are computed while round r rotates the rows of Vt.
constexpr int kJacobiSmallNe = 128;

__device__ __forceinline__ int pk(int r, int c) {
  return r >= c ? r * (r + 1) / 2 + c : c * (c + 1) / 2 + r;
}

// pair m of a round: (circle_player(m), circle_player(ne - 1 - m)); round < ne - 1 and
// m < ne / 2 keep each sum below 2 (ne - 1), so one conditional subtraction is the modulo
__device__ __forceinline__ void round_pair(int m, int round, int ne, int &p, int &q) {
  int a = m - 1 + round;
  if (a >= ne - 1) a -= ne - 1;
  p = m == 0 ? 0 : 1 + a;
  int b = ne - 2 - m + round;
  if (b >= ne - 1) b -= ne - 1;
  q = 1 + b;
}

// Batched launches (grid.x problems): problem b reads A + b strideA and writes w + b strideW,
// V + b strideV and sweeps_out[b]; the strides are 0 for a single problem.
__global__ void __launch_bounds__(1024, 1)
jacobi_small_kernel(const double *__restrict__ A, int n, int lda, int ne, int max_sweeps,
                    double tol, double *__restrict__ w, double *__restrict__ V,
                    int *__restrict__ sweeps_out, int64_t strideA, int64_t strideW,
                    int64_t strideV) {
  A += blockIdx.x * strideA;
  w += blockIdx.x * strideW;
  V += blockIdx.x * strideV;
  sweeps_out += blockIdx.x;
  extern __shared__ double2 jsh2[];
  const int np = ne / 2;
  double2 *rot = jsh2;                                    // [2][np] (c, s), by round parity
  double *red = reinterpret_cast<double *>(rot + 2 * np); // [64]
  double *P = red + 64;                                   // packed lower triangle
  double *Vt = P + (size_t)ne * (ne + 1) / 2;             // ne x ne
  for (int r = threadIdx.x; r < ne; r += blockDim.x)
    for (int c = 0; c <= r; ++c)
      P[r * (r + 1) / 2 + c] = (r < n && c < n) ? A[(int64_t)r * lda + c] : 0.0;
  for (int e = threadIdx.x; e < ne * ne; e += blockDim.x) Vt[e] = (e / ne == e % ne) ? 1.0 : 0.0;
  __syncthreads();
  // rotations of `round` into dst (threads m < np: warps 0 and 1 at ne = 128)
  auto rotations = [&](int round, double2 *dst) {
    for (int m = threadIdx.x; m < np; m += blockDim.x) {
      int p, q;
      round_pair(m, round, ne, p, q);
      const double app = P[pk(p, p)], aqq = P[pk(q, q)], apq = P[pk(p, q)];
      double c = 1.0, sv = 0.0;
      if (fabs(apq) > 1e-300) {
        const double tau = (aqq - app) / (2.0 * apq);
        double t;
        if (fabs(tau) > 1e150) t = 0.5 / tau;
        else t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        c = 1.0 / sqrt(1.0 + t * t);
        sv = t * c;
      }
      dst[m] = make_double2(c, sv);
    }
  };
  // this thread's 2 x 2 blocks (i, j), i <= j over the pairs (at most 3 at ne = 128), fixed
  // for the whole solve: enumerate the upper triangle of pairs row by row
  constexpr int kMaxB = 3;
  const int nblk = np * (np + 1) / 2;
  int bi[kMaxB], bj[kMaxB];
  int nb = 0;
  for (int b = threadIdx.x; b < nblk && nb < kMaxB; b += blockDim.x, ++nb) {
    int i = 0, rem = b;
    while (rem >= np - i) { rem -= np - i; ++i; }
    bi[nb] = i;
    bj[nb] = i + rem;
  }
  // this thread's Vt elements: e = tid + 1024 u, pair e / ne, column e % ne
  const int m0 = threadIdx.x / ne, col0 = threadIdx.x % ne;
  const int dm = blockDim.x / ne, dc = blockDim.x % ne;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    rotations(0, rot);
    __syncthreads();
    for (int round = 0; round < ne - 1; ++round) {
      const double2 *cur = rot + (round & 1) * np;
      for (int u = 0; u < nb; ++u) {
        const int i = bi[u], j = bj[u];
        int pi, qi, pj, qj;
        round_pair(i, round, ne, pi, qi);
        round_pair(j, round, ne, pj, qj);
        const double2 ri = cur[i], rj = cur[j];
        const double ci = ri.x, si = ri.y, cj = rj.x, sj = rj.y;
        const int i00 = pk(pi, pj), i01 = pk(pi, qj), i10 = pk(qi, pj), i11 = pk(qi, qj);
        const double a00 = P[i00], a01 = P[i01], a10 = P[i10], a11 = P[i11];
        // columns of pair j: (x_p, x_q) -> (c x_p - s x_q, s x_p + c x_q)
        const double b00 = cj * a00 - sj * a01, b01 = sj * a00 + cj * a01;
        const double b10 = cj * a10 - sj * a11, b11 = sj * a10 + cj * a11;
        // rows of pair i
        const double n00 = ci * b00 - si * b10, n10 = si * b00 + ci * b10;
        const double n01 = ci * b01 - si * b11, n11 = si * b01 + ci * b11;
        if (i == j) {
          P[i00] = n00;
          P[i01] = 0.5 * (n01 + n10);
          P[i11] = n11;
        } else {
          P[i00] = n00;
          P[i01] = n01;
          P[i10] = n10;
          P[i11] = n11;
        }
      }
      __syncthreads();
      // the next round's rotations read the updated P and write the other parity slot, which
      // nothing reads until the barrier below; Vt only needs this round's rotations
      if (round + 1 < ne - 1) rotations(round + 1, rot + ((round + 1) & 1) * np);
      for (int m = m0, col = col0; m < np;) {
        const double2 r = cur[m];
        int p, q;
        round_pair(m, round, ne, p, q);
        double *vp = Vt + (size_t)p * ne, *vq = Vt + (size_t)q * ne;
        const double a = vp[col], bq = vq[col];
        vp[col] = r.x * a - r.y * bq;
        vq[col] = r.y * a + r.x * bq;
        m += dm;
        col += dc;
        if (col >= ne) { col -= ne; ++m; }
      }
      __syncthreads();
    }
    // convergence: off-diagonal mass against the diagonal
    double off = 0.0, dia = 0.0;
    for (int r = threadIdx.x; r < ne; r += blockDim.x) {
      const double *row = P + r * (r + 1) / 2;
      for (int c = 0; c < r; ++c) off += 2.0 * row[c] * row[c];
      dia += row[r] * row[r];
    }
    off = warp_sum(off);
    dia = warp_sum(dia);
    if ((threadIdx.x & 31) == 0) {
      red[threadIdx.x >> 5] = off;
      red[32 + (threadIdx.x >> 5)] = dia;
    }
    __syncthreads();
    double o = 0.0, dsum = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      o += red[k];
      dsum += red[32 + k];
    }
    __syncthreads();
    if (o <= tol * tol * (dsum + o)) { ++sweep; break; }
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e % n;
    V[e] = Vt[(size_t)c * ne + r];
    if (c == 0) w[r] = P[r * (r + 1) / 2 + r];
  }
  if (threadIdx.x == 0) *sweeps_out = sweep;
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

tsvm_status chol_fp64(tsvm_context *ctx, double *A, int n, int lda, int *info_dev, double *Dinv,
                      cudaStream_t stream) {
  if (n < 1 || n > kMaxDense) return TSVM_ERR_UNSUPPORTED;  // panel must fit shared memory
  if (n <= kClusterMaxN) {   // one block row per CTA of a cluster, all of it on chip
    const size_t smem = sizeof(ClusterSmem);
    TSVM_CUDA(cudaFuncSetAttribute(chol_cluster_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    chol_cluster_kernel<<<kClusterCTAs, kClusterThreads, smem, stream ? stream : ctx->stream>>>(
        A, n, lda, Dinv, info_dev);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
  // the panel rows padded to an even length, plus the slack the 4-row reads of a ragged last
  // block run into
  const size_t ldp = ((size_t)(n > kNB ? n - kNB : 1) + 1) & ~(size_t)1;
  const size_t smem = sizeof(double) * ((size_t)kNB * ldp + 64);
  TSVM_CUDA(cudaFuncSetAttribute(chol_la_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  chol_la_kernel<<<1, kCholLAThreads, smem, stream ? stream : ctx->stream>>>(A, n, lda, Dinv,
                                                                             info_dev);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

int chol_fp64_sms(int n) { return n <= kClusterMaxN ? kClusterCTAs : 1; }

tsvm_status chol_fp64_same(tsvm_context *ctx, double *A, int n, int lda, int64_t strideA,
                           int *info_dev, double *Dinv, int64_t strideD, int count,
                           const int *active, const std::vector<int> &pending) {
  if (n < 1 || n > kMaxDense || count < 1) return TSVM_ERR_UNSUPPORTED;
  if (n <= kCholSmallN) {   // one CTA per problem, the single-launch kernel's arithmetic
    const size_t smem = chol_small_smem(n);
    TSVM_CUDA(cudaFuncSetAttribute(chol_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    chol_small_kernel<<<count, kCholSmallThreads, smem, ctx->stream>>>(A, n, lda, Dinv, info_dev,
                                                                       strideA, strideD, active);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
  for (int p : pending)
    TSVM_TRY(chol_fp64(ctx, A + p * strideA, n, lda, info_dev + p, Dinv + p * strideD));
  return TSVM_OK;
}

tsvm_status chol_fp64_batched(tsvm_context *ctx, double *A, int n, int lda, int64_t strideA,
                              int *info_dev, double *Dinv, int64_t strideD, int count,
                              const int *active) {
  if (n < 1 || n > kMaxDense || count < 1) return TSVM_ERR_UNSUPPORTED;
  // (chol_small_kernel, one CTA a problem, measured slower here: 142 against 124 us for 64
  // problems at n = 128, its trailing update reading each panel row once per entry)
  const size_t smem = sizeof(double) * (size_t)kNB * (size_t)(n > kNB ? n - kNB : 1);
  TSVM_CUDA(cudaFuncSetAttribute(chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  chol_kernel<<<count, kCholThreads, smem, ctx->stream>>>(A, n, lda, Dinv, info_dev, strideA, strideD,
                                                  active);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status tri_diag_inverse(tsvm_context *ctx, const double *L, int n, int lda, double *Dinv) {
  if (n < 1) return TSVM_ERR_INVALID_ARGUMENT;
  diag_inverse_kernel<<<(unsigned)ceil_div(n, kNB), 1024, 0, ctx->stream>>>(L, n, lda, Dinv);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status potrs_fp64(tsvm_context *ctx, const double *L, int n, int lda, const double *Dinv,
                       double *B, int nrhs, int ldb) {
  if (nrhs < 1 || nrhs > 4 || n < 1 || n > kMaxDense) return TSVM_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * ((size_t)nrhs * n + 32 * 4 * kNB);
  TSVM_CUDA(cudaFuncSetAttribute(potrs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  potrs_kernel<<<1, 1024, smem, ctx->stream>>>(L, n, lda, Dinv, B, nrhs, ldb, 0, 0, 0, nullptr);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status potrs_fp64_batched(tsvm_context *ctx, const double *L, int n, int lda,
                               int64_t strideA, const double *Dinv, int64_t strideD, double *B,
                               int nrhs, int ldb, int64_t strideB, int count, const int *active) {
  if (nrhs < 1 || nrhs > 4 || n < 1 || n > kMaxDense || count < 1) return TSVM_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * ((size_t)nrhs * n + 32 * 4 * kNB);
  TSVM_CUDA(cudaFuncSetAttribute(potrs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  potrs_kernel<<<count, 1024, smem, ctx->stream>>>(L, n, lda, Dinv, B, nrhs, ldb, strideA,
                                                   strideD, strideB, active);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status trinv_lower_fp64(tsvm_context *ctx, const double *L, int n, int lda,
                             const double *Dinv, double *Linv) {
  if (n < 1) return TSVM_ERR_INVALID_ARGUMENT;
  trinv_kernel<<<(unsigned)ceil_div(n, kNB), 1024, 0, ctx->stream>>>(L, n, lda, Dinv, Linv);
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
  if (ne <= kJacobiSmallNe) {
    int *sweeps_dev = nullptr;
    TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, 4, &sweeps_dev));
    const int np = ne / 2;
    const size_t smem = sizeof(double2) * 2 * np +
                        sizeof(double) * (64 + (size_t)ne * (ne + 1) / 2 + (size_t)ne * ne);
    TSVM_CUDA(cudaFuncSetAttribute(jacobi_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    jacobi_small_kernel<<<1, 1024, smem, ctx->stream>>>(A, n, lda, ne, 40, 1e-13, w, V,
                                                         sweeps_dev, 0, 0, 0);
    TSVM_LAUNCHED(ctx);
    int sweeps = 0;
    TSVM_CUDA(cudaMemcpyAsync(&sweeps, sweeps_dev, sizeof(int), cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (sweeps_out) *sweeps_out = sweeps;
    return TSVM_OK;
  }
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
  if (sweeps < 0) return timeout_status("eig_jacobi_fp64 (grid barrier)");
  return TSVM_OK;
}

// count eigenproblems of width n (A: count x n x n row-major, contiguous; w: count x n;
// V: count x n x n): one CTA per problem in one launch for n <= kJacobiSmallNe (the CTAs run
// side by side on their own SMs), else one grid eigensolver after the other.
tsvm_status eig_jacobi_fp64_batched(tsvm_context *ctx, double *A, int n, int count, double *w,
                                    double *V, int *max_sweeps_out) {
  if (n < 1 || n > 1024 || count < 1) return TSVM_ERR_UNSUPPORTED;
  int ne = n + (n & 1);
  if (ne < 2) ne = 2;
  const int64_t nn = (int64_t)n * n;
  if (ne > kJacobiSmallNe) {
    int worst = 0;
    for (int b = 0; b < count; ++b) {
      int sw = 0;
      TSVM_TRY(eig_jacobi_fp64(ctx, A + b * nn, n, n, w + (int64_t)b * n, V + b * nn, &sw));
      worst = sw > worst ? sw : worst;
    }
    if (max_sweeps_out) *max_sweeps_out = worst;
    return TSVM_OK;
  }
  int *sweeps_dev = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_B_EIGSW, (size_t)count, &sweeps_dev));
  const int np = ne / 2;
  const size_t smem = sizeof(double2) * 2 * np +
                      sizeof(double) * (64 + (size_t)ne * (ne + 1) / 2 + (size_t)ne * ne);
  TSVM_CUDA(cudaFuncSetAttribute(jacobi_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  jacobi_small_kernel<<<count, 1024, smem, ctx->stream>>>(A, n, n, ne, 40, 1e-13, w, V,
                                                           sweeps_dev, nn, n, nn);
  TSVM_LAUNCHED(ctx);
  std::vector<int> sw(count);
  TSVM_CUDA(cudaMemcpyAsync(sw.data(), sweeps_dev, sizeof(int) * count, cudaMemcpyDeviceToHost,
                            ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  int worst = 0;
  for (int v : sw) worst = v > worst ? v : worst;
  if (max_sweeps_out) *max_sweeps_out = worst;
  return TSVM_OK;
}

}  // namespace tsvm
