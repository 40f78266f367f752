// Mehrotra predictor-corrector interior-point solver for the SVM dual, on the device.
//
// Replaces mpc / NewtonStep / SMWSolve (tensorsvm-train.cu:1507-1840), which run on the host
// in FP64 with about 16 GEMV passes over Z per iteration.  Here:
//   * Z (n x k) stays resident in HBM in FP32; all vectors (x = alpha, s, xi, D^-1, residuals,
//     directions) are FP64 on the device; reductions are FP64 with a fixed order.
//   * Every pass over Z is a fused streaming kernel: `zt_kernel` accumulates Z^T [v1 v2] with a
//     per-row functor producing v (and side reductions); `zw_kernel` forms Z w per row and runs
//     a per-row epilogue (residuals, SMW back-substitution, dot products).
//   * The reference's three SMW solves per NewtonStep become two: by linearity
//     dx = dy (D+Q)^-1 a - (D+Q)^-1 r5, and (D+Q)^-1 a is shared by predictor and corrector.
//     Per iteration: 5 streaming passes over Z plus one Z^T D^-1 Z pass (vs ~16 + DSYRK).
//   * Scalars (mu, dy, step lengths, sigma) are computed on the device by the finalize
//     kernels; the host synchronises once per iteration to evaluate the stopping rules.
//   * M = I + Z^T D^-1 Z is accumulated in FP64 and factored by the FP64 Cholesky in dense.cu.
#include <math.h>
#include <stdio.h>

#include <chrono>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
namespace {

enum ScalarIdx : int {
  I_C = 0, I_N, I_Y, I_MU, I_RP, I_DMAX, I_DMIN, I_COND, I_SUMX, I_SUMXI,
  I_NORMRD, I_XQX, I_POBJ, I_DOBJ, I_RELGAP,
  I_ATR7, I_ATB, I_DYA, I_ALPHA_AFF, I_MUAFF, I_SIGMA, I_ATR7C, I_DYC, I_ALPHA,
  I_E2SUM, I_E2SQ, I_INFO, I_RESMAX, I_RESPREV, I_COUNT
};
constexpr int kNScal = 32;

enum Stage : int {
  ST_NONE = 0, ST_BEGIN, ST_RESID, ST_DYA, ST_ALPHA_AFF, ST_SIGMA, ST_DYC, ST_ALPHA, ST_INIT
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct Vecs {
  double *x, *s, *xi, *dinv, *t1, *t2, *r7, *b, *dx, *ds, *dxi;
  const float *a;  // labels
};

// ---------------------------------------------------------------------------------------
// Per-row operations.  R: right-hand sides (zt) or dot products (zw); NS sums, NM minima.
// ---------------------------------------------------------------------------------------
struct InitRhsOp {  // v = e (RBF init: q = Z^T e), tensorsvm-train.cu:1536
  static constexpr int R = 1, NS = 0, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void rhs(int64_t, double *v, double *, double *) const { v[0] = 1.0; }
};
struct InitRbfRowOp {  // e2 = Z q; sums e2 and e2^2 for ox = sum(e2)/||e2||^2 (T:1537-1542)
  static constexpr int R = 1, NS = 2, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void row(int64_t, const double *dot, double *sums, double *) const {
    sums[0] += dot[0];
    sums[1] += dot[0] * dot[0];
  }
};
struct XRhsOp {  // v = x
  static constexpr int R = 1, NS = 0, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void rhs(int64_t i, double *v, double *, double *) const { v[0] = V.x[i]; }
};
struct InitLinearRowOp {  // shift s, xi so the first rd is 0 (T:1572-1578), y = 0
  static constexpr int R = 1, NS = 0, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void row(int64_t i, const double *dot, double *, double *) const {
    const double t = dot[0] - 1.0;
    if (t > 0) V.s[i] += t;
    else V.xi[i] -= t;
  }
};
// Iteration start: D, D^-1, mu, sums, a^T x, min/max D; v = x for q = Z^T x (T:1606-1631).
struct BeginOp {
  static constexpr int R = 1, NS = 4, NM = 2;
  Vecs V;
  double C;
  __device__ void load(const double *sc) { C = sc[I_C]; }
  __device__ void rhs(int64_t i, double *v, double *sums, double *mins) const {
    const double x = V.x[i], s = V.s[i], xi = V.xi[i];
    const double D = s / x + xi / (C - x);
    V.dinv[i] = 1.0 / D;
    sums[0] += x * s + (C - x) * xi;
    sums[1] += x;
    sums[2] += xi;
    sums[3] += (double)V.a[i] * x;
    mins[0] = fmin(mins[0], -D);
    mins[1] = fmin(mins[1], D);
    v[0] = x;
  }
};
// Residuals from Qx = Z q: rd = Qx - a y - s + xi - e (T:1616-1618), ||rd||, x^T Q x; the SMW
// right-hand sides r5/D and a/D of the predictor (r5 = rd - rs/x + rxi/(C-x) = Qx - a y - 1).
struct ResidOp {
  static constexpr int R = 1, NS = 2, NM = 0;
  Vecs V;
  double y;
  __device__ void load(const double *sc) { y = sc[I_Y]; }
  __device__ void row(int64_t i, const double *dot, double *sums, double *) const {
    const double Qx = dot[0], a = (double)V.a[i];
    const double rd = Qx - a * y - V.s[i] + V.xi[i] - 1.0;
    sums[0] += rd * rd;
    sums[1] += V.x[i] * Qx;
    const double r5 = Qx - a * y - 1.0;
    const double di = V.dinv[i];
    V.t1[i] = r5 * di;
    V.t2[i] = a * di;
  }
};
struct SmwRhs2Op {  // v = (t1, t2)
  static constexpr int R = 2, NS = 0, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void rhs(int64_t i, double *v, double *, double *) const {
    v[0] = V.t1[i];
    v[1] = V.t2[i];
  }
};
// SMW back-substitution (T:1836-1838): r7 = t1 - (Z g1)/D, b = t2 - (Z g2)/D; a^T r7, a^T b.
struct SmwBack2Op {
  static constexpr int R = 2, NS = 2, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void row(int64_t i, const double *dot, double *sums, double *) const {
    const double di = V.dinv[i], a = (double)V.a[i];
    const double r7 = V.t1[i] - dot[0] * di;
    const double b = V.t2[i] - dot[1] * di;
    V.r7[i] = r7;
    V.b[i] = b;
    sums[0] += a * r7;
    sums[1] += a * b;
  }
};
__device__ __forceinline__ void ratio_update(double &m, double x, double s, double xi, double dx,
                                             double ds, double dxi, double C) {
  if (dx < 0) m = fmin(m, -x / dx);
  else if (dx > 0) m = fmin(m, (C - x) / dx);
  if (ds < 0) m = fmin(m, -s / ds);
  if (dxi < 0) m = fmin(m, -xi / dxi);
}
// Affine direction (T:1815-1820 with dx = dy b - r7) and its ratio test (T:1733-1739).
struct AffineOp {
  static constexpr int R = 0, NS = 0, NM = 1;
  Vecs V;
  double C, dy;
  __device__ void load(const double *sc) { C = sc[I_C]; dy = sc[I_DYA]; }
  __device__ void row(int64_t i, double *, double *mins) const {
    const double x = V.x[i], s = V.s[i], xi = V.xi[i];
    const double dx = dy * V.b[i] - V.r7[i];
    const double rs = -s * x, rxi = -xi * (C - x);
    const double ds = (rs - s * dx) / x;
    const double dxi = (rxi + xi * dx) / (C - x);
    V.dx[i] = dx;
    V.ds[i] = ds;
    V.dxi[i] = dxi;
    ratio_update(mins[0], x, s, xi, dx, ds, dxi, C);
  }
};
struct MuAffOp {  // T:1741-1745
  static constexpr int R = 0, NS = 1, NM = 0;
  Vecs V;
  double C, al;
  __device__ void load(const double *sc) { C = sc[I_C]; al = sc[I_ALPHA_AFF]; }
  __device__ void row(int64_t i, double *sums, double *) const {
    const double x = V.x[i], dx = V.dx[i];
    sums[0] += (x + al * dx) * (V.s[i] + al * V.ds[i]) + (C - x - al * dx) * (V.xi[i] + al * V.dxi[i]);
  }
};
// Corrector right-hand side (T:1752-1757): rs = sigma mu - dx ds, rxi = sigma mu + dx dxi,
// rd = rp = 0; r5 = -rs/x + rxi/(C-x); v = r5/D.
struct CorrRhsOp {
  static constexpr int R = 1, NS = 0, NM = 0;
  Vecs V;
  double C, smu;
  __device__ void load(const double *sc) { C = sc[I_C]; smu = sc[I_SIGMA] * sc[I_MU]; }
  __device__ void rhs(int64_t i, double *v, double *, double *) const {
    const double x = V.x[i], dx = V.dx[i];
    const double rs = smu - dx * V.ds[i];
    const double rxi = smu + dx * V.dxi[i];
    const double r5 = 0.0 - rs / x + rxi / (C - x);
    const double t = r5 * V.dinv[i];
    V.t1[i] = t;
    v[0] = t;
  }
};
struct CorrBackOp {
  static constexpr int R = 1, NS = 1, NM = 0;
  Vecs V;
  __device__ void load(const double *) {}
  __device__ void row(int64_t i, const double *dot, double *sums, double *) const {
    const double r7 = V.t1[i] - dot[0] * V.dinv[i];
    V.r7[i] = r7;
    sums[0] += (double)V.a[i] * r7;
  }
};
// Corrector direction, sum with the affine one (T:1759-1761), ratio test (T:1762-1769).
struct CombineOp {
  static constexpr int R = 0, NS = 0, NM = 1;
  Vecs V;
  double C, smu, dyc;
  __device__ void load(const double *sc) {
    C = sc[I_C];
    smu = sc[I_SIGMA] * sc[I_MU];
    dyc = sc[I_DYC];
  }
  __device__ void row(int64_t i, double *, double *mins) const {
    const double x = V.x[i], s = V.s[i], xi = V.xi[i];
    const double dxa = V.dx[i], dsa = V.ds[i], dxia = V.dxi[i];
    const double rs = smu - dxa * dsa, rxi = smu + dxa * dxia;
    const double dxc = dyc * V.b[i] - V.r7[i];
    const double dsc = (rs - s * dxc) / x;
    const double dxic = (rxi + xi * dxc) / (C - x);
    const double dx = dxc + dxa, ds = dsc + dsa, dxi = dxic + dxia;
    V.dx[i] = dx;
    V.ds[i] = ds;
    V.dxi[i] = dxi;
    ratio_update(mins[0], x, s, xi, dx, ds, dxi, C);
  }
};
struct UpdateOp {  // T:1772-1776; skipped when the Cholesky failed this iteration
  static constexpr int R = 0, NS = 0, NM = 0;
  Vecs V;
  double al;
  bool ok;
  __device__ void load(const double *sc) { al = sc[I_ALPHA]; ok = sc[I_INFO] == 0.0; }
  __device__ void row(int64_t i, double *, double *) const {
    if (!ok) return;
    V.x[i] += al * V.dx[i];
    V.s[i] += al * V.ds[i];
    V.xi[i] += al * V.dxi[i];
  }
};
struct FillOp {  // x = ox, s = xi = 1
  static constexpr int R = 0, NS = 0, NM = 0;
  Vecs V;
  double ox;
  __device__ void load(const double *sc) { ox = sc[I_Y]; }
  __device__ void row(int64_t i, double *, double *) const {
    V.x[i] = ox;
    V.s[i] = 1.0;
    V.xi[i] = 1.0;
  }
};
// Bias (T:355-376): counts of SVs / free SVs; v = alpha on SVs for v = sum alpha_i Z_i.
struct BiasCountOp {
  static constexpr int R = 0, NS = 2, NM = 0;
  const double *alpha;
  double C;
  __device__ void load(const double *) {}
  __device__ void row(int64_t i, double *sums, double *) const {
    const double a = alpha[i];
    if (a > 1e-6) {
      sums[0] += 1.0;
      if (a < C - 1e-6) sums[1] += 1.0;
    }
  }
};
struct BiasRhsOp {
  static constexpr int R = 1, NS = 0, NM = 0;
  const double *alpha;
  __device__ void load(const double *) {}
  __device__ void rhs(int64_t i, double *v, double *, double *) const {
    const double a = alpha[i];
    v[0] = a > 1e-6 ? a : 0.0;
  }
};

// ---------------------------------------------------------------------------------------
// Streaming kernels.  Rows are processed in batches of 32 per warp: lane L evaluates the
// per-row vector functor of row base+L (coalesced vector traffic) while the Z rows are read
// by segments of LPR lanes (CPL float4 groups per lane), RPW = 32/LPR rows per step.
// ---------------------------------------------------------------------------------------
template <int NS, int NM>
__device__ __forceinline__ void block_partials(double *sums, double *mins, double *part_s,
                                               double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    const double v = warp_sum(sums[j]);
    if (lane == 0) sh[j * kWarps + warp] = v;
  }
#pragma unroll
  for (int j = 0; j < NM; ++j) {
    const double v = warp_min(mins[j]);
    if (lane == 0) sh[(NS + j) * kWarps + warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < NS + NM) {
    const int j = threadIdx.x;
    double r = j < NS ? 0.0 : INFINITY;
    for (int w = 0; w < kWarps; ++w) r = j < NS ? r + sh[j * kWarps + w] : fmin(r, sh[j * kWarps + w]);
    part_s[(int64_t)blockIdx.x * (NS + NM) + j] = r;
  }
}

template <class Op, int LPR, int CPL>
__global__ void __launch_bounds__(kThreads)
zt_kernel(const float *__restrict__ Z, int64_t ldz, int k, int64_t n, Op op,
          const double *__restrict__ scal, double *__restrict__ part_vec, int kz,
          double *__restrict__ part_s) {
  constexpr int R = Op::R, NS = Op::NS, NM = Op::NM;
  constexpr int RPW = 32 / LPR;
  constexpr int NC = CPL * 4;
  extern __shared__ double zsh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / LPR, sl = lane % LPR;
  op.load(scal);
  double acc[NC][R];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[c][r] = 0.0;
  double sums[NS > 0 ? NS : 1], mins[NM > 0 ? NM : 1];
#pragma unroll
  for (int j = 0; j < (NS > 0 ? NS : 1); ++j) sums[j] = 0.0;
#pragma unroll
  for (int j = 0; j < (NM > 0 ? NM : 1); ++j) mins[j] = INFINITY;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
  const int64_t stride = (int64_t)gridDim.x * kWarps * 32;
  for (int64_t base = gw * 32; base < n; base += stride) {
    double v[R];
    const int64_t my = base + lane;
    if (my < n) op.rhs(my, v, sums, mins);
    else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = 0.0;
    }
#pragma unroll 4
    for (int step = 0; step < 32 / RPW; ++step) {
      const int src = step * RPW + slot;
      const int64_t row = base + src;
      double vr[R];
#pragma unroll
      for (int r = 0; r < R; ++r) vr[r] = __shfl_sync(0xffffffffu, v[r], src);
      if (row < n) {
        const float4 *zr = reinterpret_cast<const float4 *>(Z + row * ldz);
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const int g = sl + c * LPR;
          if (4 * g < k) {
            float4 z = __ldg(zr + g);
            if (4 * g + 3 >= k) {
              if (4 * g + 1 >= k) z.y = 0.f;
              if (4 * g + 2 >= k) z.z = 0.f;
              z.w = 0.f;
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
              acc[4 * c + 0][r] = fma((double)z.x, vr[r], acc[4 * c + 0][r]);
              acc[4 * c + 1][r] = fma((double)z.y, vr[r], acc[4 * c + 1][r]);
              acc[4 * c + 2][r] = fma((double)z.z, vr[r], acc[4 * c + 2][r]);
              acc[4 * c + 3][r] = fma((double)z.w, vr[r], acc[4 * c + 3][r]);
            }
          }
        }
      }
    }
  }
  // reduce the (warp, slot) partial column sums through shared memory
  const int ncol = LPR * NC;                      // columns covered by one segment
  double *red = zsh;                              // [kWarps*RPW][R][ncol]
#pragma unroll
  for (int c = 0; c < CPL; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r)
        red[((warp * RPW + slot) * R + r) * ncol + 4 * (sl + c * LPR) + q] = acc[4 * c + q][r];
  __syncthreads();
  for (int e = threadIdx.x; e < R * kz; e += kThreads) {
    const int r = e / kz, col = e % kz;
    double s = 0.0;
    if (col < ncol)
      for (int ws = 0; ws < kWarps * RPW; ++ws) s += red[(ws * R + r) * ncol + col];
    part_vec[(int64_t)blockIdx.x * R * kz + e] = s;
  }
  if (NS + NM > 0) {
    __syncthreads();
    block_partials<NS, NM>(sums, mins, part_s, zsh);
  }
}

template <class Op, int LPR, int CPL>
__global__ void __launch_bounds__(kThreads)
zw_kernel(const float *__restrict__ Z, int64_t ldz, int k, int64_t n, Op op,
          const double *__restrict__ scal, const double *__restrict__ w, int kz,
          double *__restrict__ part_s) {
  constexpr int R = Op::R, NS = Op::NS, NM = Op::NM;
  constexpr int RPW = 32 / LPR;
  constexpr int NC = CPL * 4;
  __shared__ double zsh[(NS + NM > 0 ? NS + NM : 1) * kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / LPR, sl = lane % LPR;
  op.load(scal);
  double wr[NC][R];
#pragma unroll
  for (int c = 0; c < CPL; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int col = 4 * (sl + c * LPR) + q;
#pragma unroll
      for (int r = 0; r < R; ++r) wr[4 * c + q][r] = col < k ? w[r * kz + col] : 0.0;
    }
  double sums[NS > 0 ? NS : 1], mins[NM > 0 ? NM : 1];
#pragma unroll
  for (int j = 0; j < (NS > 0 ? NS : 1); ++j) sums[j] = 0.0;
#pragma unroll
  for (int j = 0; j < (NM > 0 ? NM : 1); ++j) mins[j] = INFINITY;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
  const int64_t stride = (int64_t)gridDim.x * kWarps * 32;
  for (int64_t base = gw * 32; base < n; base += stride) {
    double mine[R];
#pragma unroll
    for (int r = 0; r < R; ++r) mine[r] = 0.0;
#pragma unroll 4
    for (int step = 0; step < 32 / RPW; ++step) {
      const int64_t row = base + step * RPW + slot;
      double d[R];
#pragma unroll
      for (int r = 0; r < R; ++r) d[r] = 0.0;
      if (row < n) {
        const float4 *zr = reinterpret_cast<const float4 *>(Z + row * ldz);
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const int g = sl + c * LPR;
          if (4 * g < k) {
            const float4 z = __ldg(zr + g);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              d[r] = fma((double)z.x, wr[4 * c + 0][r], d[r]);
              d[r] = fma((double)z.y, wr[4 * c + 1][r], d[r]);
              d[r] = fma((double)z.z, wr[4 * c + 2][r], d[r]);
              d[r] = fma((double)z.w, wr[4 * c + 3][r], d[r]);
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) d[r] += __shfl_xor_sync(0xffffffffu, d[r], o);
        const double got = __shfl_sync(0xffffffffu, d[r], (lane % RPW) * LPR);
        if (lane / RPW == step) mine[r] = got;
      }
    }
    const int64_t my = base + lane;
    if (my < n) op.row(my, mine, sums, mins);
  }
  if (NS + NM > 0) block_partials<NS, NM>(sums, mins, part_s, zsh);
}

template <class Op>
__global__ void __launch_bounds__(kThreads)
vec_kernel(int64_t n, Op op, const double *__restrict__ scal, double *__restrict__ part_s) {
  constexpr int NS = Op::NS, NM = Op::NM;
  __shared__ double vsh[(NS + NM > 0 ? NS + NM : 1) * kWarps];
  op.load(scal);
  double sums[NS > 0 ? NS : 1], mins[NM > 0 ? NM : 1];
#pragma unroll
  for (int j = 0; j < (NS > 0 ? NS : 1); ++j) sums[j] = 0.0;
#pragma unroll
  for (int j = 0; j < (NM > 0 ? NM : 1); ++j) mins[j] = INFINITY;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * kThreads)
    op.row(i, sums, mins);
  if (NS + NM > 0) block_partials<NS, NM>(sums, mins, part_s, vsh);
}

// Refinement pass: w_r = Z^T D^-1 (Z g_r) for R vectors g_r (kz apart) in one read of Z.  Per
// row the dot products z . g_r are reduced over the LPR lanes that hold the row, scaled by
// dinv, and accumulated into the lanes' column sums (FP64, block partials as in zt_kernel).
template <int R, int LPR, int CPL>
__global__ void __launch_bounds__(kThreads)
zgz_kernel(const float *__restrict__ Z, int64_t ldz, int k, int64_t n,
           const double *__restrict__ dinv, const double *__restrict__ g, int kz,
           double *__restrict__ part_vec) {
  constexpr int RPW = 32 / LPR;
  constexpr int NC = CPL * 4;
  extern __shared__ double zsh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / LPR, sl = lane % LPR;
  double gr[NC][R], acc[NC][R];
#pragma unroll
  for (int c = 0; c < CPL; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int col = 4 * (sl + c * LPR) + q;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        gr[4 * c + q][r] = col < k ? g[r * kz + col] : 0.0;
        acc[4 * c + q][r] = 0.0;
      }
    }
  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
  const int64_t stride = (int64_t)gridDim.x * kWarps * 32;
  for (int64_t base = gw * 32; base < n; base += stride) {
#pragma unroll 2
    for (int step = 0; step < 32 / RPW; ++step) {
      const int64_t row = base + step * RPW + slot;
      if (row < n) {
        const float4 *zr = reinterpret_cast<const float4 *>(Z + row * ldz);
        float4 z[CPL];
        double d[R];
#pragma unroll
        for (int r = 0; r < R; ++r) d[r] = 0.0;
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const int gq = sl + c * LPR;
          z[c] = 4 * gq < k ? __ldg(zr + gq) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            d[r] = fma((double)z[c].x, gr[4 * c + 0][r], d[r]);
            d[r] = fma((double)z[c].y, gr[4 * c + 1][r], d[r]);
            d[r] = fma((double)z[c].z, gr[4 * c + 2][r], d[r]);
            d[r] = fma((double)z[c].w, gr[4 * c + 3][r], d[r]);
          }
        }
        const double di = dinv[row];
#pragma unroll
        for (int r = 0; r < R; ++r) {
#pragma unroll
          for (int o = LPR / 2; o > 0; o >>= 1) d[r] += __shfl_xor_sync(0xffffffffu, d[r], o);
          d[r] *= di;
        }
#pragma unroll
        for (int c = 0; c < CPL; ++c)
#pragma unroll
          for (int r = 0; r < R; ++r) {
            acc[4 * c + 0][r] = fma((double)z[c].x, d[r], acc[4 * c + 0][r]);
            acc[4 * c + 1][r] = fma((double)z[c].y, d[r], acc[4 * c + 1][r]);
            acc[4 * c + 2][r] = fma((double)z[c].z, d[r], acc[4 * c + 2][r]);
            acc[4 * c + 3][r] = fma((double)z[c].w, d[r], acc[4 * c + 3][r]);
          }
      }
    }
  }
  const int ncol = LPR * NC;
  double *red = zsh;  // [kWarps*RPW][R][ncol]
#pragma unroll
  for (int c = 0; c < CPL; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r)
        red[((warp * RPW + slot) * R + r) * ncol + 4 * (sl + c * LPR) + q] = acc[4 * c + q][r];
  __syncthreads();
  for (int e = threadIdx.x; e < R * kz; e += kThreads) {
    const int r = e / kz, col = e % kz;
    double sum = 0.0;
    if (col < ncol)
      for (int ws = 0; ws < kWarps * RPW; ++ws) sum += red[(ws * R + r) * ncol + col];
    part_vec[(int64_t)blockIdx.x * R * kz + e] = sum;
  }
}

// c = h0 - (g + w) (the residual h0 - M g of the capacitance solve, M g = g + Z^T D^-1 Z g);
// with `record`, the relative residual max_r ||c_r|| / ||h0_r|| goes into I_RESMAX, and a value
// above 0.5 (refinement cannot be trusted to converge) marks the iteration as failed.
__global__ void refine_resid_kernel(const double *__restrict__ h0, const double *__restrict__ g,
                                    const double *__restrict__ w, double *__restrict__ c, int R,
                                    int kz, int k, double *__restrict__ sc, int *__restrict__ info,
                                    int record) {
  __shared__ double red[2][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double worst = 0.0;
  for (int r = 0; r < R; ++r) {
    double sc2 = 0.0, sh2 = 0.0;
    for (int e = threadIdx.x; e < kz; e += blockDim.x) {
      const int i = r * kz + e;
      const double v = e < k ? h0[i] - (g[i] + w[i]) : 0.0;
      c[i] = v;
      sc2 += v * v;
      sh2 += h0[i] * h0[i];
    }
    sc2 = warp_sum(sc2);
    sh2 = warp_sum(sh2);
    if (lane == 0) {
      red[0][warp] = sc2;
      red[1][warp] = sh2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int j = 0; j < (int)(blockDim.x >> 5); ++j) {
        a += red[0][j];
        b += red[1][j];
      }
      const double rel = b > 0.0 ? sqrt(a / b) : 0.0;
      worst = fmax(worst, isfinite(rel) ? rel : INFINITY);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && record) {
    sc[I_RESMAX] = fmax(sc[I_RESMAX], worst);
    if (!(worst <= 0.5)) {
      *info = -1;
      sc[I_INFO] = -1.0;
    }
  }
}

__global__ void kvec_add(double *__restrict__ g, const double *__restrict__ c, int count) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) g[e] += c[e];
}

// Sum block partials in fixed order; the last block also reduces the scalars and runs the
// scalar stage of the iteration.
__global__ void finalize_kernel(const double *__restrict__ part_vec, int nblk, int nvec,
                                double *__restrict__ out_vec, const double *__restrict__ part_s,
                                int ns, int nm, double *__restrict__ sc, int stage,
                                const int *__restrict__ info) {
  const int vb = (nvec + 127) / 128;
  if ((int)blockIdx.x < vb) {
    const int e = blockIdx.x * 128 + threadIdx.x;
    if (e < nvec) {
      double s = 0.0;
      for (int b = 0; b < nblk; ++b) s += part_vec[(int64_t)b * nvec + e];
      out_vec[e] = s;
    }
    return;
  }
  __shared__ double red[16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = warp; j < ns + nm; j += 4) {
    double r = j < ns ? 0.0 : INFINITY;
    for (int b = lane; b < nblk; b += 32) {
      const double v = part_s[(int64_t)b * (ns + nm) + j];
      r = j < ns ? r + v : fmin(r, v);
    }
    r = j < ns ? warp_sum(r) : warp_min(r);
    if (lane == 0) red[j] = r;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double n = sc[I_N], C = sc[I_C];
  switch (stage) {
    case ST_INIT:
      sc[I_E2SUM] = red[0];
      sc[I_E2SQ] = red[1];
      break;
    case ST_BEGIN:
      sc[I_RESPREV] = sc[I_RESMAX];
      sc[I_RESMAX] = 0.0;
      sc[I_MU] = red[0] / (2.0 * n);
      sc[I_SUMX] = red[1];
      sc[I_SUMXI] = red[2];
      sc[I_RP] = -red[3];
      sc[I_DMAX] = -red[4];
      sc[I_DMIN] = red[5];
      sc[I_COND] = -red[4] / red[5];
      break;
    case ST_RESID: {
      sc[I_NORMRD] = sqrt(red[0]);
      sc[I_XQX] = red[1];
      const double tmp = 0.5 * red[1];
      const double pobj = tmp - sc[I_SUMX], dobj = -tmp - C * sc[I_SUMXI];
      sc[I_POBJ] = pobj;
      sc[I_DOBJ] = dobj;
      sc[I_RELGAP] = (pobj - dobj) / fmax(1.0, fabs(pobj));
      break;
    }
    case ST_DYA:
      sc[I_ATR7] = red[0];
      sc[I_ATB] = red[1];
      sc[I_DYA] = (sc[I_RP] + red[0]) / red[1];
      sc[I_INFO] = (double)(*info);
      break;
    case ST_ALPHA_AFF:
      sc[I_ALPHA_AFF] = fmin(1.0, red[0]);
      break;
    case ST_SIGMA: {
      const double mua = red[0] / (2.0 * n);
      sc[I_MUAFF] = mua;
      const double r = mua / sc[I_MU];
      sc[I_SIGMA] = r * r * r;
      break;
    }
    case ST_DYC:
      sc[I_ATR7C] = red[0];
      sc[I_DYC] = red[0] / sc[I_ATB];
      break;
    case ST_ALPHA: {
      const double al = 0.99 * fmin(1.0, red[0]);
      sc[I_ALPHA] = al;
      if (sc[I_INFO] == 0.0) sc[I_Y] += al * (sc[I_DYA] + sc[I_DYC]);
      break;
    }
    default:
      break;
  }
}

// ---------------------------------------------------------------------------------------
// Host-side driver
// ---------------------------------------------------------------------------------------
struct Geometry {
  int lpr, cpl, kz;
};

Geometry geometry(int k) {
  const int k4 = (k + 3) / 4;
  Geometry g;
  g.kz = 4 * k4;
  if (k4 <= 8) { g.lpr = 8; g.cpl = 1; }
  else if (k4 <= 16) { g.lpr = 16; g.cpl = 1; }
  else if (k4 <= 32) { g.lpr = 32; g.cpl = 1; }
  else if (k4 <= 64) { g.lpr = 32; g.cpl = 2; }
  else if (k4 <= 128) { g.lpr = 32; g.cpl = 4; }
  else { g.lpr = 32; g.cpl = 8; }
  return g;
}

struct Runner {
  tsvm_context *ctx;
  const float *Z;
  int64_t ldz, n;
  int k;
  Geometry geo;
  int nblk;
  double *scal;       // device scalars
  double *part_vec, *part_s;
  int *info;
  const double *dinv;

  template <class Op, int LPR, int CPL>
  tsvm_status zt_launch(const Op &op, double *out_vec, int stage) {
    constexpr int R = Op::R;
    constexpr int RPW = 32 / LPR;
    const size_t smem_red = sizeof(double) * (size_t)kWarps * RPW * R * LPR * CPL * 4;
    const size_t smem = smem_red > sizeof(double) * 64 ? smem_red : sizeof(double) * 64;
    auto kern = zt_kernel<Op, LPR, CPL>;
    if (smem > 48 * 1024)
      TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<nblk, kThreads, smem, ctx->stream>>>(Z, ldz, k, n, op, scal, part_vec, geo.kz, part_s);
    TSVM_LAUNCHED(ctx);
    return finalize(R * geo.kz, out_vec, Op::NS, Op::NM, stage);
  }
  template <class Op>
  tsvm_status zt(const Op &op, double *out_vec, int stage) {
    switch (geo.lpr * 10 + geo.cpl) {
      case 81: return zt_launch<Op, 8, 1>(op, out_vec, stage);
      case 161: return zt_launch<Op, 16, 1>(op, out_vec, stage);
      case 321: return zt_launch<Op, 32, 1>(op, out_vec, stage);
      case 322: return zt_launch<Op, 32, 2>(op, out_vec, stage);
      case 324: return zt_launch<Op, 32, 4>(op, out_vec, stage);
      case 328: return zt_launch<Op, 32, 8>(op, out_vec, stage);
    }
    return TSVM_ERR_UNSUPPORTED;
  }
  template <class Op, int LPR, int CPL>
  tsvm_status zw_launch(const Op &op, const double *w, int stage) {
    zw_kernel<Op, LPR, CPL><<<nblk, kThreads, 0, ctx->stream>>>(Z, ldz, k, n, op, scal, w, geo.kz,
                                                                 part_s);
    TSVM_LAUNCHED(ctx);
    return finalize(0, nullptr, Op::NS, Op::NM, stage);
  }
  template <class Op>
  tsvm_status zw(const Op &op, const double *w, int stage) {
    switch (geo.lpr * 10 + geo.cpl) {
      case 81: return zw_launch<Op, 8, 1>(op, w, stage);
      case 161: return zw_launch<Op, 16, 1>(op, w, stage);
      case 321: return zw_launch<Op, 32, 1>(op, w, stage);
      case 322: return zw_launch<Op, 32, 2>(op, w, stage);
      case 324: return zw_launch<Op, 32, 4>(op, w, stage);
      case 328: return zw_launch<Op, 32, 8>(op, w, stage);
    }
    return TSVM_ERR_UNSUPPORTED;
  }
  template <int R, int LPR, int CPL>
  tsvm_status zgz_launch(const double *g, double *w) {
    constexpr int RPW = 32 / LPR;
    const size_t smem_red = sizeof(double) * (size_t)kWarps * RPW * R * LPR * CPL * 4;
    auto kern = zgz_kernel<R, LPR, CPL>;
    if (smem_red > 48 * 1024)
      TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_red));
    kern<<<nblk, kThreads, smem_red, ctx->stream>>>(Z, ldz, k, n, dinv, g, geo.kz, part_vec);
    TSVM_LAUNCHED(ctx);
    return finalize(R * geo.kz, w, 0, 0, ST_NONE);
  }
  template <int R>
  tsvm_status zgz(const double *g, double *w) {
    switch (geo.lpr * 10 + geo.cpl) {
      case 81: return zgz_launch<R, 8, 1>(g, w);
      case 161: return zgz_launch<R, 16, 1>(g, w);
      case 321: return zgz_launch<R, 32, 1>(g, w);
      case 322: return zgz_launch<R, 32, 2>(g, w);
      case 324: return zgz_launch<R, 32, 4>(g, w);
      case 328: return zgz_launch<R, 32, 8>(g, w);
    }
    return TSVM_ERR_UNSUPPORTED;
  }
  // Iterative refinement of the capacitance solve M g = h0 against the exact M (M~ factored in
  // M_fac): per sweep one pass over Z for w = Z^T D^-1 Z g, then g += M~^-1 (h0 - g - w).
  template <int R>
  tsvm_status refine(const double *M_fac, const double *h0, double *g, double *w, double *c,
                     int sweeps) {
    for (int sweep = 0; sweep < sweeps; ++sweep) {
      TSVM_TRY(zgz<R>(g, w));
      refine_resid_kernel<<<1, 256, 0, ctx->stream>>>(h0, g, w, c, R, geo.kz, k, scal, info,
                                                        sweep == 0 ? 1 : 0);
      TSVM_LAUNCHED(ctx);
      TSVM_TRY(potrs_fp64(ctx, M_fac, k, k, c, R, geo.kz));
      kvec_add<<<(unsigned)ceil_div(R * geo.kz, 256), 256, 0, ctx->stream>>>(g, c, R * geo.kz);
      TSVM_LAUNCHED(ctx);
    }
    return TSVM_OK;
  }
  template <class Op>
  tsvm_status vec(const Op &op, int stage) {
    vec_kernel<Op><<<nblk, kThreads, 0, ctx->stream>>>(n, op, scal, part_s);
    TSVM_LAUNCHED(ctx);
    if (Op::NS + Op::NM == 0 && stage == ST_NONE) return TSVM_OK;
    return finalize(0, nullptr, Op::NS, Op::NM, stage);
  }
  tsvm_status finalize(int nvec, double *out_vec, int ns, int nm, int stage) {
    const int vb = (nvec + 127) / 128;
    finalize_kernel<<<vb + 1, 128, 0, ctx->stream>>>(part_vec, nblk, nvec, out_vec, part_s, ns, nm,
                                                      scal, stage, info);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
};

}  // namespace

tsvm_status ipm_solve(tsvm_context *ctx, const float *Z, int ldz, const float *y, int64_t n,
                      int k, double C, const tsvm_ipm_options &opt, double *alpha_out,
                      double *xi_out, double *ymult_out, tsvm_ipm_stats *stats) {
  const auto t_start = std::chrono::steady_clock::now();
  Runner run;
  run.ctx = ctx;
  run.Z = Z;
  run.ldz = ldz;
  run.n = n;
  run.k = k;
  run.geo = geometry(k);
  if (run.geo.kz > 1024) return TSVM_ERR_UNSUPPORTED;
  run.nblk = (int)std::min<int64_t>((int64_t)ctx->num_sms * 4, ceil_div(n, kWarps * 32));
  if (run.nblk < 1) run.nblk = 1;
  const int kz = run.geo.kz;

  double *vecbuf = nullptr, *sbuf = nullptr, *M = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_VEC, (size_t)11 * n, &vecbuf));
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_SCAL, (size_t)kNScal + 10 * (size_t)kz + 64, &sbuf));
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)k * k, &M));
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_PART, (size_t)run.nblk * (2 * kz + 16), &part));
  run.part_vec = part;
  run.part_s = part + (size_t)run.nblk * 2 * kz;
  run.scal = sbuf;
  double *q = sbuf + kNScal;          // kz
  double *h = q + kz;                  // 2 x kz (right-hand sides, then solutions)
  double *h0 = h + 2 * kz;             // 2 x kz copy of the right-hand sides (refinement)
  double *wv = h0 + 2 * kz;            // 2 x kz  Z^T D^-1 Z g
  double *cv = wv + 2 * kz;            // 2 x kz  residual / correction
  run.info = reinterpret_cast<int *>(cv + 2 * kz);   // [0] Cholesky/refinement status,
  int *big_count = run.info + 1;                     // [1] rows summed exactly in FP64

  Vecs V;
  V.x = vecbuf;
  V.s = V.x + n;
  V.xi = V.s + n;
  V.dinv = V.xi + n;
  V.t1 = V.dinv + n;
  V.t2 = V.t1 + n;
  V.r7 = V.t2 + n;
  V.b = V.r7 + n;
  V.dx = V.b + n;
  V.ds = V.dx + n;
  V.dxi = V.ds + n;
  V.a = y;
  run.dinv = V.dinv;

  // Mixed-precision capacitance matrix: tensor-core SYRK of the rows with dinv <= tau, exact
  // FP64 sum of the others, refinement of every solve against the exact operator.  tau adapts
  // to the refinement residual of the previous iteration.
  const bool mixed = opt.precision != TSVM_PREC_FP32 && syrk_tc_supported(k) && k >= 32;
  const int sweeps = mixed ? std::max(1, std::min(2, (int)opt.refine_sweeps)) : 0;
  double tau = 64.0;
  int64_t *big_idx = nullptr;
  double *G64 = nullptr;
  if (mixed) {
    TSVM_TRY(scratch_t(ctx, SLOT_IPM_IDX, (size_t)n + 8, &big_idx));
    TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, (size_t)k * k, &G64));
  }
  int host_info[2] = {0, 0};
  int64_t exact_rows_sum = 0;
  int exact_rows_max = 0, syrk_retries = 0, mixed_iters = 0;
  double res_max = 0.0;

  double hsc[kNScal] = {0};
  hsc[I_C] = C;
  hsc[I_N] = (double)n;
  TSVM_CUDA(cudaMemcpyAsync(run.scal, hsc, sizeof(hsc), cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemsetAsync(run.info, 0, sizeof(int), ctx->stream));

  // ---- initial point (tensorsvm-train.cu:1535-1579) ----
  double ox;
  if (opt.kernel == TSVM_KERNEL_RBF) {
    TSVM_TRY(run.zt(InitRhsOp{V}, q, ST_NONE));
    TSVM_TRY(run.zw(InitRbfRowOp{V}, q, ST_INIT));
    double e2[2];
    TSVM_CUDA(cudaMemcpyAsync(e2, run.scal + I_E2SUM, sizeof(e2), cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    ox = e2[0] / e2[1];
  } else {
    ox = (double)n / (double)n;  // sum(e) / ||e||^2 with e the ones vector
  }
  if (opt.verbose) printf("ox=%f\n", ox);
  if (ox < 0.99 * C && ox > 0.01 * C) {
  } else if (ox > 0.99 * C) {
    ox = 0.99 * C;
  } else {
    ox = 0.01 * C;
  }
  {
    double oxv = ox;
    TSVM_CUDA(cudaMemcpyAsync(run.scal + I_Y, &oxv, sizeof(double), cudaMemcpyHostToDevice,
                              ctx->stream));
    TSVM_TRY(run.vec(FillOp{V}, ST_NONE));
    double zero = 0.0;
    TSVM_CUDA(cudaMemcpyAsync(run.scal + I_Y, &zero, sizeof(double), cudaMemcpyHostToDevice,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  if (opt.kernel != TSVM_KERNEL_RBF) {
    TSVM_TRY(run.zt(XRhsOp{V}, q, ST_NONE));
    TSVM_TRY(run.zw(InitLinearRowOp{V}, q, ST_NONE));
  }

  cudaEvent_t ev_syrk0 = ctx->ev[0], ev_syrk1 = ctx->ev[1], ev_chol1 = ctx->ev[2];
  double ms_syrk = 0, ms_factor = 0;
  bool pending_events = false;
  tsvm_status result = TSVM_WARN_MAX_ITER;
  int iter = 0;
  double sc[kNScal];
  double t_gap = -1.0;
  for (iter = 0; iter < opt.max_iter; ++iter) {
    TSVM_TRY(run.zt(BeginOp{V, C}, q, ST_BEGIN));
    TSVM_TRY(run.zw(ResidOp{V, 0.0}, q, ST_RESID));
    TSVM_CUDA(cudaMemcpyAsync(ctx->host_scalars, run.scal, sizeof(double) * kNScal,
                              cudaMemcpyDeviceToHost, ctx->stream));
    if (mixed)
      TSVM_CUDA(cudaMemcpyAsync(host_info, run.info, sizeof(host_info), cudaMemcpyDeviceToHost,
                                ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(sc, ctx->host_scalars, sizeof(sc));
    if (pending_events) {
      ms_syrk += event_ms(ev_syrk0, ev_syrk1);
      ms_factor += event_ms(ev_syrk1, ev_chol1);
      pending_events = false;
    }
    bool retry = false;
    if (mixed && iter > 0) {  // bookkeeping of the previous iteration's mixed SYRK
      exact_rows_sum += host_info[1];
      exact_rows_max = std::max(exact_rows_max, host_info[1]);
      ++mixed_iters;
      if (sc[I_INFO] == 0.0) res_max = std::max(res_max, sc[I_RESPREV]);
    }
    if (iter > 0 && sc[I_INFO] != 0.0) {  // Cholesky (or refinement) failed last iteration
      if (mixed && tau > 0.0) {
        // the step was not taken: redo the iteration with more rows summed exactly
        ++syrk_retries;
        tau = tau > 1e-6 ? tau / 64.0 : 0.0;
        retry = true;
        if (opt.verbose) printf("mixed SYRK: retry with tau=%.3e\n", tau);
      } else {
        if (opt.verbose)
          printf("Cholesky fact info error %d; solver becomes unstable. Terminate.\n",
                 (int)sc[I_INFO]);
        result = TSVM_ERR_NOT_SPD;
        break;
      }
    } else if (mixed && iter > 0) {
      const double r = sc[I_RESPREV];
      if (r > 1e-4) tau /= 8.0;
      else if (r < 1e-6 && tau < 1e30) tau *= 2.0;
    }
    (void)retry;
    const double mu = sc[I_MU], nrd = sc[I_NORMRD], nrp = fabs(sc[I_RP]), cond = sc[I_COND];
    if (t_gap < 0 && sc[I_RELGAP] <= 1e-6) {
      const double scale = 1.0 + sqrt((double)n);
      if (nrd / scale <= 1e-6 && nrp / scale <= 1e-6)
        t_gap = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    }
    if (opt.verbose && iter % 5 == 0)
      printf("iter %d, mu=%.3e, normdx=%.3e, normdy=%.3e max/min(D)=%.3e pobj=%.9e dobj=%.9e\n",
             iter, mu, nrd, nrp, cond, sc[I_POBJ], sc[I_DOBJ]);
    if (mu < opt.tol && nrd < opt.tol && nrp < opt.tol) {
      if (opt.verbose) {
        printf("Converged!\n");
        printf("iter %d, mu=%.3e, normdx=%.3e, normdy=%.3e max/min(D)=%.3e pobj=%.9e dobj=%.9e\n",
               iter, mu, nrd, nrp, cond, sc[I_POBJ], sc[I_DOBJ]);
      }
      result = TSVM_OK;
      break;
    }
    if (opt.rel_gap_tol > 0) {
      const double scale = 1.0 + sqrt((double)n);
      if (sc[I_RELGAP] <= opt.rel_gap_tol && nrd / scale <= opt.rel_gap_tol &&
          nrp / scale <= opt.rel_gap_tol) {
        result = TSVM_OK;
        break;
      }
    }
    if (cond > 1e18) {
      if (opt.verbose) {
        printf("D is too ill-conditioned %.3e! Terminating.\n", cond);
        printf("iter %d, mu=%.3e, normdx=%.3e, normdy=%.3e max/min(D)=%.3e pobj=%.9e dobj=%.9e\n",
               iter, mu, nrd, nrp, cond, sc[I_POBJ], sc[I_DOBJ]);
      }
      result = TSVM_WARN_ILL_CONDITIONED;
      break;
    }
    // M = I + Z^T D^-1 Z (FP64 accumulation), Cholesky (T:1674-1714)
    TSVM_CUDA(cudaEventRecord(ev_syrk0, ctx->stream));
    if (mixed) {
      TSVM_TRY(big_rows(ctx, V.dinv, n, tau, big_idx, big_count));
      TSVM_TRY(gram_fp64_rows(ctx, Z, ldz, n, k, big_idx, big_count, V.dinv, G64));
      TSVM_TRY(syrk_capacitance_tc(ctx, Z, ldz, n, k, V.dinv, tau, 2, G64, M));
    } else {
      TSVM_TRY(gram_fp64(ctx, Z, ldz, Z, ldz, n, k, k, true, M, V.dinv));
      TSVM_TRY(small_add_diag(ctx, M, k, k, 1.0));
    }
    TSVM_CUDA(cudaEventRecord(ev_syrk1, ctx->stream));
    TSVM_TRY(chol_fp64(ctx, M, k, k, run.info));
    TSVM_CUDA(cudaEventRecord(ev_chol1, ctx->stream));
    pending_events = true;
    // predictor: r7 = SMW(r5), b = SMW(a) in one pair of passes
    TSVM_TRY(run.zt(SmwRhs2Op{V}, h, ST_NONE));
    if (sweeps)
      TSVM_CUDA(cudaMemcpyAsync(h0, h, sizeof(double) * 2 * kz, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    TSVM_TRY(potrs_fp64(ctx, M, k, k, h, 2, kz));
    if (sweeps) TSVM_TRY(run.refine<2>(M, h0, h, wv, cv, sweeps));
    TSVM_TRY(run.zw(SmwBack2Op{V}, h, ST_DYA));
    TSVM_TRY(run.vec(AffineOp{V, C, 0.0}, ST_ALPHA_AFF));
    TSVM_TRY(run.vec(MuAffOp{V, C, 0.0}, ST_SIGMA));
    // corrector
    TSVM_TRY(run.zt(CorrRhsOp{V, C, 0.0}, h, ST_NONE));
    if (sweeps)
      TSVM_CUDA(cudaMemcpyAsync(h0, h, sizeof(double) * kz, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    TSVM_TRY(potrs_fp64(ctx, M, k, k, h, 1, kz));
    if (sweeps) TSVM_TRY(run.refine<1>(M, h0, h, wv, cv, sweeps));
    TSVM_TRY(run.zw(CorrBackOp{V}, h, ST_DYC));
    TSVM_TRY(run.vec(CombineOp{V, C, 0.0, 0.0}, ST_ALPHA));
    TSVM_TRY(run.vec(UpdateOp{V, 0.0, true}, ST_NONE));
  }
  if (iter >= opt.max_iter) result = TSVM_WARN_MAX_ITER;
  TSVM_CUDA(cudaMemcpyAsync(alpha_out, V.x, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  if (xi_out)
    TSVM_CUDA(cudaMemcpyAsync(xi_out, V.xi, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                              ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (pending_events) {
    ms_syrk += event_ms(ev_syrk0, ev_syrk1);
    ms_factor += event_ms(ev_syrk1, ev_chol1);
  }
  if (ymult_out) *ymult_out = sc[I_Y];
  if (stats) {
    stats->iters = iter;
    stats->status = result;
    stats->mu = sc[I_MU];
    stats->norm_rd = sc[I_NORMRD];
    stats->norm_rp = fabs(sc[I_RP]);
    stats->cond_d = sc[I_COND];
    stats->pobj = sc[I_POBJ];
    stats->dobj = sc[I_DOBJ];
    stats->rel_gap = sc[I_RELGAP];
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    stats->ms_syrk = ms_syrk;
    stats->ms_factor = ms_factor;
    stats->ms_streams = stats->ms_total - ms_syrk - ms_factor;
    stats->t_rel_gap_1e6_ms = t_gap;
    stats->mixed_syrk = mixed ? 1 : 0;
    stats->syrk_retries = syrk_retries;
    stats->exact_rows_max = exact_rows_max;
    stats->exact_rows_mean = mixed_iters ? (double)exact_rows_sum / mixed_iters : 0.0;
    stats->refine_res_max = res_max;
  }
  return result;
}

// ---------------------------------------------------------------------------------------
// Bias of the RBF model (tensorsvm-train.cu:355-376), reassociated:
//   sum_{i in SV} alpha_i y_j (Z_i . Z_j) = y_j (v . Z_j),  v = sum_{i in SV} alpha_i Z_i,
// so one pass over Z replaces the reference's 50 x nSV x k host loop.
// ---------------------------------------------------------------------------------------
namespace {

__global__ void first_free_kernel(const double *__restrict__ alpha, int64_t n, double C, int want,
                                  int *__restrict__ idx, int *__restrict__ count) {
  __shared__ int found;
  __shared__ int wcnt[32];
  if (threadIdx.x == 0) found = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < n; base += blockDim.x) {
    if (found >= want) break;
    const int64_t i = base + threadIdx.x;
    bool f = false;
    if (i < n) {
      const double a = alpha[i];
      f = a > 1e-6 && a < C - 1e-6;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int off = found;
    for (int w = 0; w < warp; ++w) off += wcnt[w];
    off += __popc(bal & ((1u << lane) - 1u));
    if (f && off < want) idx[off] = (int)i;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += wcnt[w];
      found += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = found < want ? found : want;
}

__global__ void bias_terms_kernel(const float *__restrict__ Z, int64_t ldz, int k,
                                  const float *__restrict__ y, const double *__restrict__ v,
                                  const int *__restrict__ idx, const int *__restrict__ count,
                                  double *__restrict__ out) {
  // one warp per selected free SV j: b_j = y_j - y_j (v . Z_j); out[0..1] = mean, std
  __shared__ double bj[64];
  const int m = *count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = warp; t < m; t += nw) {
    const int64_t j = idx[t];
    double s = 0.0;
    for (int c = lane; c < k; c += 32) s += v[c] * (double)Z[j * ldz + c];
    s = warp_sum(s);
    if (lane == 0) bj[t] = (double)y[j] - (double)y[j] * s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (m == 0) {
      out[0] = NAN;
      out[1] = NAN;
      return;
    }
    double mean = 0.0;
    for (int t = 0; t < m; ++t) mean += bj[t];
    mean /= m;
    double ss = 0.0;
    for (int t = 0; t < m; ++t) ss += (bj[t] - mean) * (bj[t] - mean);
    out[0] = mean;
    out[1] = sqrt(ss / m);
  }
}

}  // namespace

tsvm_status bias_rbf(tsvm_context *ctx, const float *Z, int ldz, const float *y,
                     const double *alpha, int64_t n, int k, double C, double *b, double *bstd,
                     int32_t *nsv, int32_t *nfree) {
  Runner run;
  run.ctx = ctx;
  run.Z = Z;
  run.ldz = ldz;
  run.n = n;
  run.k = k;
  run.geo = geometry(k);
  run.nblk = (int)std::min<int64_t>((int64_t)ctx->num_sms * 4, ceil_div(n, kWarps * 32));
  if (run.nblk < 1) run.nblk = 1;
  const int kz = run.geo.kz;
  double *sbuf = nullptr, *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_MISC, (size_t)kNScal + kz + 256, &sbuf));
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_PART, (size_t)run.nblk * (2 * kz + 16), &part));
  run.part_vec = part;
  run.part_s = part + (size_t)run.nblk * 2 * kz;
  run.scal = sbuf;
  double *v = sbuf + kNScal;
  double *out = v + kz;
  int *idx = reinterpret_cast<int *>(out + 4);
  int *cnt = idx + 64;
  run.info = cnt + 1;
  TSVM_TRY(run.vec(BiasCountOp{alpha, C}, ST_INIT));  // counts into I_E2SUM / I_E2SQ slots
  TSVM_TRY(run.zt(BiasRhsOp{alpha}, v, ST_NONE));
  first_free_kernel<<<1, 1024, 0, ctx->stream>>>(alpha, n, C, 50, idx, cnt);
  TSVM_LAUNCHED(ctx);
  bias_terms_kernel<<<1, 256, 0, ctx->stream>>>(Z, ldz, k, y, v, idx, cnt, out);
  TSVM_LAUNCHED(ctx);
  double hs[2], hb[2];
  TSVM_CUDA(cudaMemcpyAsync(hs, run.scal + I_E2SUM, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(hb, out, sizeof(hb), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (nsv) *nsv = (int32_t)hs[0];
  if (nfree) *nfree = (int32_t)hs[1];
  if (b) *b = hb[0];
  if (bstd) *bstd = hb[1];
  return TSVM_OK;
}

}  // namespace tsvm
