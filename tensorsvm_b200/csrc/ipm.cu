// Mehrotra predictor-corrector interior-point solver for the SVM dual, on the device.
//
// Replaces mpc / NewtonStep / SMWSolve (tensorsvm-train.cu:1507-1840), which run on the host
// in FP64 with about 16 GEMV passes over Z per iteration.  Here:
//   * Z (n x k) stays resident in HBM in FP32; all vectors (x = alpha, s, xi, D^-1, residuals,
//     directions) are FP64 on the device; reductions are FP64 with a fixed order.
//   * Every pass over Z is one persistent streaming kernel (`stream_kernel`, chunks of Z rows
//     brought into shared memory by bulk copies): Z^T v with a per-row functor producing v
//     (and side reductions), Z w per row followed by a per-row epilogue (residuals, SMW
//     back-substitution, dot products), or Z^T D^-1 Z g for the refinement of the SMW solves.
//   * The reference's three SMW solves per NewtonStep become two: by linearity
//     dx = dy (D+Q)^-1 a - (D+Q)^-1 r5, and (D+Q)^-1 a is shared by predictor and corrector.
//     Per iteration: 5 streaming passes over Z plus one Z^T D^-1 Z pass (vs ~16 + DSYRK).
//   * Scalars (mu, dy, step lengths, sigma) are computed on the device by the finalize
//     kernels; the host synchronises once per iteration to evaluate the stopping rules.
//   * M = I + Z^T D^-1 Z is accumulated in FP64 and factored by the FP64 Cholesky in dense.cu.
#include <math.h>
#include <stdio.h>

#include <string.h>

#include <algorithm>
#include <chrono>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"
#include "tc_common.cuh"
#include "trace.h"

namespace tsvm {
namespace {

enum ScalarIdx : int {
  I_C = 0, I_N, I_Y, I_MU, I_RP, I_DMAX, I_DMIN, I_COND, I_SUMX, I_SUMXI,
  I_NORMRD, I_XQX, I_POBJ, I_DOBJ, I_RELGAP,
  I_ATR7, I_ATB, I_DYA, I_ALPHA_AFF, I_MUAFF, I_SIGMA, I_ATR7C, I_DYC, I_ALPHA,
  I_E2SUM, I_E2SQ, I_INFO, I_RESMAX, I_RESPREV,
  I_TAU, I_TAUIT,   // batched mixed-precision solves: the iteration's tau, iterations counted
  I_COUNT
};
constexpr int kNScal = 32;

enum Stage : int {
  ST_NONE = 0, ST_BEGIN, ST_RESID, ST_DYA, ST_ALPHA_AFF, ST_SIGMA, ST_DYC, ST_ALPHA, ST_INIT,
  ST_ADJ
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
  static constexpr int NS = 0, NM = 1;
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
  static constexpr int NS = 1, NM = 0;
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
  static constexpr int NS = 0, NM = 1;
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
  static constexpr int NS = 0, NM = 0;
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
  static constexpr int NS = 0, NM = 0;
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
  static constexpr int NS = 2, NM = 0;
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

// ---- KKT adjoint of the converged dual (tsvm_hypergrad) ----
struct VecRhsOp {  // v = src (Z^T src)
  static constexpr int R = 1, NS = 0, NM = 0;
  const double *src;
  __device__ void load(const double *) {}
  __device__ void rhs(int64_t i, double *v, double *, double *) const { v[0] = src[i]; }
};
struct StoreRowOp {  // dst = Z g
  static constexpr int R = 1, NS = 0, NM = 0;
  double *dst;
  __device__ void load(const double *) {}
  __device__ void row(int64_t i, const double *dot, double *, double *) const { dst[i] = dot[0]; }
};
// At the solution: D = s/x + xi/(C - x) of the final iterate, D^-1, and the SMW right-hand
// sides c/D and a/D.
struct AdjRowOp {
  static constexpr int NS = 0, NM = 0;
  Vecs V;
  const double *c;
  double C;
  __device__ void load(const double *sc) { C = sc[I_C]; }
  __device__ void row(int64_t i, double *, double *) const {
    const double x = V.x[i], xi = V.xi[i], a = (double)V.a[i];
    const double D = V.s[i] / x + xi / (C - x);
    V.dinv[i] = 1.0 / D;
    V.t1[i] = c[i] / D;
    V.t2[i] = a / D;
  }
};
// Refinement of the adjoint against the exact operator: rho = c - D lambda - Z Z^T lambda - a nu
// (dot = (Z Z^T lambda)_i), t1 = rho / D, and a^T lambda for the equality row.
struct AdjResidOp {
  static constexpr int R = 1, NS = 1, NM = 0;
  Vecs V;
  const double *c, *lam;
  double nu;
  __device__ void load(const double *sc) { nu = sc[I_Y]; }
  __device__ void row(int64_t i, const double *dot, double *sums, double *) const {
    const double a = (double)V.a[i], di = V.dinv[i];
    const double rho = c[i] - lam[i] / di - dot[0] - a * nu;
    V.t1[i] = rho * di;
    sums[0] += a * lam[i];
  }
};
// lambda += t - dnu u with dnu = (a^T t + a^T lambda) / a^T u (t = S^-1 rho in r7, u in b)
struct AdjUpdateOp {
  static constexpr int NS = 0, NM = 0;
  Vecs V;
  double *lam;
  double dnu;
  __device__ void load(const double *sc) { dnu = sc[I_DYC] + sc[I_RP] / sc[I_ATB]; }
  __device__ void row(int64_t i, double *, double *) const { lam[i] += V.r7[i] - dnu * V.b[i]; }
};
struct AdjLambdaOp {  // lambda = (D+Q)^-1 c - nu (D+Q)^-1 a, nu = a^T(D+Q)^-1 c / a^T(D+Q)^-1 a
  static constexpr int NS = 0, NM = 0;
  Vecs V;
  double *lam;
  double nu;
  __device__ void load(const double *sc) { nu = sc[I_DYA]; }
  __device__ void row(int64_t i, double *, double *) const { lam[i] = V.r7[i] - nu * V.b[i]; }
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
  if constexpr (NS + NM > 0) {
    if (threadIdx.x < NS + NM) {
      const int j = threadIdx.x;
      double r = j < NS ? 0.0 : INFINITY;
      for (int w = 0; w < kWarps; ++w)
        r = j < NS ? r + sh[j * kWarps + w] : fmin(r, sh[j * kWarps + w]);
      part_s[(int64_t)blockIdx.x * (NS + NM) + j] = r;
    }
  }
}

template <class Op>
__global__ void __launch_bounds__(kThreads)
vec_kernel(int64_t n, Op op, const double *__restrict__ scal, double *__restrict__ part_s,
           const WorkUnit *__restrict__ units, const int *__restrict__ active) {
  constexpr int NS = Op::NS, NM = Op::NM;
  __shared__ double vsh[(NS + NM > 0 ? NS + NM : 1) * kWarps];
  int64_t i0 = (int64_t)blockIdx.x * kThreads, i1 = n, istep = (int64_t)gridDim.x * kThreads;
  if (units) {  // batched: the rows of one work unit, that problem's scalars
    const WorkUnit u = units[blockIdx.x];
    if (active && !active[u.p]) return;
    scal += (size_t)u.p * kNScal;
    i0 = u.goff;
    i1 = u.goff + u.rows;
    istep = kThreads;
  }
  op.load(scal);
  double sums[NS > 0 ? NS : 1], mins[NM > 0 ? NM : 1];
#pragma unroll
  for (int j = 0; j < (NS > 0 ? NS : 1); ++j) sums[j] = 0.0;
#pragma unroll
  for (int j = 0; j < (NM > 0 ? NM : 1); ++j) mins[j] = INFINITY;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += istep) op.row(i, sums, mins);
  if (NS + NM > 0) block_partials<NS, NM>(sums, mins, part_s, vsh);
}

// ---------------------------------------------------------------------------------------
// Streaming passes over Z, fed by bulk (TMA) copies.  Persistent: one CTA per SM walks its
// CR-row chunks c, c + G, ...; a producer warp keeps up to `stages` chunks in flight (one
// contiguous cp.async.bulk per chunk, completion on an mbarrier) and the 8 consumer warps take
// whole chunks in turn (the j-th chunk of the CTA goes to warp j % 8), so each warp runs the
// per-row functor for CR rows at once (lane = row, one round trip to the vectors) and then
// streams the CR rows out of shared memory while the other warps wait on theirs:
//   MODE_ZT : v = op.rhs(row), acc += z_row v             (Z^T v, row functor)
//   MODE_ZW : d = z_row . w, then op.row(row, d)            (Z w, row epilogue)
//   MODE_ZGZ: d = z_row . g, acc += z_row (dinv_row d)      (Z^T D^-1 Z g)
// Column sums are reduced over the warps in shared memory into one FP64 partial per CTA (fixed
// order); side sums / minima likewise.  Waits are bounded; a CTA that gives up sets *err.
// ---------------------------------------------------------------------------------------
enum StreamMode : int { MODE_ZT = 0, MODE_ZW = 1, MODE_ZGZ = 2 };
constexpr int kSConsumers = 8;
constexpr int kSThreads = (kSConsumers + 1) * 32;

struct GramVecOp {  // no per-row functor (MODE_ZGZ)
  static constexpr int NS = 0, NM = 0;
  __device__ void load(const double *) {}
};

template <int MODE, class Op, int R, int CR, int LPR, int CPL>
__global__ void __launch_bounds__(kSThreads, 1)
stream_kernel(const float *__restrict__ Z, int64_t ldz, int k, int64_t n, Op op,
              const double *__restrict__ scal, const double *__restrict__ w,
              const double *__restrict__ dinv, int kz, int stages,
              double *__restrict__ part_vec, double *__restrict__ part_s, int *__restrict__ err,
              const WorkUnit *__restrict__ units, const float *const *__restrict__ Zs,
              const int *__restrict__ active) {
  constexpr int NS = Op::NS, NM = Op::NM;
  constexpr int RPW = 32 / LPR;          // rows per warp step
  constexpr int RW = CR;                 // rows per chunk, all taken by one warp
  constexpr int STEPS = RW / RPW;
  static_assert(RW % RPW == 0 && RW <= 32, "chunk rows must be a multiple of rows per step");
  constexpr int NC = CPL * 4;
  constexpr bool ACC = MODE != MODE_ZW;
  constexpr bool DOT = MODE != MODE_ZT;
  extern __shared__ __align__(128) uint8_t ssm[];
  const uint32_t chunk_bytes = (uint32_t)(CR * ldz * 4);
  float *stage0 = reinterpret_cast<float *>(ssm);
  uint64_t *bars = reinterpret_cast<uint64_t *>(ssm + (size_t)stages * chunk_bytes);
  const uint32_t b_full = tc::su32(bars), b_empty = b_full + 8 * stages;
  volatile int *abort = reinterpret_cast<volatile int *>(bars + 2 * stages);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / LPR, sl = lane % LPR;
  // this CTA's rows: the persistent slice of Z (chunks blockIdx.x, + gridDim.x, ...) or, in a
  // batched pass, all chunks of one work unit of one problem
  int64_t goff = 0, q0 = blockIdx.x, qs = gridDim.x;
  if (units) {
    const WorkUnit u = units[blockIdx.x];
    if (active && !active[u.p]) return;
    Z = Zs[u.p] + u.row0 * ldz;
    n = u.rows;
    goff = u.goff;
    scal += (size_t)u.p * kNScal;
    if (DOT) w += (size_t)u.p * R * kz;
    q0 = 0;
    qs = 1;
  }
  const int64_t nchunks = (n + CR - 1) / CR;
  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      tc::mbar_init(b_full + 8 * s, 1);
      tc::mbar_init(b_empty + 8 * s, 1);
    }
    *abort = 0;
    tc::fence_barrier_init();
  }
  __syncthreads();
  op.load(scal);
  double sums[NS > 0 ? NS : 1], mins[NM > 0 ? NM : 1];
#pragma unroll
  for (int j = 0; j < (NS > 0 ? NS : 1); ++j) sums[j] = 0.0;
#pragma unroll
  for (int j = 0; j < (NM > 0 ? NM : 1); ++j) mins[j] = INFINITY;
  double acc[ACC ? NC : 1][R];
  double wr[DOT ? NC : 1][R];
#pragma unroll
  for (int c = 0; c < CPL; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int col = 4 * (sl + c * LPR) + q;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (ACC) acc[4 * c + q][r] = 0.0;
        if constexpr (DOT) wr[4 * c + q][r] = col < k ? w[r * kz + col] : 0.0;
      }
    }

  if (warp == kSConsumers) {
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      for (int64_t q = q0; q < nchunks; q += qs) {
        if (!tc::mbar_wait(b_empty + 8 * st, ph ^ 1, abort)) break;
        const int64_t r0 = q * CR;
        const uint32_t bytes = (uint32_t)((n - r0 < CR ? n - r0 : CR) * ldz * 4);
        tc::mbar_expect_tx(b_full + 8 * st, bytes);
        tc::bulk_load(tc::su32(stage0) + st * chunk_bytes, Z + r0 * ldz, bytes, b_full + 8 * st);
        if (++st == stages) { st = 0; ph ^= 1; }
      }
    }
  } else {
    int64_t j = warp;   // index of the chunk among this CTA's chunks
    for (int64_t q = q0 + (int64_t)warp * qs; q < nchunks;
         q += (int64_t)kSConsumers * qs, j += kSConsumers) {
      const int st = (int)(j % stages);
      const uint32_t ph = (uint32_t)((j / stages) & 1);
      const int64_t r0 = q * CR;   // first row of the chunk
      // The per-row work that does not read the chunk goes before its wait, so that its vector
      // loads overlap the chunk's arrival: the right-hand side of Z^T v (lane = row) ...
      double v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = 0.0;
      if constexpr (MODE == MODE_ZT) {
        if (lane < RW && r0 + lane < n) op.rhs(goff + r0 + lane, v, sums, mins);
      }
      // ... and, for Z^T D^-1 Z g, the chunk's D^-1 values (lane = row), passed to each row's
      // lanes by a shuffle off the per-row dependency chain
      double dch = 0.0;
      if constexpr (MODE == MODE_ZGZ) {
        if (lane < RW && r0 + lane < n) dch = dinv[goff + r0 + lane];
      }
      if (!tc::mbar_wait(b_full + 8 * st, ph, abort)) break;
      const float *S = stage0 + (size_t)st * CR * ldz;
      double mine[R];
#pragma unroll
      for (int r = 0; r < R; ++r) mine[r] = 0.0;
      if constexpr (MODE == MODE_ZW && LPR == 32) {
        // Z w with whole rows per lane group: every lane keeps its partial dot products for all
        // RW rows of the chunk, then one recursive-halving exchange leaves each row's total in
        // 32 / RW lanes (about one double shuffle per row instead of a 5-level tree per row).
        constexpr int B = RW == 32 ? 5 : RW == 16 ? 4 : RW == 8 ? 3 : RW == 4 ? 2 : RW == 2 ? 1 : 0;
        static_assert((1 << B) == RW, "chunk rows must be a power of two");
        double pr[RW][R];
#pragma unroll
        for (int rr = 0; rr < RW; ++rr)
#pragma unroll
          for (int r = 0; r < R; ++r) pr[rr][r] = 0.0;
#pragma unroll
        for (int rr = 0; rr < RW; ++rr) {
          const bool in = r0 + rr < n;
          const float4 *zr = reinterpret_cast<const float4 *>(S + (size_t)rr * ldz);
#pragma unroll
          for (int c = 0; c < CPL; ++c) {
            const int g = lane + c * 32;
            float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in && 4 * g < k) {
              t = zr[g];
              if (4 * g + 3 >= k) {
                if (4 * g + 1 >= k) t.y = 0.f;
                if (4 * g + 2 >= k) t.z = 0.f;
                t.w = 0.f;
              }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
              pr[rr][r] = fma((double)t.x, wr[4 * c + 0][r], pr[rr][r]);
              pr[rr][r] = fma((double)t.y, wr[4 * c + 1][r], pr[rr][r]);
              pr[rr][r] = fma((double)t.z, wr[4 * c + 2][r], pr[rr][r]);
              pr[rr][r] = fma((double)t.w, wr[4 * c + 3][r], pr[rr][r]);
            }
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(b_empty + 8 * st);   // the chunk is in registers now
        // step s (lane offset 16 >> s) keeps the upper half of the rows where the lane bit is set
#pragma unroll
        for (int sb = 0; sb < B; ++sb) {
          const int off = 16 >> sb;
          const int half = RW >> (sb + 1);
          const bool upper = (lane & off) != 0;
#pragma unroll
          for (int i = 0; i < half; ++i)
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const double keep = upper ? pr[half + i][r] : pr[i][r];
              const double send = upper ? pr[i][r] : pr[half + i][r];
              pr[i][r] = keep + __shfl_xor_sync(0xffffffffu, send, off);
            }
        }
#pragma unroll
        for (int off = 16 >> B; off > 0; off >>= 1)
#pragma unroll
          for (int r = 0; r < R; ++r) pr[0][r] += __shfl_xor_sync(0xffffffffu, pr[0][r], off);
        const int myrow = (lane >> (5 - B)) & (RW - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) mine[r] = pr[0][r];
        if ((lane & ((32 >> B) - 1)) == 0 && r0 + myrow < n)
          op.row(goff + r0 + myrow, mine, sums, mins);
      } else {
        constexpr int UNR = CPL >= 4 ? 1 : 4;   // wide rows: keep the register footprint bounded
  #pragma unroll UNR
        for (int step = 0; step < STEPS; ++step) {
          const int rw = step * RPW + slot;
          const int64_t row = r0 + rw;
          const bool in = row < n;
          const float4 *zr = reinterpret_cast<const float4 *>(S + (size_t)rw * ldz);
          float4 z[CPL];
  #pragma unroll
          for (int c = 0; c < CPL; ++c) {
            const int g = sl + c * LPR;
            float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in && 4 * g < k) {
              t = zr[g];
              if (4 * g + 3 >= k) {
                if (4 * g + 1 >= k) t.y = 0.f;
                if (4 * g + 2 >= k) t.z = 0.f;
                t.w = 0.f;
              }
            }
            z[c] = t;
          }
          double vr[R];
          if constexpr (DOT) {
            double d[R];
  #pragma unroll
            for (int r = 0; r < R; ++r) d[r] = 0.0;
  #pragma unroll
            for (int c = 0; c < CPL; ++c)
  #pragma unroll
              for (int r = 0; r < R; ++r) {
                d[r] = fma((double)z[c].x, wr[4 * c + 0][r], d[r]);
                d[r] = fma((double)z[c].y, wr[4 * c + 1][r], d[r]);
                d[r] = fma((double)z[c].z, wr[4 * c + 2][r], d[r]);
                d[r] = fma((double)z[c].w, wr[4 * c + 3][r], d[r]);
              }
  #pragma unroll
            for (int r = 0; r < R; ++r) {
  #pragma unroll
              for (int o = LPR / 2; o > 0; o >>= 1) d[r] += __shfl_xor_sync(0xffffffffu, d[r], o);
            }
            if constexpr (MODE == MODE_ZW) {
  #pragma unroll
              for (int s2 = 0; s2 < RPW; ++s2)
  #pragma unroll
                for (int r = 0; r < R; ++r) {
                  const double got = __shfl_sync(0xffffffffu, d[r], s2 * LPR);
                  if (lane == step * RPW + s2) mine[r] = got;
                }
            } else {
              const double di = __shfl_sync(0xffffffffu, dch, rw);
  #pragma unroll
              for (int r = 0; r < R; ++r) vr[r] = d[r] * di;
            }
          } else {
  #pragma unroll
            for (int r = 0; r < R; ++r) vr[r] = __shfl_sync(0xffffffffu, v[r], rw);
          }
          if constexpr (ACC) {
  #pragma unroll
            for (int c = 0; c < CPL; ++c)
  #pragma unroll
              for (int r = 0; r < R; ++r) {
                acc[4 * c + 0][r] = fma((double)z[c].x, vr[r], acc[4 * c + 0][r]);
                acc[4 * c + 1][r] = fma((double)z[c].y, vr[r], acc[4 * c + 1][r]);
                acc[4 * c + 2][r] = fma((double)z[c].z, vr[r], acc[4 * c + 2][r]);
                acc[4 * c + 3][r] = fma((double)z[c].w, vr[r], acc[4 * c + 3][r]);
              }
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(b_empty + 8 * st);
        if constexpr (MODE == MODE_ZW) {
          if (lane < RW && r0 + lane < n) op.row(goff + r0 + lane, mine, sums, mins);
        }
      }
    }
  }
  __syncthreads();  // every chunk consumed: the stage memory is free for the reductions
  double *red = reinterpret_cast<double *>(ssm);
  if constexpr (ACC) {
    constexpr int ncol = LPR * NC;
    if (warp < kSConsumers) {
#pragma unroll
      for (int c = 0; c < CPL; ++c)
#pragma unroll
        for (int qq = 0; qq < 4; ++qq)
#pragma unroll
          for (int r = 0; r < R; ++r)
            red[((warp * RPW + slot) * R + r) * ncol + 4 * (sl + c * LPR) + qq] = acc[4 * c + qq][r];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < R * kz; e += blockDim.x) {
      const int r = e / kz, col = e % kz;
      double sum = 0.0;
      if (col < ncol)
        for (int ws = 0; ws < kSConsumers * RPW; ++ws) sum += red[(ws * R + r) * ncol + col];
      part_vec[(int64_t)blockIdx.x * R * kz + e] = sum;
    }
  }
  if constexpr (NS + NM > 0) {
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const double t = warp_sum(sums[j]);
      if (lane == 0) red[j * (kSConsumers + 1) + warp] = t;
    }
#pragma unroll
    for (int j = 0; j < NM; ++j) {
      const double t = warp_min(mins[j]);
      if (lane == 0) red[(NS + j) * (kSConsumers + 1) + warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < NS + NM) {
      const int j = threadIdx.x;
      double t = j < NS ? 0.0 : INFINITY;
      for (int ww = 0; ww < kSConsumers + 1; ++ww)
        t = j < NS ? t + red[j * (kSConsumers + 1) + ww]
                   : fmin(t, red[j * (kSConsumers + 1) + ww]);
      part_s[(int64_t)blockIdx.x * (NS + NM) + j] = t;
    }
  }
  if (threadIdx.x == 0 && *abort) atomicExch(err, 1);
}

// c = h0 - (g + w) (the residual h0 - M g of the capacitance solve, M g = g + Z^T D^-1 Z g);
// with `record`, the relative residual max_r ||c_r|| / ||h0_r|| goes into I_RESMAX, and a value
// above 0.5 (refinement cannot be trusted to converge) marks the iteration as failed.
__device__ void refine_resid_block(const double *__restrict__ h0, const double *__restrict__ g,
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

__global__ void refine_resid_kernel(const double *__restrict__ h0, const double *__restrict__ g,
                                    const double *__restrict__ w, double *__restrict__ c, int R,
                                    int kz, int k, double *__restrict__ sc, int *__restrict__ info,
                                    int record) {
  refine_resid_block(h0, g, w, c, R, kz, k, sc, info, record);
}

// The same per problem of a batch (block p; R kz entries per problem).
__global__ void refine_resid_batched(const double *__restrict__ h0, const double *__restrict__ g,
                                     const double *__restrict__ w, double *__restrict__ c, int R,
                                     int kz, int k, double *__restrict__ sc, int *__restrict__ info,
                                     const int *__restrict__ active) {
  const int p = blockIdx.x;
  if (active && !active[p]) return;
  const size_t o = (size_t)p * R * kz;
  refine_resid_block(h0 + o, g + o, w + o, c + o, R, kz, k, sc + (size_t)p * kNScal, info + p, 1);
}

// tau of each problem of a batched mixed-precision solve, as the single-problem solver adapts
// it: 64 at the first iteration; after a failed step (Cholesky or refinement, the step not
// taken) tau / 64 (0 below 1e-6: every row exact); else / 8 above a refinement residual of 1e-4
// and x 2 below 1e-6.  Also kept in the problem's scalars (I_TAU) for the host.
__global__ void tau_update_batched(double *__restrict__ sc, double *__restrict__ taus, int P,
                                   const int *__restrict__ active) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P || (active && !active[p])) return;
  double *s = sc + (size_t)p * kNScal;
  double tau = taus[p];
  if (s[I_TAUIT] == 0.0) {
    tau = 64.0;
  } else if (s[I_INFO] != 0.0) {
    tau = tau > 1e-6 ? tau / 64.0 : 0.0;
  } else {
    const double r = s[I_RESPREV];
    if (r > 1e-4) tau /= 8.0;
    else if (r < 1e-6 && tau < 1e30) tau *= 2.0;
  }
  taus[p] = tau;
  s[I_TAU] = tau;
  s[I_TAUIT] += 1.0;
}

__global__ void kvec_add(double *__restrict__ g, const double *__restrict__ c, int count) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) g[e] += c[e];
}

// The scalar algebra of one iteration stage on the reduced sums / minima `red`.
__device__ void scalar_stage(double *__restrict__ sc, const double *red, int stage,
                             const int *__restrict__ info) {
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
    case ST_ADJ:  // a^T lambda of the adjoint's current iterate
      sc[I_RP] = red[0];
      break;
    default:
      break;
  }
}

// Sum block partials in fixed order; the last block also reduces the scalars and runs the
// scalar stage of the iteration -- or, with red_out set (row-sharded solves), stores the
// reduced sums and minima there for the collective, after which scalar_stage_kernel runs.
__global__ void finalize_kernel(const double *__restrict__ part_vec, int nblk, int nvec,
                                double *__restrict__ out_vec, const double *__restrict__ part_s,
                                int ns, int nm, double *__restrict__ sc, int stage,
                                const int *__restrict__ info, double *__restrict__ red_out) {
  // vector blocks: 32 entries each, the partials split over 8 warps (strided), then summed in
  // warp order -- a fixed order, independent of timing
  const int vb = (nvec + 31) / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if ((int)blockIdx.x < vb) {
    __shared__ double vsum[8][32];
    const int e = blockIdx.x * 32 + lane;
    double s = 0.0;
    if (e < nvec) {
#pragma unroll 4
      for (int b = warp; b < nblk; b += 8) s += part_vec[(int64_t)b * nvec + e];
    }
    vsum[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && e < nvec) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += vsum[w][lane];
      out_vec[e] = t;
    }
    return;
  }
  __shared__ double red[16];
  for (int j = warp; j < ns + nm; j += 8) {
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
  if (red_out) {
    for (int j = 0; j < ns + nm; ++j) red_out[j] = red[j];
    return;
  }
  scalar_stage(sc, red, stage, info);
}

// The scalar stage on sums / minima completed across the ranks (row-sharded solves).
__global__ void scalar_stage_kernel(double *__restrict__ sc, const double *__restrict__ red,
                                    int stage, const int *__restrict__ info) {
  if (threadIdx.x == 0) scalar_stage(sc, red, stage, info);
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

  int *err;   // set by a streaming pass that timed out
  // SMs left free by the streaming passes (1 while the k x k Cholesky runs beside one)
  int sm_reserve = 0;
  // row-sharded solves: every finalize completes its sums / minima across the ranks
  bool shard = false;
  double *red_buf = nullptr;   // 16 doubles

  // One streaming pass (stream_kernel) with this solve's geometry: one CTA per SM, as many
  // chunk stages as fit in ~192 KB of shared memory (at least 2, at most 16, and room for the
  // reduction).
  template <int MODE, class Op, int R, int CR, int LPR, int CPL>
  tsvm_status pass_launch(const Op &op, const double *w, double *out_vec, int stage) {
    constexpr int RPW = 32 / LPR;
    const size_t chunk = (size_t)CR * ldz * 4;
    size_t stages = std::min<size_t>(16, std::max<size_t>(2, (192 * 1024) / chunk));
    const size_t red = sizeof(double) * std::max<size_t>(
        MODE != MODE_ZW ? (size_t)kSConsumers * RPW * R * LPR * CPL * 4 : 0,
        16 * (kSConsumers + 1));
    while (stages * chunk < red) ++stages;
    const size_t smem = stages * chunk + 8 * (2 * stages + 2);
    auto kern = stream_kernel<MODE, Op, R, CR, LPR, CPL>;
    TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(std::min(nblk, ctx->num_sms - sm_reserve), ceil_div(n, CR)));
    kern<<<grid, kSThreads, smem, ctx->stream>>>(Z, ldz, k, n, op, scal, w, dinv, geo.kz,
                                                 (int)stages, part_vec, part_s, err, nullptr,
                                                 nullptr, nullptr);
    TSVM_LAUNCHED(ctx);
    return finalize(grid, MODE != MODE_ZW ? R * geo.kz : 0, out_vec, Op::NS, Op::NM, stage);
  }
  template <int MODE, class Op, int R>
  tsvm_status pass(const Op &op, const double *w, double *out_vec, int stage) {
    switch (geo.lpr * 10 + geo.cpl) {
      case 81: return pass_launch<MODE, Op, R, 32, 8, 1>(op, w, out_vec, stage);
      case 161: return pass_launch<MODE, Op, R, 32, 16, 1>(op, w, out_vec, stage);
      case 321: return pass_launch<MODE, Op, R, 32, 32, 1>(op, w, out_vec, stage);
      case 322: return pass_launch<MODE, Op, R, 16, 32, 2>(op, w, out_vec, stage);
      case 324: return pass_launch<MODE, Op, R, 8, 32, 4>(op, w, out_vec, stage);
      case 328: return pass_launch<MODE, Op, R, 8, 32, 8>(op, w, out_vec, stage);
    }
    return TSVM_ERR_UNSUPPORTED;
  }
  // Z^T v with v from the per-row functor (plus its side reductions)
  template <class Op>
  tsvm_status zt(const Op &op, double *out_vec, int stage) {
    return pass<MODE_ZT, Op, Op::R>(op, nullptr, out_vec, stage);
  }
  // Z w per row, then the per-row functor
  template <class Op>
  tsvm_status zw(const Op &op, const double *w, int stage) {
    return pass<MODE_ZW, Op, Op::R>(op, w, nullptr, stage);
  }
  // Z^T D^-1 Z g for R vectors g
  template <int R>
  tsvm_status zgz(const double *g, double *w) {
    return pass<MODE_ZGZ, GramVecOp, R>(GramVecOp{}, g, w, ST_NONE);
  }
  // Iterative refinement of the capacitance solve M g = h0 against the exact M (M~ factored in
  // M_fac): per sweep one pass over Z for w = Z^T D^-1 Z g, then g += M~^-1 (h0 - g - w).
  template <int R>
  tsvm_status refine(const double *M_fac, const double *M_dinv, const double *h0, double *g,
                     double *w, double *c, int sweeps) {
    for (int sweep = 0; sweep < sweeps; ++sweep) {
      TSVM_TRY(zgz<R>(g, w));
      refine_resid_kernel<<<1, 256, 0, ctx->stream>>>(h0, g, w, c, R, geo.kz, k, scal, info,
                                                        sweep == 0 ? 1 : 0);
      TSVM_LAUNCHED(ctx);
      TSVM_TRY(potrs_fp64(ctx, M_fac, k, k, M_dinv, c, R, geo.kz));
      kvec_add<<<(unsigned)ceil_div(R * geo.kz, 256), 256, 0, ctx->stream>>>(g, c, R * geo.kz);
      TSVM_LAUNCHED(ctx);
    }
    return TSVM_OK;
  }
  template <class Op>
  tsvm_status vec(const Op &op, int stage) {
    auto kern = vec_kernel<Op>;
    const int grid = grid_for(reinterpret_cast<const void *>(kern), 0);
    kern<<<grid, kThreads, 0, ctx->stream>>>(n, op, scal, part_s, nullptr, nullptr);
    TSVM_LAUNCHED(ctx);
    if (Op::NS + Op::NM == 0 && stage == ST_NONE) return TSVM_OK;
    return finalize(grid, 0, nullptr, Op::NS, Op::NM, stage);
  }
  // Grid of an elementwise launch: all blocks resident at once (the kernels stride over the
  // rows), at most nblk (the capacity of the partial-sum buffers).
  std::unordered_map<const void *, int> occ_cache;
  int grid_for(const void *kern, size_t smem) {
    auto it = occ_cache.find(kern);
    int occ;
    if (it != occ_cache.end()) {
      occ = it->second;
    } else {
      occ = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem) != cudaSuccess)
        occ = 1;
      occ = std::max(1, occ);
      occ_cache[kern] = occ;
    }
    return std::max(1, std::min(nblk, occ * ctx->num_sms));
  }
  tsvm_status finalize(int nparts, int nvec, double *out_vec, int ns, int nm, int stage) {
    const int vb = (nvec + 31) / 32;
    finalize_kernel<<<vb + 1, 256, 0, ctx->stream>>>(part_vec, nparts, nvec, out_vec, part_s, ns,
                                                      nm, scal, stage, info,
                                                      shard ? red_buf : nullptr);
    TSVM_LAUNCHED(ctx);
    if (!shard) return TSVM_OK;
    // the same collectives on every rank: the vector, the sums, the minima
    TSVM_TRY(comm_allreduce(ctx, out_vec, nvec, 0, COMM_SUM));
    TSVM_TRY(comm_allreduce(ctx, red_buf, ns, 0, COMM_SUM));
    TSVM_TRY(comm_allreduce(ctx, red_buf + ns, nm, 0, COMM_MIN));
    scalar_stage_kernel<<<1, 32, 0, ctx->stream>>>(scal, red_buf, stage, info);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
};

// Sum of the k x k matrix over the ranks when each rank's copy holds I + its rows' sum: the
// identity is counted once.
tsvm_status comm_capacitance(tsvm_context *ctx, double *M, int k) {
  if (!sharded(ctx)) return TSVM_OK;
  TSVM_TRY(comm_allreduce(ctx, M, (int64_t)k * k, 0, COMM_SUM));
  return small_add_diag(ctx, M, k, k, -(double)(ctx->comm.world - 1));
}

}  // namespace

tsvm_status ipm_solve(tsvm_context *ctx, const float *Z, int ldz, const float *y, int64_t n,
                      int k, double C, const tsvm_ipm_options &opt, double *alpha_out,
                      double *xi_out, double *s_out, double *ymult_out, tsvm_ipm_stats *stats) {
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
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)k * k + (size_t)ceil_div(k, 32) * 1024, &M));
  double *Mdinv = M + (size_t)k * k;   // inverses of the 32 x 32 diagonal blocks of chol(M)
  static_assert(3 * sizeof(int) <= 8 * sizeof(double), "status words before red_buf");
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
  int *big_count = run.info + 1;                     // [1] rows summed exactly in FP64,
  run.err = run.info + 2;                            // [2] streaming-pass timeout
  run.red_buf = cv + 2 * kz + 8;                     // 16 doubles (row-sharded solves)
  run.shard = sharded(ctx);
  // rows of the whole problem (this rank's n when the problem is not sharded)
  double n_global = (double)n;
  TSVM_TRY(comm_sum_host(ctx, &n_global));

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
  int host_info[3] = {0, 0, 0};
  int64_t exact_rows_sum = 0;
  int exact_rows_max = 0, syrk_retries = 0, mixed_iters = 0;
  double res_max = 0.0;

  double hsc[kNScal] = {0};
  hsc[I_C] = C;
  hsc[I_N] = n_global;
  TSVM_CUDA(cudaMemcpyAsync(run.scal, hsc, sizeof(hsc), cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemsetAsync(run.info, 0, 3 * sizeof(int), ctx->stream));

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
    TSVM_TRY(run.vec(FillOp{V, 0.0}, ST_NONE));
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
    TraceRange trace_iter("ipm iteration");
    TSVM_TRY(run.zt(BeginOp{V, C}, q, ST_BEGIN));
    TSVM_TRY(run.zw(ResidOp{V, 0.0}, q, ST_RESID));
    TSVM_CUDA(cudaMemcpyAsync(ctx->host_scalars, run.scal, sizeof(double) * kNScal,
                              cudaMemcpyDeviceToHost, ctx->stream));
    TSVM_CUDA(cudaMemcpyAsync(host_info, run.info, sizeof(host_info), cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(sc, ctx->host_scalars, sizeof(sc));
    if (run.shard) {   // a rank whose pass timed out takes the others out with it
      double e = host_info[2] ? 1.0 : 0.0;
      TSVM_TRY(comm_sum_host(ctx, &e));
      if (e > 0.0) return timeout_status("ipm streaming pass (another rank)");
    }
    if (host_info[2]) return timeout_status("ipm streaming pass");
    if (pending_events) {
      ms_syrk += event_ms(ev_syrk0, ev_syrk1);
      ms_factor += event_ms(ev_syrk1, ev_chol1);
      pending_events = false;
    }
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
    const double mu = sc[I_MU], nrd = sc[I_NORMRD], nrp = fabs(sc[I_RP]), cond = sc[I_COND];
    if (t_gap < 0 && sc[I_RELGAP] <= 1e-6) {
      const double scale = 1.0 + sqrt(n_global);
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
      const double scale = 1.0 + sqrt(n_global);
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
      TSVM_TRY(comm_capacitance(ctx, M, k));
    } else {
      TSVM_TRY(gram_fp64(ctx, Z, ldz, Z, ldz, n, k, k, true, M, V.dinv));
      TSVM_TRY(comm_allreduce(ctx, M, (int64_t)k * k, 0, COMM_SUM));
      TSVM_TRY(small_add_diag(ctx, M, k, k, 1.0));
    }
    TSVM_CUDA(cudaEventRecord(ev_syrk1, ctx->stream));
    // predictor: r7 = SMW(r5), b = SMW(a) in one pair of passes.  The right-hand sides
    // Z^T [r5/D, a/D] do not need M.  Above k = 256 the Cholesky (one CTA, latency-bound) runs
    // on the high-priority side stream on one SM while that pass streams Z on the others.  Up to
    // k = 256 it is the cluster kernel, which needs eight free SMs of one GPC: beside the
    // persistent pass it only started once the pass had ended, so it runs in line before it.
    if (!run.shard && chol_fp64_sms(k) == 1) {
      TSVM_CUDA(cudaEventRecord(ctx->fork_ev, ctx->stream));
      TSVM_CUDA(cudaStreamWaitEvent(ctx->side_stream, ctx->fork_ev, 0));
      TSVM_TRY(chol_fp64(ctx, M, k, k, run.info, Mdinv, ctx->side_stream));
      TSVM_CUDA(cudaEventRecord(ev_chol1, ctx->side_stream));
      run.sm_reserve = 1;
      const tsvm_status st_rhs = run.zt(SmwRhs2Op{V}, h, ST_NONE);
      run.sm_reserve = 0;
      TSVM_CUDA(cudaStreamWaitEvent(ctx->stream, ev_chol1, 0));
      TSVM_TRY(st_rhs);
    } else {
      TSVM_TRY(chol_fp64(ctx, M, k, k, run.info, Mdinv));
      TSVM_CUDA(cudaEventRecord(ev_chol1, ctx->stream));
      TSVM_TRY(run.zt(SmwRhs2Op{V}, h, ST_NONE));
    }
    pending_events = true;
    if (sweeps)
      TSVM_CUDA(cudaMemcpyAsync(h0, h, sizeof(double) * 2 * kz, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    TSVM_TRY(potrs_fp64(ctx, M, k, k, Mdinv, h, 2, kz));
    if (sweeps) TSVM_TRY(run.refine<2>(M, Mdinv, h0, h, wv, cv, sweeps));
    TSVM_TRY(run.zw(SmwBack2Op{V}, h, ST_DYA));
    TSVM_TRY(run.vec(AffineOp{V, C, 0.0}, ST_ALPHA_AFF));
    TSVM_TRY(run.vec(MuAffOp{V, C, 0.0}, ST_SIGMA));
    // corrector
    TSVM_TRY(run.zt(CorrRhsOp{V, C, 0.0}, h, ST_NONE));
    if (sweeps)
      TSVM_CUDA(cudaMemcpyAsync(h0, h, sizeof(double) * kz, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    TSVM_TRY(potrs_fp64(ctx, M, k, k, Mdinv, h, 1, kz));
    if (sweeps) TSVM_TRY(run.refine<1>(M, Mdinv, h0, h, wv, cv, sweeps));
    TSVM_TRY(run.zw(CorrBackOp{V}, h, ST_DYC));
    TSVM_TRY(run.vec(CombineOp{V, C, 0.0, 0.0}, ST_ALPHA));
    TSVM_TRY(run.vec(UpdateOp{V, 0.0, true}, ST_NONE));
  }
  if (iter >= opt.max_iter) result = TSVM_WARN_MAX_ITER;
  TSVM_CUDA(cudaMemcpyAsync(alpha_out, V.x, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  if (s_out)
    TSVM_CUDA(cudaMemcpyAsync(s_out, V.s, sizeof(double) * n, cudaMemcpyDeviceToDevice,
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
                                  int64_t *__restrict__ idx, int *__restrict__ count) {
  // The first `want` free SVs (1e-6 < alpha < C - 1e-6) in index order.  Each thread keeps its
  // own running count, updated from the same per-warp counts after the same barrier, so the
  // loop-top test is uniform over the block.
  __shared__ int wcnt[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int found = 0;
  for (int64_t base = 0; base < n && found < want; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    bool f = false;
    if (i < n) {
      const double a = alpha[i];
      f = a > 1e-6 && a < C - 1e-6;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int off = found, tot = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) off += wcnt[w];
      tot += wcnt[w];
    }
    off += __popc(bal & ((1u << lane) - 1u));
    if (f && off < want) idx[off] = i;
    found += tot;
    __syncthreads();  // wcnt is rewritten by the next round
  }
  if (threadIdx.x == 0) *count = found < want ? found : want;
}

__global__ void bias_terms_kernel(const float *__restrict__ Z, int64_t ldz, int k,
                                  const float *__restrict__ y, const double *__restrict__ v,
                                  const int64_t *__restrict__ idx, const int *__restrict__ count,
                                  double *__restrict__ out, double *__restrict__ slot) {
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
    if (slot) {   // row-sharded: this rank's terms, merged across the ranks afterwards
      slot[0] = (double)m;
      for (int t = 0; t < m; ++t) slot[1 + t] = bj[t];
      return;
    }
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

// Row-sharded bias: terms[r * 51] = rank r's count m_r (<= 50), then its m_r terms in index
// order.  The ranks hold consecutive row ranges in rank order, so the first <= 50 free SVs of
// the whole problem are the ranks' terms taken in rank order.
__global__ void bias_merge_kernel(const double *__restrict__ terms, int world, double *out) {
  if (threadIdx.x != 0) return;
  double take[50];
  int m = 0;
  for (int r = 0; r < world && m < 50; ++r) {
    const int mr = (int)terms[(int64_t)r * 51];
    for (int t = 0; t < mr && m < 50; ++t) take[m++] = terms[(int64_t)r * 51 + 1 + t];
  }
  if (m == 0) {
    out[0] = NAN;
    out[1] = NAN;
    return;
  }
  double mean = 0.0;
  for (int t = 0; t < m; ++t) mean += take[t];
  mean /= m;
  double ss = 0.0;
  for (int t = 0; t < m; ++t) ss += (take[t] - mean) * (take[t] - mean);
  out[0] = mean;
  out[1] = sqrt(ss / m);
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
  int64_t *idx = reinterpret_cast<int64_t *>(out + 4);
  int *cnt = reinterpret_cast<int *>(idx + 64);
  run.info = cnt + 1;
  run.err = cnt + 2;
  run.red_buf = out + 4 + 64 + 8;   // 16 doubles after idx and the status words
  run.shard = sharded(ctx);
  TSVM_CUDA(cudaMemsetAsync(run.err, 0, sizeof(int), ctx->stream));
  TSVM_TRY(run.vec(BiasCountOp{alpha, C}, ST_INIT));  // counts into I_E2SUM / I_E2SQ slots
  TSVM_TRY(run.zt(BiasRhsOp{alpha}, v, ST_NONE));
  first_free_kernel<<<1, 1024, 0, ctx->stream>>>(alpha, n, C, 50, idx, cnt);
  TSVM_LAUNCHED(ctx);
  if (run.shard) {
    const int world = ctx->comm.world;
    double *terms = nullptr;
    TSVM_TRY(scratch_t(ctx, SLOT_COMM, (size_t)world * 51 + 8, &terms));
    TSVM_CUDA(cudaMemsetAsync(terms, 0, sizeof(double) * world * 51, ctx->stream));
    bias_terms_kernel<<<1, 256, 0, ctx->stream>>>(Z, ldz, k, y, v, idx, cnt, out,
                                                    terms + (size_t)ctx->comm.rank * 51);
    TSVM_LAUNCHED(ctx);
    TSVM_TRY(comm_allreduce(ctx, terms, (int64_t)world * 51, 0, COMM_SUM));
    bias_merge_kernel<<<1, 32, 0, ctx->stream>>>(terms, world, out);
    TSVM_LAUNCHED(ctx);
  } else {
    bias_terms_kernel<<<1, 256, 0, ctx->stream>>>(Z, ldz, k, y, v, idx, cnt, out, nullptr);
    TSVM_LAUNCHED(ctx);
  }
  double hs[2], hb[2];
  int herr = 0;
  TSVM_CUDA(cudaMemcpyAsync(hs, run.scal + I_E2SUM, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(hb, out, sizeof(hb), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(&herr, run.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (herr) return timeout_status("bias pass");
  if (nsv) *nsv = (int32_t)hs[0];
  if (nfree) *nfree = (int32_t)hs[1];
  if (b) *b = hb[0];
  if (bstd) *bstd = hb[1];
  return TSVM_OK;
}


// ---------------------------------------------------------------------------------------
// Linear algebra of the KKT adjoint (tsvm_hypergrad)
// ---------------------------------------------------------------------------------------
namespace {

// nu of the adjoint: after the first solve nu = I_DYA; each refinement adds dnu.
__global__ void adj_nu_kernel(double *sc, int first) {
  if (threadIdx.x != 0) return;
  if (first) sc[I_Y] = sc[I_DYA];
  else sc[I_Y] += sc[I_DYC] + sc[I_RP] / sc[I_ATB];
}

__global__ void add_relative_diag(double *A, int k, double rel) {
  __shared__ double tr;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < k; ++i) t += A[(int64_t)i * k + i];
    tr = t;
  }
  __syncthreads();
  const double shift = rel * tr / k + 1e-300;
  for (int i = threadIdx.x; i < k; i += blockDim.x) A[(int64_t)i * k + i] += shift;
}

// A Runner over Z with its own scratch (the adjoint's vectors live in SLOT_IPM_VEC like the
// solver's: call it after tsvm_ipm, not during).
tsvm_status make_runner(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k, Runner &run,
                        double **sbuf) {
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
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_SCAL, (size_t)kNScal + 10 * (size_t)kz + 64, sbuf));
  double *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_PART, (size_t)run.nblk * (2 * kz + 16), &part));
  run.part_vec = part;
  run.part_s = part + (size_t)run.nblk * 2 * kz;
  run.scal = *sbuf;
  run.info = reinterpret_cast<int *>(*sbuf + kNScal + 9 * kz);
  run.err = run.info + 2;
  TSVM_CUDA(cudaMemsetAsync(run.info, 0, 3 * sizeof(int), ctx->stream));
  return TSVM_OK;
}

tsvm_status check_runner(tsvm_context *ctx, Runner &run) {
  int h[3] = {0, 0, 0};
  TSVM_CUDA(cudaMemcpyAsync(h, run.info, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h[2]) return timeout_status("ipm runner pass");
  if (h[0]) return TSVM_ERR_NOT_SPD;
  return TSVM_OK;
}

}  // namespace

tsvm_status zt_vec(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k, const double *v,
                   double *out) {
  Runner run;
  double *sbuf = nullptr;
  TSVM_TRY(make_runner(ctx, Z, ldz, n, k, run, &sbuf));
  run.dinv = nullptr;
  TSVM_TRY(run.zt(VecRhsOp{v}, out, ST_NONE));
  return check_runner(ctx, run);
}

tsvm_status zw_vec(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k, const double *g,
                   double *out) {
  Runner run;
  double *sbuf = nullptr;
  TSVM_TRY(make_runner(ctx, Z, ldz, n, k, run, &sbuf));
  run.dinv = nullptr;
  TSVM_TRY(run.zw(StoreRowOp{out}, g, ST_NONE));
  return check_runner(ctx, run);
}

tsvm_status kkt_adjoint(tsvm_context *ctx, const float *Z, int ldz, const float *y, int64_t n,
                        int k, double C, const double *alpha, const double *xi, const double *s,
                        const double *c, double *lambda) {
  Runner run;
  double *sbuf = nullptr;
  TSVM_TRY(make_runner(ctx, Z, ldz, n, k, run, &sbuf));
  const int kz = run.geo.kz;
  double *vecbuf = nullptr, *M = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_VEC, (size_t)11 * n, &vecbuf));
  TSVM_TRY(scratch_t(ctx, SLOT_IPM_M, (size_t)k * k + (size_t)ceil_div(k, 32) * 1024, &M));
  double *Mdinv = M + (size_t)k * k;
  Vecs V;
  V.x = const_cast<double *>(alpha);
  V.xi = const_cast<double *>(xi);
  V.s = const_cast<double *>(s);
  V.dinv = vecbuf + n;
  V.t1 = V.dinv + n;
  V.t2 = V.t1 + n;
  V.r7 = V.t2 + n;
  V.b = V.r7 + n;
  V.dx = V.b + n;
  V.ds = V.dx + n;
  V.dxi = V.ds + n;
  V.a = y;
  run.dinv = V.dinv;
  double hsc[kNScal] = {0};
  hsc[I_C] = C;
  hsc[I_N] = (double)n;
  hsc[I_RP] = 0.0;
  TSVM_CUDA(cudaMemcpyAsync(run.scal, hsc, sizeof(hsc), cudaMemcpyHostToDevice, ctx->stream));
  double *h = sbuf + kNScal + kz;
  TSVM_TRY(run.vec(AdjRowOp{V, c, 0.0}, ST_NONE));         // D, c/D, a/D
  TSVM_TRY(gram_fp64(ctx, Z, ldz, Z, ldz, n, k, k, true, M, V.dinv));
  TSVM_TRY(small_add_diag(ctx, M, k, k, 1.0));
  TSVM_TRY(chol_fp64(ctx, M, k, k, run.info, Mdinv));
  TSVM_TRY(run.zt(SmwRhs2Op{V}, h, ST_NONE));
  TSVM_TRY(potrs_fp64(ctx, M, k, k, Mdinv, h, 2, kz));
  TSVM_TRY(run.zw(SmwBack2Op{V}, h, ST_DYA));
  TSVM_TRY(run.vec(AdjLambdaOp{V, lambda, 0.0}, ST_NONE));
  adj_nu_kernel<<<1, 32, 0, ctx->stream>>>(run.scal, 1);
  TSVM_LAUNCHED(ctx);
  // The SMW back-substitution loses accuracy where D is tiny (free support vectors at the end
  // of the solve: D^-1 ~ 1/mu); refine in n-space against the exact operator D + Z Z^T.
  for (int sweep = 0; sweep < 3; ++sweep) {
    TSVM_TRY(run.zt(VecRhsOp{lambda}, h, ST_NONE));                  // Z^T lambda
    TSVM_TRY(run.zw(AdjResidOp{V, c, lambda, 0.0}, h, ST_ADJ));      // rho / D, a^T lambda
    TSVM_TRY(run.zt(VecRhsOp{V.t1}, h, ST_NONE));
    TSVM_TRY(potrs_fp64(ctx, M, k, k, Mdinv, h, 1, kz));
    TSVM_TRY(run.zw(CorrBackOp{V}, h, ST_DYC));                       // t = S^-1 rho
    TSVM_TRY(run.vec(AdjUpdateOp{V, lambda, 0.0}, ST_NONE));
    adj_nu_kernel<<<1, 32, 0, ctx->stream>>>(run.scal, 0);
    TSVM_LAUNCHED(ctx);
  }
  return check_runner(ctx, run);
}

tsvm_status project_range(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k,
                          const double *v, double *out) {
  Runner run;
  double *sbuf = nullptr;
  TSVM_TRY(make_runner(ctx, Z, ldz, n, k, run, &sbuf));
  const int kz = run.geo.kz;
  double *G = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SMALL3, (size_t)k * k + (size_t)ceil_div(k, 32) * 1024, &G));
  double *Gdinv = G + (size_t)k * k;
  run.dinv = nullptr;
  double *q = sbuf + kNScal;
  TSVM_TRY(gram_fp64(ctx, Z, ldz, Z, ldz, n, k, k, true, G));
  add_relative_diag<<<1, 256, 0, ctx->stream>>>(G, k, 1e-12);  // clipped (zero) columns
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(chol_fp64(ctx, G, k, k, run.info, Gdinv));
  TSVM_TRY(run.zt(VecRhsOp{v}, q, ST_NONE));
  TSVM_TRY(potrs_fp64(ctx, G, k, k, Gdinv, q, 1, kz));
  TSVM_TRY(run.zw(StoreRowOp{out}, q, ST_NONE));
  return check_runner(ctx, run);
}

// ---------------------------------------------------------------------------------------
// Batched interior-point solve: every pass is one launch over the work units (row ranges of
// one problem) of all unconverged problems; k x k work is one launch with a CTA per problem.
// ---------------------------------------------------------------------------------------
namespace {

// Per-problem reduction of the unit partials (units of problem p are ubeg[p] .. ubeg[p+1]-1,
// summed in that order) and the scalar stage of each active problem.  One block per problem.
__global__ void finalize_batched_kernel(const double *__restrict__ part_vec,
                                        const double *__restrict__ part_s,
                                        const int *__restrict__ ubeg, int nvec,
                                        double *__restrict__ out_vec, int ns, int nm,
                                        double *__restrict__ sc, int stage,
                                        const int *__restrict__ info,
                                        const int *__restrict__ active) {
  const int p = blockIdx.x;
  if (active && !active[p]) return;
  const int u0 = ubeg[p], u1 = ubeg[p + 1];
  for (int e = threadIdx.x; e < nvec; e += blockDim.x) {
    double s = 0.0;
    for (int u = u0; u < u1; ++u) s += part_vec[(int64_t)u * nvec + e];
    out_vec[(int64_t)p * nvec + e] = s;
  }
  __shared__ double red[16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = warp; j < ns + nm; j += nw) {
    double r = j < ns ? 0.0 : INFINITY;
    for (int u = u0 + lane; u < u1; u += 32) {
      const double v = part_s[(int64_t)u * (ns + nm) + j];
      r = j < ns ? r + v : fmin(r, v);
    }
    r = j < ns ? warp_sum(r) : warp_min(r);
    if (lane == 0) red[j] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) scalar_stage(sc + (size_t)p * kNScal, red, stage, info + p);
}

// M_p = I + sum over the units of p of their partial Gram matrices (lower tiles), mirrored.
__global__ void gram_units_reduce(const double *__restrict__ part, const int *__restrict__ ubeg,
                                  int k, const int *__restrict__ active, double *__restrict__ M,
                                  int64_t strideM) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)k * k) return;
  const int r = (int)(e / k), c = (int)(e % k);
  if (c > r) return;
  double s = r == c ? 1.0 : 0.0;
  for (int u = ubeg[p]; u < ubeg[p + 1]; ++u) s += part[(int64_t)u * k * k + (int64_t)r * k + c];
  double *Mp = M + p * strideM;
  Mp[(int64_t)r * k + c] = s;
  Mp[(int64_t)c * k + r] = s;
}

// Mixed-precision capacitance matrices of a batch: M_p = I + sum over the units of p of the
// tensor-core partials (FP32, KP x KP, lower block strips) and the exactly summed rows' partials
// (FP64, k x k, lower tiles), in unit order; NaN if a tensor-core block timed out.
__global__ void mixed_units_reduce(const float *__restrict__ part_tc, int KP,
                                   const double *__restrict__ part64, const int *__restrict__ ubeg,
                                   int k, const int *__restrict__ active,
                                   const int *__restrict__ err, double *__restrict__ M,
                                   int64_t strideM, const int *__restrict__ counts, int parts) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)k * k) return;
  const int r = (int)(e / k), c = (int)(e % k);
  if (c > r) return;
  double s = r == c ? 1.0 : 0.0;
  for (int u = ubeg[p]; u < ubeg[p + 1]; ++u) {
    s += (double)part_tc[(int64_t)u * KP * KP + (int64_t)r * KP + c];
    const int cnt = counts[u];
    for (int j = 0; j < parts; ++j)   // the pieces of the unit's exact rows that hold any
      if (gram_units_piece_rows(cnt, parts, j))
        s += part64[((int64_t)u * parts + j) * k * k + (int64_t)r * k + c];
  }
  if (*err) s = NAN;
  double *Mp = M + p * strideM;
  Mp[(int64_t)r * k + c] = s;
  Mp[(int64_t)c * k + r] = s;
}

// Stages and shared memory of one streaming pass (see Runner::pass_launch).
template <int MODE, int R, int CR, int LPR, int CPL>
void stream_config(int64_t ldz, size_t *stages_out, size_t *smem_out) {
  constexpr int RPW = 32 / LPR;
  const size_t chunk = (size_t)CR * ldz * 4;
  size_t stages = std::min<size_t>(16, std::max<size_t>(2, (192 * 1024) / chunk));
  const size_t red = sizeof(double) * std::max<size_t>(
      MODE != MODE_ZW ? (size_t)kSConsumers * RPW * R * LPR * CPL * 4 : 0,
        16 * (kSConsumers + 1));
  while (stages * chunk < red) ++stages;
  *stages_out = stages;
  *smem_out = stages * chunk + 8 * (2 * stages + 2);
}

struct BRunner {
  tsvm_context *ctx;
  const float *const *Zs;   // device table of the problems' Z
  int64_t ldz;
  int k, P, nunits;
  Geometry geo;
  const WorkUnit *units;
  const int *ubeg, *active;
  double *scal, *part_vec, *part_s;
  int *info, *err;
  const double *dinv;

  template <int MODE, class Op, int R, int CR, int LPR, int CPL>
  tsvm_status pass_launch(const Op &op, const double *w, double *out_vec, int stage) {
    size_t stages, smem;
    stream_config<MODE, R, CR, LPR, CPL>(ldz, &stages, &smem);
    auto kern = stream_kernel<MODE, Op, R, CR, LPR, CPL>;
    TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<nunits, kSThreads, smem, ctx->stream>>>(nullptr, ldz, k, 0, op, scal, w, dinv, geo.kz,
                                                   (int)stages, part_vec, part_s, err, units, Zs,
                                                   active);
    TSVM_LAUNCHED(ctx);
    return finalize(MODE != MODE_ZW ? R * geo.kz : 0, out_vec, Op::NS, Op::NM, stage);
  }
  template <int MODE, class Op, int R>
  tsvm_status pass(const Op &op, const double *w, double *out_vec, int stage) {
    switch (geo.lpr * 10 + geo.cpl) {
      case 81: return pass_launch<MODE, Op, R, 32, 8, 1>(op, w, out_vec, stage);
      case 161: return pass_launch<MODE, Op, R, 32, 16, 1>(op, w, out_vec, stage);
      case 321: return pass_launch<MODE, Op, R, 32, 32, 1>(op, w, out_vec, stage);
      case 322: return pass_launch<MODE, Op, R, 16, 32, 2>(op, w, out_vec, stage);
      case 324: return pass_launch<MODE, Op, R, 8, 32, 4>(op, w, out_vec, stage);
      case 328: return pass_launch<MODE, Op, R, 8, 32, 8>(op, w, out_vec, stage);
    }
    return TSVM_ERR_UNSUPPORTED;
  }
  template <class Op>
  tsvm_status zt(const Op &op, double *out_vec, int stage) {
    return pass<MODE_ZT, Op, Op::R>(op, nullptr, out_vec, stage);
  }
  template <class Op>
  tsvm_status zw(const Op &op, const double *w, int stage) {
    return pass<MODE_ZW, Op, Op::R>(op, w, nullptr, stage);
  }
  // per problem: w_p = Z_p^T D_p^-1 Z_p g_p for R vectors (R kz entries per problem)
  template <int R>
  tsvm_status zgz(const double *g, double *w) {
    return pass<MODE_ZGZ, GramVecOp, R>(GramVecOp{}, g, w, ST_NONE);
  }
  // One refinement sweep of every problem's capacitance solve M_p g_p = h0_p against the exact
  // operator (M~_p factored in M, one CTA per problem): g_p += M~_p^-1 (h0_p - g_p - w_p).
  template <int R>
  tsvm_status refine(const double *M, int64_t strideM, const double *Mdinv, const double *h0,
                     double *g, double *w, double *c) {
    TSVM_TRY(zgz<R>(g, w));
    refine_resid_batched<<<P, 256, 0, ctx->stream>>>(h0, g, w, c, R, geo.kz, k, scal, info,
                                                      active);
    TSVM_LAUNCHED(ctx);
    TSVM_TRY(potrs_fp64_batched(ctx, M, k, k, strideM, Mdinv, strideM, c, R, geo.kz,
                                (int64_t)R * geo.kz, P, active));
    kvec_add<<<(unsigned)ceil_div((int64_t)P * R * geo.kz, 256), 256, 0, ctx->stream>>>(
        g, c, P * R * geo.kz);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
  template <class Op>
  tsvm_status vec(const Op &op, int stage) {
    vec_kernel<Op><<<nunits, kThreads, 0, ctx->stream>>>(0, op, scal, part_s, units, active);
    TSVM_LAUNCHED(ctx);
    if (Op::NS + Op::NM == 0 && stage == ST_NONE) return TSVM_OK;
    return finalize(0, nullptr, Op::NS, Op::NM, stage);
  }
  tsvm_status finalize(int nvec, double *out_vec, int ns, int nm, int stage) {
    finalize_batched_kernel<<<P, 256, 0, ctx->stream>>>(part_vec, part_s, ubeg, nvec, out_vec, ns,
                                                         nm, scal, stage, info, active);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
};

// Work units of at most `rows` rows (a multiple of 32), each within one problem.
void build_units(const std::vector<int64_t> &off, int rows, std::vector<WorkUnit> &units,
                 std::vector<int> &ubeg) {
  units.clear();
  ubeg.assign(off.size(), 0);
  const int P = (int)off.size() - 1;
  for (int p = 0; p < P; ++p) {
    ubeg[p] = (int)units.size();
    const int64_t n = off[p + 1] - off[p];
    for (int64_t r = 0; r < n; r += rows) {
      WorkUnit u;
      u.p = p;
      u.row0 = r;
      u.rows = (int32_t)std::min<int64_t>(rows, n - r);
      u.goff = off[p] + r;
      units.push_back(u);
    }
  }
  ubeg[P] = (int)units.size();
}

}  // namespace

tsvm_status ipm_solve_batched(tsvm_context *ctx, const tsvm_ipm_problem *pr, int P, int k,
                              int ldz, const tsvm_ipm_options &opt, tsvm_ipm_stats *stats,
                              tsvm_batch_info *binfo) {
  const auto t_start = std::chrono::steady_clock::now();
  const Geometry geo = geometry(k);
  if (geo.kz > 1024 || k > ldz) return TSVM_ERR_UNSUPPORTED;
  const int kz = geo.kz;
  std::vector<int64_t> off(P + 1, 0);
  for (int p = 0; p < P; ++p) off[p + 1] = off[p] + pr[p].n;
  const int64_t N = off[P];

  // autotuner candidates for the rows per unit; tables sized for the smallest
  const int cand[] = {4096, 8192, 16384, 32768};
  std::vector<WorkUnit> units;
  std::vector<int> ubeg;
  build_units(off, cand[0], units, ubeg);
  const int max_units = (int)units.size();
  if (max_units > 65535) return TSVM_ERR_UNSUPPORTED;

  // device tables: units | ubeg | Z pointers | active | info (P) + err
  const size_t tb_units = sizeof(WorkUnit) * max_units;
  const size_t tb_ubeg = sizeof(int) * (P + 1);
  const size_t tb_z = sizeof(float *) * P;
  const size_t tb_act = sizeof(int) * P;
  const size_t tb_info = sizeof(int) * (P + 1);
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  uint8_t *tab = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_B_TABLE,
                     al(tb_units) + al(tb_ubeg) + al(tb_z) + al(tb_act) + al(tb_info), &tab));
  WorkUnit *d_units = reinterpret_cast<WorkUnit *>(tab);
  int *d_ubeg = reinterpret_cast<int *>(tab + al(tb_units));
  const float **d_z = reinterpret_cast<const float **>(tab + al(tb_units) + al(tb_ubeg));
  int *d_active = reinterpret_cast<int *>(tab + al(tb_units) + al(tb_ubeg) + al(tb_z));
  int *d_info =
      reinterpret_cast<int *>(tab + al(tb_units) + al(tb_ubeg) + al(tb_z) + al(tb_act));

  // Mixed-precision capacitance matrices (16-bit precisions, k <= 256): per unit, the rows with
  // dinv <= tau_p through the fused tensor-core SYRK and the others exactly in FP64; every
  // capacitance solve refined once against the exact operator; tau_p adapted on the device.
  const bool mixed = opt.precision != TSVM_PREC_FP32 && syrk_tc_supported(k) && k >= 32 &&
                     k <= 256 && ldz <= syrk_units_kp(k) && ldz % 4 == 0;
  const int KPs = syrk_units_kp(k);
  double *vec = nullptr, *sbuf = nullptr, *Mall = nullptr, *gpart = nullptr, *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_B_VEC, (size_t)11 * N + (size_t)N / 2 + 8, &vec));
  TSVM_TRY(scratch_t(ctx, SLOT_B_SCAL, (size_t)P * (kNScal + (mixed ? 9 : 3) * kz), &sbuf));
  float *part_tc = nullptr;
  int *xcounts = nullptr;
  double *taus = nullptr;
  int64_t *xidx = nullptr;
  if (mixed) {   // [tensor-core partials | 16 words | exact-row counts | tau per problem]
    const size_t ntc = (size_t)max_units * KPs * KPs;
    TSVM_TRY(scratch_t(ctx, SLOT_B_SYRK, ntc + 64 + (size_t)max_units + 2 * (size_t)P, &part_tc));
    xcounts = reinterpret_cast<int *>(part_tc + ntc) + 16;
    taus = reinterpret_cast<double *>(part_tc + ntc + 32 + (((size_t)max_units + 1) & ~(size_t)1));
    TSVM_TRY(scratch_t(ctx, SLOT_B_IDX, (size_t)N, &xidx));
  }
  const int64_t strideD = (int64_t)ceil_div(k, 32) * 1024;
  const int64_t strideM = (int64_t)k * k + strideD;
  TSVM_TRY(scratch_t(ctx, SLOT_B_M, (size_t)P * strideM, &Mall));
  // the exactly summed rows of a unit (mixed) in kExactParts pieces of one partial each
  constexpr int kExactParts = 4;
  TSVM_TRY(scratch_t(ctx, SLOT_B_GPART, (size_t)max_units * k * k * (mixed ? kExactParts : 1),
                     &gpart));
  TSVM_TRY(scratch_t(ctx, SLOT_B_PART, (size_t)max_units * (2 * kz + 16), &part));
  float *labels = reinterpret_cast<float *>(vec + (size_t)11 * N);
  double *scal = sbuf, *q = sbuf + (size_t)P * kNScal, *h = q + (size_t)P * kz;
  // mixed: copies of the right-hand sides, Z^T D^-1 Z g and the corrections (2 kz per problem)
  double *h0 = h + (size_t)P * 2 * kz, *wv = h0 + (size_t)P * 2 * kz, *cv = wv + (size_t)P * 2 * kz;

  Vecs V;
  V.x = vec;
  V.s = V.x + N;
  V.xi = V.s + N;
  V.dinv = V.xi + N;
  V.t1 = V.dinv + N;
  V.t2 = V.t1 + N;
  V.r7 = V.t2 + N;
  V.b = V.r7 + N;
  V.dx = V.b + N;
  V.ds = V.dx + N;
  V.dxi = V.ds + N;
  V.a = labels;

  std::vector<const float *> hz(P);
  std::vector<int> hact(P, 1);
  std::vector<double> hsc((size_t)P * kNScal, 0.0);
  for (int p = 0; p < P; ++p) {
    hz[p] = pr[p].Z;
    hsc[(size_t)p * kNScal + I_C] = pr[p].C;
    hsc[(size_t)p * kNScal + I_N] = (double)pr[p].n;
    TSVM_CUDA(cudaMemcpyAsync(labels + off[p], pr[p].y, sizeof(float) * pr[p].n,
                              cudaMemcpyDeviceToDevice, ctx->stream));
  }
  TSVM_CUDA(cudaMemcpyAsync(d_units, units.data(), sizeof(WorkUnit) * units.size(),
                            cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(d_ubeg, ubeg.data(), tb_ubeg, cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(d_z, hz.data(), tb_z, cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(d_active, hact.data(), tb_act, cudaMemcpyHostToDevice, ctx->stream));
  TSVM_CUDA(cudaMemsetAsync(d_info, 0, tb_info, ctx->stream));
  TSVM_CUDA(cudaMemcpyAsync(scal, hsc.data(), sizeof(double) * hsc.size(), cudaMemcpyHostToDevice,
                            ctx->stream));

  BRunner br;
  br.ctx = ctx;
  br.Zs = d_z;
  br.ldz = ldz;
  br.k = k;
  br.P = P;
  br.nunits = (int)units.size();
  br.geo = geo;
  br.units = d_units;
  br.ubeg = d_ubeg;
  br.active = d_active;
  br.scal = scal;
  br.part_vec = part;
  br.part_s = part + (size_t)max_units * 2 * kz;
  br.info = d_info;
  br.err = d_info + P;
  br.dinv = V.dinv;

  auto pull = [&]() -> tsvm_status {  // scalars + info of every problem to the host
    TSVM_CUDA(cudaMemcpyAsync(hsc.data(), scal, sizeof(double) * hsc.size(),
                              cudaMemcpyDeviceToHost, ctx->stream));
    return TSVM_OK;
  };
  std::vector<int> hinfo(P + 1, 0);

  // ---- initial points (tensorsvm-train.cu:1535-1579), per problem ----
  if (opt.kernel == TSVM_KERNEL_RBF) {
    TSVM_TRY(br.zt(InitRhsOp{V}, q, ST_NONE));
    TSVM_TRY(br.zw(InitRbfRowOp{V}, q, ST_INIT));
  }
  TSVM_TRY(pull());
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int p = 0; p < P; ++p) {
    double *sp = &hsc[(size_t)p * kNScal];
    const double C = pr[p].C;
    double ox = opt.kernel == TSVM_KERNEL_RBF ? sp[I_E2SUM] / sp[I_E2SQ] : 1.0;
    if (!(ox < 0.99 * C && ox > 0.01 * C)) ox = ox > 0.99 * C ? 0.99 * C : 0.01 * C;
    sp[I_Y] = ox;
  }
  TSVM_CUDA(cudaMemcpyAsync(scal, hsc.data(), sizeof(double) * hsc.size(), cudaMemcpyHostToDevice,
                            ctx->stream));
  TSVM_TRY(br.vec(FillOp{V, 0.0}, ST_NONE));
  for (int p = 0; p < P; ++p) hsc[(size_t)p * kNScal + I_Y] = 0.0;
  TSVM_CUDA(cudaMemcpyAsync(scal, hsc.data(), sizeof(double) * hsc.size(), cudaMemcpyHostToDevice,
                            ctx->stream));
  if (opt.kernel != TSVM_KERNEL_RBF) {
    TSVM_TRY(br.zt(XRhsOp{V}, q, ST_NONE));
    TSVM_TRY(br.zw(InitLinearRowOp{V}, q, ST_NONE));
  }

  // ---- autotune the rows per unit on the first pass of the iteration (idempotent) ----
  const auto t_tune0 = std::chrono::steady_clock::now();
  int best_rows = cand[0];
  {
    float best_ms = 1e30f;
    cudaEvent_t e0 = ctx->ev[4], e1 = ctx->ev[5];
    std::vector<WorkUnit> cu;
    std::vector<int> cb;
    for (int rows : cand) {
      build_units(off, rows, cu, cb);
      TSVM_CUDA(cudaMemcpyAsync(d_units, cu.data(), sizeof(WorkUnit) * cu.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
      TSVM_CUDA(cudaMemcpyAsync(d_ubeg, cb.data(), tb_ubeg, cudaMemcpyHostToDevice, ctx->stream));
      br.nunits = (int)cu.size();
      float ms = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        TSVM_CUDA(cudaEventRecord(e0, ctx->stream));
        TSVM_TRY(br.zt(BeginOp{V, 0.0}, q, ST_BEGIN));
        TSVM_CUDA(cudaEventRecord(e1, ctx->stream));
        ms = std::min(ms, event_ms(e0, e1));
      }
      if (ms < best_ms) {
        best_ms = ms;
        best_rows = rows;
      }
    }
    build_units(off, best_rows, units, ubeg);
    TSVM_CUDA(cudaMemcpyAsync(d_units, units.data(), sizeof(WorkUnit) * units.size(),
                              cudaMemcpyHostToDevice, ctx->stream));
    TSVM_CUDA(cudaMemcpyAsync(d_ubeg, ubeg.data(), tb_ubeg, cudaMemcpyHostToDevice, ctx->stream));
    br.nunits = (int)units.size();
  }
  const double ms_tune =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_tune0).count();

  // one iteration after the host's stopping decisions, ending with the next iteration's
  // Begin/Resid passes (captured once, then replayed)
  double *M = Mall;
  double *Mdinv_base = Mall + (size_t)k * k;
  auto body = [&]() -> tsvm_status {
    if (mixed) {
      tau_update_batched<<<(unsigned)ceil_div(P, 128), 128, 0, ctx->stream>>>(scal, taus, P,
                                                                               d_active);
      TSVM_LAUNCHED(ctx);
      TSVM_TRY(big_rows_units(ctx, V.dinv, d_units, br.nunits, d_active, taus, xidx, xcounts));
      TSVM_TRY(gram_fp64_units(ctx, d_z, ldz, k, d_units, br.nunits, d_active, V.dinv, gpart,
                               xidx, xcounts, kExactParts));
      // a tensor-core block that timed out raises the streaming passes' flag (the host reports
      // TSVM_ERR_TIMEOUT) and poisons M
      TSVM_TRY(syrk_units_tc(ctx, d_z, ldz, k, d_units, br.nunits, d_active, V.dinv, taus,
                             part_tc, br.err));
      mixed_units_reduce<<<dim3((unsigned)ceil_div((int64_t)k * k, 256), P), 256, 0,
                           ctx->stream>>>(part_tc, KPs, gpart, d_ubeg, k, d_active, br.err, M,
                                          strideM, xcounts, kExactParts);
    } else {
      TSVM_TRY(gram_fp64_units(ctx, d_z, ldz, k, d_units, br.nunits, d_active, V.dinv, gpart));
      gram_units_reduce<<<dim3((unsigned)ceil_div((int64_t)k * k, 256), P), 256, 0,
                          ctx->stream>>>(gpart, d_ubeg, k, d_active, M, strideM);
    }
    TSVM_LAUNCHED(ctx);
    TSVM_TRY(chol_fp64_batched(ctx, M, k, k, strideM, d_info, Mdinv_base, strideM, P, d_active));
    TSVM_TRY(br.zt(SmwRhs2Op{V}, h, ST_NONE));
    if (mixed)
      TSVM_CUDA(cudaMemcpyAsync(h0, h, sizeof(double) * P * 2 * kz, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    TSVM_TRY(potrs_fp64_batched(ctx, M, k, k, strideM, Mdinv_base, strideM, h, 2, kz,
                                (int64_t)2 * kz, P, d_active));
    if (mixed) TSVM_TRY(br.refine<2>(M, strideM, Mdinv_base, h0, h, wv, cv));
    TSVM_TRY(br.zw(SmwBack2Op{V}, h, ST_DYA));
    TSVM_TRY(br.vec(AffineOp{V, 0.0, 0.0}, ST_ALPHA_AFF));
    TSVM_TRY(br.vec(MuAffOp{V, 0.0, 0.0}, ST_SIGMA));
    TSVM_TRY(br.zt(CorrRhsOp{V, 0.0, 0.0}, h, ST_NONE));
    if (mixed)
      TSVM_CUDA(cudaMemcpyAsync(h0, h, sizeof(double) * P * kz, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    TSVM_TRY(potrs_fp64_batched(ctx, M, k, k, strideM, Mdinv_base, strideM, h, 1, kz, kz, P,
                                d_active));
    if (mixed) TSVM_TRY(br.refine<1>(M, strideM, Mdinv_base, h0, h, wv, cv));
    TSVM_TRY(br.zw(CorrBackOp{V}, h, ST_DYC));
    TSVM_TRY(br.vec(CombineOp{V, 0.0, 0.0, 0.0}, ST_ALPHA));
    TSVM_TRY(br.vec(UpdateOp{V, 0.0, true}, ST_NONE));
    TSVM_TRY(br.zt(BeginOp{V, 0.0}, q, ST_BEGIN));
    TSVM_TRY(br.zw(ResidOp{V, 0.0}, q, ST_RESID));
    return TSVM_OK;
  };

  TSVM_TRY(br.zt(BeginOp{V, 0.0}, q, ST_BEGIN));
  TSVM_TRY(br.zw(ResidOp{V, 0.0}, q, ST_RESID));

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool graph_failed = false;
  int64_t graph_launches = 0;
  std::vector<int> done_iter(P, -1), status(P, TSVM_WARN_MAX_ITER);
  std::vector<double> t_gap(P, -1.0), last(P * kNScal, 0.0);
  int iter = 0, iters_max = 0;
  tsvm_status result = TSVM_OK;
  for (iter = 0;; ++iter) {
    TraceRange trace_iter("batched ipm iteration");
    TSVM_TRY(pull());
    TSVM_CUDA(cudaMemcpyAsync(hinfo.data(), d_info, sizeof(int) * (P + 1), cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (hinfo[P]) {
      result = timeout_status("batched ipm streaming pass");
      break;
    }
    const double tnow =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    bool changed = false;
    int nactive = 0;
    for (int p = 0; p < P; ++p) {
      if (!hact[p]) continue;
      const double *sp = &hsc[(size_t)p * kNScal];
      const double scale = 1.0 + sqrt((double)pr[p].n);
      const double nrd = sp[I_NORMRD], nrp = fabs(sp[I_RP]);
      int st = -1;
      // a failed step (Cholesky, or the refinement of the mixed form) ends the problem, unless
      // the mixed form can retry it with more rows summed exactly (the step was not taken; the
      // device divides tau by 64, down to 0)
      if (iter > 0 && sp[I_INFO] != 0.0 && !(mixed && sp[I_TAU] > 0.0)) st = TSVM_ERR_NOT_SPD;
      if (st < 0 && t_gap[p] < 0 && sp[I_RELGAP] <= 1e-6 && nrd / scale <= 1e-6 &&
          nrp / scale <= 1e-6)
        t_gap[p] = tnow;
      if (st < 0 && sp[I_MU] < opt.tol && nrd < opt.tol && nrp < opt.tol) st = TSVM_OK;
      if (st < 0 && opt.rel_gap_tol > 0 && sp[I_RELGAP] <= opt.rel_gap_tol &&
          nrd / scale <= opt.rel_gap_tol && nrp / scale <= opt.rel_gap_tol)
        st = TSVM_OK;
      if (st < 0 && sp[I_COND] > 1e18) st = TSVM_WARN_ILL_CONDITIONED;
      if (st < 0 && iter >= opt.max_iter) st = TSVM_WARN_MAX_ITER;
      if (st >= 0) {
        status[p] = st;
        done_iter[p] = iter;
        hact[p] = 0;
        changed = true;
        std::copy(sp, sp + kNScal, last.begin() + (size_t)p * kNScal);
      } else {
        ++nactive;
      }
    }
    if (nactive == 0) break;
    if (changed)
      TSVM_CUDA(cudaMemcpyAsync(d_active, hact.data(), tb_act, cudaMemcpyHostToDevice,
                                ctx->stream));
    if (gexec) {
      TSVM_CUDA(cudaGraphLaunch(gexec, ctx->stream));
      ctx->launches += graph_launches;
      continue;
    }
    if (iter >= 1 && !graph_failed) {
      // capture this iteration's launches (all scratch exists after the first iteration)
      const int64_t l0 = ctx->launches;
      if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const tsvm_status cst = body();
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
        if (cst == TSVM_OK && ce == cudaSuccess && g &&
            cudaGraphInstantiate(&gexec, g, 0) == cudaSuccess) {
          graph = g;
          graph_launches = ctx->launches - l0;
          ctx->launches = l0;
          TSVM_CUDA(cudaGraphLaunch(gexec, ctx->stream));
          ctx->launches += graph_launches;
          continue;
        }
        if (g) cudaGraphDestroy(g);
        gexec = nullptr;
        ctx->launches = l0;
        cudaGetLastError();
      }
      graph_failed = true;
    }
    TSVM_TRY(body());
  }
  iters_max = iter;
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  if (result != TSVM_OK) return result;
  for (int p = 0; p < P; ++p) {
    if (pr[p].alpha_out)
      TSVM_CUDA(cudaMemcpyAsync(pr[p].alpha_out, V.x + off[p], sizeof(double) * pr[p].n,
                                cudaMemcpyDeviceToDevice, ctx->stream));
    if (pr[p].xi_out)
      TSVM_CUDA(cudaMemcpyAsync(pr[p].xi_out, V.xi + off[p], sizeof(double) * pr[p].n,
                                cudaMemcpyDeviceToDevice, ctx->stream));
  }
  TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
  const double ms_total =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  for (int p = 0; p < P; ++p) {
    const double *sp = &last[(size_t)p * kNScal];
    if (stats) {
      tsvm_ipm_stats &st = stats[p];
      memset(&st, 0, sizeof(st));
      st.iters = done_iter[p];
      st.status = status[p];
      st.mu = sp[I_MU];
      st.norm_rd = sp[I_NORMRD];
      st.norm_rp = fabs(sp[I_RP]);
      st.cond_d = sp[I_COND];
      st.pobj = sp[I_POBJ];
      st.dobj = sp[I_DOBJ];
      st.rel_gap = sp[I_RELGAP];
      st.ms_total = ms_total;
      st.t_rel_gap_1e6_ms = t_gap[p];
    }
    if (result == TSVM_OK && status[p] != TSVM_OK && status[p] != TSVM_WARN_MAX_ITER &&
        status[p] != TSVM_WARN_ILL_CONDITIONED)
      result = (tsvm_status)status[p];
  }
  if (binfo) {
    binfo->units = br.nunits;
    binfo->unit_rows = best_rows;
    binfo->graph_used = gexec || graph ? 1 : 0;
    binfo->iters_max = iters_max;
    binfo->ms_total = ms_total;
    binfo->ms_autotune = ms_tune;
  }
  return result;
}

}  // namespace tsvm
