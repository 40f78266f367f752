// Hypergradient of a validation loss through the trained SVM (tsvm_hypergrad).
//
// The reference has no counterpart; this is the KKT-adjoint extension of its training path
// (LRA T:1941-2374, mpc T:1507-1840, the bias of writemodel T:355-376).  With the model
// f(x) = sum_i alpha_i y_i K(x_i, x) + b (exact RBF kernel), the validation loss
// L = (1/m) sum_v max(0, 1 - y_v f(x_v))^2 and the dual solved on Q = Z Z^T = P Ky P
// (Ky = Y K Y, P the projector onto range(B), B = Ky Omega the first pass of the factor):
//
//   g_v      = dL/df_v = -(2/m) y_v max(0, 1 - y_v f_v),        G_b = sum_v g_v
//   c_i      = dL/dalpha_i = y_i sum_v K(x_i, x_v) g_v - G_b (Z_i . z_F) / |F|
//              (b = mean over the first <= 50 free SVs F of y_j - y_j sum_i alpha_i Z_i.Z_j,
//               z_F = sum_{j in F} y_j Z_j)
//   lambda   = adjoint: [Q + D, a; a^T, 0][lambda; nu] = [c; 0] (kkt_adjoint, SMW as in the IPM)
//   dL/dlogC = lambda . (C xi / (C - alpha))     (C enters the barrier complementarity
//                                                  xi (C - alpha) = mu; exact for fixed Z)
//   r        = dQ/dgamma alpha, differentiating the range finder with the sketch fixed:
//              dQ = dP Ky P + P dKy P + P Ky dP,  dP x = (I-P) dB B+ x + B+^T dB^T (I-P) x,
//              dB = dKy Omega, B+ = R^-1 W^T (B = W R, W orthonormal), dKy = Y K' Y,
//              K' = dK/dgamma = -||x_i - x_j||^2 K
//   dL/dlogg = -gamma lambda . r - G_b gamma mean_{j in F} y_j r_j
//              + gamma sum_v g_v sum_i alpha_i y_i K'_iv
//   dL/dXv   = g_v sum_i alpha_i y_i K_iv (-2 gamma)(x_v - x_i)
// The factor (Omega, W, R and Z) is recomputed here rather than stored by the forward pass.
// Eigenvalues of W^T Ky W clipped at 0 are taken as fixed.  Kernel products are FP32
// (distances from differences, no cancellation) accumulated in FP64 per 64-column tile.
#include <math.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"
#include "trace.h"

namespace tsvm {
namespace {

constexpr int kKP = 256;   // threads per block
constexpr int kKT = 64;    // rows of B staged per tile
constexpr int kKMaxD = 64;

// out[i][c] = sum_j w_ij exp(-gamma ||a_i - b_j||^2) U[j][c], w_ij = 1 or -||a_i - b_j||^2
// (DERIV), for NU columns of U (FP64, nb x nu_total) and out (FP64, na x nu_total).  Each thread
// keeps R rows of A in registers (rows blockIdx * 256 R + threadIdx + 256 r); a tile of 64 rows
// of B (with their squared norms) and of U sits in shared memory and is read as broadcasts, four
// features per load.  DC is d rounded up to a multiple of 4 (16 ... 32, or 64), so no FMA is
// spent on padding at d = 18 or 28.  The exponent -gamma log2(e) ||a - b||^2 is one FMA chain:
// it starts at -g (||a||^2 + ||b||^2) (g = gamma log2 e) and adds (2 g a) . b, the A rows being
// scaled by 2 g once; it is clamped at 0 (the relative error of the kernel value stays ~1e-7
// gamma ||a||^2).  DERIV weights by the exponent t = -g ||a - b||^2 and divides by g at the
// end (t / g = -||a - b||^2).  Each tile's 64 terms are summed in FP32, the tiles in FP64.  Block (x, y) sums the B
// rows [y jc, (y + 1) jc): with gridDim.y > 1 its sums go to out + y * na * nu_total and
// kprod_reduce adds the splits in order.
template <int DC, int R, int NU, bool DERIV>
__global__ void __launch_bounds__(kKP)
kprod_kernel(const float *__restrict__ A, int64_t na, const float *__restrict__ B, int64_t nb,
             int d, float gl2 /* gamma log2 e */, const double *__restrict__ U, int nu_total,
             int c0, int64_t jc, double *__restrict__ out) {
  static_assert(DC % 4 == 0, "B rows are read as float4");
  __shared__ __align__(16) float Bs[kKT][DC];
  __shared__ float Bn[kKT];
  __shared__ float Us[kKT][NU];
  float a[R][DC], an[R];
  const float g2 = 2.f * gl2;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = (int64_t)blockIdx.x * kKP * R + threadIdx.x + kKP * r;
    float t = 0.f;
#pragma unroll
    for (int c = 0; c < DC; ++c) {
      const float v = (i < na && c < d) ? A[i * d + c] : 0.f;
      t = fmaf(v, v, t);
      a[r][c] = g2 * v;
    }
    an[r] = -gl2 * t;
  }
  double acc[R][NU];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int u = 0; u < NU; ++u) acc[r][u] = 0.0;
  const int64_t jbeg = (int64_t)blockIdx.y * jc;
  const int64_t jend = jbeg + jc < nb ? jbeg + jc : nb;
  out += (int64_t)blockIdx.y * na * nu_total;
  for (int64_t j0 = jbeg; j0 < jend; j0 += kKT) {
    __syncthreads();
    for (int e = threadIdx.x; e < kKT * DC; e += kKP) {
      const int r = e / DC, c = e % DC;
      const int64_t j = j0 + r;
      Bs[r][c] = (j < jend && c < d) ? B[j * d + c] : 0.f;
    }
    for (int e = threadIdx.x; e < kKT * NU; e += kKP) {
      const int r = e / NU, u = e % NU;
      const int64_t j = j0 + r;
      Us[r][u] = (j < jend && c0 + u < nu_total) ? (float)U[j * nu_total + c0 + u] : 0.f;
    }
    __syncthreads();
    if (threadIdx.x < kKT) {
      float t = 0.f;
#pragma unroll
      for (int c = 0; c < DC; ++c) t = fmaf(Bs[threadIdx.x][c], Bs[threadIdx.x][c], t);
      Bn[threadIdx.x] = -gl2 * t;
    }
    __syncthreads();
    float part[R][NU];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int u = 0; u < NU; ++u) part[r][u] = 0.f;
    const int jn = (int)(jend - j0 < kKT ? jend - j0 : kKT);
    for (int jj = 0; jj < jn; ++jj) {
      const float bn = Bn[jj];
      float ex[R];
#pragma unroll
      for (int r = 0; r < R; ++r) ex[r] = an[r] + bn;
      const float4 *brow = reinterpret_cast<const float4 *>(&Bs[jj][0]);
#pragma unroll
      for (int c4 = 0; c4 < DC / 4; ++c4) {
        const float4 bv = brow[c4];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          ex[r] = fmaf(a[r][4 * c4], bv.x, ex[r]);
          ex[r] = fmaf(a[r][4 * c4 + 1], bv.y, ex[r]);
          ex[r] = fmaf(a[r][4 * c4 + 2], bv.z, ex[r]);
          ex[r] = fmaf(a[r][4 * c4 + 3], bv.w, ex[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float t = fminf(ex[r], 0.f);
        float e;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(t));
        if (DERIV) e *= t;
#pragma unroll
        for (int u = 0; u < NU; ++u) part[r][u] = fmaf(e, Us[jj][u], part[r][u]);
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int u = 0; u < NU; ++u) acc[r][u] += (double)part[r][u];
  }
  const double w = DERIV ? 1.0 / (double)gl2 : 1.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = (int64_t)blockIdx.x * kKP * R + threadIdx.x + kKP * r;
    if (i < na) {
#pragma unroll
      for (int u = 0; u < NU; ++u)
        if (c0 + u < nu_total) out[i * nu_total + c0 + u] = DERIV ? w * acc[r][u] : acc[r][u];
    }
  }
}

__global__ void kprod_reduce(const double *__restrict__ part, int nsplit, int64_t count,
                             double *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  double t = 0.0;
  for (int y = 0; y < nsplit; ++y) t += part[(int64_t)y * count + e];
  out[e] = t;
}

template <int DC, int R, int NU, bool DERIV>
tsvm_status kprod_launch(tsvm_context *ctx, const float *A, int64_t na, const float *B, int64_t nb,
                         int d, float gl2, const double *U, int nu_total, double *out) {
  // split B over gridDim.y so that the grid covers the SMs about eight times over
  const int64_t rowblocks = ceil_div(na, (int64_t)kKP * R);
  int64_t split = ceil_div((int64_t)ctx->num_sms * 8, rowblocks);
  split = std::max<int64_t>(1, std::min<int64_t>({split, 64, ceil_div(nb, (int64_t)kKT * 4)}));
  const int64_t jc = round_up(ceil_div(nb, split), kKT);
  split = ceil_div(nb, jc);
  double *dst = out;
  if (split > 1)
    TSVM_TRY(scratch_t(ctx, SLOT_HG_KPART, (size_t)split * na * nu_total, &dst));
  for (int c0 = 0; c0 < nu_total; c0 += NU) {
    kprod_kernel<DC, R, NU, DERIV><<<dim3((unsigned)rowblocks, (unsigned)split), kKP, 0,
                                     ctx->stream>>>(A, na, B, nb, d, gl2, U, nu_total, c0, jc, dst);
    TSVM_LAUNCHED(ctx);
  }
  if (split > 1) {
    const int64_t count = na * nu_total;
    kprod_reduce<<<(unsigned)ceil_div(count, 256), 256, 0, ctx->stream>>>(dst, (int)split, count,
                                                                           out);
    TSVM_LAUNCHED(ctx);
  }
  return TSVM_OK;
}

// NU: columns of U handled per launch (1, 8 or 32); d <= kKMaxD.
template <int NU, bool DERIV>
tsvm_status kprod(tsvm_context *ctx, const float *A, int64_t na, const float *B, int64_t nb,
                  int d, double gamma, const double *U, int nu_total, double *out) {
  const float gl2 = (float)(gamma * 1.4426950408889634);
  constexpr int R32 = NU == 1 ? 4 : NU == 8 ? 2 : 1;
  constexpr int R64 = NU == 1 ? 2 : 1;
  if (d <= 16) return kprod_launch<16, R32, NU, DERIV>(ctx, A, na, B, nb, d, gl2, U, nu_total, out);
  if (d <= 20) return kprod_launch<20, R32, NU, DERIV>(ctx, A, na, B, nb, d, gl2, U, nu_total, out);
  if (d <= 24) return kprod_launch<24, R32, NU, DERIV>(ctx, A, na, B, nb, d, gl2, U, nu_total, out);
  if (d <= 28) return kprod_launch<28, R32, NU, DERIV>(ctx, A, na, B, nb, d, gl2, U, nu_total, out);
  if (d <= 32) return kprod_launch<32, R32, NU, DERIV>(ctx, A, na, B, nb, d, gl2, U, nu_total, out);
  return kprod_launch<64, R64, NU, DERIV>(ctx, A, na, B, nb, d, gl2, U, nu_total, out);
}

// U (nb x nu FP64) -> Uf (nb x kp FP32, zero columns past nu)
__global__ void u_to_float(const double *__restrict__ U, int64_t nb, int nu, int kp,
                           float *__restrict__ Uf) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nb * kp) return;
  const int64_t j = e / kp;
  const int c = (int)(e % kp);
  Uf[e] = c < nu ? (float)U[j * nu + c] : 0.f;
}
// out (na x nu FP64) = scale * W (na x kp FP32)
__global__ void w_to_out(const float *__restrict__ W, int64_t na, int kp, int nu, double scale,
                         double *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= na * nu) return;
  const int64_t i = e / nu;
  const int c = (int)(e % nu);
  out[e] = scale * (double)W[i * kp + c];
}

// The kernel-vector product of kprod on the tensor cores (kermatmul_tc_core with the kernel
// block and U both split hi + lo, FP32 accumulation): out = [K or K'](A, B) U.  Both row sets
// are centred by B's mean; K' = -||a - b||^2 K is the kernel's S exp2(S) entries
// (S = -gamma log2(e) ||a - b||^2) divided by gamma log2 e.
tsvm_status kprod_tc(tsvm_context *ctx, const float *A, int64_t na, const float *B, int64_t nb,
                     int d, double gamma, const double *U, int nu, double *out, bool deriv) {
  const int kp = (int)round_up(nu, 64);
  const size_t oa = 0, ob = round_up((size_t)na * d, 64), ou = ob + round_up((size_t)nb * d, 64);
  const size_t ow = ou + round_up((size_t)nb * kp, 64);
  float *buf = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_HG_TC, ow + (size_t)na * kp, &buf));
  float *Ac = buf + oa, *Bc = buf + ob, *Uf = buf + ou, *Wt = buf + ow;
  TSVM_TRY(centre_pair(ctx, B, nb, A, na, d, Bc, Ac));
  u_to_float<<<(unsigned)ceil_div(nb * kp, 256), 256, 0, ctx->stream>>>(U, nb, nu, kp, Uf);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(kermatmul_tc_core(ctx, Ac, nullptr, na, Bc, nullptr, nb, d, gamma, Uf, kp, Wt,
                             TSVM_PREC_FP16, nullptr, nullptr, 3, deriv));
  const double scale = deriv ? 1.0 / (gamma * 1.4426950408889634) : 1.0;
  w_to_out<<<(unsigned)ceil_div(na * (int64_t)nu, 256), 256, 0, ctx->stream>>>(Wt, na, kp, nu,
                                                                              scale, out);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

__global__ void beta_kernel(const double *alpha, const float *y, int64_t n, double *beta) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) beta[i] = alpha[i] * (double)y[i];
}
// f = s + b; g = -(2/m) y max(0, 1 - y f); loss partials
__global__ void val_loss_kernel(const double *s, const float *yv, int64_t m, double b,
                                double *f, double *g) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m) return;
  const double fv = s[v] + b, yy = (double)yv[v];
  const double h = fmax(0.0, 1.0 - yy * fv);
  f[v] = h * h / (double)m;   // per-point loss
  g[v] = -2.0 * yy * h / (double)m;
}
// beta_x[j][0] = beta_j, beta_x[j][1 + c] = beta_j x_jc
__global__ void beta_x_kernel(const double *beta, const float *X, int64_t n, int d, double *bx) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  bx[j * (d + 1)] = beta[j];
  for (int c = 0; c < d; ++c) bx[j * (d + 1) + 1 + c] = beta[j] * (double)X[j * d + c];
}
// dXv[v][c] = -2 gamma g_v (x_vc S0_v - S_c,v)
__global__ void dxv_kernel(const double *S, const float *Xv, const double *g, int64_t m, int d,
                           double gamma, float *dXv) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m) return;
  const double s0 = S[v * (d + 1)];
  for (int c = 0; c < d; ++c)
    dXv[v * d + c] =
        (float)(-2.0 * gamma * g[v] * ((double)Xv[v * d + c] * s0 - S[v * (d + 1) + 1 + c]));
}
// c_i = y_i r_i - Gb/|F| (Z_i . zF)
__global__ void adj_rhs_kernel(const double *r, const float *y, const float *Z, int64_t ldz,
                               int k, int64_t n, const double *zF, double coef, double *c) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dot = 0.0;
  for (int q = 0; q < k; ++q) dot += (double)Z[i * ldz + q] * zF[q];
  c[i] = (double)y[i] * r[i] + coef * dot;
}
__global__ void zf_kernel(const float *Z, int64_t ldz, int k, const float *y, const int64_t *F,
                          int nf, double *zF) {
  for (int q = threadIdx.x; q < k; q += blockDim.x) {
    double s = 0.0;
    for (int t = 0; t < nf; ++t) s += (double)y[F[t]] * (double)Z[F[t] * ldz + q];
    zF[q] = s;
  }
}
// y_i v_i
__global__ void yscale_kernel(const double *v, const float *y, int64_t n, double *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)y[i] * v[i];
}
// fixed-order block sums of up to 4 dot products: part[b][q] = sum_i terms_q(i)
//   q0: lambda . (C xi / (C - alpha)), q1: lambda . pw, q2: per-point loss, q3: g . t
__global__ void dots_kernel(const double *lam, const double *xi, const double *alpha, double C,
                            const double *pw, int64_t n, const double *lossv, const double *g,
                            const double *t, int64_t m, double *part) {
  __shared__ double sh[4][256];
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    s0 += lam[i] * C * xi[i] / (C - alpha[i]);
    s1 += lam[i] * pw[i];
  }
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < m;
       v += (int64_t)gridDim.x * blockDim.x) {
    s2 += lossv[v];
    s3 += g[v] * t[v];
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  sh[2][threadIdx.x] = s2;
  sh[3][threadIdx.x] = s3;
  __syncthreads();
  if (threadIdx.x < 4) {
    double a = 0;
    for (int t2 = 0; t2 < (int)blockDim.x; ++t2) a += sh[threadIdx.x][t2];
    part[blockIdx.x * 4 + threadIdx.x] = a;
  }
}

// R (k x k upper) x = b (trans = 0) or R^T x = b (trans = 1), in place; one block.
__global__ void tri_solve_upper(const double *__restrict__ R, int k, double *__restrict__ x,
                                int trans) {
  __shared__ double xs[1024];
  for (int t = threadIdx.x; t < k; t += blockDim.x) xs[t] = x[t];
  __syncthreads();
  if (!trans) {
    for (int i = k - 1; i >= 0; --i) {
      if (threadIdx.x == 0) xs[i] /= R[(int64_t)i * k + i];
      __syncthreads();
      for (int j = threadIdx.x; j < i; j += blockDim.x) xs[j] -= R[(int64_t)j * k + i] * xs[i];
      __syncthreads();
    }
  } else {
    for (int i = 0; i < k; ++i) {
      if (threadIdx.x == 0) xs[i] /= R[(int64_t)i * k + i];
      __syncthreads();
      for (int j = i + 1 + threadIdx.x; j < k; j += blockDim.x)
        xs[j] -= R[(int64_t)i * k + j] * xs[i];
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < k; t += blockDim.x) x[t] = xs[t];
}
// out = a + s * b (elementwise over n)
__global__ void axpy_kernel(const double *a, double s, const double *b, int64_t n, double *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + s * b[i];
}
// column c of an n x 5 block (row-major) from v, scaled by y
__global__ void pack_col(const double *v, const float *y, int64_t n, double *U, int nu, int c) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) U[i * nu + c] = (double)y[i] * v[i];
}
__global__ void unpack_col(const double *U, const float *y, int64_t n, int nu, int c, double *v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (double)y[i] * U[i * nu + c];
}

}  // namespace

// Test hook (tsvm_test_kprod): out = [K or K'](A, B) U by the SIMT or the tensor-core products.
tsvm_status kprod_any(tsvm_context *ctx, const float *A, int64_t na, const float *B, int64_t nb,
                      int d, double gamma, const double *U, int nu, double *out, bool deriv,
                      bool tc) {
  if (tc) {
    if (!kermatmul_tc_supported(d, 64)) return TSVM_ERR_UNSUPPORTED;
    return kprod_tc(ctx, A, na, B, nb, d, gamma, U, nu, out, deriv);
  }
  if (d > kKMaxD) return TSVM_ERR_UNSUPPORTED;
  if (nu == 1)
    return deriv ? kprod<1, true>(ctx, A, na, B, nb, d, gamma, U, nu, out)
                 : kprod<1, false>(ctx, A, na, B, nb, d, gamma, U, nu, out);
  if (nu <= 8)
    return deriv ? kprod<8, true>(ctx, A, na, B, nb, d, gamma, U, nu, out)
                 : kprod<8, false>(ctx, A, na, B, nb, d, gamma, U, nu, out);
  return deriv ? kprod<32, true>(ctx, A, na, B, nb, d, gamma, U, nu, out)
               : kprod<32, false>(ctx, A, na, B, nb, d, gamma, U, nu, out);
}

}  // namespace tsvm

using namespace tsvm;

namespace {

// Linear maps of the kept factorisation (W, R, Omega; all n x kp float, R k x k).
struct RangeOps {
  tsvm_context *ctx;
  const float *W, *Om;
  int kp, k;
  int64_t n;
  double *kv1, *kv2;   // k-vectors (kp doubles each)
  // out = P x = W W^T x
  tsvm_status P(const double *x, double *out) {
    TSVM_TRY(zt_vec(ctx, W, kp, n, k, x, kv1));
    return zw_vec(ctx, W, kp, n, k, kv1, out);
  }
  // out = Omega B+ x = Omega R^-1 W^T x
  tsvm_status OmBp(const double *x, double *out) {
    TSVM_TRY(zt_vec(ctx, W, kp, n, k, x, kv1));
    tri_solve_upper<<<1, 256, 0, ctx->stream>>>(Rm, k, kv1, 0);
    TSVM_LAUNCHED(ctx);
    return zw_vec(ctx, Om, kp, n, k, kv1, out);
  }
  // out = B+^T Omega^T x = W R^-T Omega^T x
  tsvm_status BpTOmT(const double *x, double *out) {
    TSVM_TRY(zt_vec(ctx, Om, kp, n, k, x, kv2));
    tri_solve_upper<<<1, 256, 0, ctx->stream>>>(Rm, k, kv2, 1);
    TSVM_LAUNCHED(ctx);
    return zw_vec(ctx, W, kp, n, k, kv2, out);
  }
  const double *Rm;
};

}  // namespace

extern "C" tsvm_status tsvm_hypergrad(tsvm_context *ctx, const float *X, const float *y,
                                      int64_t n, int32_t d, const float *Xv, const float *yv,
                                      int64_t nv, double gamma, double C, int32_t k,
                                      int32_t precision, const double *alpha, const double *xi,
                                      const double *s, double ymult, double b,
                                      tsvm_hypergrad_result *res, float *dXv) {
  (void)ymult;  // the equality multiplier enters only through s (dual feasibility)
  if (!ctx || !X || !y || !Xv || !yv || !alpha || !xi || !s || !res || n < 2 || nv < 1 || d < 1 ||
      d > kKMaxD || k < 1 || k > 1000 || k > n || !(gamma > 0) || !(C > 0))
    return TSVM_ERR_INVALID_ARGUMENT;
  if (!precision_valid(precision)) return TSVM_ERR_INVALID_ARGUMENT;
  if (ctx && sharded(ctx)) return TSVM_ERR_UNSUPPORTED;
  TSVM_CUDA(cudaSetDevice(ctx->device));
  TraceRange trace_call("tsvm_hypergrad");
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = ctx->stream;
  const int kp = (int)round_up(k, 64);
  // the factorisation with its sketch Omega, R and unrounded W: kept by tsvm_factor (with
  // tsvm_set_factor_keep) for these very inputs, or recomputed here
  const bool reuse = ctx->kept.valid && ctx->kept.X == X && ctx->kept.y == y && ctx->kept.n == n &&
                     ctx->kept.d == d && ctx->kept.k == k && ctx->kept.precision == precision &&
                     ctx->kept.gamma == gamma;
  if (!reuse) TSVM_TRY(factor_rbf_keep(ctx, X, y, n, d, gamma, k, precision, nullptr, kp, nullptr));
  float *Zf = nullptr, *Om = nullptr, *Wk = nullptr;
  double *Rbuf = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_HG_Z, (size_t)n * kp, &Zf));
  TSVM_TRY(scratch_t(ctx, SLOT_HG_OMEGA, (size_t)n * kp, &Om));
  TSVM_TRY(scratch_t(ctx, SLOT_HG_R, (size_t)2 * k * k + 2 * (size_t)kp + 64, &Rbuf));
  TSVM_TRY(scratch_t(ctx, SLOT_HG_W, (size_t)n * kp, &Wk));
  FactorKeep keep{Om, Rbuf, Wk};
  res->factor_reused = reuse ? 1 : 0;
  // scratch: n-vectors beta, c, lam, u, E1, tmp, t2, s2, r + U5/D5 (5 n each); nv-vectors
  const int nb = 148;
  double *buf = nullptr;
  const size_t need = (size_t)19 * n + (size_t)4 * nv + (size_t)k + 4 * nb + 64 + 64;
  TSVM_TRY(scratch_t(ctx, SLOT_DEV_OUT, need, &buf));
  double *beta = buf, *c = beta + n, *lam = c + n, *u = lam + n, *E1 = u + n, *tmp = E1 + n;
  double *t2 = tmp + n, *s2 = t2 + n, *r = s2 + n, *U5 = r + n, *D5 = U5 + 5 * n;
  double *sv = D5 + 5 * n, *lossv = sv + nv, *g = lossv + nv, *tv = g + nv;
  double *zF = tv + nv, *part = zF + k;
  const unsigned gn = (unsigned)ceil_div(n, 256), gv = (unsigned)ceil_div(nv, 256);
  RangeOps ro{ctx, keep.W, Om, kp, k, n, Rbuf + 2 * (size_t)k * k,
              Rbuf + 2 * (size_t)k * k + kp, Rbuf};

  // free set F of the bias (first <= 50 SVs with 1e-6 < alpha < C - 1e-6, index order)
  std::vector<double> ha(n);
  TSVM_CUDA(cudaMemcpyAsync(ha.data(), alpha, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  TSVM_CUDA(cudaStreamSynchronize(st));
  std::vector<int64_t> F;
  for (int64_t i = 0; i < n && F.size() < 50; ++i)
    if (ha[i] > 1e-6 && ha[i] < C - 1e-6) F.push_back(i);
  // the free-set indices live in this call's own buffer: the kernel-vector products below grow
  // the shared scratch slots (a regrown slot is freed and reallocated)
  int64_t *dF = reinterpret_cast<int64_t *>(part + 4 * nb);
  if (!F.empty())
    TSVM_CUDA(cudaMemcpyAsync(dF, F.data(), sizeof(int64_t) * F.size(), cudaMemcpyHostToDevice, st));
  const int nf = (int)F.size();

  // kernel-vector products: the tensor cores for the 16-bit precisions (the FP32 form keeps the
  // SIMT products); the loss's own forward product below stays on the FP64-accumulating SIMT
  // kernel, which holds the loss to ~1e-7
  const bool tc_products = precision != TSVM_PREC_FP32 && kermatmul_tc_supported(d, 64);
  auto kp1 = [&](const float *A_, int64_t na_, const float *B_, int64_t nb_, const double *U_,
                 double *out_, bool deriv) -> tsvm_status {
    if (tc_products) return kprod_tc(ctx, A_, na_, B_, nb_, d, gamma, U_, 1, out_, deriv);
    return deriv ? kprod<1, true>(ctx, A_, na_, B_, nb_, d, gamma, U_, 1, out_)
                 : kprod<1, false>(ctx, A_, na_, B_, nb_, d, gamma, U_, 1, out_);
  };

  // forward on the validation set: f = K(Xv, X) beta + b, loss, g
  beta_kernel<<<gn, 256, 0, st>>>(alpha, y, n, beta);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY((kprod<1, false>(ctx, Xv, nv, X, n, d, gamma, beta, 1, sv)));
  val_loss_kernel<<<gv, 256, 0, st>>>(sv, yv, nv, b, lossv, g);
  TSVM_LAUNCHED(ctx);
  std::vector<double> hg(nv);
  TSVM_CUDA(cudaMemcpyAsync(hg.data(), g, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
  TSVM_TRY(kp1(X, n, Xv, nv, g, tmp, false));
  TSVM_CUDA(cudaStreamSynchronize(st));
  double Gb = 0.0;
  for (double v : hg) Gb += v;
  if (nf > 0) {
    zf_kernel<<<1, 256, 0, st>>>(Zf, kp, k, y, dF, nf, zF);
    TSVM_LAUNCHED(ctx);
  } else {
    TSVM_CUDA(cudaMemsetAsync(zF, 0, sizeof(double) * k, st));
  }
  adj_rhs_kernel<<<gn, 256, 0, st>>>(tmp, y, Zf, kp, k, n, zF, nf > 0 ? -Gb / nf : 0.0, c);
  TSVM_LAUNCHED(ctx);
  // adjoint
  TSVM_TRY(kkt_adjoint(ctx, Zf, kp, y, n, k, C, alpha, xi, s, c, lam));

  // r = dQ/dgamma alpha through the range finder
  TSVM_TRY(ro.P(alpha, u));                                              // u = P alpha
  yscale_kernel<<<gn, 256, 0, st>>>(u, y, n, tmp);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(kp1(X, n, X, n, tmp, E1, false));
  yscale_kernel<<<gn, 256, 0, st>>>(E1, y, n, E1);                       // E1 = Ky u
  TSVM_LAUNCHED(ctx);
  // the five vectors dKy is applied to: Om B+ E1, (I-P) E1, u, Om B+ alpha, (I-P) alpha
  TSVM_TRY(ro.OmBp(E1, tmp));
  pack_col<<<gn, 256, 0, st>>>(tmp, y, n, U5, 5, 0);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.P(E1, tmp));
  axpy_kernel<<<gn, 256, 0, st>>>(E1, -1.0, tmp, n, tmp);
  pack_col<<<gn, 256, 0, st>>>(tmp, y, n, U5, 5, 1);
  pack_col<<<gn, 256, 0, st>>>(u, y, n, U5, 5, 2);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.OmBp(alpha, tmp));
  pack_col<<<gn, 256, 0, st>>>(tmp, y, n, U5, 5, 3);
  axpy_kernel<<<gn, 256, 0, st>>>(alpha, -1.0, u, n, tmp);
  pack_col<<<gn, 256, 0, st>>>(tmp, y, n, U5, 5, 4);
  TSVM_LAUNCHED(ctx);
  if (tc_products)                                                       // D_j = K' (Y v_j)
    TSVM_TRY(kprod_tc(ctx, X, n, X, n, d, gamma, U5, 5, D5, true));
  else
    TSVM_TRY((kprod<8, true>(ctx, X, n, X, n, d, gamma, U5, 5, D5)));
  // s2 = (I-P) D4 + B+^T Om^T D5 ; E2 = Ky s2
  unpack_col<<<gn, 256, 0, st>>>(D5, y, n, 5, 3, tmp);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.P(tmp, s2));
  axpy_kernel<<<gn, 256, 0, st>>>(tmp, -1.0, s2, n, s2);
  unpack_col<<<gn, 256, 0, st>>>(D5, y, n, 5, 4, tmp);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.BpTOmT(tmp, t2));
  axpy_kernel<<<gn, 256, 0, st>>>(s2, 1.0, t2, n, s2);
  yscale_kernel<<<gn, 256, 0, st>>>(s2, y, n, tmp);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(kp1(X, n, X, n, tmp, s2, false));
  yscale_kernel<<<gn, 256, 0, st>>>(s2, y, n, s2);                       // s2 <- E2 = Ky s2
  TSVM_LAUNCHED(ctx);
  // r = (I-P) D1 + B+^T Om^T D2 + P D3 + P E2
  unpack_col<<<gn, 256, 0, st>>>(D5, y, n, 5, 2, tmp);
  axpy_kernel<<<gn, 256, 0, st>>>(tmp, 1.0, s2, n, tmp);                  // D3 + E2
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.P(tmp, r));                                                // P (D3 + E2)
  unpack_col<<<gn, 256, 0, st>>>(D5, y, n, 5, 0, tmp);                   // D1
  TSVM_LAUNCHED(ctx);
  axpy_kernel<<<gn, 256, 0, st>>>(r, 1.0, tmp, n, r);
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.P(tmp, t2));
  axpy_kernel<<<gn, 256, 0, st>>>(r, -1.0, t2, n, r);                    // + (I-P) D1
  unpack_col<<<gn, 256, 0, st>>>(D5, y, n, 5, 1, tmp);                   // D2
  TSVM_LAUNCHED(ctx);
  TSVM_TRY(ro.BpTOmT(tmp, t2));
  axpy_kernel<<<gn, 256, 0, st>>>(r, 1.0, t2, n, r);
  TSVM_LAUNCHED(ctx);

  // validation-kernel gamma term: t_v = sum_i beta_i K'_iv
  TSVM_TRY(kp1(Xv, nv, X, n, beta, tv, true));
  dots_kernel<<<nb, 256, 0, st>>>(lam, xi, alpha, C, r, n, lossv, g, tv, nv, part);
  TSVM_LAUNCHED(ctx);
  std::vector<double> hp(4 * nb), hr(nf > 0 ? nf : 1);
  TSVM_CUDA(cudaMemcpyAsync(hp.data(), part, sizeof(double) * 4 * nb, cudaMemcpyDeviceToHost, st));
  for (int t = 0; t < nf; ++t)
    TSVM_CUDA(cudaMemcpyAsync(&hr[t], r + F[t], sizeof(double), cudaMemcpyDeviceToHost, st));
  std::vector<float> hyF(nf > 0 ? nf : 1);
  for (int t = 0; t < nf; ++t)
    TSVM_CUDA(cudaMemcpyAsync(&hyF[t], y + F[t], sizeof(float), cudaMemcpyDeviceToHost, st));
  // dL/dXv
  if (dXv) {
    double *bx = nullptr, *S = nullptr;
    TSVM_TRY(scratch_t(ctx, SLOT_W2, (size_t)n * (d + 1) + (size_t)nv * (d + 1), &bx));
    S = bx + (size_t)n * (d + 1);
    beta_x_kernel<<<gn, 256, 0, st>>>(beta, X, n, d, bx);
    TSVM_LAUNCHED(ctx);
    if (tc_products)
      TSVM_TRY(kprod_tc(ctx, Xv, nv, X, n, d, gamma, bx, d + 1, S, false));
    else
      TSVM_TRY((kprod<32, false>(ctx, Xv, nv, X, n, d, gamma, bx, d + 1, S)));
    dxv_kernel<<<gv, 256, 0, st>>>(S, Xv, g, nv, d, gamma, dXv);
    TSVM_LAUNCHED(ctx);
  }
  TSVM_CUDA(cudaStreamSynchronize(st));
  double q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  for (int bb = 0; bb < nb; ++bb) {
    q0 += hp[bb * 4 + 0];
    q1 += hp[bb * 4 + 1];
    q2 += hp[bb * 4 + 2];
    q3 += hp[bb * 4 + 3];
  }
  double fr = 0.0;
  for (int t = 0; t < nf; ++t) fr += (double)hyF[t] * hr[t];
  res->loss = q2;
  res->dloss_dlog_C = q0;
  res->dloss_dlog_gamma = -gamma * q1 - (nf > 0 ? Gb * gamma * fr / nf : 0.0) + gamma * q3;
  res->n_free_bias = nf;
  res->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return TSVM_OK;
}
