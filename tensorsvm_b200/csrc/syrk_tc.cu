// Mixed-precision Gram of the SMW capacitance matrix, M = I + Z^T D^-1 Z, on the tensor cores.
//
// Replaces the DSYRK of mpc (tensorsvm-train.cu:1674-1697, FP64 on host or cublasDsyrk).  Rows
// are split by their weight dinv_j = 1/D_j:
//   * rows with dinv_j <= tau: z~_j = sqrt(dinv_j) z_j is split into WAYS BF16 terms
//     (hi = bf16(z~), lo = bf16(z~ - hi), ...) and G_tc = sum_{a+b<WAYS} P_a^T P_b is
//     accumulated by tcgen05 MMAs in FP32 (TMEM), per CTA over a contiguous range of rows;
//   * rows with dinv_j > tau (in late iterations the free support vectors, whose weights grow
//     like 1/mu and would dominate the FP32 rounding) are gathered in index order and summed
//     exactly in FP64 (gram_fp64_rows);
// and M = I + G_tc + G_64 is reduced in FP64 in a fixed order.  The IPM refines every SMW
// solve against the exact operator (one extra pass over Z) and adapts tau from the observed
// residual, so M only has to be a good preconditioner.
//
// TC kernel: persistent CTAs (one per SM), each streams its row chunks of 64 rows; per chunk
// WAYS tiles [KP rows][64 cols] BF16, K-major with the 128-byte swizzle, arrive by TMA and
// feed 128 x N x 16 MMAs for the lower block strips (rows 0-127 x cols 0-127, rows 128-255 x
// cols 0-255).  Warp 0 issues TMA, warp 1 owns TMEM and issues MMAs, warps 2-5 drain the
// FP32 accumulators to per-CTA partials.  All waits are bounded.
//
// k > 256 (up to 425): the columns are cut into groups and covered by windows of at most 256
// columns such that every pair of groups shares a window (3 groups, windows of 2, for k <= 384;
// 5 groups, windows of 3, for k <= 425: {0,1,2} {0,3,4} {1,3,4} {2,3,4}); each window is one
// gather + split + tensor-core SYRK of its columns, and each block of M is written by the first
// window that holds both of its groups.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace tsvm {
namespace {

using namespace tc;

constexpr int kSJ = 64;              // rows of Z per chunk (MMA K of one chunk, 4 x 16)
constexpr int kSyrkMaxK = 425;       // widest capacitance matrix the windows cover
constexpr int kSyrkThreads = 192;
constexpr int kSyrkFusedThreads = 320;   // producer, MMA issuer, 8 converter warps

template <int WAYS, int KP>
struct SyrkCfg {
  static constexpr uint32_t kTile = KP * kSJ * 2;          // bytes of one part tile
  static constexpr uint32_t kStage = WAYS * kTile;
  static constexpr int kStages = (200 * 1024) / kStage > 4 ? 4 : (200 * 1024) / kStage;
  static constexpr int kSegs = KP / 128;                   // 128-row strips of the output
  static constexpr uint32_t kTmemCols = KP == 256 ? 512 : 128;
  static constexpr uint32_t kBars = kStages * kStage;      // barrier area offset
  static constexpr uint32_t kSmem = kBars + 256 + 1024;    // + alignment slack
};

// parts[w][t][c][jl] (BF16): WAYS-term split of sqrt(dinv_j) Z[j][c], j = 64 t + jl; zero for
// rows with dinv_j > tau, rows j >= n and columns c >= k.  grid (T, KP / 128), block (32, 8).
// cols (may be null: the identity) maps the KP columns of the operand to columns of Z; columns
// c >= k (k = the window's width) are zero.
template <int WAYS>
__global__ void __launch_bounds__(256)
syrk_prep(const float *__restrict__ Z, int64_t ldz, int k, int64_t n, int64_t T, int KP,
          const double *__restrict__ dinv, double tau, const int *__restrict__ cols,
          __nv_bfloat16 *__restrict__ parts) {
  // a block takes 64 rows x 128 columns: 32 loads in flight per thread (one 128-byte row
  // segment per warp and load), written back as WAYS BF16 tiles of 128 columns x 64 rows
  constexpr int kPC = 128;
  __shared__ float tile[kSJ][kPC + 1];
  __shared__ float wrow[kSJ];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int64_t t = blockIdx.x;
  const int c0 = blockIdx.y * kPC;
  if (tid < kSJ) {
    const int64_t j = t * kSJ + tid;
    float w = 0.f;
    if (j < n) {
      const double d = dinv[j];
      if (d <= tau) w = (float)sqrt(d);
    }
    wrow[tid] = w;
  }
  __syncthreads();
#pragma unroll
  for (int r = ty; r < kSJ; r += 8) {
    const int64_t j = t * kSJ + r;
    const float w = wrow[r];
#pragma unroll
    for (int g = 0; g < kPC / 32; ++g) {
      const int c = c0 + 32 * g + tx;
      float v = 0.f;
      if (w != 0.f && c < k) v = Z[j * ldz + (cols ? cols[c] : c)] * w;
      tile[r][32 * g + tx] = v;
    }
  }
  __syncthreads();
  const size_t part_stride = (size_t)T * KP * kSJ;
  for (int cc = ty; cc < kPC && c0 + cc < KP; cc += 8) {
    const int c = c0 + cc;
    float v0 = tile[2 * tx][cc], v1 = tile[2 * tx + 1][cc];
    __nv_bfloat162 *dst =
        reinterpret_cast<__nv_bfloat162 *>(parts + ((size_t)t * KP + c) * kSJ) + tx;
#pragma unroll
    for (int w = 0; w < WAYS; ++w) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
      dst[w * part_stride / 2] = h;
      v0 -= __low2float(h);
      v1 -= __high2float(h);
    }
  }
}

template <int WAYS, int KP>
__global__ void __launch_bounds__(kSyrkThreads, 1)
syrk_tc_kernel(const __grid_constant__ CUtensorMap map, int T, float *__restrict__ part,
               int *__restrict__ err) {
  using Cfg = SyrkCfg<WAYS, KP>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const uint32_t raw = su32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *sbase = smem_raw + (base - raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sbase + Cfg::kBars);
  const uint32_t b_full = su32(bars);                    // [kStages]
  const uint32_t b_empty = b_full + 8 * Cfg::kStages;    // [kStages]
  const uint32_t b_done = b_empty + 8 * Cfg::kStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * Cfg::kStages + 1);
  volatile int *abort = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = gridDim.x;
  const int t0 = (int)((int64_t)T * blockIdx.x / G), t1 = (int)((int64_t)T * (blockIdx.x + 1) / G);

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::kStages; ++s) {
      mbar_init(b_full + 8 * s, 1);
      mbar_init(b_empty + 8 * s, 1);
    }
    mbar_init(b_done, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(tmem_slot)),
                 "r"(Cfg::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&map) : "memory");
      int st = 0;
      uint32_t ph = 0;
      for (int t = t0; t < t1; ++t) {
        if (!mbar_wait(b_empty + 8 * st, ph ^ 1, abort)) break;
        mbar_expect_tx(b_full + 8 * st, Cfg::kStage);
        const uint32_t dst = base + st * Cfg::kStage;
#pragma unroll
        for (int w = 0; w < WAYS; ++w)
          tma_load_2d(&map, b_full + 8 * st, dst + w * Cfg::kTile, 0, (w * T + t) * KP);
        if (++st == Cfg::kStages) { st = 0; ph ^= 1; }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint64_t d0 = desc_sw128(base);
      int st = 0;
      uint32_t ph = 0;
      bool first = true, ok = true;
      for (int t = t0; t < t1; ++t) {
        if (!mbar_wait(b_full + 8 * st, ph, abort)) { ok = false; break; }
        tc_fence_after();
        const uint64_t ds = d0 + (uint64_t)((st * Cfg::kStage) >> 4);
#pragma unroll
        for (int a = 0; a < WAYS; ++a)
#pragma unroll
          for (int b = 0; a + b < WAYS; ++b)
#pragma unroll
            for (int mb = 0; mb < Cfg::kSegs; ++mb) {
              const uint32_t idesc = idesc_f16(128, (mb + 1) * 128, 1u);
              const uint64_t da = ds + (uint64_t)((a * Cfg::kTile + mb * 128 * 128) >> 4);
              const uint64_t db = ds + (uint64_t)((b * Cfg::kTile) >> 4);
              const uint32_t dt = tmem + (mb == 0 ? 0u : 128u);
#pragma unroll
              for (int kk = 0; kk < kSJ / 16; ++kk)
                umma(dt, da + 2 * kk, db + 2 * kk, idesc,
                     (first && a == 0 && b == 0 && kk == 0) ? 0u : 1u);
            }
        first = false;
        umma_commit(b_empty + 8 * st);
        if (++st == Cfg::kStages) { st = 0; ph ^= 1; }
      }
      if (ok) umma_commit(b_done);
    }
  } else {
    // epilogue: warps 2-5, lane quarter q = warp % 4
    const int q = warp & 3;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    const bool have = t1 > t0;
    if (!have || mbar_wait(b_done, 0, abort)) {
      tc_fence_after();
      float *P = part + (size_t)blockIdx.x * KP * KP;
#pragma unroll
      for (int mb = 0; mb < Cfg::kSegs; ++mb) {
        const int r = mb * 128 + q * 32 + lane;
        const uint32_t tcol = tmem + (mb == 0 ? 0u : 128u);
        for (int c0 = 0; c0 < (mb + 1) * 128; c0 += 32) {
          uint32_t v[32];
          if (have) {
            tmem_ld32(tcol + c0 + lane_off, v);
            tmem_wait_ld();
          } else {
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = 0u;
          }
          float4 *dst = reinterpret_cast<float4 *>(P + (size_t)r * KP + c0);
#pragma unroll
          for (int i = 0; i < 8; ++i)
            dst[i] = make_float4(__uint_as_float(v[4 * i]), __uint_as_float(v[4 * i + 1]),
                                 __uint_as_float(v[4 * i + 2]), __uint_as_float(v[4 * i + 3]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && *abort) atomicExch(err, 1);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(Cfg::kTmemCols));
  }
}

// ---------------------------------------------------------------------------------------
// Fused 2-way SYRK for k <= 256 (one column window, ldz <= KP): the rows of Z arrive as FP32 by
// bulk copies and are scaled by sqrt(dinv), split into BF16 hi + lo and written into the
// swizzled K-major operand tiles by the converter warps inside the kernel, so the operand never
// goes through HBM (syrk_prep + syrk_tc_kernel read Z, write the BF16 parts and read them back).
//   warp 0      bulk copies of 16-row sub-chunks of Z into a 6-slot FP32 ring
//   warp 1      TMEM owner and MMA issuer (as syrk_tc_kernel), 2 operand stages of 64 rows
//   warps 2-9   converters (warp w handles 8-row group (w - 2) % 2 of sub-chunk (w - 2) / 2 of
//               every chunk; four converter warps could not keep the tensor pipe busy), then
//               the epilogue (TMEM -> per-CTA FP32 partials)
// Element (c, j) of a part tile (Z column c, row j of the 64-row chunk) sits at byte
// c * 128 + ((j / 8) ^ (c % 8)) * 16 + (j % 8) * 2: the layout the 128-byte-swizzle TMA load of
// syrk_tc_kernel produces, read by the same MMA descriptors.
template <int KP>
struct FusedCfg {
  static constexpr uint32_t kTile = KP * kSJ * 2;           // one BF16 part tile
  static constexpr uint32_t kPartStage = 2 * kTile;         // hi + lo
  static constexpr int kParts = 2;
  // FP32 sub-chunks of 16 rows in a 6-slot ring: finer slots than half-chunks keep more of the
  // ring's 96 KB in flight (a slot is held while it is converted)
  static constexpr uint32_t kHalfRows = 16;
  static constexpr uint32_t kHalf = kHalfRows * KP * 4;     // FP32 sub-chunk (ldz <= KP)
  static constexpr int kHalves = 6;
  static constexpr int kSubs = kSJ / kHalfRows;             // sub-chunks per 64-row chunk
  static constexpr int kSubWarps = kHalfRows / 8;           // converter warps per sub-chunk
  static constexpr int kSegs = KP / 128;
  static constexpr uint32_t kTmemCols = KP == 256 ? 512 : 128;
  static constexpr uint32_t kStaging = kParts * kPartStage;
  static constexpr uint32_t kBars = kStaging + kHalves * kHalf;
  static constexpr uint32_t kSmem = kBars + 256 + 1024;
};

// Work-unit mode (units non-null, the batched interior-point solve): block b sums the rows of
// unit b alone -- Z = Zs[p] + row0 ldz, its rows, their weights at dinv + goff, the problem's own
// tau -- into partial b; a block whose problem is inactive returns at once.
template <int KP>
__global__ void __launch_bounds__(kSyrkFusedThreads, 1)
syrk_fused_kernel(const float *__restrict__ Z, int64_t ldz, int k, int64_t n, int T,
                  const double *__restrict__ dinv, double tau, float *__restrict__ part,
                  int *__restrict__ err, const WorkUnit *__restrict__ units,
                  const float *const *__restrict__ Zs, const double *__restrict__ taus,
                  const int *__restrict__ active) {
  using Cfg = FusedCfg<KP>;
  int t0, t1;
  if (units) {
    const WorkUnit u = units[blockIdx.x];
    if (active && !active[u.p]) return;   // the whole block, before any barrier or TMEM
    Z = Zs[u.p] + u.row0 * ldz;
    n = u.rows;
    dinv += u.goff;
    tau = taus[u.p];
    t0 = 0;
    t1 = (int)((n + kSJ - 1) / kSJ);
  } else {
    t0 = (int)((int64_t)T * blockIdx.x / gridDim.x);
    t1 = (int)((int64_t)T * (blockIdx.x + 1) / gridDim.x);
  }
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const uint32_t raw = su32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *sbase = smem_raw + (base - raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sbase + Cfg::kBars);
  const uint32_t b_hfull = su32(bars);                       // [kHalves] FP32 half-chunk landed
  const uint32_t b_hempty = b_hfull + 8 * Cfg::kHalves;      // [kHalves] converted
  const uint32_t b_pfull = b_hempty + 8 * Cfg::kHalves;      // [kParts] operand stage written
  const uint32_t b_pempty = b_pfull + 8 * Cfg::kParts;       // [kParts] operand stage consumed
  const uint32_t b_done = b_pempty + 8 * Cfg::kParts;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * Cfg::kHalves + 2 * Cfg::kParts + 1);
  volatile int *abort = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const float *staging = reinterpret_cast<const float *>(sbase + Cfg::kStaging);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::kHalves; ++s) {
      mbar_init(b_hfull + 8 * s, 1);
      mbar_init(b_hempty + 8 * s, Cfg::kSubWarps);
    }
    for (int s = 0; s < Cfg::kParts; ++s) {
      mbar_init(b_pfull + 8 * s, 8);
      mbar_init(b_pempty + 8 * s, 1);
    }
    mbar_init(b_done, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(tmem_slot)),
                 "r"(Cfg::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int t = t0; ok && t < t1; ++t) {
        for (int h = 0; h < Cfg::kSubs; ++h) {
          if (!mbar_wait(b_hempty + 8 * s, ph ^ 1, abort)) { ok = false; break; }
          const int64_t r0 = (int64_t)t * kSJ + h * Cfg::kHalfRows;
          const int64_t rows = n - r0 < (int64_t)Cfg::kHalfRows ? n - r0 : Cfg::kHalfRows;
          if (rows > 0) {
            const uint32_t bytes = (uint32_t)(rows * ldz * 4);
            mbar_expect_tx(b_hfull + 8 * s, bytes);
            bulk_load(base + Cfg::kStaging + s * Cfg::kHalf, Z + r0 * ldz, bytes, b_hfull + 8 * s);
          } else {
            mbar_arrive(b_hfull + 8 * s);   // nothing to copy: the converters zero these rows
          }
          if (++s == Cfg::kHalves) { s = 0; ph ^= 1; }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint64_t d0 = desc_sw128(base);
      int st = 0;
      uint32_t ph = 0;
      bool first = true, ok = true;
      for (int t = t0; t < t1; ++t) {
        if (!mbar_wait(b_pfull + 8 * st, ph, abort)) { ok = false; break; }
        tc_fence_after();
        const uint64_t ds = d0 + (uint64_t)((st * Cfg::kPartStage) >> 4);
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; a + b < 2; ++b)
#pragma unroll
            for (int mb = 0; mb < Cfg::kSegs; ++mb) {
              const uint32_t idesc = idesc_f16(128, (mb + 1) * 128, 1u);
              const uint64_t da = ds + (uint64_t)((a * Cfg::kTile + mb * 128 * 128) >> 4);
              const uint64_t db = ds + (uint64_t)((b * Cfg::kTile) >> 4);
              const uint32_t dt = tmem + (mb == 0 ? 0u : 128u);
#pragma unroll
              for (int kk = 0; kk < kSJ / 16; ++kk)
                umma(dt, da + 2 * kk, db + 2 * kk, idesc,
                     (first && a == 0 && b == 0 && kk == 0) ? 0u : 1u);
            }
        first = false;
        umma_commit(b_pempty + 8 * st);
        if (++st == Cfg::kParts) { st = 0; ph ^= 1; }
      }
      if (ok) umma_commit(b_done);
    }
  } else {
    // converters: warp cw = warp - 2 takes rows 8 g .. 8 g + 7 (g = cw % 2) of sub-chunk h = cw / 2
    // of every chunk, lane = column within each 32-column block
    const int cw = warp - 2, g = cw % Cfg::kSubWarps, h = cw / Cfg::kSubWarps;
    int ps = 0;
    uint32_t pph = 0;
    bool ok = true;
    // lane l < 8 holds dinv of row l of this warp's 8-row group in chunk tt, loaded one chunk
    // ahead so that the load is off the conversion's path
    auto fetch = [&](int tt) -> double {
      const int64_t row = (int64_t)tt * kSJ + h * Cfg::kHalfRows + 8 * g + lane;
      return (lane < 8 && tt < t1 && row < n) ? dinv[row] : 0.0;
    };
    double dv_next = fetch(t0);
    for (int t = t0; ok && t < t1; ++t) {
      const double dv = dv_next;
      dv_next = fetch(t + 1);
      if (!mbar_wait(b_pempty + 8 * ps, pph ^ 1, abort)) { ok = false; break; }
      uint8_t *tile = sbase + ps * Cfg::kPartStage;
      // this sub-chunk's slot of the ring (sub-chunks in the order (t, 0), (t, 1), ...)
      const int hidx = Cfg::kSubs * (t - t0) + h;
      const int hs = hidx % Cfg::kHalves;
      const uint32_t hph = (uint32_t)((hidx / Cfg::kHalves) & 1);
      if (!mbar_wait(b_hfull + 8 * hs, hph, abort)) { ok = false; break; }
      const int64_t r0 = (int64_t)t * kSJ + h * Cfg::kHalfRows + 8 * g;   // this warp's rows
      float wr = 0.f;   // lane l < 8: the weight of row r0 + l (0 for exact rows and padding)
      if (lane < 8 && r0 + lane < n && dv <= tau) wr = (float)sqrt(dv);
      float wj[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) wj[q] = __shfl_sync(0xffffffffu, wr, q);
      const float *src = staging + (size_t)hs * (Cfg::kHalf / 4) + (size_t)(8 * g) * ldz;
      const int jg = h * Cfg::kSubWarps + g;   // 8-row group of the 64-row chunk
#pragma unroll 2
      for (int cb = 0; cb < KP; cb += 32) {
        const int c = cb + lane;
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float x = c < k ? src[(size_t)q * ldz + c] : 0.f;
          v[q] = wj[q] != 0.f ? x * wj[q] : 0.f;   // select: padding rows may hold anything
        }
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const __nv_bfloat162 hv = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
          const float2 hf = __bfloat1622float2(hv);
          const __nv_bfloat162 lv = __floats2bfloat162_rn(v[2 * q] - hf.x, v[2 * q + 1] - hf.y);
          hi[q] = *reinterpret_cast<const uint32_t *>(&hv);
          lo[q] = *reinterpret_cast<const uint32_t *>(&lv);
        }
        const uint32_t off = (uint32_t)c * 128u + (uint32_t)((jg ^ (c & 7)) << 4);
        *reinterpret_cast<uint4 *>(tile + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4 *>(tile + Cfg::kTile + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(b_hempty + 8 * hs);
      // the generic-proxy stores must be visible to the tensor cores' async-proxy reads
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(b_pfull + 8 * ps);
      if (++ps == Cfg::kParts) { ps = 0; pph ^= 1; }
    }
    // epilogue (lane quarter q = warp % 4; the two warps of a quarter take alternate 32-column
    // blocks)
    const int q = warp & 3;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    const bool have = t1 > t0;
    if (ok && (!have || mbar_wait(b_done, 0, abort))) {
      tc_fence_after();
      float *P = part + (size_t)blockIdx.x * KP * KP;
#pragma unroll
      for (int mb = 0; mb < Cfg::kSegs; ++mb) {
        const int r = mb * 128 + q * 32 + lane;
        const uint32_t tcol = tmem + (mb == 0 ? 0u : 128u);
        for (int c0 = 32 * (cw >> 2); c0 < (mb + 1) * 128; c0 += 64) {
          uint32_t v[32];
          if (have) {
            tmem_ld32(tcol + c0 + lane_off, v);
            tmem_wait_ld();
          } else {
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = 0u;
          }
          float4 *dst = reinterpret_cast<float4 *>(P + (size_t)r * KP + c0);
#pragma unroll
          for (int i = 0; i < 8; ++i)
            dst[i] = make_float4(__uint_as_float(v[4 * i]), __uint_as_float(v[4 * i + 1]),
                                 __uint_as_float(v[4 * i + 2]), __uint_as_float(v[4 * i + 3]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && *abort) atomicExch(err, 1);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(Cfg::kTmemCols));
  }
}

// M[R][C] = M[C][R] = (R == C) + G64[R][C] + sum_g part[g][r][c] (FP64) for the window entries
// r >= c, R = cols[r], C = cols[c] (identity when cols is null), k the full width, wl the
// window's.  With a window plan only the entries whose group pair this window owns
// (owner[gid[R] * ng + gid[C]] == win) are written.  A timed-out tensor-core launch (err set)
// poisons M with NaN.  A block takes 32 consecutive entries (coalesced rows of the partials);
// its 8 warps sum the CTA partials g = w, w + 8, ... (four loads in flight per thread), and the
// eight sums are added in warp order: the same order on every run.
constexpr int kReduceEntries = 32;
__global__ void __launch_bounds__(256)
syrk_reduce(const float *__restrict__ part, int G, int KP, int k, int wl,
            const int *__restrict__ cols, const int *__restrict__ gid,
            const int *__restrict__ owner, int ng, int win, const double *__restrict__ G64,
            const int *__restrict__ err, double *__restrict__ M) {
  __shared__ double red[8][kReduceEntries + 1];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t e = (int64_t)blockIdx.x * kReduceEntries + tx;
  const bool valid = e < (int64_t)wl * wl;
  const int r = valid ? (int)(e / wl) : 0, c = valid ? (int)(e % wl) : 0;
  const bool want = valid && c <= r;
  double s = 0.0;
  if (want) {
    const float *p = part + (size_t)r * KP + c;
    const size_t stride = (size_t)KP * KP;
    int g = ty;
    for (; g + 24 < G; g += 32) {
      const float a0 = __ldcs(p + (size_t)g * stride), a1 = __ldcs(p + (size_t)(g + 8) * stride);
      const float a2 = __ldcs(p + (size_t)(g + 16) * stride);
      const float a3 = __ldcs(p + (size_t)(g + 24) * stride);
      s += (double)a0;
      s += (double)a1;
      s += (double)a2;
      s += (double)a3;
    }
    for (; g < G; g += 8) s += (double)__ldcs(p + (size_t)g * stride);
  }
  red[ty][tx] = s;
  __syncthreads();
  if (ty != 0 || !want) return;
  const int R = cols ? cols[r] : r, C = cols ? cols[c] : c;
  if (owner && owner[gid[R] * ng + gid[C]] != win) return;
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < 8; ++w) t += red[w][tx];
  if (G64) t += G64[(size_t)R * k + C];
  if (R == C) t += 1.0;
  if (*err) t = NAN;
  M[(size_t)R * k + C] = t;
  M[(size_t)C * k + R] = t;
}

// Rows with dinv > tau, in index order: per-block counts over contiguous row ranges, then each
// block writes its rows at the prefix offset.  count_out[0] = total.
__global__ void __launch_bounds__(256)
big_rows_count(const double *__restrict__ dinv, int64_t n, double tau, int *__restrict__ counts) {
  __shared__ int wsum[8];
  const int64_t rows = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * rows, r1 = min(n, r0 + rows);
  int c = 0;
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) c += dinv[i] > tau ? 1 : 0;
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < 8; ++w) s += wsum[w];
    counts[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(256)
big_rows_index(const double *__restrict__ dinv, int64_t n, double tau,
               const int *__restrict__ counts, int64_t *__restrict__ idx,
               int *__restrict__ count_out) {
  __shared__ int wcnt[8];
  __shared__ int base_sh;
  const int64_t rows = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * rows, r1 = min(n, r0 + rows);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    int s = 0;
    for (int b = 0; b < (int)blockIdx.x; ++b) s += counts[b];
    base_sh = s;
    if (blockIdx.x == gridDim.x - 1) count_out[0] = s + counts[blockIdx.x];
  }
  __syncthreads();
  int base = base_sh;
  for (int64_t b0 = r0; b0 < r1; b0 += blockDim.x) {
    const int64_t i = b0 + threadIdx.x;
    const bool f = i < r1 && dinv[i] > tau;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += wcnt[w];
    off += __popc(bal & ((1u << lane) - 1u));
    if (f) idx[off] = i;
    int tot = 0;
    for (int w = 0; w < 8; ++w) tot += wcnt[w];
    __syncthreads();
    base += tot;
  }
}

// Batched form: block u lists the rows of work unit u with dinv > taus[p] (indices within the
// unit, in index order) at rowidx + goff and their count in counts[u].
__global__ void __launch_bounds__(256)
big_rows_units_kernel(const double *__restrict__ dinv, const WorkUnit *__restrict__ units,
                      const int *__restrict__ active, const double *__restrict__ taus,
                      int64_t *__restrict__ rowidx, int *__restrict__ counts) {
  __shared__ int wcnt[8];
  const WorkUnit u = units[blockIdx.x];
  if (active && !active[u.p]) {
    if (threadIdx.x == 0) counts[blockIdx.x] = 0;
    return;
  }
  const double tau = taus[u.p];
  const double *dv = dinv + u.goff;
  int64_t *idx = rowidx + u.goff;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int base = 0;   // the same in every thread: updated from the same shared counts
  for (int b0 = 0; b0 < u.rows; b0 += 256) {
    const int i = b0 + (int)threadIdx.x;
    const bool f = i < u.rows && dv[i] > tau;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += wcnt[w];
    off += __popc(bal & ((1u << lane) - 1u));
    if (f) idx[off] = i;
    int tot = 0;
    for (int w = 0; w < 8; ++w) tot += wcnt[w];
    __syncthreads();
    base += tot;
  }
  if (threadIdx.x == 0) counts[blockIdx.x] = base;
}

// Column windows for k > 256 (see the file comment).
struct SyrkPlan {
  int ng = 1, nw = 1;
  int gbeg[6] = {0};                 // group g = columns [gbeg[g], gbeg[g + 1])
  int wg[4][3] = {{0}};              // groups of each window
  int wn[4] = {1};                   // groups per window
};

SyrkPlan syrk_plan(int k) {
  SyrkPlan p;
  if (k <= 256) {
    p.gbeg[1] = k;
    return p;
  }
  if (k <= 384) {
    p.ng = 3;
    p.nw = 3;
    const int w[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int i = 0; i < 3; ++i) {
      p.wn[i] = 2;
      p.wg[i][0] = w[i][0];
      p.wg[i][1] = w[i][1];
    }
  } else {
    p.ng = 5;
    p.nw = 4;
    const int w[4][3] = {{0, 1, 2}, {0, 3, 4}, {1, 3, 4}, {2, 3, 4}};
    for (int i = 0; i < 4; ++i) {
      p.wn[i] = 3;
      for (int j = 0; j < 3; ++j) p.wg[i][j] = w[i][j];
    }
  }
  const int gs = (k + p.ng - 1) / p.ng;
  for (int g = 0; g <= p.ng; ++g) p.gbeg[g] = std::min(k, g * gs);
  return p;
}

template <int WAYS, int KP>
tsvm_status launch_syrk_tc(tsvm_context *ctx, const CUtensorMap &map, int T, int G, float *part,
                           int *err) {
  using Cfg = SyrkCfg<WAYS, KP>;
  auto kern = syrk_tc_kernel<WAYS, KP>;
  TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::kSmem));
  kern<<<G, kSyrkThreads, Cfg::kSmem, ctx->stream>>>(map, T, part, err);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

template <int KP>
tsvm_status launch_syrk_fused(tsvm_context *ctx, const float *Z, int64_t ldz, int k, int64_t n,
                              int T, const double *dinv, double tau, int G, float *part,
                              int *err) {
  using Cfg = FusedCfg<KP>;
  auto kern = syrk_fused_kernel<KP>;
  TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::kSmem));
  kern<<<G, kSyrkFusedThreads, Cfg::kSmem, ctx->stream>>>(Z, ldz, k, n, T, dinv, tau, part, err,
                                                          nullptr, nullptr, nullptr, nullptr);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

template <int KP>
tsvm_status launch_syrk_fused_units(tsvm_context *ctx, const float *const *Zs, int64_t ldz,
                                    int k, const WorkUnit *units, int nunits, const int *active,
                                    const double *dinv, const double *taus, float *part,
                                    int *err) {
  using Cfg = FusedCfg<KP>;
  auto kern = syrk_fused_kernel<KP>;
  TSVM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::kSmem));
  kern<<<nunits, kSyrkFusedThreads, Cfg::kSmem, ctx->stream>>>(
      nullptr, ldz, k, 0, 0, dinv, 0.0, part, err, units, Zs, taus, active);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

}  // namespace

bool syrk_tc_supported(int k) { return k >= 1 && k <= kSyrkMaxK && tc::encode_fn() != nullptr; }

tsvm_status big_rows(tsvm_context *ctx, const double *dinv, int64_t n, double tau, int64_t *idx,
                     int *count_dev) {
  const int nb = ctx->num_sms * 4;
  int *counts = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SYRK_CNT, (size_t)nb, &counts));
  big_rows_count<<<nb, 256, 0, ctx->stream>>>(dinv, n, tau, counts);
  TSVM_LAUNCHED(ctx);
  big_rows_index<<<nb, 256, 0, ctx->stream>>>(dinv, n, tau, counts, idx, count_dev);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

tsvm_status big_rows_units(tsvm_context *ctx, const double *dinv, const WorkUnit *units,
                           int nunits, const int *active, const double *taus, int64_t *rowidx,
                           int *counts) {
  if (nunits < 1) return TSVM_ERR_INVALID_ARGUMENT;
  big_rows_units_kernel<<<nunits, 256, 0, ctx->stream>>>(dinv, units, active, taus, rowidx,
                                                         counts);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

int syrk_units_kp(int k) { return k <= 128 ? 128 : 256; }

tsvm_status syrk_units_tc(tsvm_context *ctx, const float *const *Zs, int64_t ldz, int k,
                          const WorkUnit *units, int nunits, const int *active,
                          const double *dinv, const double *taus, float *part_tc, int *err) {
  const int KP = syrk_units_kp(k);
  if (!syrk_tc_supported(k) || k > 256 || ldz > KP || ldz % 4 != 0 || nunits < 1)
    return TSVM_ERR_UNSUPPORTED;
  return KP == 128 ? launch_syrk_fused_units<128>(ctx, Zs, ldz, k, units, nunits, active, dinv,
                                                  taus, part_tc, err)
                   : launch_syrk_fused_units<256>(ctx, Zs, ldz, k, units, nunits, active, dinv,
                                                  taus, part_tc, err);
}

tsvm_status syrk_capacitance_tc(tsvm_context *ctx, const float *Z, int ldz, int64_t n, int k,
                                const double *dinv, double tau, int ways, const double *G64,
                                double *M) {
  if (!syrk_tc_supported(k) || (ways != 2 && ways != 3)) return TSVM_ERR_UNSUPPORTED;
  const SyrkPlan plan = syrk_plan(k);
  // per window: its columns (device table), width and tensor-core width
  int *dplan = nullptr;   // [nw][256] columns | gid[k] | owner[ng][ng]
  const int *dgid = nullptr, *downer = nullptr;
  std::vector<int> wl(plan.nw), hplan;
  if (plan.nw > 1) {
    hplan.assign((size_t)plan.nw * 256 + k + plan.ng * plan.ng, 0);
    std::vector<int> owner(plan.ng * plan.ng, -1);
    for (int w = 0; w < plan.nw; ++w) {
      int c = 0;
      for (int j = 0; j < plan.wn[w]; ++j) {
        const int g = plan.wg[w][j];
        for (int col = plan.gbeg[g]; col < plan.gbeg[g + 1]; ++col) hplan[(size_t)w * 256 + c++] = col;
        for (int j2 = 0; j2 < plan.wn[w]; ++j2) {
          const int g2 = plan.wg[w][j2];
          if (owner[g * plan.ng + g2] < 0) owner[g * plan.ng + g2] = w;
        }
      }
      wl[w] = c;
    }
    for (int g = 0; g < plan.ng; ++g)
      for (int col = plan.gbeg[g]; col < plan.gbeg[g + 1]; ++col) hplan[(size_t)plan.nw * 256 + col] = g;
    std::copy(owner.begin(), owner.end(), hplan.begin() + (size_t)plan.nw * 256 + k);
    TSVM_TRY(scratch_t(ctx, SLOT_SYRK_PLAN, hplan.size(), &dplan));
    if (ctx->syrk_plan_k != k) {   // the table depends on k only: upload once per width
      TSVM_CUDA(cudaMemcpyAsync(dplan, hplan.data(), sizeof(int) * hplan.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
      TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
      ctx->syrk_plan_k = k;
    }
    dgid = dplan + (size_t)plan.nw * 256;
    downer = dgid + k;
  } else {
    wl[0] = k;
  }
  int wmax = 0;
  for (int w = 0; w < plan.nw; ++w) wmax = std::max(wmax, wl[w]);
  const int KPmax = wmax <= 128 ? 128 : 256;
  const int64_t T = ceil_div(n, (int64_t)kSJ);
  // One window, 2-way split, rows of at most KP floats on 16-byte boundaries: scale and split
  // inside the tensor-core kernel (no BF16 operand in HBM).
  if (ways == 2 && plan.nw == 1 && ldz <= KPmax && ldz % 4 == 0 &&
      (reinterpret_cast<uintptr_t>(Z) & 15) == 0 && T <= (int64_t)INT32_MAX) {
    const int G = (int)std::min<int64_t>(ctx->num_sms, T);
    float *part = nullptr;
    TSVM_TRY(scratch_t(ctx, SLOT_SYRK_PART, (size_t)G * KPmax * KPmax + 64, &part));
    int *err = reinterpret_cast<int *>(part + (size_t)G * KPmax * KPmax);
    TSVM_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    const tsvm_status st =
        KPmax == 128 ? launch_syrk_fused<128>(ctx, Z, ldz, k, n, (int)T, dinv, tau, G, part, err)
                     : launch_syrk_fused<256>(ctx, Z, ldz, k, n, (int)T, dinv, tau, G, part, err);
    if (st != TSVM_OK) return st;
    syrk_reduce<<<(unsigned)ceil_div((int64_t)k * k, kReduceEntries), 256, 0, ctx->stream>>>(
        part, G, KPmax, k, k, nullptr, nullptr, nullptr, plan.ng, 0, G64, err, M);
    TSVM_LAUNCHED(ctx);
    return TSVM_OK;
  }
  if ((int64_t)ways * T * KPmax > (int64_t)INT32_MAX) return TSVM_ERR_UNSUPPORTED;
  __nv_bfloat16 *parts = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SYRK_OP, (size_t)ways * T * KPmax * kSJ, &parts));
  const int G = (int)std::min<int64_t>(ctx->num_sms, T);
  float *part = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_SYRK_PART, (size_t)G * KPmax * KPmax + 64, &part));
  int *err = reinterpret_cast<int *>(part + (size_t)G * KPmax * KPmax);
  TSVM_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
  for (int w = 0; w < plan.nw; ++w) {
    const int KP = wl[w] <= 128 ? 128 : 256;
    const int *cols = plan.nw > 1 ? dplan + (size_t)w * 256 : nullptr;
    const dim3 pgrid((unsigned)T, (unsigned)(KP / 128));
    if (ways == 2)
      syrk_prep<2><<<pgrid, dim3(32, 8), 0, ctx->stream>>>(Z, ldz, wl[w], n, T, KP, dinv, tau,
                                                           cols, parts);
    else
      syrk_prep<3><<<pgrid, dim3(32, 8), 0, ctx->stream>>>(Z, ldz, wl[w], n, T, KP, dinv, tau,
                                                           cols, parts);
    TSVM_LAUNCHED(ctx);
    CUtensorMap map;
    if (!tc::make_map(&map, parts, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, kSJ,
                      (uint64_t)ways * T * KP, kSJ, KP))
      return TSVM_ERR_CUDA;
    tsvm_status st;
    if (ways == 2)
      st = KP == 128 ? launch_syrk_tc<2, 128>(ctx, map, (int)T, G, part, err)
                     : launch_syrk_tc<2, 256>(ctx, map, (int)T, G, part, err);
    else
      st = KP == 128 ? launch_syrk_tc<3, 128>(ctx, map, (int)T, G, part, err)
                     : launch_syrk_tc<3, 256>(ctx, map, (int)T, G, part, err);
    if (st != TSVM_OK) return st;
    syrk_reduce<<<(unsigned)ceil_div((int64_t)wl[w] * wl[w], kReduceEntries), 256, 0,
                  ctx->stream>>>(
        part, G, KP, k, wl[w], cols, dgid, downer, plan.ng, w, G64, err, M);
    TSVM_LAUNCHED(ctx);
  }
  return TSVM_OK;
}

}  // namespace tsvm
