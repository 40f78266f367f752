// Gaussian sketch identical to the reference's gaussrand() stream, generated on the GPU.
//
// The reference (tensorsvm-train.cu:2621-2643, filled at 1966-1974) draws Q (n x k, row-major)
// one value at a time on the host with the Marsaglia polar method over glibc rand() from the
// default seed.  That stream is reproduced here in four steps:
//
//  1. glibc's TYPE_3 generator is the additive lagged-Fibonacci recurrence
//        r[i] = r[i-31] + r[i-3]  (mod 2^32),   rand() #m = r[m+344] >> 1,
//     which is linear over Z/2^32 in its 31-word state.  The host raises the 31x31 transition
//     matrix T to the powers T^(L*2^m) once per context; `sketch_seed` gives every segment of
//     L = 2048 outputs its start state by multiplying the base state by the matrices of the
//     set bits of its segment index.
//  2. `sketch_generate` runs the recurrence for each segment with a fully unrolled 32-word
//     register ring and writes the raw rand() stream.
//  3. The polar method consumes rand() in pairs and accepts a pair when 0 < S < 1, where
//     S = V1^2 + V2^2 in float.  Every attempt uses exactly two draws, so attempt j is draws
//     (2j, 2j+1); `sketch_count` + `sketch_scan` + `sketch_emit` compact the accepted attempts
//     in order (a three-kernel stream compaction).
//  4. Each accepted pair yields V1*f and V2*f with f = sqrt(-2 log S / S), in the same float
//     operation order as the reference's host code (explicit round-to-nearest intrinsics, no
//     contraction).  log is evaluated in double and rounded to float; that equals glibc's
//     logf except for rare 1-ulp cases, so the sketch matches the reference bit for bit in
//     the accept pattern and to <= 1 ulp in value.
#include <math.h>

#include <algorithm>
#include <array>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {

namespace {

constexpr int kSegWords = 2048;       // rand() outputs generated per segment (thread)
constexpr int kPairsPerBlock = 4096;  // attempts handled per block in count/emit
constexpr int kMaxLevels = 28;        // segments up to 2^28 (far beyond any device memory)

__global__ void __launch_bounds__(256) sketch_seed(const uint32_t *__restrict__ jump, int levels,
                                                   const uint32_t *__restrict__ state0,
                                                   uint32_t *__restrict__ states, int64_t nseg) {
  __shared__ uint32_t J[31 * 31];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t s[31];
#pragma unroll
  for (int w = 0; w < 31; ++w) s[w] = state0[w];
  for (int m = 0; m < levels; ++m) {
    __syncthreads();
    for (int i = threadIdx.x; i < 31 * 31; i += blockDim.x) J[i] = jump[m * 961 + i];
    __syncthreads();
    if (t < nseg && ((t >> m) & 1)) {
      uint32_t ns[31];
#pragma unroll
      for (int r = 0; r < 31; ++r) {
        uint32_t acc = 0;
#pragma unroll
        for (int c = 0; c < 31; ++c) acc += J[r * 31 + c] * s[c];
        ns[r] = acc;
      }
#pragma unroll
      for (int r = 0; r < 31; ++r) s[r] = ns[r];
    }
  }
  if (t < nseg) {
#pragma unroll
    for (int w = 0; w < 31; ++w) states[(int64_t)w * nseg + t] = s[w];
  }
}

__global__ void __launch_bounds__(128) sketch_generate(const uint32_t *__restrict__ states,
                                                       int64_t nseg, uint32_t *__restrict__ R) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nseg) return;
  // ring slot of relative index j is (j & 31); the state word w is relative index w - 31
  uint32_t b[32];
  b[0] = 0;
#pragma unroll
  for (int w = 0; w < 31; ++w) b[(w + 1) & 31] = states[(int64_t)w * nseg + t];
  uint4 *out = reinterpret_cast<uint4 *>(R + t * kSegWords);
  for (int blk = 0; blk < kSegWords / 32; ++blk) {
#pragma unroll
    for (int i = 0; i < 32; ++i) b[i] = b[(i + 1) & 31] + b[(i + 29) & 31];
#pragma unroll
    for (int q = 0; q < 8; ++q)
      out[blk * 8 + q] = make_uint4(b[4 * q] >> 1, b[4 * q + 1] >> 1, b[4 * q + 2] >> 1,
                                    b[4 * q + 3] >> 1);
  }
}

struct Polar {
  float v1, v2, s;
  bool ok;
};

__device__ __forceinline__ Polar polar_attempt(uint2 r) {
  // (float)rand() / RAND_MAX with RAND_MAX promoted to 2^31: exact scaling of float(r)
  const float u1 = __fmul_rn(__uint2float_rn(r.x), 4.656612873077392578125e-10f);
  const float u2 = __fmul_rn(__uint2float_rn(r.y), 4.656612873077392578125e-10f);
  Polar p;
  p.v1 = __fsub_rn(__fmul_rn(2.0f, u1), 1.0f);
  p.v2 = __fsub_rn(__fmul_rn(2.0f, u2), 1.0f);
  p.s = __fadd_rn(__fmul_rn(p.v1, p.v1), __fmul_rn(p.v2, p.v2));
  p.ok = (p.s < 1.0f) && (p.s != 0.0f);
  return p;
}

__global__ void __launch_bounds__(256) sketch_count(const uint2 *__restrict__ R2,
                                                    int64_t attempts,
                                                    unsigned long long *__restrict__ counts) {
  __shared__ double sh[8];
  const int64_t base = (int64_t)blockIdx.x * kPairsPerBlock;
  double c = 0;
  for (int i = 0; i < kPairsPerBlock / 256; ++i) {
    const int64_t p = base + i * 256 + threadIdx.x;
    if (p < attempts && polar_attempt(R2[p]).ok) c += 1.0;
  }
  double v[1] = {c};
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) counts[blockIdx.x] = (unsigned long long)v[0];
}

// Exclusive scan of per-block counts (one block); offsets[nb] receives the total.
__global__ void __launch_bounds__(1024) sketch_scan(unsigned long long *__restrict__ counts,
                                                    int64_t nb) {
  __shared__ unsigned long long part[1024];
  const int64_t per = (nb + 1023) / 1024;
  const int64_t lo = threadIdx.x * per, hi = min(nb, lo + per);
  unsigned long long s = 0;
  for (int64_t i = lo; i < hi; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    unsigned long long v = threadIdx.x >= off ? part[threadIdx.x - off] : 0ull;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned long long run = part[threadIdx.x] - s;  // exclusive prefix of this thread's range
  for (int64_t i = lo; i < hi; ++i) {
    const unsigned long long c = counts[i];
    counts[i] = run;
    run += c;
  }
  if (threadIdx.x == 1023) counts[nb] = part[1023];
}

__global__ void __launch_bounds__(256) sketch_emit(const uint2 *__restrict__ R2, int64_t attempts,
                                                   const unsigned long long *__restrict__ offsets,
                                                   int64_t count, float *__restrict__ Q) {
  __shared__ unsigned int wcount[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kPairsPerBlock;
  unsigned long long run = offsets[blockIdx.x];
  for (int i = 0; i < kPairsPerBlock / 256; ++i) {
    const int64_t p = base + i * 256 + threadIdx.x;
    Polar a;
    a.ok = false;
    if (p < attempts) a = polar_attempt(R2[p]);
    const unsigned ballot = __ballot_sync(0xffffffffu, a.ok);
    if (lane == 0) wcount[warp] = __popc(ballot);
    __syncthreads();
    unsigned int woff = 0, total = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      woff += (w < warp) ? wcount[w] : 0u;
      total += wcount[w];
    }
    const unsigned long long idx = run + woff + __popc(ballot & ((1u << lane) - 1u));
    if (a.ok) {
      const float lg = (float)log((double)a.s);
      const float f = __fsqrt_rn(__fdiv_rn(__fmul_rn(-2.0f, lg), a.s));
      const int64_t o = (int64_t)(2 * idx);
      if (o + 1 < count) {
        *reinterpret_cast<float2 *>(Q + o) = make_float2(__fmul_rn(a.v1, f), __fmul_rn(a.v2, f));
      } else if (o < count) {
        Q[o] = __fmul_rn(a.v1, f);
      }
    }
    run += total;
    __syncthreads();
  }
}

using Mat31 = std::array<uint32_t, 961>;

Mat31 mat_mul(const Mat31 &A, const Mat31 &B) {
  Mat31 C{};
  for (int r = 0; r < 31; ++r)
    for (int m = 0; m < 31; ++m) {
      const uint32_t a = A[r * 31 + m];
      if (!a) continue;
      for (int c = 0; c < 31; ++c) C[r * 31 + c] += a * B[m * 31 + c];
    }
  return C;
}

// glibc rand() initial table from seed 1 and the 31-word state before output 0.
std::array<uint32_t, 31> glibc_state0() {
  std::vector<uint32_t> r(344);
  int32_t word = 1;
  r[0] = 1;
  for (int i = 1; i < 31; ++i) {
    const int32_t hi = word / 127773, lo = word % 127773;
    word = 16807 * lo - 2836 * hi;
    if (word < 0) word += 2147483647;
    r[i] = (uint32_t)word;
  }
  for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
  for (int i = 34; i < 344; ++i) r[i] = r[i - 31] + r[i - 3];
  std::array<uint32_t, 31> s{};
  for (int w = 0; w < 31; ++w) s[w] = r[313 + w];
  return s;
}

tsvm_status ensure_jump_tables(tsvm_context *ctx, uint32_t **dev) {
  uint32_t *d = nullptr;
  TSVM_TRY(scratch_t(ctx, SLOT_JUMP, (size_t)(kMaxLevels * 961 + 64), &d));
  if (ctx->jump_levels != kMaxLevels) {
    Mat31 T{};
    for (int w = 0; w < 30; ++w) T[w * 31 + w + 1] = 1;
    T[30 * 31 + 0] = 1;
    T[30 * 31 + 28] = 1;
    Mat31 P = T;  // T^(2^i); L = 2048 = 2^11
    for (int i = 0; i < 11; ++i) P = mat_mul(P, P);
    std::vector<uint32_t> host((size_t)kMaxLevels * 961 + 64, 0);
    for (int m = 0; m < kMaxLevels; ++m) {
      std::copy(P.begin(), P.end(), host.begin() + (size_t)m * 961);
      P = mat_mul(P, P);
    }
    const auto s0 = glibc_state0();
    std::copy(s0.begin(), s0.end(), host.begin() + (size_t)kMaxLevels * 961);
    TSVM_CUDA(cudaMemcpyAsync(d, host.data(), host.size() * sizeof(uint32_t),
                              cudaMemcpyHostToDevice, ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->jump_levels = kMaxLevels;
  }
  *dev = d;
  return TSVM_OK;
}

tsvm_status rand_stream_segments(tsvm_context *ctx, int64_t nseg, uint32_t **R_out) {
  uint32_t *jump = nullptr, *states = nullptr, *R = nullptr;
  TSVM_TRY(ensure_jump_tables(ctx, &jump));
  TSVM_TRY(scratch_t(ctx, SLOT_STATES, (size_t)nseg * 31, &states));
  TSVM_TRY(scratch_t(ctx, SLOT_RAND, (size_t)nseg * kSegWords, &R));
  int levels = 0;
  while (levels < kMaxLevels && (int64_t(1) << levels) < nseg) ++levels;
  sketch_seed<<<(unsigned)ceil_div(nseg, 256), 256, 0, ctx->stream>>>(
      jump, levels, jump + (size_t)kMaxLevels * 961, states, nseg);
  TSVM_LAUNCHED(ctx);
  sketch_generate<<<(unsigned)ceil_div(nseg, 128), 128, 0, ctx->stream>>>(states, nseg, R);
  TSVM_LAUNCHED(ctx);
  *R_out = R;
  return TSVM_OK;
}

}  // namespace

tsvm_status glibc_rand_stream(tsvm_context *ctx, int64_t count, uint32_t *out) {
  if (count <= 0) return TSVM_OK;
  const int64_t nseg = ceil_div(count, kSegWords);
  uint32_t *R = nullptr;
  TSVM_TRY(rand_stream_segments(ctx, nseg, &R));
  TSVM_CUDA(cudaMemcpyAsync(out, R, (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            ctx->stream));
  return TSVM_OK;
}

tsvm_status sketch_glibc(tsvm_context *ctx, int64_t count, float *Q) {
  if (count <= 0) return TSVM_OK;
  const int64_t npairs = (count + 1) / 2;
  // acceptance probability pi/4; margin of many standard deviations
  double attempts_d = (double)npairs * (4.0 / M_PI) + 10.0 * sqrt((double)npairs) + 4096.0;
  for (int retry = 0; retry < 4; ++retry) {
    const int64_t nseg = ceil_div((int64_t)(2.0 * attempts_d), kSegWords);
    const int64_t attempts = nseg * kSegWords / 2;
    uint32_t *R = nullptr;
    TSVM_TRY(rand_stream_segments(ctx, nseg, &R));
    const int64_t nb = ceil_div(attempts, kPairsPerBlock);
    unsigned long long *counts = nullptr;
    TSVM_TRY(scratch_t(ctx, SLOT_COUNTS, (size_t)nb + 1, &counts));
    const uint2 *R2 = reinterpret_cast<const uint2 *>(R);
    sketch_count<<<(unsigned)nb, 256, 0, ctx->stream>>>(R2, attempts, counts);
    TSVM_LAUNCHED(ctx);
    sketch_scan<<<1, 1024, 0, ctx->stream>>>(counts, nb);
    TSVM_LAUNCHED(ctx);
    unsigned long long total = 0;
    TSVM_CUDA(cudaMemcpyAsync(&total, counts + nb, sizeof(total), cudaMemcpyDeviceToHost,
                              ctx->stream));
    TSVM_CUDA(cudaStreamSynchronize(ctx->stream));
    if ((int64_t)total >= npairs) {
      sketch_emit<<<(unsigned)nb, 256, 0, ctx->stream>>>(R2, attempts, counts, count, Q);
      TSVM_LAUNCHED(ctx);
      return TSVM_OK;
    }
    attempts_d *= 1.25;
  }
  return TSVM_ERR_SKETCH;
}

}  // namespace tsvm

// ---------------------------------------------------------------------------------------
// Counter-based Gaussian sketch (TSVM_SKETCH_PHILOX): Philox4x32-10 (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011) keyed by the 64-bit seed,
// counter (block, 0, 0, 0) for the block of four entries 4 block .. 4 block + 3 of the
// row-major n x k sketch; the four words become two Box-Muller pairs.  Every entry depends only
// on (seed, index), not on the launch shape, so any grid reproduces the same matrix.
// ---------------------------------------------------------------------------------------
namespace tsvm {
namespace {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// (0, 1): the top 24 bits of the word, centred on their cell
__device__ __forceinline__ float philox_uniform(uint32_t x) {
  return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

__global__ void __launch_bounds__(256) sketch_philox_kernel(uint64_t seed, int64_t count,
                                                            float *__restrict__ Q) {
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  const int64_t blocks = (count + 3) / 4;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < blocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    const uint4 r = philox4x32_10(make_uint4((uint32_t)b, (uint32_t)(b >> 32), 0u, 0u), key);
    float z[4];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const float u0 = philox_uniform(p == 0 ? r.x : r.z);
      const float u1 = philox_uniform(p == 0 ? r.y : r.w);
      const float rad = sqrtf(-2.0f * logf(u0));
      float s, c;
      sincospif(2.0f * u1, &s, &c);
      z[2 * p] = rad * c;
      z[2 * p + 1] = rad * s;
    }
    const int64_t e = 4 * b;
    if (e + 3 < count) {
      reinterpret_cast<float4 *>(Q)[b] = make_float4(z[0], z[1], z[2], z[3]);
    } else {
      for (int q = 0; q < 4 && e + q < count; ++q) Q[e + q] = z[q];
    }
  }
}

}  // namespace

tsvm_status sketch_philox(tsvm_context *ctx, uint64_t seed, int64_t count, float *Q) {
  if (count < 0 || !Q || (reinterpret_cast<uintptr_t>(Q) & 15) != 0)
    return TSVM_ERR_INVALID_ARGUMENT;
  if (count == 0) return TSVM_OK;
  const int64_t blocks = (count + 3) / 4;
  const unsigned grid = (unsigned)std::min<int64_t>((int64_t)ctx->num_sms * 8, (blocks + 255) / 256);
  sketch_philox_kernel<<<grid, 256, 0, ctx->stream>>>(seed, count, Q);
  TSVM_LAUNCHED(ctx);
  return TSVM_OK;
}

}  // namespace tsvm
