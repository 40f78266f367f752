// Shared helpers for the tensorsvm B200 kernels: status plumbing, launch accounting,
// warp/block reductions and a bounded grid barrier.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "tensorsvm.h"

namespace tsvm {

// ---------------------------------------------------------------------------------------
// Error plumbing: every internal routine returns tsvm_status; no exit().
// ---------------------------------------------------------------------------------------
tsvm_status cuda_status(cudaError_t e, const char *what, const char *file, int line);
// TSVM_ERR_TIMEOUT, naming the wait that gave up on stderr when TSVM_DEBUG is set.
tsvm_status timeout_status(const char *where);

#define TSVM_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return ::tsvm::cuda_status(e_, #call, __FILE__, __LINE__);     \
  } while (0)

#define TSVM_TRY(expr)                                                                    \
  do {                                                                                    \
    tsvm_status s_ = (expr);                                                              \
    if (s_ != TSVM_OK) return s_;                                                         \
  } while (0)

// Check the last launch and count it (the launch counter backs tsvm_kernel_launches()).
#define TSVM_LAUNCHED(ctx)                                                                \
  do {                                                                                    \
    (ctx)->launches++;                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) return ::tsvm::cuda_status(e_, "kernel launch", __FILE__, __LINE__); \
  } while (0)

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
static inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// ---------------------------------------------------------------------------------------
// Device reductions (FP64), deterministic: fixed shuffle trees, fixed block order.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum of NV doubles per thread; result valid in thread 0. `sh` needs
// NV * (blockDim.x/32) doubles.  Ends with a __syncthreads so `sh` can be reused.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) sh[i * nw + warp] = v[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sh[i * nw + w];
      v[i] = s;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------
// Grid barrier for cooperative launches.  Every wait is bounded: after `max_spins` polls
// the waiting block records an error flag and the barrier returns false; callers then
// leave the kernel, so no launch can hang the device.
// ---------------------------------------------------------------------------------------
struct GridBarrier {
  unsigned int count;
  unsigned int generation;
  int error;
  int pad;
};

__device__ __forceinline__ bool grid_sync(GridBarrier *gb, unsigned int nblocks,
                                          long long max_spins = (1ll << 24)) {
  __syncthreads();
  __shared__ int ok_sh;
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned int *gen = &gb->generation;
    unsigned int g = *gen;
    __threadfence();
    if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
      gb->count = 0;
      __threadfence();
      atomicAdd(&gb->generation, 1u);
    } else {
      long long spins = 0;
      while (*gen == g) {
        if (++spins > max_spins || *((volatile int *)&gb->error)) {
          atomicExch(&gb->error, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (*((volatile int *)&gb->error)) ok = 0;
    ok_sh = ok;
  }
  __syncthreads();
  return ok_sh != 0;
}

}  // namespace tsvm
