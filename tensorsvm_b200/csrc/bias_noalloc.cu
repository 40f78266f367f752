// Allocation-free variant of the RBF bias computation (tsvm_bias_noalloc).
//
// Why it exists: some callers cannot let a library call cudaMalloc -- a serving process whose
// device memory is carved up in advance by its own pool, a host framework that forbids
// allocations from plug-ins, or a caller that has already committed all of HBM and would see
// the allocation fail.  tsvm_bias (bias_rbf in ipm.cu) keeps its split-n partial sums in
// scratch owned by a tsvm_context, which is allocated on demand.  This variant keeps that
// scratch in a fixed file-scope __device__ array instead, so a call allocates nothing: the
// caller passes the inputs and a 4-double device output buffer, plus the stream to use.
//
// Limits and sharing rules:
//   * k <= kNoAllocMaxK (1024); larger k is rejected with TSVM_ERR_INVALID_ARGUMENT.
//   * The array (about 2.4 MB) exists once per device that loads this library and stays
//     resident until the process exits.
//   * The host needs the array's device address, which is not the address of the host-side
//     symbol: the first call on each device looks it up with cudaGetSymbolAddress (with that
//     device current) and caches it.  Make that first call before any stream capture.
//   * Every call uses the same array and it keeps the previous call's contents; everything a
//     call reads from it is written earlier in the same call.  Two calls whose kernels overlap
//     on the GPU (for example on two streams without ordering) race on the array.
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "tensorsvm.h"

namespace {

constexpr int kNoAllocMaxK = 1024;    // largest factor width accepted
constexpr int kNoAllocBlocks = 296;   // fixed split of the rows (2 blocks per B200 SM)
constexpr int kNoAllocThreads = 256;
constexpr int kMaxFree = 50;          // first <= 50 free SVs, as the reference's bias

// [block][0..kNoAllocMaxK): partial sum_i alpha_i Z_i over the block's rows (alpha > 1e-6)
// [block][kNoAllocMaxK], [block][kNoAllocMaxK+1]: partial SV / free-SV counts
constexpr size_t kPartStride = kNoAllocMaxK + 8;
constexpr size_t kScratchDoubles = (size_t)kNoAllocBlocks * kPartStride;

static __device__ __align__(256) double g_bias_scratch[kScratchDoubles];

__global__ void __launch_bounds__(kNoAllocThreads)
noalloc_bias_partial(const float *__restrict__ Z, int64_t ldz, int k, int64_t n,
                     const double *__restrict__ alpha, double C, double *__restrict__ scratch) {
  const int64_t rows = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * rows;
  const int64_t r1 = min(n, r0 + rows);
  double acc[kNoAllocMaxK / kNoAllocThreads];
#pragma unroll
  for (int q = 0; q < kNoAllocMaxK / kNoAllocThreads; ++q) acc[q] = 0.0;
  double nsv = 0.0, nfree = 0.0;
  for (int64_t i = r0; i < r1; ++i) {
    const double a = alpha[i];
    if (!(a > 1e-6)) continue;
    if (threadIdx.x == 0) {
      nsv += 1.0;
      if (a < C - 1e-6) nfree += 1.0;
    }
#pragma unroll
    for (int q = 0; q < kNoAllocMaxK / kNoAllocThreads; ++q) {
      const int c = threadIdx.x + q * kNoAllocThreads;
      if (c < k) acc[q] += a * (double)Z[i * ldz + c];
    }
  }
  double *part = scratch + (size_t)blockIdx.x * kPartStride;
#pragma unroll
  for (int q = 0; q < kNoAllocMaxK / kNoAllocThreads; ++q) {
    const int c = threadIdx.x + q * kNoAllocThreads;
    if (c < k) part[c] = acc[q];
  }
  if (threadIdx.x == 0) {
    part[kNoAllocMaxK] = nsv;
    part[kNoAllocMaxK + 1] = nfree;
  }
}

// One block: reduce the partials in block order into v (kept in shared memory), find the
// first <= 50 free SVs in index order, then b_j = y_j - y_j (v . Z_j); out = {mean, std, nsv,
// nfree}.  Mean and std are NaN when there is no free SV.
__global__ void __launch_bounds__(1024)
noalloc_bias_final(const float *__restrict__ Z, int64_t ldz, int k, int64_t n,
                   const float *__restrict__ y, const double *__restrict__ alpha, double C,
                   const double *__restrict__ scratch, double *__restrict__ out) {
  __shared__ double v[kNoAllocMaxK];
  __shared__ double bj[kMaxFree];
  __shared__ int64_t idx[kMaxFree];
  __shared__ int wcnt[32];
  __shared__ double counts[2];
  for (int c = threadIdx.x; c < k; c += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < kNoAllocBlocks; ++b) s += scratch[(size_t)b * kPartStride + c];
    v[c] = s;
  }
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int b = 0; b < kNoAllocBlocks; ++b)
      s += scratch[(size_t)b * kPartStride + kNoAllocMaxK + threadIdx.x];
    counts[threadIdx.x] = s;
  }
  // Every thread keeps its own copy of the running count of free SVs, updated from the same
  // per-warp counts after the same barrier, so the loop-top test is uniform over the block.
  int found = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t base = 0; base < n && found < kMaxFree; base += blockDim.x) {
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
    if (f && off < kMaxFree) idx[off] = i;
    found += tot;
    __syncthreads();  // wcnt is rewritten by the next round; idx is read after the loop
  }
  const int m = found < kMaxFree ? found : kMaxFree;
  for (int t = warp; t < m; t += nw) {
    const int64_t j = idx[t];
    double s = 0.0;
    for (int c = lane; c < k; c += 32) s += v[c] * (double)Z[j * ldz + c];
    s = tsvm::warp_sum(s);
    if (lane == 0) bj[t] = (double)y[j] - (double)y[j] * s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mean = NAN, sd = NAN;
    if (m > 0) {
      mean = 0.0;
      for (int t = 0; t < m; ++t) mean += bj[t];
      mean /= m;
      double ss = 0.0;
      for (int t = 0; t < m; ++t) ss += (bj[t] - mean) * (bj[t] - mean);
      sd = sqrt(ss / m);
    }
    out[0] = mean;
    out[1] = sd;
    out[2] = counts[0];
    out[3] = counts[1];
  }
}

// Device address of g_bias_scratch, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
double *g_addr[kMaxDevices] = {};

tsvm_status scratch_address(int device, double **out) {
  if (device < 0 || device >= kMaxDevices) return TSVM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[device]) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_bias_scratch);
    if (e != cudaSuccess || p == nullptr) return TSVM_ERR_CUDA;
    g_addr[device] = p;
  }
  *out = g_addr[device];
  return TSVM_OK;
}

}  // namespace

extern "C" tsvm_status tsvm_bias_noalloc(const float *Z, int32_t ldz, const float *y,
                                         const double *alpha, int64_t n, int32_t k, double C,
                                         double *out, void *stream) {
  if (!Z || !y || !alpha || !out || n < 1 || k < 1 || ldz < k) return TSVM_ERR_INVALID_ARGUMENT;
  if (k > kNoAllocMaxK) return TSVM_ERR_INVALID_ARGUMENT;  // beyond the static scratch capacity
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return TSVM_ERR_NO_DEVICE;
  double *scratch = nullptr;
  const tsvm_status st = scratch_address(device, &scratch);
  if (st != TSVM_OK) return st;
  // An error left by an earlier, unrelated launch of the caller is not this call's failure:
  // clear it so that the check after the launches reports only these two kernels.
  (void)cudaGetLastError();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  noalloc_bias_partial<<<kNoAllocBlocks, kNoAllocThreads, 0, s>>>(Z, ldz, k, n, alpha, C,
                                                                   scratch);
  noalloc_bias_final<<<1, 1024, 0, s>>>(Z, ldz, k, n, y, alpha, C, scratch, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return TSVM_ERR_CUDA;
  return TSVM_OK;
}
