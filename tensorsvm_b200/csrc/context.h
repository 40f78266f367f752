// The tsvm_context behind the C ABI: device, stream, launch counter and a slot-keyed
// device scratch arena (grown on demand, never shrunk, freed by tsvm_destroy).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "tensorsvm.h"

namespace tsvm {

enum Slot : int {
  SLOT_RAND = 0,      // sketch: raw rand() stream
  SLOT_STATES,        // sketch: per-segment generator states
  SLOT_COUNTS,        // sketch: per-block accept counts / offsets
  SLOT_JUMP,          // sketch: jump-ahead matrices
  SLOT_Q,             // factor: sketch / pass-2 output (n x kp fp32)
  SLOT_W,             // factor: pass-1 output, orthonormalised in place (n x kp fp32)
  SLOT_W2,            // factor: scratch n x kp fp32
  SLOT_OPA,           // factor: tensor-core B operand (kp x n fp16/bf16, labels folded in)
  SLOT_OPX,           // factor: tensor-core split features (n x Kg fp16)
  SLOT_XC,            // factor: centred features + norms
  SLOT_PART,          // split-n partial sums (fp64)
  SLOT_SMALL,         // k x k fp64 work (Gram, Cholesky, eigen)
  SLOT_SMALL2,
  SLOT_SMALL3,
  SLOT_IPM_VEC,       // IPM fp64 vectors
  SLOT_IPM_SCAL,      // IPM device scalars
  SLOT_IPM_M,         // IPM capacitance matrix + factor
  SLOT_SYRK_OP,       // IPM: BF16 split operand of the tensor-core SYRK
  SLOT_SYRK_PART,     // IPM: per-CTA FP32 partial Gram matrices of the tensor-core SYRK
  SLOT_SYRK_CNT,      // IPM: per-block counts of the exactly summed (large-weight) rows
  SLOT_IPM_IDX,       // IPM: indices of the exactly summed rows
  SLOT_SYRK_PLAN,     // IPM: column windows of the tensor-core SYRK for k > 256
  SLOT_IPM_PART,      // IPM / bias streaming partial sums (kept apart from SLOT_PART, which the
                      // Z^T D^-1 Z accumulation may regrow inside the iteration)
  SLOT_MISC,
  SLOT_B_VEC,         // batched IPM: concatenated fp64 vectors and labels of all problems
  SLOT_B_TABLE,       // batched IPM: work units, unit offsets, Z pointers, flags
  SLOT_B_SCAL,        // batched IPM: per-problem scalars and k-vectors
  SLOT_B_M,           // batched IPM: per-problem capacitance matrices and factors
  SLOT_B_GPART,       // batched IPM: per-unit partial Gram matrices
  SLOT_B_PART,        // batched IPM: per-unit streaming partial sums
  SLOT_B_SYRK,        // batched mixed IPM: per-unit tensor-core partials, error flag, exact-row
                      // counts, per-problem tau
  SLOT_B_IDX,         // batched mixed IPM: exactly summed rows of every unit
  SLOT_HG_OMEGA,      // hypergradient: copy of the factor's sketch
  SLOT_HG_R,          // hypergradient: combined CholeskyQR factor and k-vectors
  SLOT_HG_KPART,      // hypergradient: per-split partial kernel-vector products
  SLOT_HG_W,          // hypergradient: the factor's orthonormal basis before rounding
  SLOT_HG_Z,          // hypergradient: the factor Z it differentiates (kept or recomputed)
  SLOT_HG_TC,         // hypergradient: centred rows, FP32 operand and product of the tensor-core
                      // kernel-vector products
  SLOT_DEV_IN,        // tsvm_train: device copies of host inputs
  SLOT_DEV_Z,         // tsvm_train: factor Z
  SLOT_DEV_OUT,       // tsvm_train: device alpha
  SLOT_PRED_IN,       // tsvm_predict: device copies of the model and the rows
  SLOT_PRED_OUT,      // tsvm_predict: decision values
  SLOT_B_EIG,         // batched factor: projections C, eigenvectors, eigenvalues
  SLOT_B_FXC,         // batched factor: centred rows and row norms of every problem
  SLOT_B_FACG,        // batched factor: CholeskyQR Gram matrices / factors, Dinv blocks, status
  SLOT_B_EIGSW,       // batched factor: per-problem sweep counts
  SLOT_COMM,          // row-sharded path: staging of host values for the collectives
  SLOT_SHARD_A,       // row-sharded factor: the all-gathered kernel-block operand (all rows)
  SLOT_COUNT_
};

}  // namespace tsvm

struct tsvm_context {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the context's own stream
  // high-priority side stream (and the event that forks it off `stream`): the interior-point
  // iteration's k x k Cholesky runs there beside the next streaming pass over Z
  cudaStream_t side_stream = nullptr;
  cudaEvent_t fork_ev = nullptr;
  int64_t launches = 0;
  void *buf[tsvm::SLOT_COUNT_] = {};
  size_t bytes[tsvm::SLOT_COUNT_] = {};
  cudaEvent_t ev[8] = {};
  // sketch jump-ahead tables, keyed by the number of segments they cover
  int jump_levels = 0;
  // pinned host staging for small device->host reads
  double *host_scalars = nullptr;
  // width k whose column-window table SLOT_SYRK_PLAN holds (-1: none)
  int syrk_plan_k = -1;
  // test hook: scratch growth fails with TSVM_ERR_OUT_OF_MEMORY after this many more device
  // allocations (-1: never)
  int alloc_fail_after = -1;
  // seed of the Philox sketch (tsvm_set_sketch_seed)
  uint64_t sketch_seed = 0;
  // row-sharded solves (tsvm_set_comm): the caller's communicator
  bool has_comm = false;
  tsvm_comm comm = {};
  // tsvm_set_factor_keep: tsvm_factor keeps what tsvm_hypergrad needs of the factor (sketch,
  // CholeskyQR R, unrounded basis, Z in SLOT_HG_*), and which inputs it belongs to
  int keep_factor = 0;
  struct {
    bool valid = false;
    const float *X = nullptr, *y = nullptr;
    int64_t n = 0;
    int d = 0, k = 0, precision = 0;
    double gamma = 0.0;
  } kept;
  // the last RBF tsvm_train (its X, y in SLOT_DEV_IN and Z in SLOT_DEV_Z), for -analysis
  struct {
    bool valid = false;
    int64_t n = 0;
    int d = 0, k = 0, ldz = 0;
    double gamma = 0.0;
  } last_train;
};

namespace tsvm {

// Ensure slot `s` holds at least `bytes` bytes; returns the device pointer (or null + status).
tsvm_status scratch(tsvm_context *ctx, Slot s, size_t bytes, void **out);

template <class T>
inline tsvm_status scratch_t(tsvm_context *ctx, Slot s, size_t count, T **out) {
  void *p = nullptr;
  tsvm_status st = scratch(ctx, s, count * sizeof(T), &p);
  *out = static_cast<T *>(p);
  return st;
}

// Elapsed ms between two recorded events (synchronises on the second).
float event_ms(cudaEvent_t a, cudaEvent_t b);

// Collectives of the row-sharded path: no-ops without a communicator.  dtype 0 double,
// 1 float; op 0 sum, 1 min.
enum CommOp : int { COMM_SUM = 0, COMM_MIN = 1 };
tsvm_status comm_allreduce(tsvm_context *ctx, void *buf, int64_t count, int dtype, int op);
inline bool sharded(const tsvm_context *ctx) { return ctx->has_comm && ctx->comm.world > 1; }
// Sum of a host value over the ranks (through a device staging word).
tsvm_status comm_sum_host(tsvm_context *ctx, double *value);

}  // namespace tsvm
