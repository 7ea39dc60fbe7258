// sr_adjoint.hpp — launchers of the forward+adjoint kernel, the gradient
// finalize kernel and the on-device Adam step (sr_adjoint.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "sr_internal.hpp"
#include "sr_kernels.hpp"

namespace sr {

struct AdjArgs {
  EvalArgs e;                 // forward part (dataset, programs, groups, spans, MSE partials)
  const int64_t *const_off;   // [E] first constant (global index) of each expression
  const int32_t *const_cnt;   // [E] constants of each expression
  const int32_t *bwd_lo;      // [E] lowest instruction holding a constant (code_len: none)
  double *grad_acc;           // [C] FP64 gradient sums, zeroed before the launch
  float *gtape;               // per-warp tapes in global memory, or null (shared memory)
  int32_t tape_len;           // tape entries per warp (>= the tape of any program)
  int32_t gmax;               // gradient accumulators per warp (>= constants of any program)
  int32_t seg_cap;            // recompute mode: segment-tape entries (min(segment, longest))
  int32_t reserved0;
};

// Forward-mode (tangent) launch: the expressions with at most
// kMaxTangentConsts constants.  Per instruction one mask word: bits 0..7 A
// (constants under the accumulator before the operator), 8..15 B (constants
// under the operand b), bit 24 set when the instruction loads a constant leaf
// (its bit in A).
constexpr int kMaxTangentConsts = 8;
constexpr uint32_t kTanLoadConst = 1u << 24;

struct TanArgs {
  EvalArgs e;                 // forward part (dataset, programs, group table, spans, MSE sums)
  const uint32_t *tmask;      // [instructions + 1] mask words, aligned with the code
  const int64_t *const_off;   // [E] first constant (global index) of each expression
  const int32_t *const_cnt;   // [E] constants of each expression
  double *gout;               // [span groups][C] gradient sums per span group
  int64_t C;                  // constants of the population
  int32_t n_valid;            // expressions in the group table
  int32_t K;                  // tangent rows per warp (>= the constants of any expression)
};

int tan_dpt();         // datapoints per thread
int tan_warps(int K);  // evaluating warps per block (at most) for K tangent rows
size_t tan_smem_bytes(int K, int W, int V, int s_smem, int span, int G);
cudaError_t tan_configure(int K, size_t smem, int W, int *blocks_per_sm);
// The launchers below leave the kernels' maximum dynamic shared memory as it
// is: a launch sequence raises it first to the largest size any of its
// launches of that kernel needs (tan_set_smem_limit / adj_set_smem_limit;
// limits only ever grow, raise_smem_limit), so every launch of a captured
// sequence is valid on its own.
cudaError_t tan_set_smem_limit(int K, size_t smem);
cudaError_t launch_tangent(const TanArgs &args, int blocks, size_t smem, cudaStream_t stream);
cudaError_t launch_tan_finalize(const double2 *partial, const double *gout, int n_groups, int E,
                                int64_t C, const int32_t *exprs, int n_exprs,
                                const int64_t *const_off, const int32_t *const_cnt, int K,
                                float *mse, float *grad, double *gsum, double2 *sums,
                                cudaStream_t stream);

// Datapoints per thread of the adjoint kernel.
int adj_dpt();
size_t adj_smem_bytes(int W, int V, int s_smem, int span, int tape_len, int gmax,
                      bool global_tape);
// Instructions per recompute segment.
int adj_segment();
cudaError_t adj_configure(size_t smem, int W, bool global_tape, bool recompute,
                          int *blocks_per_sm);
cudaError_t adj_set_smem_limit(bool global_tape, bool recompute, size_t smem);
cudaError_t launch_adjoint(const AdjArgs &args, bool recompute, int blocks, size_t smem,
                           cudaStream_t stream);
// mse / grad (and the (sum, count) sums) of the n_exprs reverse-mode
// expressions listed in exprs.
cudaError_t launch_grad_finalize(const double2 *partial, int n_spans, int E,
                                 const int32_t *exprs, int n_exprs, const int64_t *const_off,
                                 const int32_t *const_cnt, const double *grad_acc, float *mse,
                                 float *grad, double2 *sums, cudaStream_t stream);
cudaError_t launch_adam(int64_t C, const float *grad, float *m, float *v, float *consts,
                        const int64_t *loc, Instr *code, int step, float lr, float beta1,
                        float beta2, float eps, cudaStream_t stream);

}  // namespace sr
