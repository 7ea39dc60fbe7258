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

// Datapoints per thread of the adjoint kernel.
int adj_dpt();
size_t adj_smem_bytes(int W, int V, int s_smem, int span, int tape_len, int gmax,
                      bool global_tape);
// Instructions per recompute segment.
int adj_segment();
cudaError_t adj_configure(size_t smem, int W, bool global_tape, bool recompute,
                          int *blocks_per_sm);
cudaError_t launch_adjoint(const AdjArgs &args, bool recompute, int blocks, size_t smem,
                           cudaStream_t stream);
cudaError_t launch_grad_finalize(const double2 *partial, int n_spans, int E,
                                 const int64_t *const_off, const int32_t *const_cnt,
                                 const double *grad_acc, float *mse, float *grad,
                                 cudaStream_t stream);
cudaError_t launch_adam(int64_t C, const float *grad, float *m, float *v, float *consts,
                        const int64_t *loc, Instr *code, int step, float lr, float beta1,
                        float beta2, float eps, cudaStream_t stream);

}  // namespace sr
