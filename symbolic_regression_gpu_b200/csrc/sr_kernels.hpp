// sr_kernels.hpp — host-callable launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "sr_internal.hpp"

namespace sr {

constexpr int kMaxWarps = 16;                       // evaluating warps per block
constexpr int kMaxBlockThreads = (kMaxWarps + 1) * 32;  // + producer warp
// Evaluating warps per block of an MSE interpreter launch at 8 datapoints per
// thread: 31 + the producer warp = 1,024 threads, one block per SM.
constexpr int kMaxInterpWarps = 31;
constexpr int64_t kDataAlign = 4096;               // X / cache row stride multiple
constexpr int kPlainStack = 128;                    // plain kernel stack depth
constexpr int kFp64Stack = 96;                      // FP64 reference kernel stack depth

// Dynamic shared memory of interp_kernel for a launch shape.
size_t interp_smem_bytes(int dpt, int W, int V, int s_smem, int span, int G, bool pred);
// Spill slots per warp kept in shared memory for a datapoints-per-thread
// choice (deeper slots go to global scratch).
inline int smem_spill_slots(int dpt) { return dpt >= 16 ? 2 : (dpt == 8 ? 4 : 8); }
// Raises fn's maximum dynamic shared memory to at least `smem` bytes (never
// lowers it): a kernel launched by several prepared sequences with different
// shared-memory sizes keeps a limit that admits every launch already
// captured, however they are replayed.
cudaError_t raise_smem_limit(const void *fn, size_t smem);
// Sets the dynamic-smem attribute and returns resident blocks per SM.
// `ops` is the operator profile (kOpsAll / kOpsProtected) and `cache` whether
// the programs read cached subtrees (MSE mode only; prediction launches use
// kOpsAll without cached operands).
cudaError_t interp_configure(int dpt, bool pred, int ops, bool cache, size_t smem, int W,
                             int *blocks_per_sm);
cudaError_t launch_interp(int dpt, bool pred, int ops, bool cache, const EvalArgs &args,
                          int blocks, size_t smem, cudaStream_t stream);
cudaError_t launch_finalize(const double2 *partial, int n_spans, int E,
                            float *mse, cudaStream_t stream);
// The interpreter's MSE entries ([n_groups][E] x 2 double2 per span group,
// see EvalArgs::span_per_item): mse = sum / count (NaN without a valid
// datapoint) into `mse`, and (sum, count) into `sums`; either may be NULL.
cudaError_t launch_finalize_groups(const double2 *partial, int n_groups, int E, float *mse,
                                   double2 *sums, cudaStream_t stream);
// (sum of valid squared errors, valid count) per expression, combined over
// the span partials in the order launch_finalize uses (plain and gradient
// launches).
cudaError_t launch_sums(const double2 *partial, int n_spans, int E, double2 *sums,
                        cudaStream_t stream);
cudaError_t launch_plain(const int32_t *tok, const float *val, const int64_t *off,
                         const int32_t *len, const float *X, int64_t ldx, int V,
                         int64_t N, int E, double2 *partial, int n_dpblocks,
                         cudaStream_t stream);
// FP64 evaluation of the plain set (accuracy report): mse64[e] in double.
cudaError_t launch_fp64(const int32_t *tok, const float *val, const int64_t *off,
                       const int32_t *len, const float *X, int64_t ldx, int V, int64_t N, int E,
                       double2 *partial, int n_dpblocks, double *mse64, cudaStream_t stream);
// Operator-throughput microbenchmark (op_rate_kernel<op>); op 0 times the
// harness alone.  cudaErrorInvalidValue for an opcode without an instance.
cudaError_t launch_op_rate(int op, float *out, int blocks, int threads, int iters,
                           cudaStream_t stream);
cudaError_t launch_pipe_bench(bool mufu, float *out, int blocks, int threads,
                              int iters, cudaStream_t stream);

}  // namespace sr
