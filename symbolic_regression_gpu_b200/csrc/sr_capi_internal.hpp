// sr_capi_internal.hpp — helpers shared by the translation units of the C ABI:
// sr_capi.cpp (context, dataset, forward prepare / launch / read-back),
// sr_capi_grad.cpp (fused forward + adjoint, Adam) and sr_capi_tools.cpp (FP64
// reference, device generation loop, microbenchmarks, detection and host-only
// helpers).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "sr_context.hpp"
#include "sr_kernels.hpp"

namespace sr {
namespace capi {

double now_ms();
// Milliseconds between two events, 0 when either was never recorded.
float elapsed_ms(cudaEvent_t a, cudaEvent_t b);
// Records a CUDA failure on ctx (and clears a non-sticky error); returns its status.
sr_status cuda_fail(sr_context *ctx, cudaError_t e, const char *what);

// Makes ctx->device current for the scope of an API call.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

int host_threads(const sr_context *ctx);
int64_t round_up(int64_t a, int64_t b);
sr_status check_population(sr_context *ctx, const sr_population *pop);
sr_status compile_set(sr_context *ctx, int E, const int32_t *tok, const double *val,
                      const int64_t *off, const int32_t *hints, ProgramSet &ps);
// Operator profile of a compiled set (evaluation launches).
bool protected_profile(const ProgramSet &ps);
// Launch shape: groups of G cost-sorted expressions x spans of datapoints.
// `split`: spill slots per warp kept in shared memory (-1 = the default for
// the dpt); `per_warp`: expressions per group and evaluating warp.
sr_status plan_set(sr_context *ctx, ProgramSet &ps, bool pred, int dpt, int W, int split = -1,
                   int per_warp = 4, int span_target = 1024);
sr_status upload_groups(sr_context *ctx, ProgramSet &ps);
sr_status upload_code(sr_context *ctx, ProgramSet &ps);
EvalArgs make_args(sr_context *ctx, ProgramSet &ps, int32_t *counter);
sr_status launch_set(sr_context *ctx, ProgramSet &ps, bool pred, int32_t *counter,
                     float *pred_out, int64_t ldp, const int32_t *pred_row);
sr_status prepare_main_shape(sr_context *ctx, bool allow_tune);
cudaError_t record_event(sr_context *ctx, int k);
void reset_prepared(sr_context *ctx);
void invalidate_data(sr_context *ctx);
sr_status check_device_error(sr_context *ctx);
void fill_stats(sr_context *ctx, sr_stats *st);
sr_status prepare_plain(sr_context *ctx, const sr_population *pop);
sr_status detect_on_device(sr_context *ctx, int E, const int32_t *tok, const double *val,
                           const int64_t *off, int min_size, int min_freq, Detection &out);
sr_status prepare_grad(sr_context *ctx, const sr_population *pop, bool recompute,
                       bool reverse_only);
sr_status launch_grad(sr_context *ctx);
int grad_launch_count(const sr::GradSet &g);

}  // namespace capi
}  // namespace sr

#define SR_TRY_CUDA(ctx, call)                                         \
  do {                                                                 \
    const cudaError_t e_ = (call);                                     \
    if (e_ != cudaSuccess) return sr::capi::cuda_fail(ctx, e_, #call); \
  } while (0)

#define SR_TRY(call)                  \
  do {                                \
    const sr_status s_ = (call);      \
    if (s_ != SR_OK) return s_;       \
  } while (0)
