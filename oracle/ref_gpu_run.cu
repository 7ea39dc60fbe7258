// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// The reference's own GPU evaluators, compiled unchanged for sm_100a from
// where they lie in the reference tree, as a same-GPU comparison point for
// the bench: the subtree-cache path evaluate_gpu_mse_wrapper
// (src/cleaned/cl_gpu_eval.cu:332-592: eval_subtrees_kernel,
// eval_skeletons_kernel, reduce_mse_kernel) in this file and the plain path
// evaluate_gpu_simple_wrapper (src/cleaned/cl_gpu_simple.cu:187-336) in
// ref_gpu_run_simple.cu.  Built into its own library with hidden
// visibility (the project's library exports the same C++ entry points).
//
// The reference kernels index with int32 (expr_idx * total_dps,
// cache_idx * total_dps): callers run them only on expression chunks with
// E_chunk * N < 2^31, N < 1,048,576 for the cache path, and populations
// whose variable indices are below the variable count and whose stack depth
// stays within MAX_STACK_SIZE (60); oracle/ref_gpu.py checks all of that
// before any call.
#include "cl_gpu_eval.cu"

#include "ref_pack.hpp"

#define REFG_EXPORT extern "C" __attribute__((visibility("default")))

REFG_EXPORT void *refg_subtree_create() { return create_gpu_context(); }
REFG_EXPORT void refg_subtree_destroy(void *ctx) { destroy_gpu_context(ctx); }

// One evaluate_gpu_mse_wrapper call.  stats_out: total ms (the wrapper's wall
// clock), transfer ms, kernel ms (the reference's own event timings),
// detection ms.
REFG_EXPORT void refg_subtree_eval(void *ctx, int E, const int *tok, const double *val,
                                   const long long *off, int V, int N, const float *X,
                                   float *mse_out, int upload_X, int clear_cache,
                                   double *stats_out) {
  refpack::PackedInfo p(E, tok, val, off, V, N, X);
  std::vector<float> mses;
  RunStats st;
  evaluate_gpu_mse_wrapper(p.info, p.all.data(), mses, ctx, upload_X != 0, clear_cache != 0, st);
  for (int i = 0; i < E && i < static_cast<int>(mses.size()); ++i) mse_out[i] = mses[i];
  stats_out[0] = st.total_eval_time_ms;
  stats_out[1] = st.data_transfer_time_ms;
  stats_out[2] = st.gpu_kernel_time_ms;
  stats_out[3] = st.drift_detect_time_ms;
}
