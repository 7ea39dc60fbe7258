// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// The reference's plain GPU evaluator (src/cleaned/cl_gpu_simple.cu:57-336:
// eval_simple_kernel, reduce_mse_kernel_simple, evaluate_gpu_simple_wrapper)
// compiled unchanged for sm_100a; see ref_gpu_run.cu for the limits its
// callers respect.
#include "cl_gpu_simple.cu"

#include "ref_pack.hpp"

#define REFG_EXPORT extern "C" __attribute__((visibility("default")))

REFG_EXPORT void *refg_simple_create() { return create_gpu_simple_context(); }
REFG_EXPORT void refg_simple_destroy(void *ctx) { destroy_gpu_simple_context(ctx); }

// One evaluate_gpu_simple_wrapper call; stats_out as refg_subtree_eval.
REFG_EXPORT void refg_simple_eval(void *ctx, int E, const int *tok, const double *val,
                                  const long long *off, int V, int N, const float *X,
                                  float *mse_out, int upload_X, double *stats_out) {
  refpack::PackedInfo p(E, tok, val, off, V, N, X);
  std::vector<float> mses;
  RunStats st;
  evaluate_gpu_simple_wrapper(p.info, p.all.data(), mses, ctx, upload_X != 0, st);
  for (int i = 0; i < E && i < static_cast<int>(mses.size()); ++i) mse_out[i] = mses[i];
  stats_out[0] = st.total_eval_time_ms;
  stats_out[1] = st.data_transfer_time_ms;
  stats_out[2] = st.gpu_kernel_time_ms;
  stats_out[3] = 0.0;
}
