// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// Compiles the reference's subtree-cache evaluator (src/cleaned/cl_gpu_eval.cu)
// unchanged and exposes its file-static host helpers: the flat cache key and
// the cache marking of evaluate_gpu_mse.  Only host code is called; nothing
// here launches a kernel.
#include "cl_gpu_eval.cu"

#include <cstdint>
#include <vector>

extern "C" {

// compute_subtree_hash_gpu (cl_gpu_eval.cu:259-272)
uint64_t ref_subtree_hash_gpu(const int *tok, const double *val, int len) {
  return compute_subtree_hash_gpu(tok, val, len);
}

// compute_subtree_size_state (cl_gpu_eval.cu:279-292)
int ref_subtree_size_state(const int *tok, int start, int total) {
  return compute_subtree_size_state(tok, start, total);
}

// mark_cached_subtrees_from_state (cl_gpu_eval.cu:294-329) with a cache map
// holding keys[k] -> slots[k]; hints_out gets one entry per token.
void ref_mark_cached(int E, const int *tok, const double *val, const long long *off,
                     const uint64_t *keys, const int *slots, int n_keys, int *hints_out) {
  std::vector<int> nt(E);
  std::vector<int *> tp(E);
  std::vector<double *> vp(E);
  for (int i = 0; i < E; ++i) {
    nt[i] = static_cast<int>(off[i + 1] - off[i]);
    tp[i] = const_cast<int *>(tok + off[i]);
    vp[i] = const_cast<double *>(val + off[i]);
  }
  InputInfo info{};
  info.num_exprs = E;
  info.num_tokens = nt.data();
  info.tokens = tp.data();
  info.values = vp.data();
  GPUSubtreeStateContext ctx;  // host map only; no device buffer is touched
  for (int k = 0; k < n_keys; ++k) ctx.hash_to_idx[keys[k]] = slots[k];
  SubtreeDetectionResult result{};
  result.num_exprs = E;
  result.expr_sub_hints = new int *[E];
  for (int i = 0; i < E; ++i) result.expr_sub_hints[i] = new int[nt[i] > 0 ? nt[i] : 1];
  mark_cached_subtrees_from_state(info, ctx, result);
  for (int i = 0; i < E; ++i) {
    for (int k = 0; k < nt[i]; ++k) hints_out[off[i] + k] = result.expr_sub_hints[i][k];
    delete[] result.expr_sub_hints[i];
  }
  delete[] result.expr_sub_hints;
}

}  // extern "C"
