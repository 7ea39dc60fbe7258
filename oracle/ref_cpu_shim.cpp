// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// Compiles the reference's CPU evaluator (src/cleaned/cl_cpu_eval.cpp) and
// subtree detection (src/utils/detect.cpp) unchanged, from where they lie in
// the reference tree (include path set by oracle/Makefile), and exposes C
// entry points so that tests/golden/make_golden.py can record their outputs
// and bench.py can time evaluate_cpu_mse as the CPU baseline.  The .cpp files
// are #included because the per-datapoint evaluator and the hash helpers are
// file-static there.
#include "cl_cpu_eval.cpp"
#include "detect.cpp"

#include <cstdint>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "ref_pack.hpp"

extern "C" {

// evaluate_single_expr (cl_cpu_eval.cpp:59-90)
float ref_eval_single(const int *tok, const double *val, int n, const float *vars, int num_vars) {
  return evaluate_single_expr(tok, val, n, vars, num_vars);
}

// evaluate_cpu_mse (cl_cpu_eval.cpp:94-168) over a column-major dataset.
double ref_eval_mse(int E, const int *tok, const double *val, const long long *off, int V, int N,
                    const float *X, float *mse_out, int threads) {
  refpack::PackedInfo p(E, tok, val, off, V, N, X);
  setenv("THREADS", std::to_string(threads).c_str(), 1);
  std::vector<float> mses;
  RunStats st;
  evaluate_cpu_mse(p.info, p.all.data(), mses, st);
  for (int i = 0; i < E; ++i) mse_out[i] = mses[i];
  return st.total_eval_time_ms;
}

// evaluate_single_expr at every datapoint, out[e * N + dp], on `threads`
// threads over contiguous expression ranges.
void ref_predict_all(int E, const int *tok, const double *val, const long long *off, int V,
                     int N, const float *X, float *out, int threads) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> th;
  for (int k = 0; k < threads; ++k) {
    th.emplace_back([=]() {
      std::vector<float> dpv(V > 0 ? V : 1);
      const int e0 = static_cast<int>(static_cast<long long>(E) * k / threads);
      const int e1 = static_cast<int>(static_cast<long long>(E) * (k + 1) / threads);
      for (int e = e0; e < e1; ++e) {
        const int n = static_cast<int>(off[e + 1] - off[e]);
        for (int dp = 0; dp < N; ++dp) {
          for (int v = 0; v < V; ++v) dpv[v] = X[static_cast<size_t>(v) * N + dp];
          out[static_cast<size_t>(e) * N + dp] =
              evaluate_single_expr(tok + off[e], val + off[e], n, dpv.data(), V);
        }
      }
    });
  }
  for (auto &t : th) t.join();
}

// compute_hash (detect.cpp:50-68)
uint64_t ref_compute_hash(const int *tok, const double *val, int len) {
  return compute_hash(tok, val, len);
}

// compute_subtree_size (detect.cpp:23-47)
int ref_subtree_size(const int *tok, int start, int total) {
  return compute_subtree_size(tok, start, total);
}

// The reverse pass of detect_common_subtrees (detect.cpp:169-191), driven
// through the reference's own simple_op_arity and hash_node.
void ref_merkle(const int *tok, const double *val, int len, int *sizes, uint64_t *hashes) {
  for (int i = len - 1; i >= 0; --i) {
    if (tok[i] <= 0) {
      sizes[i] = 1;
      hashes[i] = hash_node(tok[i], val[i], {});
      continue;
    }
    const int arity = simple_op_arity(tok[i]);
    int size = 1, pos = i + 1;
    std::vector<uint64_t> ch;
    for (int k = 0; k < arity; ++k) {
      if (pos >= len) break;
      size += sizes[pos];
      ch.push_back(hashes[pos]);
      pos += sizes[pos];
    }
    sizes[i] = size;
    hashes[i] = hash_node(tok[i], val[i], ch);
  }
}

// detect_common_subtrees (detect.cpp:120-387).  Returns the group count;
// per group (up to max_groups): size, occurrences, flat key of its tokens.
// hints_out receives expr_sub_hints flattened (one entry per token).
int ref_detect(int E, const int *tok, const double *val, const long long *off, int min_size,
               int min_freq, int max_groups, int *g_size, int *g_count, uint64_t *g_key,
               int *hints_out, double *avg_size, double *coverage, long long *covered) {
  std::vector<int> nt(E);
  std::vector<const int *> tp(E);
  std::vector<const double *> vp(E);
  for (int i = 0; i < E; ++i) {
    nt[i] = static_cast<int>(off[i + 1] - off[i]);
    tp[i] = tok + off[i];
    vp[i] = val + off[i];
  }
  SubtreeDetectionResult r =
      detect_common_subtrees(E, 0, nt.data(), tp.data(), vp.data(), min_size, min_freq);
  const int n = r.num_subs;
  for (int g = 0; g < n && g < max_groups; ++g) {
    g_size[g] = r.num_sub_tokens[g];
    g_count[g] = r.num_occurrences[g];
    g_key[g] = compute_hash(r.sub_tokens[g], r.sub_values[g], r.num_sub_tokens[g]);
  }
  if (hints_out)
    for (int i = 0; i < E; ++i)
      for (int k = 0; k < nt[i]; ++k) hints_out[off[i] + k] = r.expr_sub_hints[i][k];
  *avg_size = r.avg_subtree_size;
  *coverage = r.coverage_ratio;
  *covered = r.total_covered_tokens;
  free_subtree_detection_result(r);
  return n;
}

}  // extern "C"
