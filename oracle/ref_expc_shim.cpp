// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// The reference's CPU evaluator with ONE added case: opcode 32, exp clamped
// at 80 (expf(fminf(x, 80))), the unary operator the evolution workloads use
// and the reference does not have.  oracle/Makefile copies
// src/cleaned/cl_cpu_eval.cpp from the reference tree into oracle/_ref/
// (never into the repository) and inserts that single `case` line into
// eval_op_cpu (cl_cpu_eval.cpp:16-56), after the OP_LOOSE_SQRT case; every
// other line, the right-to-left evaluation (:59-90) and the MSE rule
// (:94-168) are the reference's own.  This is the parity oracle for
// populations that contain opcode 32.
//
// Built as its own library with hidden visibility, so that its copy of
// evaluate_cpu_mse never interposes on (or is interposed by) the unchanged
// one in libref_oracle.so or this project's library.
#include "cl_cpu_eval_expc.cpp"

#include <cstdint>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "ref_pack.hpp"

#define REFX_EXPORT extern "C" __attribute__((visibility("default")))

// evaluate_single_expr (cl_cpu_eval.cpp:59-90) with the added case.
REFX_EXPORT float refx_eval_single(const int *tok, const double *val, int n, const float *vars,
                                   int num_vars) {
  return evaluate_single_expr(tok, val, n, vars, num_vars);
}

// evaluate_cpu_mse (cl_cpu_eval.cpp:94-168) over a column-major dataset.
REFX_EXPORT double refx_eval_mse(int E, const int *tok, const double *val, const long long *off,
                                 int V, int N, const float *X, float *mse_out, int threads) {
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
REFX_EXPORT void refx_predict(int E, const int *tok, const double *val, const long long *off,
                              int V, int N, const float *X, float *out, int threads) {
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
