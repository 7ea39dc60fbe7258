// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// Compiles the reference's expression generator and GP operators
// (src/utils/utils.cpp:955-1273: generate_random_expression,
// mutate_expression, crossover_expressions and the file-static subtree_size)
// and its file readers (load_data_file, parse_input_info) unchanged, from
// where they lie in the reference tree, and exposes C entry points so that
// tests/test_evolve_cpu.py can compare the device-side generation loop's
// restatement (oracle/evolve.py) with the reference's own operators and
// tests/test_io.py the parallel loaders with the reference's readers.
// utils.cpp is #included because subtree_size is file-static.
#include "utils.cpp"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {
EvolutionParams gp_params(int num_vars, int max_tokens, int max_depth) {
  EvolutionParams p;
  p.num_vars = num_vars;
  p.max_tokens = max_tokens;
  p.max_depth = max_depth;
  return p;
}
int copy_out(const std::vector<int> &t, const std::vector<float> &v, int *tok, float *val,
             int cap) {
  const int n = static_cast<int>(t.size());
  for (int i = 0; i < std::min(n, cap); ++i) {
    tok[i] = t[i];
    val[i] = v[i];
  }
  return n;
}
}  // namespace

extern "C" {

void ref_gp_seed(int seed) { set_seed(seed); }

// generate_random_expression (utils.cpp:1156-1161); returns the length.
int ref_gp_generate(int num_vars, int max_tokens, int max_depth, int *tok, float *val, int cap) {
  std::vector<int> t;
  std::vector<float> v;
  generate_random_expression(gp_params(num_vars, max_tokens, max_depth), t, v);
  return copy_out(t, v, tok, val, cap);
}

// mutate_expression (utils.cpp:1163-1204).
int ref_gp_mutate(int num_vars, int max_tokens, int max_depth, const int *ptok, const float *pval,
                  int plen, int *tok, float *val, int cap) {
  std::vector<int> pt(ptok, ptok + plen), t;
  std::vector<float> pv(pval, pval + plen), v;
  mutate_expression(gp_params(num_vars, max_tokens, max_depth), pt, pv, t, v);
  return copy_out(t, v, tok, val, cap);
}

// crossover_expressions (utils.cpp:1206-1273).
int ref_gp_crossover(int num_vars, int max_tokens, int max_depth, const int *atok,
                     const float *aval, int alen, const int *btok, const float *bval, int blen,
                     int *tok, float *val, int cap) {
  std::vector<int> at(atok, atok + alen), bt(btok, btok + blen), t;
  std::vector<float> av(aval, aval + alen), bv(bval, bval + blen), v;
  crossover_expressions(gp_params(num_vars, max_tokens, max_depth), at, av, bt, bv, t, v);
  return copy_out(t, v, tok, val, cap);
}

// load_data_file (utils.cpp:235-300): out[v * num_dps + j] = value j of column v.
void ref_load_data(const char *path, int num_vars, int num_dps, double *out) {
  double **v = load_data_file(path, num_vars, num_dps);
  for (int i = 0; i <= num_vars; ++i) {
    std::memcpy(out + static_cast<size_t>(i) * num_dps, v[i], sizeof(double) * num_dps);
    free(v[i]);
  }
  free(v);
}

// parse_input_info (utils.cpp:122-233).  With tokens == NULL: sizes only.
int ref_parse_gen(const char *path, int *num_exprs, long long *num_tokens, int *tokens,
                  double *values, long long *offsets, int *num_vars, int *num_dps) {
  InputInfo info = parse_input_info(path);
  *num_exprs = info.num_exprs;
  long long total = 0;
  for (int i = 0; i < info.num_exprs; ++i) total += info.num_tokens[i];
  *num_tokens = total;
  if (tokens) {
    long long o = 0;
    for (int i = 0; i < info.num_exprs; ++i) {
      offsets[i] = o;
      num_vars[i] = info.num_vars[i];
      num_dps[i] = info.num_dps[i];
      for (int k = 0; k < info.num_tokens[i]; ++k) {
        tokens[o + k] = info.tokens[i][k];
        values[o + k] = info.values[i][k];
      }
      o += info.num_tokens[i];
    }
    offsets[info.num_exprs] = o;
  }
  if (info.num_exprs > 0) free_input_info(info);
  return 0;
}

// The file-static subtree_size (utils.cpp:1110-1129).
int ref_gp_subtree_size(const int *tok, int len, int start) {
  std::vector<int> t(tok, tok + len);
  return subtree_size(t, start);
}

}  // extern "C"
