// ORACLE — test infrastructure only (see oracle/sr_oracle.c).
//
// Packs a CSR population (tokens, values, int64 offsets) and a column-major
// dataset into the reference's InputInfo / all_vars arguments
// (src/utils/utils.h:25-47; the layout cl_sr_system.cpp:172-202 builds), for
// the shims that call the reference's evaluators compiled unchanged.
// Include after the reference header that defines InputInfo.
#pragma once
#include <cstdint>
#include <vector>

namespace refpack {

struct PackedInfo {
  InputInfo info{};
  std::vector<int> nv, nd, nt;
  std::vector<int *> tp;
  std::vector<double *> vp;
  std::vector<float *> rows;
  std::vector<float **> all;
  PackedInfo(int E, const int *tok, const double *val, const long long *off, int V, int N,
             const float *X) {
    nv.assign(E, V);
    nd.assign(E, N);
    nt.resize(E);
    tp.resize(E);
    vp.resize(E);
    for (int i = 0; i < E; ++i) {
      nt[i] = static_cast<int>(off[i + 1] - off[i]);
      tp[i] = const_cast<int *>(tok + off[i]);
      vp[i] = const_cast<double *>(val + off[i]);
    }
    info.num_exprs = E;
    info.num_vars = nv.data();
    info.num_dps = nd.data();
    info.num_tokens = nt.data();
    info.tokens = tp.data();
    info.values = vp.data();
    info.data_filenames = nullptr;
    info.tokens_packed = nullptr;
    info.values_packed_f32 = nullptr;
    info.X_packed_f32 = nullptr;
    info.has_shared_data = true;
    rows.resize(V + 1);
    for (int v = 0; v <= V; ++v)
      rows[v] = const_cast<float *>(X) + static_cast<size_t>(v) * static_cast<size_t>(N);
    all.assign(E > 0 ? E : 1, rows.data());
  }
};

}  // namespace refpack
