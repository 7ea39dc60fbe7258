// sr_evolve.hpp — launchers of the device-side evolution step and of the
// device-side bytecode compiler (sr_evolve.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "sr_internal.hpp"

namespace sr {

// Parameters of the random-expression generator and the breeding step
// (reference EvolutionParams, src/utils/utils.h:178-187, and the loop
// constants of src/cleaned/cl_sr_system.cpp:285-330).
struct EvolveParams {
  int32_t num_vars;
  int32_t max_tokens;
  int32_t max_depth;
  int32_t tournament;
  float const_min, const_max;
  float prob_leaf, prob_const_leaf, prob_unary;
  float mutation_prob;
  int32_t n_unary, n_binary;
  int32_t unary_ops[32];
  int32_t binary_ops[16];
  uint64_t seed;
};

// Population layout shared by these kernels: expression i has len[i] tokens
// at tok[i * stride ...] and values at val[i * stride ...] (float).
constexpr int kEvolveMaxStride = 256;

// Generation 0: random expressions (reference generate_random_expression).
cudaError_t launch_evolve_init(const EvolveParams &p, int E, int stride, int32_t *tok,
                               float *val, int32_t *len, cudaStream_t s);

// Ranking: order[] = expression indices by ascending fitness, NaN last, ties
// by index; fit_sorted[j] = fitness[order[j]].  temp: cub scratch of
// rank_temp_bytes(E) bytes; keys: 2*E uint32, idx_in: E int32.
size_t rank_temp_bytes(int E);
cudaError_t launch_rank(const float *fitness, int E, void *temp, size_t temp_bytes,
                        uint32_t *keys, int32_t *idx_in, int32_t *order, float *fit_sorted,
                        cudaStream_t s);

// One breeding step (reference cl_sr_system.cpp:285-330): children[0:elites)
// are the elites in rank order, the rest tournament-selected mutations /
// crossovers.  Inputs and outputs must not alias.
cudaError_t launch_evolve_step(const EvolveParams &p, int generation, int E, int stride,
                               int elites, const int32_t *order, const float *fit_sorted,
                               const int32_t *tok, const float *val, const int32_t *len,
                               int32_t *tok_out, float *val_out, int32_t *len_out,
                               cudaStream_t s);

// Device compile of a population in the layout above into the interpreter's
// bytecode: program i at code[i * (stride + 1)], code_off / code_len per
// expression.  summary[0] = largest spill-slot need, summary[1] = error flag
// (1 = an invalid expression; its code_len is 0), summary[2..3] = total
// tokens (int64), summary[4..5] = total instructions (int64), summary[6] =
// instructions inside the kOpsProtected profile; zeroed by the launcher.
cudaError_t launch_compile_device(const int32_t *tok, const float *val, const int32_t *len,
                                  int E, int stride, int num_vars, Instr *code,
                                  int64_t *code_off, int32_t *code_len, int32_t *summary,
                                  cudaStream_t s);

}  // namespace sr
