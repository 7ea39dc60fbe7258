// sr_program.hpp — host-side validation and compilation of prefix expressions
// into the interpreter bytecode (format in sr_internal.hpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "sr_eval.h"
#include "sr_internal.hpp"

namespace sr {

// Result of compiling one expression.
struct ExprInfo {
  int32_t n_tokens = 0;   // tokens of the original expression
  int32_t n_instr = 0;    // bytecode instructions
  int32_t need = 0;       // spill slots used
  int32_t n_const = 0;    // SR_TOK_CONST tokens (adjoint numbering)
  float cost = 0.f;       // modelled device cost per datapoint (arbitrary units)
  double sfu_ops = 0.0;   // declared-roofline work per datapoint
  double fp32_ops = 0.0;
};

// Subtree size of the prefix expression starting at `pos`, with the
// reference's arity rule: token <= 0 is a leaf, 1..9 binary, anything else
// unary (reference compute_subtree_size, src/utils/detect.cpp:23-47;
// compute_subtree_size_state, src/cleaned/cl_gpu_eval.cu:279-292).
// sizes[i] for every i is produced in one reverse pass.
void subtree_sizes(const int32_t *tok, int len, int32_t *sizes);

// Validate and compile one expression.
//   hints (nullable, len entries): cache marking as produced by the subtree
//   cache: hints[i] >= 0 marks the root of a cached subtree held in cache slot
//   hints[i]; -2 marks the body of such a subtree; -1 elsewhere (reference
//   mark_cached_subtrees_from_state, src/cleaned/cl_gpu_eval.cu:294-329).
// Appends the program to `out`.  Returns SR_OK or an error with `*err` set.
sr_status compile_expression(const int32_t *tok, const double *val, int len,
                             int num_vars, const int32_t *hints,
                             std::vector<Instr> &out, ExprInfo &info,
                             std::string *err);

// Declared per-datapoint work of one operator token (project cost model:
// SFU / FP32 operation counts), used for the roofline; not CUDA's
// implementation.
void declared_op_work(int tok, double *sfu, double *fp32);

// Modelled relative device cost of one operator per datapoint (used only to
// balance warps; calibrated by hand against instruction counts).
float op_cost(int tok);

}  // namespace sr
