// sr_internal.hpp — definitions shared by the host compiler (C++) and the
// device interpreter (CUDA): the bytecode format and the kernel argument block.
//
// Bytecode.  Each prefix expression (reference token encoding,
// src/utils/opcodes.h:10-40) is compiled on the host into a short program for
// a one-accumulator machine.  The accumulator T lives in registers (DPT
// datapoints per lane); spilled intermediates live in a per-warp shared-memory
// stack S whose slot for every access is fixed at compile time, so the device
// never tracks a stack pointer.  Leaves are never instructions of their own:
// every variable / constant / cached-subtree leaf is an operand of its parent
// operator.  One instruction = one operator node of the tree (or a single MOV
// when the whole expression is a leaf).
//
//   Instr.w  bits 0..5   operator: reference token code 1..27, 32 = exp clamped
//                        at 80 (extension), 0 = MOV (T = operand A)
//            bits 6..8   kind of operand A (first popped, the left operand)
//            bits 9..11  kind of operand B (right operand; kNone for unary)
//            bit  12     spill: store T into S[spill slot] before executing
//            bits 13..17 spill slot
//   Instr.a  payload of operand A, Instr.b payload of operand B:
//            kT: unused; kS: stack slot; kX: variable row; kC: float bits of
//            the constant; kR: subtree-cache slot
//   Instr.c  bits 0..9 / 10..19: constant index (token order) of operand A / B
//            when that operand is a constant, 0x3FF otherwise (adjoint).
#pragma once
#include <cstdint>
#include <vector_types.h>

#if defined(__CUDACC__)
#define SR_HD __host__ __device__ __forceinline__
#else
#define SR_HD inline
#endif

namespace sr {

enum : uint32_t {
  kT = 0,     // accumulator
  kS = 1,     // spilled stack slot (per-warp shared memory)
  kX = 2,     // input variable row of the staged X tile (shared memory)
  kC = 3,     // immediate constant
  kR = 4,     // cached subtree value (global memory [slot][dp])
  kNone = 7,  // no operand (unary)
};

constexpr uint32_t kOpMov = 0;
constexpr uint32_t kOpExpClamp = 32;
constexpr uint32_t kSpillBit = 1u << 12;
constexpr uint32_t kNoConst = 0x3FFu;
constexpr int kMaxSpillSlots = 16;  // S slots per warp supported by the kernels
constexpr int kStages = 4;          // X tile ring depth

struct alignas(16) Instr {
  uint32_t w, a, b, c;
};

SR_HD uint32_t instr_op(uint32_t w) { return w & 63u; }
SR_HD uint32_t instr_ka(uint32_t w) { return (w >> 6) & 7u; }
SR_HD uint32_t instr_kb(uint32_t w) { return (w >> 9) & 7u; }
SR_HD bool instr_spill(uint32_t w) { return (w & kSpillBit) != 0; }
SR_HD uint32_t instr_spill_slot(uint32_t w) { return (w >> 13) & 31u; }
SR_HD uint32_t make_w(uint32_t op, uint32_t ka, uint32_t kb) {
  return (op & 63u) | ((ka & 7u) << 6) | ((kb & 7u) << 9);
}
SR_HD bool is_binary_token(int tok) { return tok >= 1 && tok <= 9; }
SR_HD bool is_unary_token(int tok) {
  return (tok >= 10 && tok <= 27) || tok == static_cast<int>(kOpExpClamp);
}

// Device-side error word bits.
enum : int32_t {
  kDevErrTimeout = 1,   // a bounded mbarrier wait gave up
  kDevErrBounds = 2,    // a device bounds check fired (debug builds)
};

// Argument block of the interpreter kernel (passed by value).
//
// Work decomposition: expressions are sorted by modelled cost and cut into
// groups of W (one expression per evaluating warp); the datapoint axis is cut
// into tiles of 32*DPT datapoints and the tiles into spans.  A work item is
// (span, group); items are numbered span-major and handed out by an atomic
// counter to persistent blocks.  Each block streams the tiles of its item
// through a kStages-deep ring of X tiles filled by the bulk-copy engine.
struct EvalArgs {
  const float *X;        // [(V+1)][ldx], y in row V
  int64_t ldx;           // row stride (floats), multiple of 256
  int64_t N;             // datapoints
  const Instr *code;     // all programs back to back
  const int64_t *code_off;   // [E] first instruction of each expression
  const int32_t *code_len;   // [E] instruction count
  const int32_t *group_expr; // [n_groups * W] expression index or -1
  double2 *partial;      // [n_spans][E] (sum of squared errors, valid count)
  int32_t *work_counter; // zeroed before each launch
  int32_t *error;        // device error word
  const float *cache;    // subtree cache [slot][ldc] (kR operands)
  int64_t ldc;
  float *pred;           // prediction output [row][ldp] (prediction mode)
  int64_t ldp;
  const int32_t *pred_row;   // [E] output row of each expression
  int32_t V;
  int32_t E;
  int32_t W;             // evaluating warps per block (block = (W+1) warps)
  int32_t smax;          // S slots per warp
  int32_t n_groups;
  int32_t n_spans;
  int32_t tiles_per_span;
  int32_t n_tiles;
};

}  // namespace sr
