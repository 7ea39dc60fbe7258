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
// operator.  One instruction = one operator node of the tree (or a single
// load when the whole expression is a leaf).  Every instruction has the
// canonical form
//
//     [spill T -> S[slot]]  [T = leaf]  [b = operand]  T = op(T, b)
//
// so the device decodes no left/right operand roles: when the accumulator is
// the right operand of a non-commutative operator the host emits the
// reversed opcode, T = f(b, T).
//
//   Instr.w  bits 0..5   device opcode: reference token 1..27 (binary 1..9
//                        as T = f(T, b), unary 10..27 as T = f(T)), 32 = exp
//                        clamped at 80 (extension), 40 + k = reversed binary
//                        k (T = f_k(b, T)) for non-commutative k, 0 = none
//            bit  6      load: T = leaf A before the operator
//            bits 7..8   kind of leaf A: 0 = variable row (shared memory),
//                        1 = constant, 2 = cached subtree (global memory)
//            bits 9..11  kind of operand b: 0 = none, 1 = spill slot,
//                        2 = variable row, 3 = constant, 4 = cached subtree
//            bit  12     spill: store T into S[spill slot] first
//            bits 13..17 spill slot
//   Instr.a  payload of leaf A, Instr.b payload of operand b: spill slot /
//            variable row / float bits of the constant / cache slot
//   Instr.c  bits 0..9 / 10..19: constant index (token order) of leaf A /
//            operand b when it is a constant, 0x3FF otherwise; bits 20..29:
//            when b is a spill slot, the program-relative index of the
//            instruction whose output was spilled there (the adjoint reads
//            that value back from its tape).
#pragma once
#include <cstdint>
#include <vector_types.h>

#if defined(__CUDACC__)
#define SR_HD __host__ __device__ __forceinline__
#else
#define SR_HD inline
#endif

namespace sr {

// Kinds of leaf A (loaded into the accumulator).
enum : uint32_t { kLeafX = 0, kLeafC = 1, kLeafR = 2 };
// Kinds of operand b.
enum : uint32_t { kBNone = 0, kBS = 1, kBX = 2, kBC = 3, kBR = 4 };

constexpr uint32_t kOpNone = 0;
constexpr uint32_t kOpExpClamp = 32;
constexpr uint32_t kOpReversed = 40;  // 40 + k: T = f_k(b, T)
constexpr uint32_t kLoadBit = 1u << 6;
constexpr uint32_t kSpillBit = 1u << 12;
constexpr uint32_t kNoConst = 0x3FFu;
constexpr int kMaxSpillSlots = 16;  // S slots per warp supported by the kernels
constexpr int kBufs = 2;            // X span buffers per block

struct alignas(16) Instr {
  uint32_t w, a, b, c;
};

SR_HD uint32_t instr_op(uint32_t w) { return w & 63u; }
SR_HD bool instr_load(uint32_t w) { return (w & kLoadBit) != 0; }
SR_HD uint32_t instr_leaf_kind(uint32_t w) { return (w >> 7) & 3u; }
SR_HD uint32_t instr_b_kind(uint32_t w) { return (w >> 9) & 7u; }
SR_HD bool instr_spill(uint32_t w) { return (w & kSpillBit) != 0; }
SR_HD uint32_t instr_spill_slot(uint32_t w) { return (w >> 13) & 31u; }
// Non-commutative binary operators get a reversed opcode.  ADD and MUL are
// exactly commutative in IEEE arithmetic; MIN/MAX are treated as
// non-commutative so that signed zeros keep the reference's operand order.
SR_HD bool is_commutative_token(int tok) { return tok == 1 || tok == 3; }
SR_HD bool is_binary_token(int tok) { return tok >= 1 && tok <= 9; }
SR_HD bool is_unary_token(int tok) {
  return (tok >= 10 && tok <= 27) || tok == static_cast<int>(kOpExpClamp);
}

// Operator profiles of the interpreter: the set of opcodes its dispatch
// switch handles inline (every other opcode goes through one out-of-line
// routine, with identical results).  kOpsAll: every operator inline.
// kOpsProtected: + - *, protected division, sin, cos, exp clamped at 80,
// protected log and sqrt|x| (and their reversed forms).  A launch uses
// kOpsProtected when at least kProtectedShare of its instructions are in it.
constexpr int kOpsAll = 0;
constexpr int kOpsProtected = 1;
constexpr double kProtectedShare = 0.9;
SR_HD bool in_protected_profile(uint32_t op) {
  return op == 0 || op == 1 || op == 2 || op == kOpReversed + 2 || op == 3 || op == 8 ||
         op == kOpReversed + 8 || op == 10 || op == 11 || op == kOpExpClamp || op == 22 ||
         op == 27;
}

// Device-side error word bits.
enum : int32_t {
  kDevErrTimeout = 1,   // a bounded mbarrier wait gave up
  kDevErrBounds = 2,    // a device bounds check fired (debug builds)
};

// Argument block of the interpreter kernel (passed by value).
//
// Work decomposition: expressions are sorted by modelled cost (descending)
// and cut into groups of G; the datapoint axis is cut into spans of `span`
// datapoints.  A work item is (span, group); items are numbered span-major
// and handed out by an atomic counter to persistent blocks.  A block's
// producer thread copies the item's X span (all V+1 rows) into one of two
// shared-memory buffers with the bulk-copy engine; the block's evaluating
// warps claim the group's expressions one at a time from a shared counter and
// run each over the whole span, tile by tile (32*DPT datapoints per tile).
// Warps never wait for each other inside an item.
struct EvalArgs {
  const float *X;        // [(V+1)][ldx], y in row V
  int64_t ldx;           // row stride (floats), multiple of 4096
  int64_t N;             // datapoints
  const Instr *code;     // all programs back to back
  const int64_t *code_off;   // [E] first instruction of each expression
  const int32_t *code_len;   // [E] instruction count
  const int32_t *group_expr; // [n_groups * G] expression index or -1 (tail)
  double2 *partial;      // [n_span_groups][E] x 2 (MSE launches; see span_per_item)
  int32_t *work_counter; // zeroed before each launch
  int32_t *error;        // device error word
  const float *cache;    // subtree cache [slot][ldc] (cached-subtree operands)
  int64_t ldc;
  float *pred;           // prediction output [row][ldp] (prediction mode)
  int64_t ldp;
  const int32_t *pred_row;   // [E] output row of each expression
  int32_t V;
  int32_t E;
  int32_t W;             // evaluating warps per block (block = (W+1) warps)
  int32_t smax;          // S slots per warp
  int32_t G;             // expressions per group
  int32_t n_groups;
  int32_t span;          // datapoints per span, multiple of 32*DPT
  int32_t n_spans;
  // Spill slots [0, s_smem) of each warp live in shared memory, slots
  // [s_smem, smax) in this global scratch: per resident warp
  // (blockIdx.x * W + warp), (smax - s_smem) tiles of 32*DPT floats.
  float *spill;
  int32_t s_smem;
  // Spans per work item: an item is (span group, expression group), a span
  // group k_spans consecutive spans.  MSE launches write one entry per (span
  // group, expression) into `partial`: two double2, (sum as hi + lo,
  // count).
  int32_t span_per_item;
};

}  // namespace sr
