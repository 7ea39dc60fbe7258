// sr_program.cpp — validation and bytecode compilation of prefix expressions.
//
// Semantics follow the reference CPU evaluator evaluate_single_expr
// (src/cleaned/cl_cpu_eval.cpp:59-90): tokens are consumed right to left, a
// constant pushes (float)value, a variable pushes x[(int)value] (0 when the
// index is not a valid input variable, cl_cpu_eval.cpp:70-76), an operator pops
// its left operand first (cl_gpu_eval.cu:98-101).
//
// The compiler builds the expression tree, labels every node with the number
// of spill slots its evaluation needs (Sethi-Ullman numbering: the child that
// needs more slots is evaluated first, which bounds the slots of a
// 127-token tree by 5), and emits one instruction per operator node with its
// leaf children folded in as operands.  Reordering the evaluation of two
// independent subtrees changes no floating-point result: every operator still
// receives exactly the same operand values.
#include "sr_program.hpp"

#include <cmath>
#include <cstring>

namespace sr {

void subtree_sizes(const int32_t *tok, int len, int32_t *sizes) {
  // Reverse pass: children of position i start at i+1.
  for (int i = len - 1; i >= 0; --i) {
    const int t = tok[i];
    if (t <= 0) {
      sizes[i] = 1;
      continue;
    }
    const int arity = (t < 10) ? 2 : 1;
    int size = 1, pos = i + 1;
    for (int k = 0; k < arity && pos < len; ++k) {
      size += sizes[pos];
      pos += sizes[pos];
    }
    sizes[i] = size;
  }
}

void declared_op_work(int tok, double *sfu, double *fp32) {
  double s = 0, f = 0;
  switch (tok) {
    case SR_OP_ADD: case SR_OP_SUB: case SR_OP_MUL: case SR_OP_NEG:
    case SR_OP_ABS: case SR_OP_MIN: case SR_OP_MAX:
      f = 1; break;
    case SR_OP_LOOSE_DIV: case SR_OP_DIV: case SR_OP_INV: case SR_OP_LOOSE_INV:
      s = 1; f = 1; break;
    case SR_OP_LOOSE_SQRT: case SR_OP_SQRT:
      s = 1; break;
    case SR_OP_SIN: case SR_OP_COS:
      s = 1; f = 1; break;
    case SR_OP_EXP: case SR_OP_EXP_CLAMP:
      s = 1; f = 2; break;
    case SR_OP_LOG: case SR_OP_LOOSE_LOG:
      s = 1; f = 1; break;
    case SR_OP_POW: case SR_OP_LOOSE_POW:
      s = 2; f = 2; break;
    case SR_OP_TAN:
      s = 3; f = 2; break;
    case SR_OP_SINH: case SR_OP_COSH: case SR_OP_TANH:
      s = 2; f = 3; break;
    case SR_OP_ASIN: case SR_OP_ACOS: case SR_OP_ATAN:
      s = 1; f = 8; break;
    default: break;  // leaves
  }
  *sfu = s;
  *fp32 = f;
}

float op_cost(int tok) {
  switch (tok) {
    case 0: return 1.f;
    case SR_OP_ADD: case SR_OP_SUB: case SR_OP_MUL: case SR_OP_MIN:
    case SR_OP_MAX: case SR_OP_NEG: case SR_OP_ABS: return 1.f;
    case SR_OP_DIV: return 10.f;
    case SR_OP_LOOSE_DIV: return 12.f;
    case SR_OP_INV: return 8.f;
    case SR_OP_LOOSE_INV: return 10.f;
    case SR_OP_SQRT: return 8.f;
    case SR_OP_LOOSE_SQRT: return 9.f;
    case SR_OP_SIN: case SR_OP_COS: return 24.f;
    case SR_OP_TAN: return 36.f;
    case SR_OP_SINH: return 26.f;
    case SR_OP_COSH: return 22.f;
    case SR_OP_TANH: return 18.f;
    case SR_OP_EXP: return 12.f;
    case SR_OP_EXP_CLAMP: return 13.f;
    case SR_OP_LOG: return 16.f;
    case SR_OP_LOOSE_LOG: return 18.f;
    case SR_OP_POW: return 50.f;
    case SR_OP_LOOSE_POW: return 52.f;
    case SR_OP_ASIN: return 20.f;
    case SR_OP_ACOS: return 22.f;
    case SR_OP_ATAN: return 22.f;
    default: return 1.f;
  }
}

namespace {

struct Node {
  bool leaf = false;
  int32_t op = 0;          // operator token
  uint32_t lk = kLeafC;    // leaf kind (kLeafX / kLeafC / kLeafR)
  uint32_t lp = 0;         // leaf payload
  uint32_t lconst = kNoConst;
  int32_t left = -1;       // first popped operand (operators)
  int32_t right = -1;      // second popped operand (binary)
  int32_t need = 0;
};

inline uint32_t float_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, sizeof u);
  return u;
}

// (int)value with the reference's truncation; values that cannot be an int
// (NaN, huge) map to -1 = "not an input variable".
inline int var_index(double v) {
  if (!(v > -2147483648.0 && v < 2147483648.0)) return -1;
  return static_cast<int>(v);
}

inline uint32_t b_kind_of_leaf(uint32_t lk) {
  return lk == kLeafX ? kBX : (lk == kLeafC ? kBC : kBR);
}

// Opcode computing T = f(b, T) for binary token f.
inline uint32_t reversed(int tok) {
  return is_commutative_token(tok) ? static_cast<uint32_t>(tok)
                                   : kOpReversed + static_cast<uint32_t>(tok);
}

struct Emitter {
  const std::vector<Node> &nodes;
  std::vector<Instr> &out;
  size_t first = 0;          // index of this program's first instruction in `out`
  int pending_spill = -1;
  int sp = 0;
  int spill_at[kMaxSpillSlots + 1] = {};  // instruction that spilled into each slot

  // [spill] [T = load] [b = operand] T = op(T, b)
  void emit(uint32_t op, const Node *load, uint32_t bk, uint32_t bp, uint32_t bc) {
    Instr ins;
    ins.w = (op & 63u) | ((bk & 7u) << 9);
    uint32_t ac = kNoConst;
    ins.a = 0;
    if (load) {
      ins.w |= kLoadBit | ((load->lk & 3u) << 7);
      ins.a = load->lp;
      ac = load->lconst;
    }
    const int index = static_cast<int>(out.size() - first);
    if (pending_spill >= 0) {
      ins.w |= kSpillBit | (static_cast<uint32_t>(pending_spill) << 13);
      spill_at[pending_spill] = index;
      pending_spill = -1;
    }
    ins.b = bp;
    // A spilled operand is the accumulator value right before its spill.
    const uint32_t producer = (bk == kBS) ? static_cast<uint32_t>(spill_at[bp] - 1) : 0u;
    ins.c = (ac & 0x3FFu) | ((bc & 0x3FFu) << 10) | ((producer & 0x3FFu) << 20);
    out.push_back(ins);
  }

  void emit_b_leaf(uint32_t op, const Node *load, const Node &b) {
    emit(op, load, b_kind_of_leaf(b.lk), b.lp, b.lconst);
  }

  void gen(int n) {
    const Node &nd = nodes[n];
    if (nd.leaf) {
      emit(kOpNone, &nd, kBNone, 0, kNoConst);
      return;
    }
    const Node &L = nodes[nd.left];
    const uint32_t op = static_cast<uint32_t>(nd.op);
    if (nd.right < 0) {  // unary
      if (L.leaf) {
        emit(op, &L, kBNone, 0, kNoConst);
      } else {
        gen(nd.left);
        emit(op, nullptr, kBNone, 0, kNoConst);
      }
      return;
    }
    const Node &R = nodes[nd.right];
    if (L.leaf && R.leaf) {
      emit_b_leaf(op, &L, R);              // T = L; T = f(T, R)
    } else if (R.leaf) {
      gen(nd.left);
      emit_b_leaf(op, nullptr, R);         // T = f(T=L, R)
    } else if (L.leaf) {
      gen(nd.right);
      emit_b_leaf(reversed(nd.op), nullptr, L);  // T = f(L, T=R)
    } else {
      // Both operands are operator subtrees: evaluate the one needing more
      // spill slots first (ties: the right one, the reference's own order),
      // park it in S[sp], evaluate the other into T, combine.
      const bool left_first = L.need > R.need;
      gen(left_first ? nd.left : nd.right);
      const int slot = sp++;
      pending_spill = slot;
      gen(left_first ? nd.right : nd.left);
      --sp;
      if (left_first)
        emit(reversed(nd.op), nullptr, kBS, static_cast<uint32_t>(slot), kNoConst);  // f(S, T)
      else
        emit(op, nullptr, kBS, static_cast<uint32_t>(slot), kNoConst);  // f(T, S)
    }
  }
};

}  // namespace

sr_status compile_expression(const int32_t *tok, const double *val, int len,
                             int num_vars, const int32_t *hints,
                             std::vector<Instr> &out, ExprInfo &info,
                             std::string *err) {
  info = ExprInfo{};
  info.n_tokens = len;
  if (len <= 0) {
    if (err) *err = "empty expression";
    return SR_ERR_MALFORMED_EXPRESSION;
  }
  if (len > SR_MAX_TOKENS) {
    if (err) *err = "expression has " + std::to_string(len) + " tokens (max " +
                    std::to_string(SR_MAX_TOKENS) + ")";
    return SR_ERR_EXPRESSION_TOO_LONG;
  }
  // Validate the original token stream: known tokens, no underflow, exactly
  // one value left.
  {
    int depth = 0;
    for (int i = len - 1; i >= 0; --i) {
      const int t = tok[i];
      if (t == SR_TOK_CONST || t == SR_TOK_VAR) {
        ++depth;
      } else if (is_binary_token(t)) {
        if (depth < 2) {
          if (err) *err = "stack underflow at token " + std::to_string(i);
          return SR_ERR_MALFORMED_EXPRESSION;
        }
        --depth;
      } else if (is_unary_token(t)) {
        if (depth < 1) {
          if (err) *err = "stack underflow at token " + std::to_string(i);
          return SR_ERR_MALFORMED_EXPRESSION;
        }
      } else {
        if (err) *err = "unknown token " + std::to_string(t) + " at position " +
                        std::to_string(i);
        return SR_ERR_BAD_TOKEN;
      }
    }
    if (depth != 1) {
      if (err) *err = "expression leaves " + std::to_string(depth) +
                      " values on the stack";
      return SR_ERR_MALFORMED_EXPRESSION;
    }
  }

  // Constant numbering in token order, and subtree sizes for cache hints.
  thread_local std::vector<int32_t> const_idx, sizes, seq;
  thread_local std::vector<Node> nodes;
  thread_local std::vector<int32_t> stk;
  const_idx.assign(len, static_cast<int32_t>(kNoConst));
  int n_const = 0;
  for (int i = 0; i < len; ++i)
    if (tok[i] == SR_TOK_CONST) const_idx[i] = n_const++;
  info.n_const = n_const;

  // Skeleton positions: cached subtrees collapse to one leaf at their root.
  seq.clear();
  if (hints) {
    sizes.resize(len);
    subtree_sizes(tok, len, sizes.data());
    for (int k = 0; k < len; ++k) {
      const int h = hints[k];
      if (h >= 0) {
        seq.push_back(-(k + 1));  // negative = cached-subtree leaf at k
        k += sizes[k] - 1;
      } else if (h == -2) {
        continue;
      } else {
        seq.push_back(k);
      }
    }
  } else {
    seq.resize(len);
    for (int k = 0; k < len; ++k) seq[k] = k;
  }

  // Parse right to left into a tree; children get lower node ids than their
  // parent, so node-id order is a post-order.
  nodes.clear();
  stk.clear();
  for (int s = static_cast<int>(seq.size()) - 1; s >= 0; --s) {
    const int e = seq[s];
    Node nd;
    if (e < 0) {
      const int k = -e - 1;
      nd.leaf = true;
      nd.lk = kLeafR;
      nd.lp = static_cast<uint32_t>(hints[k]);
    } else {
      const int t = tok[e];
      if (t == SR_TOK_CONST) {
        nd.leaf = true;
        nd.lk = kLeafC;
        nd.lp = float_bits(static_cast<float>(val[e]));
        nd.lconst = static_cast<uint32_t>(const_idx[e]);
      } else if (t == SR_TOK_VAR) {
        nd.leaf = true;
        const int v = var_index(val[e]);
        if (v >= 0 && v < num_vars) {
          nd.lk = kLeafX;
          nd.lp = static_cast<uint32_t>(v);
        } else {
          nd.lk = kLeafC;  // reference CPU pushes 0.0f (cl_cpu_eval.cpp:73-75)
          nd.lp = float_bits(0.0f);
        }
      } else {
        nd.op = t;
        if (stk.empty()) {
          if (err) *err = "cache marking produced an invalid skeleton";
          return SR_ERR_MALFORMED_EXPRESSION;
        }
        nd.left = stk.back();
        stk.pop_back();
        if (is_binary_token(t)) {
          if (stk.empty()) {
            if (err) *err = "cache marking produced an invalid skeleton";
            return SR_ERR_MALFORMED_EXPRESSION;
          }
          nd.right = stk.back();
          stk.pop_back();
        }
      }
    }
    nodes.push_back(nd);
    stk.push_back(static_cast<int32_t>(nodes.size() - 1));
  }
  if (stk.size() != 1) {
    if (err) *err = "cache marking produced an invalid skeleton";
    return SR_ERR_MALFORMED_EXPRESSION;
  }
  const int root = stk[0];

  // Spill-slot labels (post-order).
  for (auto &nd : nodes) {
    if (nd.leaf) {
      nd.need = 0;
    } else if (nd.right < 0) {
      const Node &c = nodes[nd.left];
      nd.need = c.leaf ? 0 : c.need;
    } else {
      const Node &L = nodes[nd.left];
      const Node &R = nodes[nd.right];
      if (L.leaf && R.leaf) nd.need = 0;
      else if (R.leaf) nd.need = L.need;
      else if (L.leaf) nd.need = R.need;
      else nd.need = (L.need == R.need) ? L.need + 1 : std::max(L.need, R.need);
    }
  }
  info.need = nodes[root].need;
  if (info.need > kMaxSpillSlots) {
    if (err) *err = "expression needs " + std::to_string(info.need) +
                    " spill slots (max " + std::to_string(kMaxSpillSlots) + ")";
    return SR_ERR_EXPRESSION_TOO_LONG;
  }

  const size_t first = out.size();
  Emitter em{nodes, out, first};
  em.gen(root);
  info.n_instr = static_cast<int32_t>(out.size() - first);

  // Cost model and declared work, over the executed instructions.
  float cost = 0.f;
  double sfu = 0, fp = 0;
  for (size_t i = first; i < out.size(); ++i) {
    const uint32_t w = out[i].w;
    uint32_t op = instr_op(w);
    if (op > kOpReversed) op -= kOpReversed;
    cost += 2.0f + op_cost(static_cast<int>(op));
    if (instr_load(w) && instr_leaf_kind(w) != kLeafC) cost += 0.5f;
    const uint32_t bk = instr_b_kind(w);
    if (bk == kBS || bk == kBX || bk == kBR) cost += 0.5f;
    if (instr_spill(w)) cost += 0.5f;
    double s, f;
    declared_op_work(static_cast<int>(op), &s, &f);
    sfu += s;
    fp += f;
  }
  info.cost = cost + 6.0f;  // epilogue
  info.sfu_ops = sfu;
  info.fp32_ops = fp + 3.0;  // MSE epilogue per datapoint (declared model)
  return SR_OK;
}

}  // namespace sr
