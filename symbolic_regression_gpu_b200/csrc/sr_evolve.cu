// sr_evolve.cu — the generation loop around the evaluator, on the device.
//
//   evolve_init_kernel     generation 0: one random expression per slot
//                          (reference generate_random_expression,
//                          src/utils/utils.cpp:1156-1161).
//   rank (cub radix sort)  population order by fitness, NaN last
//                          (reference std::sort with a NaN-last comparator,
//                          src/cleaned/cl_sr_system.cpp:286-290).
//   evolve_step_kernel     one thread per child: elites copied in rank order,
//                          the others bred by tournament selection and
//                          subtree mutation / subtree crossover (reference
//                          cl_sr_system.cpp:297-327, mutate_expression and
//                          crossover_expressions, src/utils/utils.cpp:1163-1273).
//   compile_kernel         one thread per expression: the host compiler's
//                          prefix -> bytecode translation (Sethi-Ullman
//                          evaluation order, leaf operands folded, reversed
//                          opcodes, spill slots), so a population bred on the
//                          device is evaluated without a host round trip.
//
// Random numbers: every child draws from its own counter-based stream (a
// SplitMix64 sequence seeded from (seed, generation, child)), so a step is
// deterministic for a given seed and independent of the launch shape.  The
// reference draws from one process-wide std::mt19937 / rand() sequence; the
// two give the same distributions, not the same samples.  The order of draws
// inside a child follows the reference's call order exactly (tournament,
// mutation-or-crossover choice, node choice, generator), which the oracle
// (oracle/evolve.py) replays draw for draw.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_eval.h"
#include "sr_evolve.hpp"
#include "sr_internal.hpp"

namespace sr {
namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// SplitMix64 stream.
struct Rng {
  uint64_t s;
  __device__ __forceinline__ uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    return mix64(s);
  }
  // [0, 1) with 24 random bits.
  __device__ __forceinline__ float unit() {
    return static_cast<float>(static_cast<uint32_t>(next() >> 40)) * (1.0f / 16777216.0f);
  }
  // [0, n) for n >= 1.
  __device__ __forceinline__ int below(int n) {
    return static_cast<int>(((next() >> 32) * static_cast<uint64_t>(n)) >> 32);
  }
  // Reference rand_int(lo, hi) (utils.cpp:972-978): no draw when hi <= lo.
  __device__ __forceinline__ int between(int lo, int hi) {
    return hi <= lo ? lo : lo + below(hi - lo + 1);
  }
  // Reference rand_uniform(lo, hi); unfused so the host replays it bit for bit.
  __device__ __forceinline__ float range(float lo, float hi) {
    return __fadd_rn(lo, __fmul_rn(__fsub_rn(hi, lo), unit()));
  }
};

__device__ __forceinline__ Rng child_stream(uint64_t seed, int generation, int child) {
  const uint64_t ctr = (static_cast<uint64_t>(static_cast<uint32_t>(generation)) << 32) |
                       static_cast<uint32_t>(child);
  return Rng{mix64(seed ^ mix64(ctr))};
}

// Arity of a token in a bred expression: binary 1..9, unary 10..27 and the
// exp-clamp extension 32, leaves otherwise (reference op_arity,
// src/utils/opcodes.h:42-80, which has no opcode 32).
__device__ __forceinline__ int gp_arity(int t) {
  return (t >= 1 && t <= 9) ? 2 : (((t >= 10 && t <= 27) || t == 32) ? 1 : 0);
}

// Length of the subtree rooted at `start` (reference subtree_size,
// utils.cpp:1110-1129, for well-formed prefix input).
__device__ int subtree_len(const int32_t *tok, int len, int start) {
  if (start < 0 || start >= len) return 0;
  int need = 1, p = start;
  while (need > 0 && p < len) {
    need += gp_arity(tok[p]) - 1;
    ++p;
  }
  return p - start;
}

constexpr int kMaxGenDepth = 64;

// Reference generate_with_limit / build_node / emit_leaf (utils.cpp:995-1108)
// as an explicit-stack walk with the same order of random draws.  Writes at
// most `cap` tokens at tok / val; returns the count, or -1 if `cap` was too
// small (the caller then keeps the parent).
__device__ int generate(Rng &r, const EvolveParams &g, int limit, int32_t *tok, float *val,
                        int cap) {
  int left = min(g.max_tokens, limit);
  if (left <= 0) return 0;
  int n = 0;
  int fdepth[kMaxGenDepth], frem[kMaxGenDepth];
  int nf = 0;
  const int nv = max(1, g.num_vars);
  // One node at `depth`: a leaf (returns 0) or an operator (returns its
  // arity, its children still to come); -1 when out of space.
  auto node = [&](int depth) -> int {
    bool must_leaf = depth >= g.max_depth || left == 1;
    if (!must_leaf && r.unit() < g.prob_leaf) must_leaf = true;
    if (n >= cap) return -1;
    if (must_leaf) {
      const bool c = r.unit() < g.prob_const_leaf;
      if (c) {
        tok[n] = SR_TOK_CONST;
        val[n] = r.range(g.const_min, g.const_max);
      } else {
        tok[n] = SR_TOK_VAR;
        val[n] = static_cast<float>(r.between(0, nv - 1));
      }
      ++n;
      --left;
      return 0;
    }
    float thresh = g.prob_unary;
    if (left < 2) thresh = 0.0f;
    if (left < 3) thresh = 1.0f;
    const bool unary = r.unit() < thresh;
    const int op = unary ? g.unary_ops[r.between(0, g.n_unary - 1)]
                         : g.binary_ops[r.between(0, g.n_binary - 1)];
    tok[n] = op;
    val[n] = 0.0f;
    ++n;
    --left;
    return unary ? 1 : 2;
  };
  int a = node(0);
  if (a < 0) return -1;
  if (a > 0) {
    fdepth[0] = 1;
    frem[0] = a;
    nf = 1;
  }
  while (nf > 0) {
    if (frem[nf - 1] == 0) {
      --nf;
      continue;
    }
    --frem[nf - 1];
    if (left <= 0) {
      // Budget exhausted with children pending: the reference appends a
      // variable-0 leaf without charging the budget (utils.cpp:1072-1078).
      if (n >= cap) return -1;
      tok[n] = SR_TOK_VAR;
      val[n] = 0.0f;
      ++n;
      continue;
    }
    const int d = fdepth[nf - 1];
    a = node(d);
    if (a < 0) return -1;
    if (a > 0) {
      if (nf >= kMaxGenDepth) return -1;
      fdepth[nf] = d + 1;
      frem[nf] = a;
      ++nf;
    }
  }
  if (n == 0) {  // utils.cpp:1102-1106
    if (cap < 1) return -1;
    tok[0] = SR_TOK_CONST;
    val[0] = 0.0f;
    n = 1;
  }
  return n;
}

__device__ __forceinline__ void copy_tokens(const int32_t *st, const float *sv, int n, int32_t *dt,
                                            float *dv) {
  for (int k = 0; k < n; ++k) {
    dt[k] = st[k];
    dv[k] = sv[k];
  }
}

__global__ void evolve_init_kernel(const EvolveParams p, int E, int stride, int32_t *tok,
                                   float *val, int32_t *len) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  Rng r = child_stream(p.seed, -1, i);
  int32_t *t = tok + static_cast<int64_t>(i) * stride;
  float *v = val + static_cast<int64_t>(i) * stride;
  int n = generate(r, p, p.max_tokens, t, v, stride);
  if (n < 0) {  // cannot happen with stride >= 2 * max_tokens + 2
    t[0] = SR_TOK_CONST;
    v[0] = 0.0f;
    n = 1;
  }
  len[i] = n;
}

// Order-preserving key of a fitness value; NaN after everything.
__global__ void fitness_keys_kernel(const float *fit, int E, uint32_t *keys, int32_t *idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  const float f = fit[i];
  const uint32_t u = __float_as_uint(f);
  keys[i] = isnan(f) ? 0xFFFFFFFFu : ((u & 0x80000000u) ? ~u : (u | 0x80000000u));
  idx[i] = i;
}

__global__ void gather_fitness_kernel(const float *fit, const int32_t *order, int E,
                                      float *fit_sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  fit_sorted[i] = fit[order[i]];
}

// Reference tournament (cl_sr_system.cpp:302-307): indices into the ranked
// population, strict `<` on fitness (a NaN never wins, a NaN incumbent is
// never replaced).
__device__ __forceinline__ int tournament(Rng &r, const float *fit, int E, int size) {
  int best = r.below(E);
  for (int k = 0; k < size - 1; ++k) {
    const int cand = r.below(E);
    if (fit[cand] < fit[best]) best = cand;
  }
  return best;
}

__global__ void evolve_step_kernel(const EvolveParams p, int generation, int E, int stride,
                                   int elites, const int32_t *__restrict__ order,
                                   const float *__restrict__ fit, const int32_t *__restrict__ tok,
                                   const float *__restrict__ val, const int32_t *__restrict__ len,
                                   int32_t *__restrict__ tok_out, float *__restrict__ val_out,
                                   int32_t *__restrict__ len_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  int32_t *ct = tok_out + static_cast<int64_t>(i) * stride;
  float *cv = val_out + static_cast<int64_t>(i) * stride;
  auto parent = [&](int rank, const int32_t *&t, const float *&v, int &n) {
    const int64_t o = static_cast<int64_t>(order[rank]) * stride;
    t = tok + o;
    v = val + o;
    n = min(max(len[order[rank]], 0), stride);
  };
  const int32_t *at;
  const float *av;
  int an;
  if (i < elites) {
    parent(i, at, av, an);
    copy_tokens(at, av, an, ct, cv);
    len_out[i] = an;
    return;
  }
  Rng r = child_stream(p.seed, generation, i);
  const int b1 = tournament(r, fit, E, p.tournament);
  parent(b1, at, av, an);
  int out = -1;
  if (r.unit() < p.mutation_prob) {
    // Subtree mutation (utils.cpp:1163-1204).
    if (an > 0) {
      const int idx = r.between(0, an - 1);
      int old = subtree_len(at, an, idx);
      if (old <= 0) old = 1;
      const int base = an - old;
      const int max_new = p.max_tokens - base;
      if (max_new > 0) {
        copy_tokens(at, av, idx, ct, cv);
        const int tail = an - idx - old;
        const int n = generate(r, p, max_new, ct + idx, cv + idx, stride - idx - tail);
        if (n >= 0) {
          copy_tokens(at + idx + old, av + idx + old, tail, ct + idx + n, cv + idx + n);
          out = idx + n + tail;
        }
      }
    }
  } else {
    // Subtree crossover (utils.cpp:1206-1273).
    const int b2 = tournament(r, fit, E, p.tournament);
    const int32_t *bt;
    const float *bv;
    int bn;
    parent(b2, bt, bv, bn);
    if (an > 0 && bn > 0) {
      const int li = r.between(0, an - 1);
      int ls = subtree_len(at, an, li);
      if (ls <= 0) ls = 1;
      const int attempts = min(bn, 32);
      for (int k = 0; k < attempts; ++k) {
        const int ri = r.between(0, bn - 1);
        const int rs = subtree_len(bt, bn, ri);
        if (rs <= 0) continue;
        const int total = an - ls + rs;
        if (total > p.max_tokens || total > stride) continue;
        copy_tokens(at, av, li, ct, cv);
        copy_tokens(bt + ri, bv + ri, rs, ct + li, cv + li);
        copy_tokens(at + li + ls, av + li + ls, an - li - ls, ct + li + rs, cv + li + rs);
        out = total;
        break;
      }
    }
  }
  if (out < 0) {  // the reference's "child = parent" fallbacks
    copy_tokens(at, av, an, ct, cv);
    out = an;
  }
  len_out[i] = out;
}

// ---- device compile ----------------------------------------------------------

struct DNode {
  int32_t op;       // operator token, or -1 for a leaf
  uint32_t lk;      // leaf kind
  uint32_t lp;      // leaf payload
  int16_t lconst;   // constant index or -1
  int16_t left, right;
  int16_t need;
};

__device__ __forceinline__ uint32_t b_kind_of(uint32_t lk) {
  return lk == kLeafX ? kBX : (lk == kLeafC ? kBC : kBR);
}
__device__ __forceinline__ uint32_t reversed_op(int tok) {
  return is_commutative_token(tok) ? static_cast<uint32_t>(tok)
                                   : kOpReversed + static_cast<uint32_t>(tok);
}

struct DEmitter {
  Instr *out;
  int count = 0;
  int pending_spill = -1;
  int spill_at[kMaxSpillSlots + 1];

  __device__ void emit(uint32_t op, const DNode *load, uint32_t bk, uint32_t bp, uint32_t bc) {
    Instr ins;
    ins.w = (op & 63u) | ((bk & 7u) << 9);
    uint32_t ac = kNoConst;
    ins.a = 0;
    if (load) {
      ins.w |= kLoadBit | ((load->lk & 3u) << 7);
      ins.a = load->lp;
      ac = load->lconst >= 0 ? static_cast<uint32_t>(load->lconst) : kNoConst;
    }
    if (pending_spill >= 0) {
      ins.w |= kSpillBit | (static_cast<uint32_t>(pending_spill) << 13);
      spill_at[pending_spill] = count;
      pending_spill = -1;
    }
    ins.b = bp;
    const uint32_t producer = (bk == kBS) ? static_cast<uint32_t>(spill_at[bp] - 1) : 0u;
    ins.c = (ac & 0x3FFu) | ((bc & 0x3FFu) << 10) | ((producer & 0x3FFu) << 20);
    out[count++] = ins;
  }
  __device__ void emit_b_leaf(uint32_t op, const DNode *load, const DNode &b) {
    emit(op, load, b_kind_of(b.lk), b.lp,
         b.lconst >= 0 ? static_cast<uint32_t>(b.lconst) : kNoConst);
  }
};

// Same translation as the host compiler (compile_expression,
// csrc/sr_program.cpp) without cache hints; returns the instruction count, or
// -1 for an invalid expression.
__device__ int compile_one(const int32_t *tok, const float *val, int len, int num_vars,
                           Instr *out, int *need_out) {
  if (len <= 0 || len > kEvolveMaxStride) return -1;
  {
    int depth = 0;
    for (int i = len - 1; i >= 0; --i) {
      const int t = tok[i];
      if (t == SR_TOK_CONST || t == SR_TOK_VAR) {
        ++depth;
      } else if (is_binary_token(t)) {
        if (depth < 2) return -1;
        --depth;
      } else if (is_unary_token(t)) {
        if (depth < 1) return -1;
      } else {
        return -1;
      }
    }
    if (depth != 1) return -1;
  }
  DNode nodes[kEvolveMaxStride];
  int16_t stk[kEvolveMaxStride];
  int ns = 0, nn = 0;
  // Constants are numbered in token order; parse right to left.
  int n_const = 0;
  for (int i = 0; i < len; ++i) n_const += tok[i] == SR_TOK_CONST ? 1 : 0;
  int cidx = n_const;
  for (int i = len - 1; i >= 0; --i) {
    const int t = tok[i];
    DNode nd;
    nd.op = -1;
    nd.lk = kLeafC;
    nd.lp = 0;
    nd.lconst = -1;
    nd.left = nd.right = -1;
    nd.need = 0;
    if (t == SR_TOK_CONST) {
      nd.lk = kLeafC;
      nd.lp = __float_as_uint(val[i]);
      --cidx;
      nd.lconst = static_cast<int16_t>(cidx < static_cast<int>(kNoConst) ? cidx : -1);
    } else if (t == SR_TOK_VAR) {
      const float v = val[i];
      const int vi = (v > -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v) : -1;
      if (vi >= 0 && vi < num_vars) {
        nd.lk = kLeafX;
        nd.lp = static_cast<uint32_t>(vi);
      } else {
        nd.lk = kLeafC;  // reference CPU pushes 0.0f (cl_cpu_eval.cpp:73-75)
        nd.lp = __float_as_uint(0.0f);
      }
    } else {
      nd.op = t;
      nd.left = stk[--ns];
      if (is_binary_token(t)) nd.right = stk[--ns];
    }
    nodes[nn] = nd;
    stk[ns++] = static_cast<int16_t>(nn);
    ++nn;
  }
  const int root = stk[0];
  for (int k = 0; k < nn; ++k) {
    DNode &nd = nodes[k];
    if (nd.op < 0) {
      nd.need = 0;
    } else if (nd.right < 0) {
      const DNode &c = nodes[nd.left];
      nd.need = c.op < 0 ? 0 : c.need;
    } else {
      const DNode &L = nodes[nd.left];
      const DNode &R = nodes[nd.right];
      if (L.op < 0 && R.op < 0) nd.need = 0;
      else if (R.op < 0) nd.need = L.need;
      else if (L.op < 0) nd.need = R.need;
      else nd.need = (L.need == R.need) ? L.need + 1 : max(L.need, R.need);
    }
  }
  if (nodes[root].need > kMaxSpillSlots) return -1;
  *need_out = nodes[root].need;
  // Emission: the host compiler's recursive walk with an explicit stack.
  DEmitter em;
  em.out = out;
  int16_t fn[kEvolveMaxStride];
  int8_t fst[kEvolveMaxStride];
  int8_t fslot[kEvolveMaxStride];
  int nf = 0, sp = 0;
  fn[0] = static_cast<int16_t>(root);
  fst[0] = 0;
  nf = 1;
  while (nf > 0) {
    const int n = fn[nf - 1];
    const int st = fst[nf - 1];
    const DNode &nd = nodes[n];
    if (nd.op < 0) {
      em.emit(kOpNone, &nd, kBNone, 0, kNoConst);
      --nf;
      continue;
    }
    const DNode &L = nodes[nd.left];
    const uint32_t op = static_cast<uint32_t>(nd.op);
    if (nd.right < 0) {
      if (L.op < 0) {
        em.emit(op, &L, kBNone, 0, kNoConst);
        --nf;
      } else if (st == 0) {
        fst[nf - 1] = 1;
        fn[nf] = nd.left;
        fst[nf] = 0;
        ++nf;
      } else {
        em.emit(op, nullptr, kBNone, 0, kNoConst);
        --nf;
      }
      continue;
    }
    const DNode &R = nodes[nd.right];
    if (L.op < 0 && R.op < 0) {
      em.emit_b_leaf(op, &L, R);
      --nf;
    } else if (R.op < 0) {
      if (st == 0) {
        fst[nf - 1] = 1;
        fn[nf] = nd.left;
        fst[nf] = 0;
        ++nf;
      } else {
        em.emit_b_leaf(op, nullptr, R);
        --nf;
      }
    } else if (L.op < 0) {
      if (st == 0) {
        fst[nf - 1] = 1;
        fn[nf] = nd.right;
        fst[nf] = 0;
        ++nf;
      } else {
        em.emit_b_leaf(reversed_op(nd.op), nullptr, L);
        --nf;
      }
    } else {
      const bool left_first = L.need > R.need;
      if (st == 0) {
        fst[nf - 1] = 1;
        fn[nf] = left_first ? nd.left : nd.right;
        fst[nf] = 0;
        ++nf;
      } else if (st == 1) {
        const int slot = sp++;
        fslot[nf - 1] = static_cast<int8_t>(slot);
        em.pending_spill = slot;
        fst[nf - 1] = 2;
        fn[nf] = left_first ? nd.right : nd.left;
        fst[nf] = 0;
        ++nf;
      } else {
        --sp;
        const uint32_t slot = static_cast<uint32_t>(fslot[nf - 1]);
        em.emit(left_first ? reversed_op(nd.op) : op, nullptr, kBS, slot, kNoConst);
        --nf;
      }
    }
  }
  return em.count;
}

__global__ void compile_kernel(const int32_t *__restrict__ tok, const float *__restrict__ val,
                               const int32_t *__restrict__ len, int E, int stride, int num_vars,
                               Instr *__restrict__ code, int64_t *__restrict__ code_off,
                               int32_t *__restrict__ code_len, int32_t *summary) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  const int64_t base = static_cast<int64_t>(i) * (stride + 1);
  const int n = len[i];
  int need = 0;
  const int count = (n >= 1 && n <= stride)
                        ? compile_one(tok + static_cast<int64_t>(i) * stride,
                                      val + static_cast<int64_t>(i) * stride, n, num_vars,
                                      code + base, &need)
                        : -1;
  code_off[i] = base;
  if (count < 0) {
    code_len[i] = 0;
    atomicOr(&summary[1], 1);
    return;
  }
  code_len[i] = count;
  int prot = 0;
  for (int k = 0; k < count; ++k) prot += in_protected_profile(instr_op(code[base + k].w)) ? 1 : 0;
  if (prot) atomicAdd(&summary[6], prot);
  atomicMax(&summary[0], need);
  atomicAdd(reinterpret_cast<unsigned long long *>(summary + 2), static_cast<unsigned long long>(n));
  atomicAdd(reinterpret_cast<unsigned long long *>(summary + 4),
            static_cast<unsigned long long>(count));
}

inline unsigned grid_for(int n, int block) { return static_cast<unsigned>((n + block - 1) / block); }

}  // namespace

cudaError_t launch_evolve_init(const EvolveParams &p, int E, int stride, int32_t *tok,
                               float *val, int32_t *len, cudaStream_t s) {
  if (E <= 0) return cudaSuccess;
  evolve_init_kernel<<<grid_for(E, 128), 128, 0, s>>>(p, E, stride, tok, val, len);
  return cudaGetLastError();
}

size_t rank_temp_bytes(int E) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const uint32_t *>(nullptr),
                                  static_cast<uint32_t *>(nullptr),
                                  static_cast<const int32_t *>(nullptr),
                                  static_cast<int32_t *>(nullptr), E);
  return bytes;
}

cudaError_t launch_rank(const float *fitness, int E, void *temp, size_t temp_bytes,
                        uint32_t *keys, int32_t *idx_in, int32_t *order, float *fit_sorted,
                        cudaStream_t s) {
  if (E <= 0) return cudaSuccess;
  fitness_keys_kernel<<<grid_for(E, 256), 256, 0, s>>>(fitness, E, keys, idx_in);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  // Radix sort is stable: equal fitness keeps index order.
  err = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys + E, idx_in, order, E, 0, 32,
                                        s);
  if (err != cudaSuccess) return err;
  gather_fitness_kernel<<<grid_for(E, 256), 256, 0, s>>>(fitness, order, E, fit_sorted);
  return cudaGetLastError();
}

cudaError_t launch_evolve_step(const EvolveParams &p, int generation, int E, int stride,
                               int elites, const int32_t *order, const float *fit_sorted,
                               const int32_t *tok, const float *val, const int32_t *len,
                               int32_t *tok_out, float *val_out, int32_t *len_out,
                               cudaStream_t s) {
  if (E <= 0) return cudaSuccess;
  evolve_step_kernel<<<grid_for(E, 128), 128, 0, s>>>(p, generation, E, stride, elites, order,
                                                      fit_sorted, tok, val, len, tok_out, val_out,
                                                      len_out);
  return cudaGetLastError();
}

cudaError_t launch_compile_device(const int32_t *tok, const float *val, const int32_t *len,
                                  int E, int stride, int num_vars, Instr *code,
                                  int64_t *code_off, int32_t *code_len, int32_t *summary,
                                  cudaStream_t s) {
  cudaError_t err = cudaMemsetAsync(summary, 0, 8 * sizeof(int32_t), s);
  if (err != cudaSuccess || E <= 0) return err;
  compile_kernel<<<grid_for(E, 64), 64, 0, s>>>(tok, val, len, E, stride, num_vars, code,
                                                code_off, code_len, summary);
  return cudaGetLastError();
}

}  // namespace sr
