// sr_tangent.cu — forward-mode (tangent) gradient of the population MSE with
// respect to the constants of expressions with at most kMaxTangentConsts
// constants.  (No reference counterpart: the reference evaluates MSE only.)
//
//   tan_kernel<DPT, MAXW, MINB>
//                       the interpreter's work decomposition (a producer
//                       thread streaming X spans into shared memory and
//                       folding span results, warps claiming expressions of a
//                       group) with, beside each datapoint's value T, one
//                       tangent row t_c = d T / d constant c per constant, in
//                       the warp's shared memory.  Per instruction the warp
//                       computes the operator's value and local partials and
//                       moves the tangents forward:
//                         t_c = dT * t_c  for the constants under the
//                                          accumulator (mask A),
//                         t_c = db * t_c  for the constants under the operand
//                                          b (mask B: the constant itself, or
//                                          a spilled subtree, whose rows
//                                          stayed where they were),
//                       and a constant that enters (a leaf or operand b)
//                       starts at t_c = 1.  The masks come from the host (one
//                       word per instruction: A, B and a constant-load flag);
//                       instructions with A = B = 0 compute no partials.
//                       At the end of a tile d MSE / d c gets sum over
//                       datapoints of seed * t_c, seed = 2 (pred - y) for valid
//                       datapoints (0 otherwise): each lane's DPT products in
//                       FP32, FP64 across lanes, tiles and spans.  No tape, no
//                       second pass.
//
// Zero rule (the mirror of the reverse sweep's "a zero adjoint times anything
// is zero"): a zero partial times anything is zero (t_c = dT == 0 ? 0 :
// dT * t_c), and the final product is zero where the seed is zero.  An
// expression is a tree, so each constant reaches the result along one path
// and the two rules give the same zeros: whichever of an infinite and a zero
// factor lies nearer the result decides, in both modes, between NaN and 0.
// Constants outside a mask are never multiplied, so an infinite partial off
// a constant's path (sqrt'(0) in a branch without that constant) does not
// reach its tangent.
//
// Values and partials are those of the reverse-mode kernel (sr_grad_ops.cuh
// formulas, the forward interpreter's routines), so the MSE equals the
// forward pass's up to summation order and the gradients differ from the
// reverse mode only by the order of the FP32 products along each path.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_adjoint.hpp"
#include "sr_kernels.hpp"
#include "sr_device.cuh"
#include "sr_grad_ops.cuh"

namespace sr {
namespace {

// How a partial is known: exactly 1, exactly -1, or computed into dT / db.
enum : int { kDOne = 0, kDNeg = 1, kDGen = 2 };

// t = d == 0 ? 0 : d * t
template <int DPT>
__device__ __forceinline__ void kill_mul(float (&t)[DPT], const float (&d)[DPT]) {
#pragma unroll
  for (int k = 0; k < DPT; k += 2) {
    const float2 r = __fmul2_rn(make_float2(d[k], d[k + 1]), make_float2(t[k], t[k + 1]));
    t[k] = (d[k] == 0.0f) ? 0.0f : r.x;
    t[k + 1] = (d[k + 1] == 0.0f) ? 0.0f : r.y;
  }
}

// Operators outside the inline set: value and partials through the
// reverse-mode kernel's routine; T, b, dT, db travel through the stack.
template <int DPT>
__device__ __noinline__ void tan_op_cold(uint32_t op, float *T, float *b, float *dT, float *db) {
  float t[DPT], bb[DPT], d1[DPT], d2[DPT];
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    t[k] = T[k];
    bb[k] = b[k];
    d1[k] = 0.0f;
    d2[k] = 0.0f;
  }
  apply_op_grad<DPT>(op, t, bb, d1, d2);
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    T[k] = t[k];
    dT[k] = d1[k];
    db[k] = d2[k];
  }
}

// sin / cos with their derivative for a lane holding an argument outside the
// fast reduction range (out of line, rare).
template <int DPT>
__device__ __noinline__ void tan_sincos_cold(float *T, float *dT, int q_offset) {
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    float s, c;
    sr_sincosf(T[k], &s, &c);
    T[k] = q_offset ? c : s;
    dT[k] = q_offset ? -s : c;
  }
}

// T = op(T, b) with the partials the tangent update needs (only when `live`:
// instructions off every constant's path skip them).  dk / bk_: how dT / db
// are known.  The IEEE divisions and reciprocals of the protected division
// (both operand orders), the protected log's and sqrt|x|'s derivatives run
// in one shared loop each after the switch, so the code holds one copy of
// each (instruction-cache footprint).
template <int DPT>
__device__ __forceinline__ void tan_apply(uint32_t op, bool live, float (&T)[DPT],
                                          float (&b)[DPT], float (&dT)[DPT], float (&db)[DPT],
                                          int &dk, int &bk_) {
  dk = kDGen;
  bk_ = kDGen;
  // post bit 1: T = T / b; bit 2: the partials from 1 / b (when live).  For
  // these operators b holds the divisor (the protected denominator) or, for
  // the unary ones, the value to invert.
  int post = 0;
  switch (op) {
    case 0:
      dk = kDOne;
      break;
    // + - * in paired FP32 instructions (each half correctly rounded, a - b
    // as a + (-b)): the forward interpreter's values.
    case 1:
#pragma unroll
      for (int k = 0; k < DPT; k += 2) {
        const float2 r = __fadd2_rn(make_float2(T[k], T[k + 1]), make_float2(b[k], b[k + 1]));
        T[k] = r.x;
        T[k + 1] = r.y;
      }
      dk = kDOne;
      bk_ = kDOne;
      break;
    case 2:
#pragma unroll
      for (int k = 0; k < DPT; k += 2) {
        const float2 r = __fadd2_rn(make_float2(T[k], T[k + 1]), make_float2(-b[k], -b[k + 1]));
        T[k] = r.x;
        T[k + 1] = r.y;
      }
      dk = kDOne;
      bk_ = kDNeg;
      break;
    case kOpReversed + 2:
#pragma unroll
      for (int k = 0; k < DPT; k += 2) {
        const float2 r = __fadd2_rn(make_float2(b[k], b[k + 1]), make_float2(-T[k], -T[k + 1]));
        T[k] = r.x;
        T[k + 1] = r.y;
      }
      dk = kDNeg;
      bk_ = kDOne;
      break;
    case 3:
#pragma unroll
      for (int k = 0; k < DPT; k += 2) {
        dT[k] = b[k];
        dT[k + 1] = b[k + 1];
        db[k] = T[k];
        db[k + 1] = T[k + 1];
        const float2 r = __fmul2_rn(make_float2(T[k], T[k + 1]), make_float2(b[k], b[k + 1]));
        T[k] = r.x;
        T[k + 1] = r.y;
      }
      break;
    case 8:  // T / protected(b)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        db[k] = fabsf(b[k]) <= 1e-9f ? 0.0f : 1.0f;  // 0: the flat region
        b[k] = loose_denom(b[k]);
      }
      post = 1 | 2;
      break;
    case kOpReversed + 8:  // b / protected(T), as T' / b' with T' = b, b' = protected(T)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        dT[k] = fabsf(T[k]) <= 1e-9f ? 0.0f : 1.0f;
        const float d = loose_denom(T[k]);
        T[k] = b[k];
        b[k] = d;
      }
      post = 1 | 2;
      break;
    case 10:
    case 11: {
      const int qoff = (op == 11) ? 1 : 0;
      bool slow = false;
#pragma unroll
      for (int k = 0; k < DPT; ++k) slow |= !sincos_fast_ok(T[k]);
      if (slow) {
        float t_[DPT], d_[DPT];
#pragma unroll
        for (int k = 0; k < DPT; ++k) t_[k] = T[k];
        tan_sincos_cold<DPT>(t_, d_, qoff);
#pragma unroll
        for (int k = 0; k < DPT; ++k) {
          T[k] = t_[k];
          dT[k] = d_[k];
        }
      } else {
#pragma unroll
        for (int k = 0; k < DPT; k += 2) {
          SinCosParts p0, p1;
          sincos_parts2(make_float2(T[k], T[k + 1]), p0, p1);
          // sin with sin(-0) = -0, as sr_sincosf returns it
          const float s0 = T[k] == 0.0f ? T[k] : sincos_pick(p0, 0);
          const float s1 = T[k + 1] == 0.0f ? T[k + 1] : sincos_pick(p1, 0);
          const float c0 = sincos_pick(p0, 1), c1 = sincos_pick(p1, 1);
          T[k] = qoff ? c0 : s0;
          T[k + 1] = qoff ? c1 : s1;
          dT[k] = qoff ? -s0 : c0;
          dT[k + 1] = qoff ? -s1 : c1;
        }
      }
      break;
    }
    case kOpExpClamp:
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        const float x = T[k];
        const float o = expf(fminf(x, 80.0f));
        dT[k] = (x < 80.0f) ? o : 0.0f;
        T[k] = o;
      }
      break;
    case 22:  // protected log: -1e9 at 0, else log|x|; derivative 0 at 0, else 1/x
#pragma unroll
      for (int k = 0; k < DPT; k += 2) {
        const float x0 = T[k], x1 = T[k + 1];
        const float2 l = sr_log_nonneg2(fabsf(x0), fabsf(x1));
        b[k] = x0;
        b[k + 1] = x1;
        T[k] = x0 == 0.0f ? -1e9f : l.x;
        T[k + 1] = x1 == 0.0f ? -1e9f : l.y;
      }
      post = 2;
      break;
    case 27:  // sqrt|x|: derivative 0 at 0, else sign(x) / (2 out)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        const float x = T[k];
        const float o = __fsqrt_rn(fabsf(x));
        b[k] = x == 0.0f ? 1.0f : 2.0f * o;  // at 0: sign 0 times 1
        dT[k] = signf(x);                     // times 1 / (2 out) below
        T[k] = o;
      }
      post = 2;
      break;
    default: {
      float t_[DPT], b_[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        t_[k] = T[k];
        b_[k] = b[k];
      }
      if (live) {
        float d1[DPT], d2[DPT];
        tan_op_cold<DPT>(op, t_, b_, d1, d2);
#pragma unroll
        for (int k = 0; k < DPT; ++k) {
          dT[k] = d1[k];
          db[k] = d2[k];
        }
      } else {
        apply_op_cold<DPT>(op, t_, b_);
      }
#pragma unroll
      for (int k = 0; k < DPT; ++k) T[k] = t_[k];
      break;
    }
  }
  if (post & 1) {
#pragma unroll
    for (int k = 0; k < DPT; ++k) T[k] = __fdiv_rn(T[k], b[k]);
  }
  if ((post & 2) && live) {
    float rc[DPT];
#pragma unroll
    for (int k = 0; k < DPT; ++k) rc[k] = __frcp_rn(b[k]);
    // Partials from the reciprocal (the reverse-mode routines' formulas).
    if (op == 8) {  // d/dT = 1/den, d/db = -out/den (0 in the flat region)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        db[k] = db[k] == 0.0f ? 0.0f : __fmul_rn(-T[k], rc[k]);
        dT[k] = rc[k];
      }
    } else if (op == kOpReversed + 8) {  // d/db = 1/den, d/dT = -out/den
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        dT[k] = dT[k] == 0.0f ? 0.0f : __fmul_rn(-T[k], rc[k]);
        db[k] = rc[k];
      }
    } else if (op == 22) {
#pragma unroll
      for (int k = 0; k < DPT; ++k) dT[k] = b[k] == 0.0f ? 0.0f : rc[k];
    } else {  // 27
#pragma unroll
      for (int k = 0; k < DPT; ++k) dT[k] = dT[k] * rc[k];
    }
  }
}

// One program over the warp's tile: values in T (registers), tangents in the
// warp's shared-memory rows tan[c][TILE] (c = constant index; the loops over
// a mask's set bits index them directly, one copy of each update in the code).
// A spilled subtree's tangents stay in their rows: the instructions that
// follow it (up to the one that takes it back as operand b) belong to other
// subtrees, whose constants are other constants, so they never write its
// rows; the instruction that consumes it multiplies them by db in place.
template <int DPT>
__device__ __forceinline__ void run_tangent_program(const Instr *__restrict__ code,
                                                    const uint32_t *__restrict__ tmask, int len,
                                                    const float *xs, int xrs,
                                                    const SpillStack &st, int lane, float *tan,
                                                    float (&T)[DPT]) {
  constexpr int TILE = 32 * DPT;
  uint4 ins = ldg_instr(code);
  uint32_t m = __ldg(tmask);
  for (int i = 0; i < len; ++i) {
    // The code and mask buffers end with a padding entry, so these prefetches
    // of the next entry are always in bounds.
    const uint4 nxt = ldg_instr(code + i + 1);
    const uint32_t mn = __ldg(tmask + i + 1);
    const uint32_t w = ins.x;
    const uint32_t A = m & 0xFFu, B = (m >> 8) & 0xFFu;
    if (w & (kLoadBit | kSpillBit)) {
      if (instr_spill(w)) spill_store<DPT>(st, instr_spill_slot(w), lane, T);
      if (instr_load(w))
        load_leaf<DPT, false>(instr_leaf_kind(w), ins.y, T, xs, xrs, lane, nullptr, 0, 0);
    }
    float b[DPT], dT[DPT], db[DPT];
    const uint32_t bk = instr_b_kind(w);
    if (bk != kBNone) load_operand<DPT, false>(bk, ins.z, b, xs, xrs, st, lane, nullptr, 0, 0);
    int dk, bkn;
    tan_apply<DPT>(instr_op(w), (A | B) != 0, T, b, dT, db, dk, bkn);
    if (A | B) {
      // Constants that enter here (a constant leaf, a constant operand b)
      // start from tangent 1; rows of an operator whose partial is exactly 1
      // stay as they are.  (One loop for both masks: a second copy of it
      // costs more in instruction-cache misses than its branches.)
      const uint32_t fresh = (m & kTanLoadConst ? A : 0u) | (bk == kBC ? B : 0u);
      for (uint32_t u = A | B; u; u &= u - 1) {
        const int c = __ffs(u) - 1;
        const bool on_b = (B >> c) & 1u;
        const int kind = on_b ? bkn : dk;
        const bool is_fresh = (fresh >> c) & 1u;
        if (kind == kDOne && !is_fresh) continue;
        float *row = tan + c * TILE;
        float tv[DPT];
        if (is_fresh) {
#pragma unroll
          for (int k = 0; k < DPT; ++k) tv[k] = 1.0f;
        } else {
          lds_vec<DPT>(row, lane, tv);
        }
        if (kind == kDNeg) {
#pragma unroll
          for (int k = 0; k < DPT; ++k) tv[k] = -tv[k];
        } else if (kind == kDGen) {
          if (on_b)
            kill_mul<DPT>(tv, db);
          else
            kill_mul<DPT>(tv, dT);
        }
        sts_vec<DPT>(row, lane, tv);
      }
    }
    ins = nxt;
    m = mn;
  }
}

// MAXW / MINB: at most MAXW evaluating warps, at least MINB resident blocks
// per SM.
template <int DPT, int MAXW, int MINB>
__global__ void __launch_bounds__((MAXW + 1) * 32, MINB) tan_kernel(const TanArgs a) {
  constexpr int TILE = 32 * DPT;
  const EvalArgs &p = a.e;
  const int K = a.K;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int W = p.W;
  const int rows = p.V + 1;
  const int span = p.span;
  float *xbuf = reinterpret_cast<float *>(smem_raw);
  float *sreg = xbuf + static_cast<size_t>(kBufs) * rows * span;
  float *tans = sreg + static_cast<size_t>(W) * p.s_smem * TILE;  // [W][K][TILE]
  double *gsm = reinterpret_cast<double *>(tans + static_cast<size_t>(W) * K * TILE);  // [W][K][32]
  ItemDesc *desc = reinterpret_cast<ItemDesc *>(gsm + static_cast<size_t>(W) * K * 32);
  uint64_t *full = reinterpret_cast<uint64_t *>(desc + kBufs);
  uint64_t *empty = full + kBufs;
  SpanPart *part = reinterpret_cast<SpanPart *>(empty + kBufs);
  GroupAcc *gacc = reinterpret_cast<GroupAcc *>(part + kBufs * p.G);
  double *gpart = reinterpret_cast<double *>(gacc + p.G);  // [kBufs][G][K]
  double *ggacc = gpart + static_cast<size_t>(kBufs) * p.G * K;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kBufs; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], static_cast<uint32_t>(W));
    }
    mbar_init_fence();
  }
  __syncthreads();

  const int k_spans = p.span_per_item;
  const int n_items = p.n_groups * ((p.n_spans + k_spans - 1) / k_spans);
  if (warp == W) {
    if (lane == 0)
      run_producer<true>(p.n_groups, n_items, k_spans, p.n_spans, p.work_counter, p.error, p.X,
                         p.ldx, rows, span, xbuf, desc, full, empty,
                         FoldArgs{part, gacc, p.partial, p.G, p.E, a.n_valid, K, gpart, ggacc,
                                  a.gout, a.const_off, a.const_cnt, a.C});
    return;
  }

  SpillStack st;  // value spill slots
  st.ss = sreg + static_cast<size_t>(warp) * p.s_smem * TILE;
  st.gs = p.spill + (static_cast<size_t>(blockIdx.x) * W + warp) *
                        static_cast<size_t>(p.smax - p.s_smem) * TILE;
  st.s_smem = p.s_smem;
  float *tan = tans + static_cast<size_t>(warp) * K * TILE;
  double *gl = gsm + static_cast<size_t>(warp) * K * 32;  // per-lane gradient sums
  const int tiles = span / TILE;
  uint32_t buf = 0, phase = 0;
  for (;;) {
    if (!mbar_wait(&full[buf], phase, p.error)) return;
    const ItemDesc d = desc[buf];
    if (d.item < 0) return;
    const float *xb = xbuf + static_cast<size_t>(buf) * rows * span;
    const int64_t dp_span = static_cast<int64_t>(d.span) * span;
    for (;;) {
      int j = 0;
      if (lane == 0) j = atomicAdd(&desc[buf].claim, 1);
      j = __shfl_sync(0xffffffffu, j, 0);
      if (j >= p.G) break;
      const int e = p.group_expr[static_cast<int64_t>(d.group) * p.G + j];
      if (e < 0) break;  // groups are padded at their end only
      const Instr *code = p.code + p.code_off[e];
      const uint32_t *tm = a.tmask + p.code_off[e];
      const int len = p.code_len[e];
      const int nconst = min(a.const_cnt[e], K);
      double acc = 0.0;
      int cnt = 0;
      for (int c = 0; c < nconst; ++c) gl[c * 32 + lane] = 0.0;
      for (int t = 0; t < tiles; ++t) {
        const int64_t dp0 = dp_span + static_cast<int64_t>(t) * TILE;
        if (dp0 >= p.N) break;  // tail of the last span
        const float *xs = xb + t * TILE;
        float T[DPT];
        run_tangent_program<DPT>(code, tm, len, xs, span, st, lane, tan, T);
        float y[DPT], sd[DPT];
        lds_vec<DPT>(xs + p.V * span, lane, y);
        const bool full_tile = dp0 + TILE <= p.N;  // warp-uniform
        float s = 0.0f, c = 0.0f;  // Kahan over the lane's DPT values
        int nv = 0;
        float dfs[DPT], dsq[DPT];
#pragma unroll
        for (int k = 0; k < DPT; k += 2) {
          const float2 df2 = __fadd2_rn(make_float2(T[k], T[k + 1]), make_float2(-y[k], -y[k + 1]));
          const float2 sq2 = __fmul2_rn(df2, df2);
          dfs[k] = df2.x;
          dfs[k + 1] = df2.y;
          dsq[k] = sq2.x;
          dsq[k + 1] = sq2.y;
        }
#pragma unroll
        for (int k = 0; k < DPT; ++k) {
          const bool valid =
              (full_tile || dp0 + (k / 4) * 128 + lane * 4 + (k % 4) < p.N) && isfinite(T[k]);
          const float df = dfs[k];
          const float sq = valid ? dsq[k] : 0.0f;
          nv += valid ? 1 : 0;
          const float yk = __fsub_rn(sq, c);
          const float tt = __fadd_rn(s, yk);
          c = __fsub_rn(__fsub_rn(tt, s), yk);
          s = tt;
          sd[k] = valid ? 2.0f * df : 0.0f;
        }
        double tile_sum = static_cast<double>(s) - static_cast<double>(c);
        if (!isfinite(tile_sum)) {
          float tc[DPT], yc[DPT];
#pragma unroll
          for (int k = 0; k < DPT; ++k) {
            tc[k] = T[k];
            yc[k] = y[k];
          }
          tile_sum = tile_sum_fp64<DPT>(tc, yc, full_tile, dp0, lane, p.N);
        }
        acc += tile_sum;
        cnt += nv;
        // d MSE / d c (times the count): seed * t_c, zero where the seed is;
        // each lane adds its DPT products in order in FP32, FP64 from there
        // on (an FP32 lane sum overflows only for products beyond ~4e37).
        for (int cc = 0; cc < nconst; ++cc) {
          float tv[DPT];
          lds_vec<DPT>(tan + cc * TILE, lane, tv);
#pragma unroll
          for (int k = 0; k < DPT; k += 2) {
            const float2 r = __fmul2_rn(make_float2(sd[k], sd[k + 1]), make_float2(tv[k], tv[k + 1]));
            tv[k] = sd[k] == 0.0f ? 0.0f : r.x;
            tv[k + 1] = sd[k + 1] == 0.0f ? 0.0f : r.y;
          }
          float g = tv[0];
#pragma unroll
          for (int k = 1; k < DPT; ++k) g = __fadd_rn(g, tv[k]);
          gl[cc * 32 + lane] += static_cast<double>(g);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      }
      double *gp = gpart + (static_cast<size_t>(buf) * p.G + j) * K;
      for (int cc = 0; cc < K; ++cc) {
        double g = cc < nconst ? gl[cc * 32 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) gp[cc] = g;
      }
      if (lane == 0) part[static_cast<size_t>(buf) * p.G + j] = SpanPart{acc, cnt, e};
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[buf]);
    if (++buf == kBufs) {
      buf = 0;
      phase ^= 1u;
    }
  }
}

// mse and grad of the expressions of one tangent launch: the span groups'
// double-double MSE sums and FP64 gradient sums added in span-group order;
// the FP64 sums themselves go to sums ((sum, count) per expression) and gsum
// (per constant).
__global__ void tan_finalize_kernel(const double2 *__restrict__ partial,
                                    const double *__restrict__ gout, int n_groups, int E,
                                    int64_t C, const int32_t *__restrict__ exprs, int n_exprs,
                                    const int64_t *__restrict__ const_off,
                                    const int32_t *__restrict__ const_cnt, int K,
                                    float *__restrict__ mse, float *__restrict__ grad,
                                    double *__restrict__ gsum, double2 *__restrict__ sums) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_exprs) return;
  const int e = exprs[q];
  double hi = 0.0, lo = 0.0, cnt = 0.0;
  for (int k = 0; k < n_groups; ++k) {
    const double2 *pp = partial + 2 * (static_cast<int64_t>(k) * E + e);
    const double2 v = pp[0];
    dd_add(hi, lo, v.x);
    dd_add(hi, lo, v.y);
    cnt += pp[1].x;
  }
  const double s = isfinite(hi) ? __dadd_rn(hi, lo) : hi;
  mse[e] = (cnt > 0.0) ? static_cast<float>(s / cnt) : qnan();
  sums[e] = make_double2(s, cnt);
  const int nc = min(const_cnt[e], K);
  const int64_t o = const_off[e];
  for (int c = 0; c < nc; ++c) {
    double g = 0.0;
    for (int k = 0; k < n_groups; ++k) g += gout[static_cast<int64_t>(k) * C + o + c];
    gsum[o + c] = g;
    grad[o + c] = (cnt > 0.0) ? static_cast<float>(g / cnt) : qnan();
  }
}

template <int DPT, int MAXW, int MINB>
const void *tan_fn() {
  return reinterpret_cast<const void *>(&tan_kernel<DPT, MAXW, MINB>);
}

// Launch shapes: 8 datapoints per thread, one block per SM with as many
// evaluating warps as the register file holds beside the producer warp: up
// to 19 (96 registers per thread) for up to 4 tangent rows, 15 (120) for more.
// The kernel is latency-bound on dependent chains; one large block keeps
// more warps resident than two blocks of 8 + 1 or 7 + 1 warps did (16 and 12
// evaluating warps per SM).
constexpr int kTanDpt = 8;
constexpr int tan_max_warps(int K) { return K <= 4 ? 19 : 15; }
const void *select_tan(int K) {
  return K <= 4 ? tan_fn<kTanDpt, 19, 1>() : tan_fn<kTanDpt, 15, 1>();
}

}  // namespace

int tan_dpt() { return kTanDpt; }
int tan_warps(int K) { return tan_max_warps(K); }

size_t tan_smem_bytes(int K, int W, int V, int s_smem, int span, int G) {
  const size_t tile = 32u * static_cast<size_t>(kTanDpt);
  return (static_cast<size_t>(kBufs) * (V + 1) * span +
          static_cast<size_t>(W) * (s_smem + K) * tile) * sizeof(float) +
         static_cast<size_t>(W) * K * 32 * sizeof(double) +
         kBufs * sizeof(ItemDesc) + 2 * kBufs * sizeof(uint64_t) +
         static_cast<size_t>(G) * (kBufs * sizeof(SpanPart) + sizeof(GroupAcc)) +
         static_cast<size_t>(G) * K * (kBufs + 1) * sizeof(double);
}

cudaError_t tan_configure(int K, size_t smem, int W, int *blocks_per_sm) {
  const void *fn = select_tan(K);
  if (W < 1 || W > tan_max_warps(K)) return cudaErrorInvalidValue;
  const cudaError_t err = raise_smem_limit(fn, smem);
  if (err != cudaSuccess) return err;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, (W + 1) * 32, smem);
}

cudaError_t tan_set_smem_limit(int K, size_t smem) {
  return raise_smem_limit(select_tan(K), smem);
}

cudaError_t launch_tangent(const TanArgs &args, int blocks, size_t smem, cudaStream_t stream) {
  if (args.K < 1 || args.K > kMaxTangentConsts) return cudaErrorInvalidValue;
  const void *fn = select_tan(args.K);
  if (args.e.W < 1 || args.e.W > tan_max_warps(args.K)) return cudaErrorInvalidValue;
  void *params[] = {const_cast<TanArgs *>(&args)};
  return cudaLaunchKernel(fn, dim3(blocks), dim3((args.e.W + 1) * 32), params, smem, stream);
}

cudaError_t launch_tan_finalize(const double2 *partial, const double *gout, int n_groups, int E,
                                int64_t C, const int32_t *exprs, int n_exprs,
                                const int64_t *const_off, const int32_t *const_cnt, int K,
                                float *mse, float *grad, double *gsum, double2 *sums,
                                cudaStream_t stream) {
  if (n_exprs <= 0) return cudaSuccess;
  tan_finalize_kernel<<<(n_exprs + 127) / 128, 128, 0, stream>>>(
      partial, gout, n_groups, E, C, exprs, n_exprs, const_off, const_cnt, K, mse, grad, gsum,
      sums);
  return cudaGetLastError();
}

}  // namespace sr
