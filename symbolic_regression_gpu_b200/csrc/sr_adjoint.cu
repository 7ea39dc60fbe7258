// sr_adjoint.cu — reverse-mode adjoint of the population MSE with respect to
// every expression's constants, and on-device Adam over those constants.
// (No reference counterpart: the reference evaluates MSE only.)
//
//   adj_kernel<GTAPE>       fused forward + backward per tile.  Same work
//                           decomposition as interp_kernel (a producer thread
//                           streaming X spans into shared memory, warps
//                           claiming expressions of a group).  Per tile a warp
//                           (1) runs the program forward; each instruction's
//                           dispatch computes its value and its local partials
//                           (d out / d T, and d out / d b when b is a constant
//                           or a spilled subtree), and the partials go to the
//                           warp's Jacobian tape;
//                           (2) forms the squared error and the seed
//                           2 (pred - y) for valid datapoints (0 otherwise);
//                           (3) sweeps the tape backwards: an adjoint
//                           accumulator gT, adjoint spill slots mirroring the
//                           forward ones, and per-lane FP64 accumulators for
//                           the constants.  The sweep has no operator code at
//                           all and stops at the lowest instruction that holds
//                           a constant.
//                           The tape lives in shared memory, or per warp in
//                           global scratch (GTAPE) for programs whose tape
//                           does not fit.  At the end of a span the constant
//                           accumulators are reduced over the warp and added
//                           to grad_acc (FP64 atomics).
//   grad_finalize_kernel    mse = sum / count per expression and
//                           grad = grad_acc / count per constant.
//   adam_kernel             one Adam step per constant, written back into the
//                           bytecode immediates (and the constant vector).
//
// Derivative conventions at non-smooth points (the FP64 gradient oracle uses
// the same): |x| and sqrt|x| have derivative 0 at 0; the protected regions of
// LOOSE_DIV / LOOSE_INV (|d| <= 1e-9) and the clamp of exp (x >= 80) have
// derivative 0; LOOSE_LOG is 0 at 0; MIN / MAX route the adjoint to the
// operand they return (the first on ties, the non-NaN one if one is NaN);
// 0^0 of LOOSE_POW has derivative 0.  A zero adjoint times an infinite or NaN
// partial is zero ("strong zero"), so datapoints and branches that do not
// reach the result contribute exactly nothing.  Values are computed exactly as
// the forward interpreter computes them (same routines, same rounding), so the
// MSE of a gradient call equals the forward MSE up to summation order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_adjoint.hpp"
#include "sr_device.cuh"
#include "sr_grad_ops.cuh"

namespace sr {
namespace {

#ifndef SR_ADJ_DPT
#define SR_ADJ_DPT 4
#endif
constexpr int kAdjDpt = SR_ADJ_DPT;  // datapoints per thread (4 or 8)
static_assert(kAdjDpt == 4 || kAdjDpt == 8, "adjoint DPT 4 or 8");

__device__ __forceinline__ float strong_mul(float g, float d) { return g == 0.0f ? 0.0f : g * d; }


// Per-lane FP64 gradient accumulator of constant c: += sum of g over DPT,
// summed in FP64 (per-datapoint adjoints can be near the FP32 range, where an
// FP32 partial sum would overflow).  Indices at or above the expression's
// constant count (none are emitted) are ignored rather than written out of
// bounds.
template <int DPT>
__device__ __forceinline__ void gacc_add(double *gacc, uint32_t c, uint32_t nconst, int lane,
                                         const float (&g)[DPT]) {
  if (c >= nconst) return;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < DPT; ++k) s += static_cast<double>(g[k]);
  gacc[c * 32 + lane] += s;
}

__device__ __forceinline__ bool needs_db(uint32_t bk) { return bk == kBC || bk == kBS; }

// One forward instruction: [spill] [T = leaf] [b = operand] T = op(T, b),
// with its local partials in dT / db.  Returns the operand kind of b.
template <int DPT>
__device__ __forceinline__ uint32_t fwd_instr(const uint4 ins, float (&T)[DPT], float (&dT)[DPT],
                                              float (&db)[DPT], const float *xs, int span,
                                              const SpillStack &st, int lane, const EvalArgs &p,
                                              int64_t dp0) {
  const uint32_t w = ins.x;
  if (instr_spill(w)) spill_store<DPT>(st, instr_spill_slot(w), lane, T);
  if (instr_load(w))
    load_leaf<DPT>(instr_leaf_kind(w), ins.y, T, xs, span, lane, p.cache, p.ldc, dp0);
  float b[DPT];
  const uint32_t bk = instr_b_kind(w);
  if (bk != kBNone) load_operand<DPT>(bk, ins.z, b, xs, span, st, lane, p.cache, p.ldc, dp0);
  apply_op_grad<DPT>(instr_op(w), T, b, dT, db);
  return bk;
}

// One backward instruction: gT is the adjoint of the instruction's output
// on entry and of its input accumulator on exit; db is read only when the
// operand b is a constant or a spilled subtree.  Adjoint spill slots: `adj`.
template <int DPT>
__device__ __forceinline__ void bwd_instr(const uint4 ins, float (&gT)[DPT], const float *dT_at,
                                          const float *db_at, const SpillStack &adj,
                                          double *gacc, uint32_t nconst, int lane) {
  const uint32_t w = ins.x;
  const uint32_t bk = instr_b_kind(w);
  float dT[DPT], gi[DPT];
  lds_vec<DPT>(dT_at, lane, dT);
#pragma unroll
  for (int k = 0; k < DPT; ++k) gi[k] = strong_mul(gT[k], dT[k]);
  if (needs_db(bk)) {
    float db[DPT], gb[DPT];
    lds_vec<DPT>(db_at, lane, db);
#pragma unroll
    for (int k = 0; k < DPT; ++k) gb[k] = strong_mul(gT[k], db[k]);
    if (bk == kBC)
      gacc_add<DPT>(gacc, (ins.w >> 10) & 0x3FFu, nconst, lane, gb);
    else
      spill_store<DPT>(adj, ins.z, lane, gb);
  }
  if (instr_load(w)) {
    if (instr_leaf_kind(w) == kLeafC) gacc_add<DPT>(gacc, ins.w & 0x3FFu, nconst, lane, gi);
    if (instr_spill(w)) {
      spill_load<DPT>(adj, instr_spill_slot(w), lane, gT);
    } else {
#pragma unroll
      for (int k = 0; k < DPT; ++k) gT[k] = 0.0f;
    }
  } else {
#pragma unroll
    for (int k = 0; k < DPT; ++k) gT[k] = gi[k];
  }
}

// GTAPE: tapes in per-warp global scratch instead of shared memory.
// RECOMP: recompute mode.  Checkpoint mode keeps the partials of every
// instruction in [lo, len) (tape: dT entries, then db entries).  Recompute
// mode splits the program into segments of kSeg instructions; the forward
// pass saves T and every forward spill slot at each segment start (after the
// first) and writes the partials of the last segment only; the backward
// sweep replays each earlier segment from its checkpoint into the segment
// tape before sweeping it.  Recompute tape per warp: segment tape (2 seg_cap
// entries, seg_cap = min(kSeg, longest program of the launch)), adjoint
// spill slots (smax), checkpoints ((segments - 1) x (1 + smax)).
constexpr int kSeg = 16;

template <bool GTAPE, bool RECOMP>
__global__ void __launch_bounds__((kMaxWarps + 1) * 32, 1) adj_kernel(const AdjArgs a) {
  constexpr int DPT = kAdjDpt;
  constexpr int TILE = 32 * DPT;
  const EvalArgs &p = a.e;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int W = p.W;
  const int rows = p.V + 1;
  const int span = p.span;
  float *xbuf = reinterpret_cast<float *>(smem_raw);
  float *sreg = xbuf + static_cast<size_t>(kBufs) * rows * span;
  float *tapes = sreg + static_cast<size_t>(W) * p.s_smem * TILE;
  const size_t smem_tape = GTAPE ? 0 : static_cast<size_t>(W) * a.tape_len * TILE;
  double *gaccs = reinterpret_cast<double *>(tapes + smem_tape);
  ItemDesc *desc = reinterpret_cast<ItemDesc *>(gaccs + static_cast<size_t>(W) * a.gmax * 32);
  uint64_t *full = reinterpret_cast<uint64_t *>(desc + kBufs);
  uint64_t *empty = full + kBufs;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kBufs; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], static_cast<uint32_t>(W));
    }
    mbar_init_fence();
  }
  __syncthreads();

  const int n_items = p.n_groups * p.n_spans;
  if (warp == W) {
    if (lane == 0)
      run_producer<false>(p.n_groups, n_items, 1, p.n_spans, p.work_counter, p.error, p.X,
                          p.ldx, rows, span, xbuf, desc, full, empty, FoldArgs{});
    return;
  }

  SpillStack st;  // forward spill slots
  st.ss = sreg + static_cast<size_t>(warp) * p.s_smem * TILE;
  st.gs = p.spill + (static_cast<size_t>(blockIdx.x) * W + warp) *
                        static_cast<size_t>(p.smax - p.s_smem) * TILE;
  st.s_smem = p.s_smem;
  float *tape = GTAPE ? a.gtape + (static_cast<size_t>(blockIdx.x) * W + warp) *
                                      static_cast<size_t>(a.tape_len) * TILE
                      : tapes + static_cast<size_t>(warp) * a.tape_len * TILE;
  // Adjoint spill slots: the forward slots in checkpoint mode (forward values
  // are no longer needed in the sweep); a region of the tape in recompute
  // mode (the replay needs the forward slots).
  SpillStack adj = st;
  float *ckpt = nullptr;
  if (RECOMP) {
    adj.ss = tape + 2 * a.seg_cap * TILE;
    adj.gs = adj.ss;
    adj.s_smem = p.smax;
    ckpt = adj.ss + static_cast<size_t>(p.smax) * TILE;
  }
  double *gacc = gaccs + static_cast<size_t>(warp) * a.gmax * 32;
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
      if (e < 0) break;
      const Instr *code = p.code + p.code_off[e];
      const int len = p.code_len[e];
      const int lo = a.bwd_lo[e];  // lowest instruction holding a constant (len: none)
      const uint32_t nconst = static_cast<uint32_t>(a.const_cnt[e]);
      // Checkpoint: partials of [t_lo, len).  Recompute: of the last segment.
      const int last_seg = RECOMP ? ((len - 1) / kSeg) * kSeg : 0;
      const int t_lo = RECOMP ? max(lo, last_seg) : lo;
      const int db_base = RECOMP ? a.seg_cap : len - lo;
      for (uint32_t c = 0; c < nconst; ++c) gacc[c * 32 + lane] = 0.0;
      double acc = 0.0;
      int cnt = 0;
      for (int t = 0; t < tiles; ++t) {
        const int64_t dp0 = dp_span + static_cast<int64_t>(t) * TILE;
        if (dp0 >= p.N) break;
        const float *xs = xb + t * TILE;
        // ---- forward: values and local partials ----
        float T[DPT];
        int kb = 0;
        {
          uint4 ins = ldg_instr(code);
          for (int i = 0; i < len; ++i) {
            const uint4 nxt = ldg_instr(code + i + 1);
            if (RECOMP && i > 0 && i % kSeg == 0 && i < last_seg && i + kSeg > lo) {
              // Checkpoint at the start of a segment the sweep replays (not
              // the last one, whose partials the forward pass keeps, and only
              // segments that reach lo).
              float *ck = ckpt + static_cast<size_t>(i / kSeg - 1) * (1 + p.smax) * TILE;
              sts_vec<DPT>(ck, lane, T);
              for (int sl = 0; sl < p.smax; ++sl) {
                float v[DPT];
                spill_load<DPT>(st, static_cast<uint32_t>(sl), lane, v);
                sts_vec<DPT>(ck + (1 + sl) * TILE, lane, v);
              }
            }
            float dT[DPT], db[DPT];
            const uint32_t bk = fwd_instr<DPT>(ins, T, dT, db, xs, span, st, lane, p, dp0);
            if (i >= t_lo) {
              sts_vec<DPT>(tape + (i - (RECOMP ? last_seg : lo)) * TILE, lane, dT);
              if (needs_db(bk)) {
                sts_vec<DPT>(tape + (db_base + kb) * TILE, lane, db);
                ++kb;
              }
            }
            ins = nxt;
          }
        }
        // ---- epilogue: squared error and seed ----
        float gT[DPT];
        {
          float y[DPT];
          lds_vec<DPT>(xs + p.V * span, lane, y);
          const bool full_tile = dp0 + TILE <= p.N;
          float s = 0.0f, c = 0.0f;
          int nv = 0;
#pragma unroll
          for (int k = 0; k < DPT; ++k) {
            const bool valid =
                (full_tile || dp0 + (k / 4) * 128 + lane * 4 + (k % 4) < p.N) && isfinite(T[k]);
            const float df = __fsub_rn(T[k], y[k]);
            const float sq = valid ? __fmul_rn(df, df) : 0.0f;
            nv += valid ? 1 : 0;
            const float yk = __fsub_rn(sq, c);
            const float tt = __fadd_rn(s, yk);
            c = __fsub_rn(__fsub_rn(tt, s), yk);
            s = tt;
            gT[k] = valid ? 2.0f * df : 0.0f;
          }
          double tile_sum = static_cast<double>(s) - static_cast<double>(c);
          if (!isfinite(tile_sum)) {
            tile_sum = 0.0;
#pragma unroll
            for (int k = 0; k < DPT; ++k) {
              const bool valid = (full_tile || dp0 + (k / 4) * 128 + lane * 4 + (k % 4) < p.N) &&
                                 isfinite(T[k]);
              const float df = __fsub_rn(T[k], y[k]);
              tile_sum += valid ? static_cast<double>(__fmul_rn(df, df)) : 0.0;
            }
          }
          acc += tile_sum;
          cnt += nv;
        }
        // ---- backward sweep ----
        if (!RECOMP) {
          for (int i = len - 1; i >= lo; --i) {
            const uint4 ins = ldg_instr(code + i);
            if (needs_db(instr_b_kind(ins.x))) --kb;
            bwd_instr<DPT>(ins, gT, tape + (i - lo) * TILE, tape + (db_base + kb) * TILE, adj,
                           gacc, nconst, lane);
          }
        } else {
          for (int s0 = last_seg; s0 >= 0 && s0 + kSeg > lo; s0 -= kSeg) {
            const int s1 = min(len, s0 + kSeg);
            if (s0 != last_seg) {
              // Replay [s0, s1) from the checkpoint at s0 (s0 > 0: segment 0
              // starts with a leaf load and needs no state).
              if (s0 > 0) {
                const float *ck = ckpt + static_cast<size_t>(s0 / kSeg - 1) * (1 + p.smax) * TILE;
                lds_vec<DPT>(ck, lane, T);
                for (int sl = 0; sl < p.smax; ++sl) {
                  float v[DPT];
                  lds_vec<DPT>(ck + (1 + sl) * TILE, lane, v);
                  spill_store<DPT>(st, static_cast<uint32_t>(sl), lane, v);
                }
              }
              kb = 0;
              for (int i = s0; i < s1; ++i) {
                const uint4 ins = ldg_instr(code + i);
                float dT[DPT], db[DPT];
                const uint32_t bk = fwd_instr<DPT>(ins, T, dT, db, xs, span, st, lane, p, dp0);
                if (i >= lo) {
                  sts_vec<DPT>(tape + (i - s0) * TILE, lane, dT);
                  if (needs_db(bk)) {
                    sts_vec<DPT>(tape + (db_base + kb) * TILE, lane, db);
                    ++kb;
                  }
                }
              }
            }
            for (int i = s1 - 1; i >= max(s0, lo); --i) {
              const uint4 ins = ldg_instr(code + i);
              if (needs_db(instr_b_kind(ins.x))) --kb;
              bwd_instr<DPT>(ins, gT, tape + (i - s0) * TILE, tape + (db_base + kb) * TILE, adj,
                             gacc, nconst, lane);
            }
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      }
      if (lane == 0)
        p.partial[static_cast<int64_t>(d.span) * p.E + e] =
            make_double2(acc, static_cast<double>(cnt));
      const int64_t coff = a.const_off[e];
      for (uint32_t c = 0; c < nconst; ++c) {
        double g = gacc[c * 32 + lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) atomicAdd(&a.grad_acc[coff + c], g);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[buf]);
    if (++buf == kBufs) {
      buf = 0;
      phase ^= 1u;
    }
  }
}

__global__ void grad_finalize_kernel(const double2 *__restrict__ partial, int n_spans, int E,
                                     const int32_t *__restrict__ exprs, int n_exprs,
                                     const int64_t *__restrict__ const_off,
                                     const int32_t *__restrict__ const_cnt,
                                     const double *__restrict__ grad_acc, float *__restrict__ mse,
                                     float *__restrict__ grad, double2 *__restrict__ sums) {
  const int q_ = blockIdx.x * blockDim.x + threadIdx.x;
  if (q_ >= n_exprs) return;
  const int e = exprs[q_];
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n_spans; ++k) {
    const double2 q = partial[static_cast<int64_t>(k) * E + e];
    s += q.x;
    c += q.y;
  }
  if (mse) mse[e] = (c > 0.0) ? static_cast<float>(s / c) : qnan();
  if (sums) sums[e] = make_double2(s, c);
  const int64_t o = const_off[e];
  for (int k = 0; k < const_cnt[e]; ++k)
    grad[o + k] = (c > 0.0) ? static_cast<float>(grad_acc[o + k] / c) : qnan();
}

// One Adam step per constant.  Non-finite gradients leave the constant and
// the moments unchanged.  The new value is written into the bytecode
// immediate that holds the constant (word loc & 1 ? b : a of instruction
// loc >> 1) and into consts[].
__global__ void adam_kernel(int64_t C, const float *__restrict__ grad, float *__restrict__ m,
                            float *__restrict__ v, float *__restrict__ consts,
                            const int64_t *__restrict__ loc, Instr *__restrict__ code, int step,
                            float lr, float beta1, float beta2, float eps) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const float g = grad[c];
  if (!isfinite(g)) return;
  const float mc = beta1 * m[c] + (1.0f - beta1) * g;
  const float vc = beta2 * v[c] + (1.0f - beta2) * g * g;
  m[c] = mc;
  v[c] = vc;
  const float bc1 = 1.0f - powf(beta1, static_cast<float>(step));
  const float bc2 = 1.0f - powf(beta2, static_cast<float>(step));
  const float mhat = mc / bc1;
  const float vhat = vc / bc2;
  const float nv = consts[c] - lr * mhat / (sqrtf(vhat) + eps);
  consts[c] = nv;
  const int64_t l = loc[c];
  uint32_t *word = reinterpret_cast<uint32_t *>(code + (l >> 1)) + ((l & 1) ? 2 : 1);
  *word = __float_as_uint(nv);
}

}  // namespace

size_t adj_smem_bytes(int W, int V, int s_smem, int span, int tape_len, int gmax,
                      bool global_tape) {
  const size_t tile = 32u * kAdjDpt;
  const size_t tape = global_tape ? 0 : static_cast<size_t>(W) * tape_len * tile;
  return (static_cast<size_t>(kBufs) * (V + 1) * span + static_cast<size_t>(W) * s_smem * tile +
          tape) * sizeof(float) +
         static_cast<size_t>(W) * gmax * 32 * sizeof(double) + kBufs * sizeof(ItemDesc) +
         2 * kBufs * sizeof(uint64_t);
}

static const void *adj_fn(bool global_tape, bool recompute) {
  if (recompute)
    return global_tape ? reinterpret_cast<const void *>(&adj_kernel<true, true>)
                       : reinterpret_cast<const void *>(&adj_kernel<false, true>);
  return global_tape ? reinterpret_cast<const void *>(&adj_kernel<true, false>)
                     : reinterpret_cast<const void *>(&adj_kernel<false, false>);
}

cudaError_t adj_set_smem_limit(bool global_tape, bool recompute, size_t smem) {
  return raise_smem_limit(adj_fn(global_tape, recompute), smem);
}

cudaError_t adj_configure(size_t smem, int W, bool global_tape, bool recompute,
                          int *blocks_per_sm) {
  const void *fn = adj_fn(global_tape, recompute);
  const cudaError_t err = raise_smem_limit(fn, smem);
  if (err != cudaSuccess) return err;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, (W + 1) * 32, smem);
}

cudaError_t launch_adjoint(const AdjArgs &args, bool recompute, int blocks, size_t smem,
                           cudaStream_t stream) {
  if (args.e.W < 1 || args.e.W > kMaxWarps) return cudaErrorInvalidValue;
  const void *fn = adj_fn(args.gtape != nullptr, recompute);
  void *params[] = {const_cast<AdjArgs *>(&args)};
  return cudaLaunchKernel(fn, dim3(blocks), dim3((args.e.W + 1) * 32), params, smem, stream);
}

int adj_segment() { return kSeg; }

cudaError_t launch_grad_finalize(const double2 *partial, int n_spans, int E,
                                 const int32_t *exprs, int n_exprs, const int64_t *const_off,
                                 const int32_t *const_cnt, const double *grad_acc, float *mse,
                                 float *grad, double2 *sums, cudaStream_t stream) {
  if (n_exprs <= 0) return cudaSuccess;
  grad_finalize_kernel<<<(n_exprs + 255) / 256, 256, 0, stream>>>(
      partial, n_spans, E, exprs, n_exprs, const_off, const_cnt, grad_acc, mse, grad, sums);
  return cudaGetLastError();
}

cudaError_t launch_adam(int64_t C, const float *grad, float *m, float *v, float *consts,
                        const int64_t *loc, Instr *code, int step, float lr, float beta1,
                        float beta2, float eps, cudaStream_t stream) {
  if (C <= 0) return cudaSuccess;
  adam_kernel<<<static_cast<unsigned>((C + 255) / 256), 256, 0, stream>>>(
      C, grad, m, v, consts, loc, code, step, lr, beta1, beta2, eps);
  return cudaGetLastError();
}

int adj_dpt() { return kAdjDpt; }

}  // namespace sr
