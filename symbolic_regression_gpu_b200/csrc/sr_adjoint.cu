// sr_adjoint.cu — reverse-mode adjoint of the population MSE with respect to
// every expression's constants, and on-device Adam over those constants.
// (No reference counterpart: the reference evaluates MSE only.)
//
//   adj_kernel<DPT=4>       fused forward + backward per tile.  Same work
//                           decomposition as interp_kernel (producer thread
//                           streaming X spans into shared memory, warps claiming
//                           expressions of a group).  Per tile a warp
//                           (1) runs the program forward, writing every
//                           instruction's output into its shared-memory tape;
//                           (2) forms the squared-error epilogue and the seed
//                           2 (pred - y) for valid datapoints (0 otherwise);
//                           (3) replays the program backwards: an adjoint
//                           accumulator gT and adjoint spill slots mirror the
//                           forward ones, each instruction's local partials
//                           come from its tape values, constant leaves
//                           accumulate gT * partial into per-lane FP64
//                           accumulators.  At the end of a span the
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
// reach the result contribute exactly nothing.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_adjoint.hpp"
#include "sr_device.cuh"

namespace sr {
namespace {

constexpr int kAdjDpt = 4;

__device__ __forceinline__ float strong_mul(float g, float d) { return g == 0.0f ? 0.0f : g * d; }

__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// Partials of f(u, v) for binary token `tok` (u first / left operand);
// `out` is f(u, v).  Transcendental pieces go through the out-of-line
// 4-wide routines.
template <int DPT>
__device__ __forceinline__ void binary_partials(int tok, const float (&u)[DPT],
                                                const float (&v)[DPT], const float (&out)[DPT],
                                                float (&du)[DPT], float (&dv)[DPT]) {
  switch (tok) {
    case 1:
#pragma unroll
      for (int k = 0; k < DPT; ++k) { du[k] = 1.0f; dv[k] = 1.0f; }
      break;
    case 2:
#pragma unroll
      for (int k = 0; k < DPT; ++k) { du[k] = 1.0f; dv[k] = -1.0f; }
      break;
    case 3:
#pragma unroll
      for (int k = 0; k < DPT; ++k) { du[k] = v[k]; dv[k] = u[k]; }
      break;
    case 4: {  // u / v
      float r[DPT];
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(r, h, v_rcp(quad<DPT>(v, h)));
#pragma unroll
      for (int k = 0; k < DPT; ++k) { du[k] = r[k]; dv[k] = -out[k] * r[k]; }
    } break;
    case 5: {  // u^v: du = v u^(v-1), dv = u^v ln u
      float vm1[DPT], pw[DPT], lg[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) vm1[k] = v[k] - 1.0f;
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) {
        unquad<DPT>(pw, h, v_pow(quad<DPT>(u, h), quad<DPT>(vm1, h)));
        unquad<DPT>(lg, h, v_log(quad<DPT>(u, h)));
      }
#pragma unroll
      for (int k = 0; k < DPT; ++k) { du[k] = v[k] * pw[k]; dv[k] = out[k] * lg[k]; }
    } break;
    case 6:  // fminf(u, v)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        const bool first = isnan(v[k]) || (!isnan(u[k]) && u[k] <= v[k]);
        du[k] = first ? 1.0f : 0.0f;
        dv[k] = first ? 0.0f : 1.0f;
      }
      break;
    case 7:  // fmaxf(u, v)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        const bool first = isnan(v[k]) || (!isnan(u[k]) && u[k] >= v[k]);
        du[k] = first ? 1.0f : 0.0f;
        dv[k] = first ? 0.0f : 1.0f;
      }
      break;
    case 8: {  // u / protected(v)
      float d[DPT], r[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) d[k] = loose_denom(v[k]);
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(r, h, v_rcp(quad<DPT>(d, h)));
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        du[k] = r[k];
        dv[k] = (fabsf(v[k]) <= 1e-9f) ? 0.0f : -out[k] * r[k];
      }
    } break;
    case 9: {  // (u == 0 && v == 0) ? 0 : |u|^v
      float a[DPT], vm1[DPT], pw[DPT], lg[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) { a[k] = fabsf(u[k]); vm1[k] = v[k] - 1.0f; }
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) {
        unquad<DPT>(pw, h, v_pow(quad<DPT>(a, h), quad<DPT>(vm1, h)));
        unquad<DPT>(lg, h, v_log(quad<DPT>(a, h)));
      }
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        const bool z = (u[k] == 0.0f && v[k] == 0.0f);
        du[k] = z ? 0.0f : v[k] * pw[k] * signf(u[k]);
        dv[k] = z ? 0.0f : out[k] * lg[k];
      }
    } break;
    default:
#pragma unroll
      for (int k = 0; k < DPT; ++k) { du[k] = 0.0f; dv[k] = 0.0f; }
      break;
  }
}

// Derivative of unary token `tok` at x, with out = f(x).
template <int DPT>
__device__ __forceinline__ void unary_partial(int tok, const float (&x)[DPT],
                                              const float (&out)[DPT], float (&dx)[DPT]) {
  switch (tok) {
    case 0:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = 1.0f;
      break;
    case 10:
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_cos(quad<DPT>(x, h)));
      break;
    case 11:
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_sin(quad<DPT>(x, h)));
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = -dx[k];
      break;
    case 12:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = 1.0f + out[k] * out[k];
      break;
    case 13:
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_cosh(quad<DPT>(x, h)));
      break;
    case 14:
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_sinh(quad<DPT>(x, h)));
      break;
    case 15:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = 1.0f - out[k] * out[k];
      break;
    case 16:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = out[k];
      break;
    case 17:
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_rcp(quad<DPT>(x, h)));
      break;
    case 18:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = -out[k] * out[k];
      break;
    case 19:
    case 20: {
      float t[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) t[k] = 1.0f - x[k] * x[k];
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(t, h, v_sqrt(quad<DPT>(t, h)));
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_rcp(quad<DPT>(t, h)));
      if (tok == 20) {
#pragma unroll
        for (int k = 0; k < DPT; ++k) dx[k] = -dx[k];
      }
    } break;
    case 21: {
      float t[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) t[k] = 1.0f + x[k] * x[k];
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_rcp(quad<DPT>(t, h)));
    } break;
    case 22:
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_rcp(quad<DPT>(x, h)));
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = (x[k] == 0.0f) ? 0.0f : dx[k];
      break;
    case 23:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = (fabsf(x[k]) <= 1e-9f) ? 0.0f : -out[k] * out[k];
      break;
    case 24:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = signf(x[k]);
      break;
    case 25:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = -1.0f;
      break;
    case 26: {
      float t[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) t[k] = 2.0f * out[k];
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_rcp(quad<DPT>(t, h)));
    } break;
    case 27: {
      float t[DPT];
#pragma unroll
      for (int k = 0; k < DPT; ++k) t[k] = 2.0f * out[k];
#pragma unroll
      for (int h = 0; h < DPT / 4; ++h) unquad<DPT>(dx, h, v_rcp(quad<DPT>(t, h)));
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = (x[k] == 0.0f) ? 0.0f : signf(x[k]) * dx[k];
    } break;
    case 32:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = (x[k] < 80.0f) ? out[k] : 0.0f;
      break;
    default:
#pragma unroll
      for (int k = 0; k < DPT; ++k) dx[k] = 0.0f;
      break;
  }
}

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
  double *gaccs = reinterpret_cast<double *>(tapes + static_cast<size_t>(W) * a.tape_len * TILE);
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
      run_producer(p.n_groups, n_items, p.work_counter, p.error, p.X, p.ldx, rows, span, xbuf,
                   desc, full, empty);
    return;
  }

  SpillStack st;  // forward spill slots, then adjoint spill slots
  st.ss = sreg + static_cast<size_t>(warp) * p.s_smem * TILE;
  st.gs = p.spill + (static_cast<size_t>(blockIdx.x) * W + warp) *
                        static_cast<size_t>(p.smax - p.s_smem) * TILE;
  st.s_smem = p.s_smem;
  float *tape = tapes + static_cast<size_t>(warp) * a.tape_len * TILE;
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
      const int nconst = a.const_cnt[e];
      for (int c = 0; c < nconst; ++c) gacc[c * 32 + lane] = 0.0;
      double acc = 0.0;
      int cnt = 0;
      for (int t = 0; t < tiles; ++t) {
        const int64_t dp0 = dp_span + static_cast<int64_t>(t) * TILE;
        if (dp0 >= p.N) break;
        const float *xs = xb + t * TILE;
        // ---- forward, recording every instruction's output ----
        float T[DPT];
        {
          uint4 ins = ldg_instr(code);
          for (int i = 0; i < len; ++i) {
            const uint4 nxt = ldg_instr(code + i + 1);
            const uint32_t w = ins.x;
            if (instr_spill(w)) spill_store<DPT>(st, instr_spill_slot(w), lane, T);
            if (instr_load(w))
              load_leaf<DPT>(instr_leaf_kind(w), ins.y, T, xs, span, lane, p.cache, p.ldc, dp0);
            float b[DPT];
            const uint32_t bk = instr_b_kind(w);
            if (bk != kBNone) load_operand<DPT>(bk, ins.z, b, xs, span, st, lane, p.cache, p.ldc, dp0);
            apply_op<DPT>(instr_op(w), T, b);
            sts_vec<DPT>(tape + i * TILE, lane, T);
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
        // ---- backward ----
        for (int i = len - 1; i >= 0; --i) {
          const uint4 ins = ldg_instr(code + i);
          const uint32_t w = ins.x;
          const uint32_t op = instr_op(w);
          const uint32_t bk = instr_b_kind(w);
          float to[DPT], ti[DPT], bv[DPT];
          lds_vec<DPT>(tape + i * TILE, lane, to);
          if (instr_load(w))
            load_leaf<DPT>(instr_leaf_kind(w), ins.y, ti, xs, span, lane, p.cache, p.ldc, dp0);
          else
            lds_vec<DPT>(tape + (i - 1) * TILE, lane, ti);
          if (bk == kBS) {
            lds_vec<DPT>(tape + ((ins.w >> 20) & 0x3FFu) * TILE, lane, bv);
          } else if (bk != kBNone) {
            load_operand<DPT>(bk, ins.z, bv, xs, span, st, lane, p.cache, p.ldc, dp0);
          } else {
#pragma unroll
            for (int k = 0; k < DPT; ++k) bv[k] = 0.0f;
          }
          float dT[DPT], db[DPT];
          if (bk == kBNone) {
            unary_partial<DPT>(static_cast<int>(op), ti, to, dT);
#pragma unroll
            for (int k = 0; k < DPT; ++k) db[k] = 0.0f;
          } else if (op > kOpReversed) {  // T = f(b, T)
            binary_partials<DPT>(static_cast<int>(op - kOpReversed), bv, ti, to, db, dT);
          } else {
            binary_partials<DPT>(static_cast<int>(op), ti, bv, to, dT, db);
          }
          float gi[DPT], gb[DPT];
#pragma unroll
          for (int k = 0; k < DPT; ++k) {
            gi[k] = strong_mul(gT[k], dT[k]);
            gb[k] = strong_mul(gT[k], db[k]);
          }
          if (bk == kBC) {
            gacc_add<DPT>(gacc, (ins.w >> 10) & 0x3FFu, static_cast<uint32_t>(nconst), lane, gb);
          } else if (bk == kBS) {
            spill_store<DPT>(st, ins.z, lane, gb);
          }
          if (instr_load(w)) {
            if (instr_leaf_kind(w) == kLeafC)
              gacc_add<DPT>(gacc, ins.w & 0x3FFu, static_cast<uint32_t>(nconst), lane, gi);
            if (instr_spill(w)) {
              spill_load<DPT>(st, instr_spill_slot(w), lane, gT);
            } else {
#pragma unroll
              for (int k = 0; k < DPT; ++k) gT[k] = 0.0f;
            }
          } else {
#pragma unroll
            for (int k = 0; k < DPT; ++k) gT[k] = gi[k];
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
      for (int c = 0; c < nconst; ++c) {
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
                                     const int64_t *__restrict__ const_off,
                                     const int32_t *__restrict__ const_cnt,
                                     const double *__restrict__ grad_acc, float *__restrict__ mse,
                                     float *__restrict__ grad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n_spans; ++k) {
    const double2 q = partial[static_cast<int64_t>(k) * E + e];
    s += q.x;
    c += q.y;
  }
  if (mse) mse[e] = (c > 0.0) ? static_cast<float>(s / c) : qnan();
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

size_t adj_smem_bytes(int W, int V, int s_smem, int span, int tape_len, int gmax) {
  const size_t tile = 32u * kAdjDpt;
  return (static_cast<size_t>(kBufs) * (V + 1) * span + static_cast<size_t>(W) * s_smem * tile +
          static_cast<size_t>(W) * tape_len * tile) * sizeof(float) +
         static_cast<size_t>(W) * gmax * 32 * sizeof(double) + kBufs * sizeof(ItemDesc) +
         2 * kBufs * sizeof(uint64_t);
}

cudaError_t adj_configure(size_t smem, int W, int *blocks_per_sm) {
  const void *fn = reinterpret_cast<const void *>(&adj_kernel);
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, (W + 1) * 32, smem);
}

cudaError_t launch_adjoint(const AdjArgs &args, int blocks, size_t smem, cudaStream_t stream) {
  if (args.e.W < 1 || args.e.W > kMaxWarps) return cudaErrorInvalidValue;
  // Each tape class has its own shared-memory size; the attribute is the
  // kernel's, so set it for this launch.
  const cudaError_t err = cudaFuncSetAttribute(reinterpret_cast<const void *>(&adj_kernel),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  adj_kernel<<<blocks, (args.e.W + 1) * 32, smem, stream>>>(args);
  return cudaGetLastError();
}

cudaError_t launch_grad_finalize(const double2 *partial, int n_spans, int E,
                                 const int64_t *const_off, const int32_t *const_cnt,
                                 const double *grad_acc, float *mse, float *grad,
                                 cudaStream_t stream) {
  if (E <= 0) return cudaSuccess;
  grad_finalize_kernel<<<(E + 255) / 256, 256, 0, stream>>>(partial, n_spans, E, const_off,
                                                             const_cnt, grad_acc, mse, grad);
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
