// sr_kernels.cu — sm_100a kernels of the population evaluator.
//
//  interp_kernel<DPT, PRED, MAXW, MINB, OPS>
//                             persistent interpreter (OPS: the operator
//                             profile its switch dispatches inline,
//                             sr_internal.hpp).  One producer thread
//                             per block claims work items (span, group) from
//                             a global counter and copies the item's X span
//                             (every row) into one of two shared-memory
//                             buffers with the bulk-copy (TMA) engine, one
//                             cp.async.bulk per row, completion tracked by
//                             mbarrier transaction counts.  The W evaluating
//                             warps claim the group's expressions from a
//                             shared counter and run each over the whole span:
//                             32 lanes x DPT datapoints per instruction fetch,
//                             accumulator in registers, spilled values in a
//                             per-warp shared stack.  The epilogue either
//                             accumulates the squared error (FP32 Kahan over a
//                             lane's DPT values, FP64 across tiles and lanes)
//                             or stores the predictions.
//  finalize_kernel            per-expression combination of span partials in
//                             a fixed order: mse = sum / count.
//  sums_kernel                the same combination kept as (sum, count), for
//                             datapoint-sharded callers.
//  fp64_kernel                the plain kernel's shape in double: the FP64
//                             reference of the accuracy report.
//  plain_kernel               baseline with the reference's launch shape
//                             (4 expressions x 128 datapoints per block, token
//                             stack in local memory), fused MSE reduction.
//  pipe microbenchmarks       FP32 FMA and MUFU throughput of the device.
//  op_rate_kernel             throughput of each operator's FP32 semantics alone
//                             (the accurate-operator bound of the interpreter).
//
// Reference counterparts: eval_subtrees_kernel / eval_skeletons_kernel /
// reduce_mse_kernel (src/cleaned/cl_gpu_eval.cu:60-245) and eval_simple_kernel
// / reduce_mse_kernel_simple (src/cleaned/cl_gpu_simple.cu:57-173).
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_device.cuh"
#include "sr_eval.h"
#include "sr_internal.hpp"
#include "sr_kernels.hpp"
#include "sr_ops.cuh"

namespace sr {

namespace {

// MAXW / MINB: launch bounds of the instantiation (at most MAXW evaluating
// warps, at least MINB resident blocks per SM), which set the register budget.
template <int DPT, bool PRED, int MAXW, int MINB, int OPS, bool CACHE>
__global__ void __launch_bounds__((MAXW + 1) * 32, MINB) interp_kernel(const EvalArgs p) {
  constexpr int TILE = 32 * DPT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int W = p.W;
  const int rows = p.V + 1;
  const int span = p.span;
  float *xbuf = reinterpret_cast<float *>(smem_raw);
  float *sreg = xbuf + static_cast<size_t>(kBufs) * rows * span;
  ItemDesc *desc =
      reinterpret_cast<ItemDesc *>(sreg + static_cast<size_t>(W) * p.s_smem * TILE);
  uint64_t *full = reinterpret_cast<uint64_t *>(desc + kBufs);
  uint64_t *empty = full + kBufs;
  SpanPart *part = reinterpret_cast<SpanPart *>(empty + kBufs);  // MSE launches only
  GroupAcc *gacc = reinterpret_cast<GroupAcc *>(part + kBufs * p.G);

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
      run_producer<!PRED>(p.n_groups, n_items, k_spans, p.n_spans, p.work_counter, p.error, p.X,
                          p.ldx, rows, span, xbuf, desc, full, empty,
                          FoldArgs{part, gacc, p.partial, p.G, p.E, p.E, 0, nullptr, nullptr, nullptr,
                                   nullptr, nullptr, 0});
    return;
  }

  // ---------------- evaluating warps ----------------
  SpillStack st;
  st.ss = sreg + static_cast<size_t>(warp) * p.s_smem * TILE;
  st.gs = p.spill + (static_cast<size_t>(blockIdx.x) * W + warp) *
                        static_cast<size_t>(p.smax - p.s_smem) * TILE;
  st.s_smem = p.s_smem;
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
      const int len = p.code_len[e];
      double acc = 0.0;
      int cnt = 0;
      for (int t = 0; t < tiles; ++t) {
        const int64_t dp0 = dp_span + static_cast<int64_t>(t) * TILE;
        if (dp0 >= p.N) break;  // tail of the last span
        const float *xs = xb + t * TILE;
        float T[DPT];
        run_program<DPT, OPS, CACHE>(code, len, xs, span, st, lane, p.cache, p.ldc, dp0, T);
        if constexpr (PRED) {
          stg_vec<DPT>(p.pred + static_cast<int64_t>(p.pred_row[e]) * p.ldp + dp0, lane, T);
        } else {
          float y[DPT];
          lds_vec<DPT>(xs + p.V * span, lane, y);
          const bool full = dp0 + TILE <= p.N;  // warp-uniform
          float s = 0.0f, c = 0.0f;  // Kahan over the lane's DPT values
          int nv = 0;
          float dsq[DPT];  // squared residuals, two datapoints per paired operation
#pragma unroll
          for (int k = 0; k < DPT; k += 2) {
            const float2 df2 =
                __fadd2_rn(make_float2(T[k], T[k + 1]), make_float2(-y[k], -y[k + 1]));
            const float2 sq2 = __fmul2_rn(df2, df2);
            dsq[k] = sq2.x;
            dsq[k + 1] = sq2.y;
          }
#pragma unroll
          for (int k = 0; k < DPT; ++k) {
            const bool valid =
                (full || dp0 + (k / 4) * 128 + lane * 4 + (k % 4) < p.N) && isfinite(T[k]);
            const float sq = valid ? dsq[k] : 0.0f;
            nv += valid ? 1 : 0;
            const float yk = __fsub_rn(sq, c);
            const float tt = __fadd_rn(s, yk);
            c = __fsub_rn(__fsub_rn(tt, s), yk);
            s = tt;
          }
          double tile_sum = static_cast<double>(s) - static_cast<double>(c);
          if (!isfinite(tile_sum)) {
            float tc[DPT], yc[DPT];
#pragma unroll
            for (int k = 0; k < DPT; ++k) {
              tc[k] = T[k];
              yc[k] = y[k];
            }
            tile_sum = tile_sum_fp64<DPT>(tc, yc, full, dp0, lane, p.N);
          }
          acc += tile_sum;
          cnt += nv;
        }
      }
      if constexpr (!PRED) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          acc += __shfl_xor_sync(0xffffffffu, acc, o);
          cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        if (lane == 0) part[static_cast<size_t>(buf) * p.G + j] = SpanPart{acc, cnt, e};
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

// The same for the interpreter's entries ([n_groups][E] x (hi, lo), (count,
// 0)): the span groups' double-double sums added in order, then mse =
// (hi + lo) / count.
__global__ void finalize_dd_kernel(const double2 *__restrict__ partial, int n_groups, int E,
                                   float *__restrict__ mse, double2 *__restrict__ sums) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double hi = 0.0, lo = 0.0, c = 0.0;
  for (int k = 0; k < n_groups; ++k) {
    const double2 *q = partial + 2 * (static_cast<int64_t>(k) * E + e);
    const double2 a = q[0];
    dd_add(hi, lo, a.x);
    dd_add(hi, lo, a.y);
    c += q[1].x;
  }
  const double s = isfinite(hi) ? __dadd_rn(hi, lo) : hi;
  if (mse) mse[e] = (c > 0.0) ? static_cast<float>(s / c) : qnan();
  if (sums) sums[e] = make_double2(s, c);
}

__global__ void finalize_kernel(const double2 *__restrict__ partial, int n_spans,
                                int E, float *__restrict__ mse) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n_spans; ++k) {
    const double2 q = partial[static_cast<int64_t>(k) * E + e];
    s += q.x;
    c += q.y;
  }
  // Reference: mses[i] = total_sq_err / valid_dps, or NaN when no datapoint
  // is valid (src/cleaned/cl_cpu_eval.cpp:154-158).
  mse[e] = (c > 0.0) ? static_cast<float>(s / c) : qnan();
}

// The same fixed-order combination as finalize_kernel, kept as (sum, count)
// for callers that add the partial sums of several datapoint shards.
__global__ void sums_kernel(const double2 *__restrict__ partial, int n_spans, int E,
                            double2 *__restrict__ sums) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n_spans; ++k) {
    const double2 q = partial[static_cast<int64_t>(k) * E + e];
    s += q.x;
    c += q.y;
  }
  sums[e] = make_double2(s, c);
}

// Plain baseline: the reference launch shape (4 expressions x 128 datapoints
// per block), raw prefix tokens interpreted right to left with a stack in
// local memory (reference eval_simple_kernel, src/cleaned/cl_gpu_simple.cu:57-120)
// but with the squared error reduced in the same kernel (per-thread FP64,
// then block) instead of an [E x N] buffer and a second pass.
__global__ void __launch_bounds__(128)
    plain_kernel(const int32_t *__restrict__ tok, const float *__restrict__ val,
                 const int64_t *__restrict__ off, const int32_t *__restrict__ len,
                 const float *__restrict__ X, int64_t ldx, int V, int64_t N,
                 int E, double2 *__restrict__ partial) {
  __shared__ double red_s[4][4];
  __shared__ int red_c[4][4];
  const int e0 = blockIdx.x * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int cnt[4] = {0, 0, 0, 0};
  for (int64_t dp = static_cast<int64_t>(blockIdx.y) * 128 + threadIdx.x; dp < N;
       dp += static_cast<int64_t>(gridDim.y) * 128) {
    float xc[SR_MAX_VARS + 1];
    for (int v = 0; v <= V; ++v) xc[v] = X[v * ldx + dp];
    const float yv = xc[V];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = e0 + j;
      if (e >= E) break;
      float stk[kPlainStack];
      int sp = 0;
      const int64_t o = off[e];
      for (int i = len[e] - 1; i >= 0; --i) {
        const int t = tok[o + i];
        if (t > 0) {
          const float v1 = stk[--sp];
          float v2 = 0.0f;
          if (t < 10) v2 = stk[--sp];
          stk[sp++] = op_apply(t, v1, v2);
        } else if (t == 0) {
          stk[sp++] = val[o + i];
        } else {
          const int vi = static_cast<int>(val[o + i]);
          stk[sp++] = (vi >= 0 && vi < V) ? xc[vi] : 0.0f;
        }
      }
      const float pred = stk[0];
      if (isfinite(pred)) {
        const float df = __fsub_rn(pred, yv);
        acc[j] += static_cast<double>(__fmul_rn(df, df));
        cnt[j] += 1;
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double s = acc[j];
    int c = cnt[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      red_s[j][warp] = s;
      red_c[j][warp] = c;
    }
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int j = threadIdx.x;
    const int e = e0 + j;
    if (e < E) {
      const double s = red_s[j][0] + red_s[j][1] + red_s[j][2] + red_s[j][3];
      const int c = red_c[j][0] + red_c[j][1] + red_c[j][2] + red_c[j][3];
      partial[static_cast<int64_t>(blockIdx.y) * E + e] =
          make_double2(s, static_cast<double>(c));
    }
  }
}

// FP64 reference evaluation for the accuracy report: the plain kernel's
// shape with every operator in double, constants entering as (double)(float)
// value and the variables as the FP32 dataset; a datapoint counts when its
// FP64 prediction would be a finite float (the FP32 path's validity rule).
__global__ void __launch_bounds__(128)
    fp64_kernel(const int32_t *__restrict__ tok, const float *__restrict__ val,
                const int64_t *__restrict__ off, const int32_t *__restrict__ len,
                const float *__restrict__ X, int64_t ldx, int V, int64_t N, int E,
                double2 *__restrict__ partial) {
  __shared__ double red_s[4][4];
  __shared__ int red_c[4][4];
  const int e0 = blockIdx.x * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int cnt[4] = {0, 0, 0, 0};
  for (int64_t dp = static_cast<int64_t>(blockIdx.y) * 128 + threadIdx.x; dp < N;
       dp += static_cast<int64_t>(gridDim.y) * 128) {
    const double yv = static_cast<double>(X[V * ldx + dp]);
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      const int e = e0 + j;
      if (e >= E) break;
      double stk[kFp64Stack];  // the frame stays below the default stack limit
      int sp = 0;
      const int64_t o = off[e];
      for (int i = len[e] - 1; i >= 0; --i) {
        const int t = tok[o + i];
        if (t > 0) {
          const double v1 = stk[--sp];
          double v2 = 0.0;
          if (t < 10) v2 = stk[--sp];
          stk[sp++] = op_apply_f64(t, v1, v2);
        } else if (t == 0) {
          stk[sp++] = static_cast<double>(val[o + i]);
        } else {
          const int vi = static_cast<int>(val[o + i]);
          stk[sp++] = (vi >= 0 && vi < V) ? static_cast<double>(X[vi * ldx + dp]) : 0.0;
        }
      }
      const double pred = stk[0];
      if (!isnan(pred) && !isinf(static_cast<float>(pred))) {
        const double d = pred - yv;
        acc[j] += d * d;
        cnt[j] += 1;
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double s = acc[j];
    int c = cnt[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      red_s[j][warp] = s;
      red_c[j][warp] = c;
    }
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int j = threadIdx.x;
    const int e = e0 + j;
    if (e < E) {
      const double s = red_s[j][0] + red_s[j][1] + red_s[j][2] + red_s[j][3];
      const int c = red_c[j][0] + red_c[j][1] + red_c[j][2] + red_c[j][3];
      partial[static_cast<int64_t>(blockIdx.y) * E + e] =
          make_double2(s, static_cast<double>(c));
    }
  }
}

__global__ void finalize_f64_kernel(const double2 *__restrict__ partial, int n_spans, int E,
                                    double *__restrict__ mse) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n_spans; ++k) {
    const double2 q = partial[static_cast<int64_t>(k) * E + e];
    s += q.x;
    c += q.y;
  }
  mse[e] = (c > 0.0) ? s / c : __longlong_as_double(0x7ff8000000000000ll);
}

// ---- pipe microbenchmarks (8 independent chains per thread) ----
__global__ void fma_pipe_kernel(float *out, int iters) {
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = threadIdx.x * 1e-3f + k;
  const float m = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fmaf(r[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 1234.5f) out[threadIdx.x] = s;  // keep the loop alive
}

__global__ void mufu_pipe_kernel(float *out, int iters) {
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = 1.0f + threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      asm volatile("rsqrt.approx.ftz.f32 %0, %0;" : "+f"(r[k]));
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 1234.5f) out[threadIdx.x] = s;
}

// Throughput of one operator's FP32 semantics with nothing around it: every
// thread evaluates OP on 8 independent operand pairs per iteration and adds
// the results.  The first operand moves by a tiny step every iteration, so no
// evaluation is loop-invariant (an empty inline-asm barrier was not enough:
// the code generator still hoisted some functions out of the loop).  With
// OP = 0 (the identity) it times the harness alone (two adds per evaluation).
template <int OP>
__global__ void op_rate_kernel(float *out, int iters) {
  float x[8], y[8], acc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 8u + static_cast<uint32_t>(k);
    h ^= h >> 16;
    h *= 0x7feb352dU;
    h ^= h >> 15;
    h *= 0x846ca68bU;
    h ^= h >> 16;
    x[k] = -3.0f + 6.0f * static_cast<float>(h & 0xFFFFFFu) * (1.0f / 16777216.0f);
    y[k] = 0.5f + 2.5f * static_cast<float>(h >> 8) * (1.0f / 16777216.0f);
    acc[k] = 0.0f;
  }
  for (int i = 0; i < iters; ++i) {
    const float step = static_cast<float>(i) * 1e-6f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float a = __fadd_rn(x[k], step);
      acc[k] = __fadd_rn(acc[k], op_apply(OP, a, y[k]));
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += acc[k];
  if (s == 1234.5f) out[threadIdx.x] = s;  // keeps the loop alive
}

template <int... OPS>
struct OpRateTable {
  static const void *get(int op) {
    const void *fn = nullptr;
    ((fn = (op == OPS) ? reinterpret_cast<const void *>(&op_rate_kernel<OPS>) : fn), ...);
    return fn;
  }
};
using OpRates = OpRateTable<0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18,
                            19, 20, 21, 22, 23, 24, 25, 26, 27, 32>;

}  // namespace

size_t interp_smem_bytes(int dpt, int W, int V, int s_smem, int span, int G, bool pred) {
  const size_t tile = 32u * static_cast<size_t>(dpt);
  return (static_cast<size_t>(kBufs) * (V + 1) * span +
          static_cast<size_t>(W) * s_smem * tile) * sizeof(float) +
         kBufs * sizeof(ItemDesc) + 2 * kBufs * sizeof(uint64_t) +
         (pred ? 0 : static_cast<size_t>(G) * (kBufs * sizeof(SpanPart) + sizeof(GroupAcc)));
}

template <int DPT, bool PRED, int MAXW, int MINB, int OPS = kOpsAll, bool CACHE = false>
static const void *interp_fn() {
  return reinterpret_cast<const void *>(&interp_kernel<DPT, PRED, MAXW, MINB, OPS, CACHE>);
}

template <int DPT, int MAXW, int MINB>
static const void *interp_mse(int ops, bool cache) {
  if (cache)
    return ops == kOpsProtected ? interp_fn<DPT, false, MAXW, MINB, kOpsProtected, true>()
                                : interp_fn<DPT, false, MAXW, MINB, kOpsAll, true>();
  return ops == kOpsProtected ? interp_fn<DPT, false, MAXW, MINB, kOpsProtected, false>()
                              : interp_fn<DPT, false, MAXW, MINB, kOpsAll, false>();
}

// Instantiations: W <= 8 uses the narrow variants (more blocks per SM, tighter
// register budget), larger W the wide ones (up to 16 warps; at 8 datapoints
// per thread MSE launches also come as 2 blocks of up to 15 + 1 warps and 1
// block of up to 31 + 1 warps, both at 64 registers: on the batched
// population the interpreter is latency-bound, and 30 or 31 evaluating warps
// per SM beat 24 at 72 registers: 65.2 -> 60.1 and 58.8 ms).  MSE launches
// come in both operator profiles, with and without cached-subtree operands;
// prediction launches (cache fills, predictions) in kOpsAll without.
static const void *select_interp(int dpt, bool pred, int ops, bool cache, int W) {
  if (W > kMaxWarps && (pred || dpt != 8)) return nullptr;
  const bool narrow = W <= 8;
  if (dpt == 16) {
    if (narrow) return pred ? interp_fn<16, true, 8, 2>() : interp_mse<16, 8, 2>(ops, cache);
    return pred ? interp_fn<16, true, 16, 1>() : interp_mse<16, 16, 1>(ops, cache);
  }
  if (dpt == 8) {
    if (narrow) return pred ? interp_fn<8, true, 8, 3>() : interp_mse<8, 8, 3>(ops, cache);
    if (pred) return interp_fn<8, true, 16, 1>();
    return W <= 15 ? interp_mse<8, 15, 2>(ops, cache) : interp_mse<8, 31, 1>(ops, cache);
  }
  if (dpt == 4) {
    if (narrow) return pred ? interp_fn<4, true, 8, 4>() : interp_mse<4, 8, 4>(ops, cache);
    return pred ? interp_fn<4, true, 16, 2>() : interp_mse<4, 16, 2>(ops, cache);
  }
  return nullptr;
}

cudaError_t raise_smem_limit(const void *fn, size_t smem) {
  cudaFuncAttributes a{};
  const cudaError_t err = cudaFuncGetAttributes(&a, fn);
  if (err != cudaSuccess) return err;
  if (static_cast<size_t>(a.maxDynamicSharedSizeBytes) >= smem) return cudaSuccess;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(smem));
}

cudaError_t interp_configure(int dpt, bool pred, int ops, bool cache, size_t smem, int W,
                             int *blocks_per_sm) {
  const void *fn = select_interp(dpt, pred, ops, cache, W);
  if (!fn || W < 1 || W > kMaxInterpWarps) return cudaErrorInvalidValue;
  const cudaError_t err = raise_smem_limit(fn, smem);
  if (err != cudaSuccess) return err;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn,
                                                       (W + 1) * 32, smem);
}

cudaError_t launch_interp(int dpt, bool pred, int ops, bool cache, const EvalArgs &args,
                          int blocks, size_t smem, cudaStream_t stream) {
  const void *fn = select_interp(dpt, pred, ops, cache, args.W);
  if (!fn || args.W < 1 || args.W > kMaxInterpWarps) return cudaErrorInvalidValue;
  // Plans of one instantiation can differ in shared-memory size (main and
  // cache-fill sets, autotune candidates); the attribute belongs to the
  // kernel, so set it for this launch.
  const cudaError_t err = raise_smem_limit(fn, smem);
  if (err != cudaSuccess) return err;
  void *params[] = {const_cast<EvalArgs *>(&args)};
  return cudaLaunchKernel(fn, dim3(blocks), dim3((args.W + 1) * 32), params, smem, stream);
}

cudaError_t launch_finalize(const double2 *partial, int n_spans, int E,
                            float *mse, cudaStream_t stream) {
  if (E <= 0) return cudaSuccess;
  finalize_kernel<<<(E + 255) / 256, 256, 0, stream>>>(partial, n_spans, E, mse);
  return cudaGetLastError();
}

cudaError_t launch_finalize_groups(const double2 *partial, int n_groups, int E, float *mse,
                                   double2 *sums, cudaStream_t stream) {
  if (E <= 0) return cudaSuccess;
  finalize_dd_kernel<<<(E + 255) / 256, 256, 0, stream>>>(partial, n_groups, E, mse, sums);
  return cudaGetLastError();
}

cudaError_t launch_plain(const int32_t *tok, const float *val, const int64_t *off,
                         const int32_t *len, const float *X, int64_t ldx, int V,
                         int64_t N, int E, double2 *partial, int n_dpblocks,
                         cudaStream_t stream) {
  if (E <= 0 || n_dpblocks <= 0) return cudaSuccess;
  const dim3 grid((E + 3) / 4, n_dpblocks);
  plain_kernel<<<grid, 128, 0, stream>>>(tok, val, off, len, X, ldx, V, N, E,
                                         partial);
  return cudaGetLastError();
}

cudaError_t launch_fp64(const int32_t *tok, const float *val, const int64_t *off,
                       const int32_t *len, const float *X, int64_t ldx, int V, int64_t N, int E,
                       double2 *partial, int n_dpblocks, double *mse64, cudaStream_t stream) {
  if (E <= 0) return cudaSuccess;
  if (n_dpblocks > 0 && N > 0) {
    const dim3 grid((E + 3) / 4, n_dpblocks);
    fp64_kernel<<<grid, 128, 0, stream>>>(tok, val, off, len, X, ldx, V, N, E, partial);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }
  finalize_f64_kernel<<<(E + 255) / 256, 256, 0, stream>>>(partial, N > 0 ? n_dpblocks : 0, E,
                                                           mse64);
  return cudaGetLastError();
}

cudaError_t launch_sums(const double2 *partial, int n_spans, int E, double2 *sums,
                        cudaStream_t stream) {
  if (E <= 0) return cudaSuccess;
  sums_kernel<<<(E + 255) / 256, 256, 0, stream>>>(partial, n_spans, E, sums);
  return cudaGetLastError();
}

cudaError_t launch_op_rate(int op, float *out, int blocks, int threads, int iters,
                           cudaStream_t stream) {
  const void *fn = OpRates::get(op);
  if (!fn) return cudaErrorInvalidValue;
  void *params[] = {&out, &iters};
  return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), params, 0, stream);
}

cudaError_t launch_pipe_bench(bool mufu, float *out, int blocks, int threads,
                              int iters, cudaStream_t stream) {
  if (mufu)
    mufu_pipe_kernel<<<blocks, threads, 0, stream>>>(out, iters);
  else
    fma_pipe_kernel<<<blocks, threads, 0, stream>>>(out, iters);
  return cudaGetLastError();
}

}  // namespace sr
