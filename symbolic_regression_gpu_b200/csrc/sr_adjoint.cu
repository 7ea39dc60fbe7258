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

namespace sr {
namespace {

#ifndef SR_ADJ_DPT
#define SR_ADJ_DPT 4
#endif
constexpr int kAdjDpt = SR_ADJ_DPT;  // datapoints per thread (4 or 8)
static_assert(kAdjDpt == 4 || kAdjDpt == 8, "adjoint DPT 4 or 8");

__device__ __forceinline__ float strong_mul(float g, float d) { return g == 0.0f ? 0.0f : g * d; }

__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// ---- value + derivative routines, out of line ------------------------------
// Each routine exists once per width SR_ADJ_WIDTH (datapoints per call: 1, 2
// or 4).  Narrow routines keep the hot code small (instruction cache); wide
// ones give the scheduler independent work inside one call.
#ifndef SR_ADJ_WIDTH
#define SR_ADJ_WIDTH 1
#endif
static_assert(SR_ADJ_WIDTH == 1 || SR_ADJ_WIDTH == 2 || SR_ADJ_WIDTH == 4, "width 1, 2 or 4");

struct VD1 {
  float v, d;
};
struct VD2 {
  float v, du, dv;
};
struct VD4 {
  float4 v, d;
};

#if SR_ADJ_WIDTH == 1
#define SR_VD1_WIDE(NAME) \
  __device__ __noinline__ VD1 NAME##_w1(float x) { return NAME##_body(x); }
#elif SR_ADJ_WIDTH == 2
#define SR_VD1_WIDE(NAME)                                            \
  __device__ __noinline__ float4 NAME##_w2(float x0, float x1) {     \
    const VD1 a = NAME##_body(x0), b = NAME##_body(x1);              \
    return make_float4(a.v, a.d, b.v, b.d);                          \
  }
#else
#define SR_VD1_WIDE(NAME)                                            \
  __device__ __noinline__ VD4 NAME##_w4(float4 x) {                 \
    const VD1 a = NAME##_body(x.x), b = NAME##_body(x.y);            \
    const VD1 c = NAME##_body(x.z), e = NAME##_body(x.w);            \
    return VD4{make_float4(a.v, b.v, c.v, e.v), make_float4(a.d, b.d, c.d, e.d)}; \
  }
#endif
#define SR_VD1(NAME, VAL, DER)                                       \
  __device__ __forceinline__ VD1 NAME##_body(float x) {              \
    const float o = (VAL);                                           \
    return VD1{o, (DER)};                                            \
  }                                                                  \
  SR_VD1_WIDE(NAME)
// sin and cos share one argument reduction through sr_sincosf (its two
// results are those of sr_sinf / sr_cosf, the forward interpreter's).
__device__ __forceinline__ VD1 g_sin_body(float x) {
  float s, c;
  sr_sincosf(x, &s, &c);
  return VD1{s, c};
}
SR_VD1_WIDE(g_sin)
__device__ __forceinline__ VD1 g_cos_body(float x) {
  float s, c;
  sr_sincosf(x, &s, &c);
  return VD1{c, -s};
}
SR_VD1_WIDE(g_cos)
SR_VD1(g_tan, tanf(x), __fadd_rn(1.0f, __fmul_rn(o, o)))
SR_VD1(g_sinh, sinhf(x), coshf(x))
SR_VD1(g_cosh, coshf(x), sinhf(x))
SR_VD1(g_tanh, tanhf(x), __fsub_rn(1.0f, __fmul_rn(o, o)))
SR_VD1(g_exp, expf(x), o)
SR_VD1(g_log, sr_logf(x), __frcp_rn(x))
SR_VD1(g_rcp, __frcp_rn(x), __fmul_rn(-o, o))
SR_VD1(g_asin, asinf(x), __frcp_rn(__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(x, x)))))
SR_VD1(g_acos, acosf(x), -__frcp_rn(__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(x, x)))))
SR_VD1(g_atan, atanf(x), __frcp_rn(__fadd_rn(1.0f, __fmul_rn(x, x))))
SR_VD1(g_llog, sr_loose_logf(x), (x == 0.0f) ? 0.0f : __frcp_rn(x))
SR_VD1(g_linv, __frcp_rn(loose_denom(x)), (fabsf(x) <= 1e-9f) ? 0.0f : __fmul_rn(-o, o))
SR_VD1(g_sqrt, __fsqrt_rn(x), __frcp_rn(2.0f * o))
SR_VD1(g_lsqrt, __fsqrt_rn(fabsf(x)), (x == 0.0f) ? 0.0f : signf(x) * __frcp_rn(2.0f * o))
SR_VD1(g_expc, expf(fminf(x, 80.0f)), (x < 80.0f) ? o : 0.0f)
#undef SR_VD1
#undef SR_VD1_WIDE

// u^v: du = v u^(v-1), dv = u^v ln u.
__device__ __forceinline__ VD2 g_pow_body(float u, float v) {
  const float o = powf(u, v);
  return VD2{o, __fmul_rn(v, powf(u, __fsub_rn(v, 1.0f))), __fmul_rn(o, logf(u))};
}
// LOOSE_POW u, v: 0^0 = 0, else |u|^v; du = v |u|^(v-1) sign(u), dv = out ln|u|.
__device__ __forceinline__ VD2 g_lpow_body(float u, float v) {
  const bool z = (u == 0.0f && v == 0.0f);
  const float a = fabsf(u);
  const float o = z ? 0.0f : powf(a, v);
  return VD2{o, z ? 0.0f : __fmul_rn(__fmul_rn(v, powf(a, __fsub_rn(v, 1.0f))), signf(u)),
             z ? 0.0f : __fmul_rn(o, logf(a))};
}
// Division u / d with 1/d reused for both partials: du = 1/d, dv = -out/d
// (0 where `flat`, the protected region of LOOSE_DIV); NaN at d == 0 when
// nan_at_zero (DIV).
__device__ __forceinline__ VD2 g_div_body(float u, float d, bool flat, bool nan_at_zero) {
  const float q = __fdiv_rn(u, d);
  const float o = (nan_at_zero && d == 0.0f) ? qnan() : q;
  const float rc = __frcp_rn(d);
  return VD2{o, rc, flat ? 0.0f : __fmul_rn(-o, rc)};
}
#if SR_ADJ_WIDTH == 1
__device__ __noinline__ VD2 g_pow_w1(float u, float v) { return g_pow_body(u, v); }
__device__ __noinline__ VD2 g_lpow_w1(float u, float v) { return g_lpow_body(u, v); }
__device__ __noinline__ VD2 g_div_w1(float u, float d, bool flat, bool nz) {
  return g_div_body(u, d, flat, nz);
}
#endif
template <int N>
struct VD2N {
  float v[N], du[N], dv[N];
};
#if SR_ADJ_WIDTH == 2
__device__ __noinline__ VD2N<2> g_pow_w2(float u0, float u1, float v0, float v1) {
  const VD2 a = g_pow_body(u0, v0), b = g_pow_body(u1, v1);
  return VD2N<2>{{a.v, b.v}, {a.du, b.du}, {a.dv, b.dv}};
}
__device__ __noinline__ VD2N<2> g_lpow_w2(float u0, float u1, float v0, float v1) {
  const VD2 a = g_lpow_body(u0, v0), b = g_lpow_body(u1, v1);
  return VD2N<2>{{a.v, b.v}, {a.du, b.du}, {a.dv, b.dv}};
}
__device__ __noinline__ VD2N<2> g_div_w2(float u0, float u1, float d0, float d1, bool f0, bool f1,
                                         bool nz) {
  const VD2 a = g_div_body(u0, d0, f0, nz), b = g_div_body(u1, d1, f1, nz);
  return VD2N<2>{{a.v, b.v}, {a.du, b.du}, {a.dv, b.dv}};
}
#endif
#if SR_ADJ_WIDTH == 4
__device__ __noinline__ VD2N<4> g_pow_w4(float4 u, float4 v) {
  const VD2 a = g_pow_body(u.x, v.x), b = g_pow_body(u.y, v.y);
  const VD2 c = g_pow_body(u.z, v.z), e = g_pow_body(u.w, v.w);
  return VD2N<4>{{a.v, b.v, c.v, e.v}, {a.du, b.du, c.du, e.du}, {a.dv, b.dv, c.dv, e.dv}};
}
__device__ __noinline__ VD2N<4> g_lpow_w4(float4 u, float4 v) {
  const VD2 a = g_lpow_body(u.x, v.x), b = g_lpow_body(u.y, v.y);
  const VD2 c = g_lpow_body(u.z, v.z), e = g_lpow_body(u.w, v.w);
  return VD2N<4>{{a.v, b.v, c.v, e.v}, {a.du, b.du, c.du, e.du}, {a.dv, b.dv, c.dv, e.dv}};
}
__device__ __noinline__ VD2N<4> g_div_w4(float4 u, float4 d, uint32_t flat, bool nz) {
  const VD2 a = g_div_body(u.x, d.x, flat & 1u, nz), b = g_div_body(u.y, d.y, flat & 2u, nz);
  const VD2 c = g_div_body(u.z, d.z, flat & 4u, nz), e = g_div_body(u.w, d.w, flat & 8u, nz);
  return VD2N<4>{{a.v, b.v, c.v, e.v}, {a.du, b.du, c.du, e.du}, {a.dv, b.dv, c.dv, e.dv}};
}
#endif

// T, dT = f(T), f'(T) for DPT datapoints through the routine of width SR_ADJ_WIDTH.
#if SR_ADJ_WIDTH == 1
#define SR_G1(FN)                                                          \
  {                                                                        \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) {                      \
      const VD1 r = FN##_w1(T[k]);                                         \
      T[k] = r.v;                                                          \
      dT[k] = r.d;                                                         \
    }                                                                      \
  }                                                                        \
  break;
#elif SR_ADJ_WIDTH == 2
#define SR_G1(FN)                                                          \
  {                                                                        \
    _Pragma("unroll") for (int k = 0; k < DPT; k += 2) {                   \
      const float4 r = FN##_w2(T[k], T[k + 1]);                            \
      T[k] = r.x;                                                          \
      dT[k] = r.y;                                                         \
      T[k + 1] = r.z;                                                      \
      dT[k + 1] = r.w;                                                     \
    }                                                                      \
  }                                                                        \
  break;
#else
#define SR_G1(FN)                                                          \
  {                                                                        \
    _Pragma("unroll") for (int h = 0; h < DPT / 4; ++h) {                  \
      const VD4 r = FN##_w4(quad<DPT>(T, h));                              \
      unquad<DPT>(T, h, r.v);                                              \
      unquad<DPT>(dT, h, r.d);                                             \
    }                                                                      \
  }                                                                        \
  break;
#endif

// (out, d/dleft, d/dright) of a binary routine for all DPT datapoints.
template <int DPT>
__device__ __forceinline__ void binary_vd(int which, const float (&u)[DPT], const float (&v)[DPT],
                                          const bool (&flat)[DPT], bool nz, float (&o)[DPT],
                                          float (&du)[DPT], float (&dv)[DPT]) {
#if SR_ADJ_WIDTH == 1
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    const VD2 r = which == 0 ? g_pow_w1(u[k], v[k])
                             : (which == 1 ? g_lpow_w1(u[k], v[k]) : g_div_w1(u[k], v[k], flat[k], nz));
    o[k] = r.v;
    du[k] = r.du;
    dv[k] = r.dv;
  }
#elif SR_ADJ_WIDTH == 2
#pragma unroll
  for (int k = 0; k < DPT; k += 2) {
    const VD2N<2> r = which == 0 ? g_pow_w2(u[k], u[k + 1], v[k], v[k + 1])
                      : which == 1 ? g_lpow_w2(u[k], u[k + 1], v[k], v[k + 1])
                                   : g_div_w2(u[k], u[k + 1], v[k], v[k + 1], flat[k], flat[k + 1], nz);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      o[k + q] = r.v[q];
      du[k + q] = r.du[q];
      dv[k + q] = r.dv[q];
    }
  }
#else
#pragma unroll
  for (int h = 0; h < DPT / 4; ++h) {
    uint32_t fl = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) fl |= flat[4 * h + q] ? (1u << q) : 0u;
    const VD2N<4> r = which == 0 ? g_pow_w4(quad<DPT>(u, h), quad<DPT>(v, h))
                      : which == 1 ? g_lpow_w4(quad<DPT>(u, h), quad<DPT>(v, h))
                                   : g_div_w4(quad<DPT>(u, h), quad<DPT>(v, h), fl, nz);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      o[4 * h + q] = r.v[q];
      du[4 * h + q] = r.du[q];
      dv[4 * h + q] = r.dv[q];
    }
  }
#endif
}

// T = op(T, b) exactly as apply_op computes it, plus dT = d out / d T and
// db = d out / d b (left unset for unary operators).
#define SR_EACH2(STMT)                                           \
  {                                                              \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) { STMT; }   \
  }                                                              \
  break;
// Binary routine `which` (0 pow, 1 loose pow, 2 division) on (left, right);
// REV: T is the right operand.
#define SR_G2(WHICH, REV, NZ)                                              \
  {                                                                        \
    float o_[DPT], dl_[DPT], dr_[DPT];                                     \
    if (REV)                                                               \
      binary_vd<DPT>(WHICH, b, T, flat, NZ, o_, dl_, dr_);                 \
    else                                                                   \
      binary_vd<DPT>(WHICH, T, b, flat, NZ, o_, dl_, dr_);                 \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) {                      \
      T[k] = o_[k];                                                        \
      dT[k] = REV ? dr_[k] : dl_[k];                                       \
      db[k] = REV ? dl_[k] : dr_[k];                                       \
    }                                                                      \
  }                                                                        \
  break;

template <int DPT>
__device__ __forceinline__ void apply_op_grad(uint32_t op, float (&T)[DPT], float (&b)[DPT],
                                              float (&dT)[DPT], float (&db)[DPT]) {
  bool flat[DPT];
#pragma unroll
  for (int k = 0; k < DPT; ++k) flat[k] = false;
  switch (op) {
    case 0: SR_EACH2(dT[k] = 1.0f)
    case 1: SR_EACH2(T[k] = __fadd_rn(T[k], b[k]); dT[k] = 1.0f; db[k] = 1.0f)
    case 2: SR_EACH2(T[k] = __fsub_rn(T[k], b[k]); dT[k] = 1.0f; db[k] = -1.0f)
    case 42: SR_EACH2(T[k] = __fsub_rn(b[k], T[k]); dT[k] = -1.0f; db[k] = 1.0f)
    case 3: SR_EACH2(db[k] = T[k]; dT[k] = b[k]; T[k] = __fmul_rn(T[k], b[k]))
    case 4: SR_G2(2, false, true)
    case 44: SR_G2(2, true, true)
    case 5: SR_G2(0, false, false)
    case 45: SR_G2(0, true, false)
    case 6:
      SR_EACH2(const bool f = isnan(b[k]) || (!isnan(T[k]) && T[k] <= b[k]);
               T[k] = fminf(T[k], b[k]); dT[k] = f ? 1.0f : 0.0f; db[k] = f ? 0.0f : 1.0f)
    case 46:
      SR_EACH2(const bool f = isnan(T[k]) || (!isnan(b[k]) && b[k] <= T[k]);
               T[k] = fminf(b[k], T[k]); db[k] = f ? 1.0f : 0.0f; dT[k] = f ? 0.0f : 1.0f)
    case 7:
      SR_EACH2(const bool f = isnan(b[k]) || (!isnan(T[k]) && T[k] >= b[k]);
               T[k] = fmaxf(T[k], b[k]); dT[k] = f ? 1.0f : 0.0f; db[k] = f ? 0.0f : 1.0f)
    case 47:
      SR_EACH2(const bool f = isnan(T[k]) || (!isnan(b[k]) && b[k] >= T[k]);
               T[k] = fmaxf(b[k], T[k]); db[k] = f ? 1.0f : 0.0f; dT[k] = f ? 0.0f : 1.0f)
    case 8: {  // T / protected(b)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        flat[k] = fabsf(b[k]) <= 1e-9f;
        b[k] = loose_denom(b[k]);
      }
    }
      SR_G2(2, false, false)
    case 48: {  // b / protected(T)
#pragma unroll
      for (int k = 0; k < DPT; ++k) {
        flat[k] = fabsf(T[k]) <= 1e-9f;
        T[k] = loose_denom(T[k]);
      }
    }
      SR_G2(2, true, false)
    case 9: SR_G2(1, false, false)
    case 49: SR_G2(1, true, false)
    case 10: SR_G1(g_sin)
    case 11: SR_G1(g_cos)
    case 12: SR_G1(g_tan)
    case 13: SR_G1(g_sinh)
    case 14: SR_G1(g_cosh)
    case 15: SR_G1(g_tanh)
    case 16: SR_G1(g_exp)
    case 17: SR_G1(g_log)
    case 18: SR_G1(g_rcp)
    case 19: SR_G1(g_asin)
    case 20: SR_G1(g_acos)
    case 21: SR_G1(g_atan)
    case 22: SR_G1(g_llog)
    case 23: SR_G1(g_linv)
    case 24: SR_EACH2(dT[k] = signf(T[k]); T[k] = fabsf(T[k]))
    case 25: SR_EACH2(T[k] = -T[k]; dT[k] = -1.0f)
    case 26: SR_G1(g_sqrt)
    case 27: SR_G1(g_lsqrt)
    case 32: SR_G1(g_expc)
    default: SR_EACH2(T[k] = 0.0f; dT[k] = 0.0f; db[k] = 0.0f)
  }
}
#undef SR_G1
#undef SR_G2
#undef SR_EACH2

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

cudaError_t adj_configure(size_t smem, int W, bool global_tape, bool recompute,
                          int *blocks_per_sm) {
  const void *fn = adj_fn(global_tape, recompute);
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, (W + 1) * 32, smem);
}

cudaError_t launch_adjoint(const AdjArgs &args, bool recompute, int blocks, size_t smem,
                           cudaStream_t stream) {
  if (args.e.W < 1 || args.e.W > kMaxWarps) return cudaErrorInvalidValue;
  const void *fn = adj_fn(args.gtape != nullptr, recompute);
  // Each tape class has its own shared-memory size; the attribute is the
  // kernel's, so set it for this launch.
  const cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  void *params[] = {const_cast<AdjArgs *>(&args)};
  return cudaLaunchKernel(fn, dim3(blocks), dim3((args.e.W + 1) * 32), params, smem, stream);
}

int adj_segment() { return kSeg; }

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
