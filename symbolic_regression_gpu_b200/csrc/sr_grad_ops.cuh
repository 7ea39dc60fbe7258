// sr_grad_ops.cuh — every operator's value together with its local partial
// derivatives (d out / d left, d out / d right), as the gradient kernels use
// them: the values are exactly the forward interpreter's (same routines, same
// rounding), the partials follow the conventions stated at the top of
// sr_adjoint.cu (derivative 0 at the non-smooth points and in the protected
// regions).  The reverse-mode kernel (sr_adjoint.cu) and the forward-mode
// kernel (sr_tangent.cu) both evaluate partials through these routines, so
// the two modes multiply the same partials.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_device.cuh"

namespace sr {
namespace {
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

}  // namespace
}  // namespace sr
