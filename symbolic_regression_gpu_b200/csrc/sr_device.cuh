// sr_device.cuh — device building blocks shared by the interpreter kernels
// (forward, prediction, forward+adjoint): mbarrier / bulk-copy helpers, the
// datapoint layout of a tile, operand loads, the spill stack, the operator
// dispatch and the program runner.  Everything sits in an unnamed namespace:
// each kernel translation unit gets its own copy.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_eval.h"
#include "sr_internal.hpp"
#include "sr_ops.cuh"

namespace sr {
namespace {

constexpr uint64_t kWaitLimitNs = 4000000000ull;  // 4 s per mbarrier wait
constexpr uint64_t kDrainLimitNs = 100000000ull;  // 100 ms on error paths

struct alignas(16) ItemDesc {
  int32_t item;   // work item, -1 = no more work
  int32_t group;
  int32_t span;
  int32_t claim;  // next expression of the group to hand out
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "  selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after kWaitLimitNs (sets kDevErrTimeout) or as soon
// as another warp has flagged an error.  Never spins forever.
__device__ __noinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                       int32_t *err) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 0) {
      if (*reinterpret_cast<volatile int32_t *>(err) != 0) return false;
      if (global_timer_ns() - t0 > kWaitLimitNs) {
        atomicOr(err, kDevErrTimeout);
        return false;
      }
    }
  }
}

// Wait used only while draining copies on an error path.
__device__ __noinline__ void mbar_drain(uint64_t *bar, uint32_t parity) {
  const uint64_t t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_timer_ns() - t0 > kDrainLimitNs) return;
  }
}

// Bulk copy global -> shared (no multicast), completion counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ uint4 ldg_instr(const Instr *p) {
  return __ldg(reinterpret_cast<const uint4 *>(p));
}

// Datapoint layout inside a tile of 32*DPT: element k of lane l is datapoint
// (k/4)*128 + 4*l + (k%4), so every vector access of a warp covers 512
// contiguous bytes (conflict-free in shared memory, coalesced in global).
template <int DPT>
__device__ __forceinline__ void lds_vec(const float *base, int lane,
                                        float (&v)[DPT]) {
#pragma unroll
  for (int h = 0; h < DPT / 4; ++h) {
    const float4 q = *reinterpret_cast<const float4 *>(base + h * 128 + lane * 4);
    v[4 * h + 0] = q.x;
    v[4 * h + 1] = q.y;
    v[4 * h + 2] = q.z;
    v[4 * h + 3] = q.w;
  }
}

template <int DPT>
__device__ __forceinline__ void sts_vec(float *base, int lane,
                                        const float (&v)[DPT]) {
#pragma unroll
  for (int h = 0; h < DPT / 4; ++h)
    *reinterpret_cast<float4 *>(base + h * 128 + lane * 4) =
        make_float4(v[4 * h + 0], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}

template <int DPT>
__device__ __forceinline__ void ldg_vec(const float *base, int lane,
                                        float (&v)[DPT]) {
#pragma unroll
  for (int h = 0; h < DPT / 4; ++h) {
    const float4 q = __ldg(reinterpret_cast<const float4 *>(base + h * 128 + lane * 4));
    v[4 * h + 0] = q.x;
    v[4 * h + 1] = q.y;
    v[4 * h + 2] = q.z;
    v[4 * h + 3] = q.w;
  }
}

template <int DPT>
__device__ __forceinline__ void stg_vec(float *base, int lane,
                                        const float (&v)[DPT]) {
#pragma unroll
  for (int h = 0; h < DPT / 4; ++h)
    *reinterpret_cast<float4 *>(base + h * 128 + lane * 4) =
        make_float4(v[4 * h + 0], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}

// ---- out-of-line operator routines -----------------------------------------
// Every routine that expands to more than a handful of instructions (CUDA's
// accurate transcendentals, IEEE division / reciprocal / square root, powf)
// exists once, SR_MATH_WIDTH datapoints wide (1, 2 or 4), instead of being
// inlined DPT times into each opcode of the dispatch switch: that keeps the
// interpreter's code small enough for the instruction cache.
#ifndef SR_MATH_WIDTH
#define SR_MATH_WIDTH 2
#endif
static_assert(SR_MATH_WIDTH == 1 || SR_MATH_WIDTH == 2 || SR_MATH_WIDTH == 4, "width 1, 2 or 4");
#if SR_MATH_WIDTH == 1
#define SR_V1(NAME, EXPR) \
  __device__ __noinline__ float NAME##_w1(float x) { return (EXPR); }
#define SR_V2(NAME, EXPR) \
  __device__ __noinline__ float NAME##_w1(float x, float y) { return (EXPR); }
#elif SR_MATH_WIDTH == 2
#define SR_V1(NAME, EXPR)                                                   \
  __device__ __noinline__ float2 NAME##_w2(float2 v) {                      \
    float2 r;                                                               \
    { const float x = v.x; r.x = (EXPR); }                                  \
    { const float x = v.y; r.y = (EXPR); }                                  \
    return r;                                                               \
  }
#define SR_V2(NAME, EXPR)                                                   \
  __device__ __noinline__ float2 NAME##_w2(float2 u, float2 v) {            \
    float2 r;                                                               \
    { const float x = u.x, y = v.x; r.x = (EXPR); }                         \
    { const float x = u.y, y = v.y; r.y = (EXPR); }                         \
    return r;                                                               \
  }
#else
#define SR_V1(NAME, EXPR)                                                   \
  __device__ __noinline__ float4 NAME##_w4(float4 v) {                      \
    float4 r;                                                               \
    { const float x = v.x; r.x = (EXPR); }                                  \
    { const float x = v.y; r.y = (EXPR); }                                  \
    { const float x = v.z; r.z = (EXPR); }                                  \
    { const float x = v.w; r.w = (EXPR); }                                  \
    return r;                                                               \
  }
#define SR_V2(NAME, EXPR)                                                   \
  __device__ __noinline__ float4 NAME##_w4(float4 u, float4 v) {            \
    float4 r;                                                               \
    { const float x = u.x, y = v.x; r.x = (EXPR); }                         \
    { const float x = u.y, y = v.y; r.y = (EXPR); }                         \
    { const float x = u.z, y = v.z; r.z = (EXPR); }                         \
    { const float x = u.w, y = v.w; r.w = (EXPR); }                         \
    return r;                                                               \
  }
#endif
SR_V1(v_sin, sr_sinf(x))
SR_V1(v_cos, sr_cosf(x))
SR_V1(v_tan, tanf(x))
SR_V1(v_sinh, sinhf(x))
SR_V1(v_cosh, coshf(x))
SR_V1(v_tanh, tanhf(x))
SR_V1(v_exp, expf(x))
SR_V1(v_log, sr_logf(x))
SR_V1(v_asin, asinf(x))
SR_V1(v_acos, acosf(x))
SR_V1(v_atan, atanf(x))
SR_V1(v_rcp, __frcp_rn(x))
SR_V1(v_sqrt, __fsqrt_rn(x))
SR_V2(v_div, __fdiv_rn(x, y))
SR_V2(v_pow, powf(x, y))
#undef SR_V1
#undef SR_V2

// Y[k] = FN(X[k]) / Y[k] = FN(X[k], Z[k]) for DPT datapoints through the
// routine of width SR_MATH_WIDTH (Y may alias X or Z).
#if SR_MATH_WIDTH == 1
#define SR_MAP1(FN, Y, X)                                                   \
  _Pragma("unroll") for (int k_ = 0; k_ < DPT; ++k_) Y[k_] = FN##_w1(X[k_]);
#define SR_MAP2(FN, Y, X, Z)                                                \
  _Pragma("unroll") for (int k_ = 0; k_ < DPT; ++k_) Y[k_] = FN##_w1(X[k_], Z[k_]);
#elif SR_MATH_WIDTH == 2
#define SR_MAP1(FN, Y, X)                                                   \
  _Pragma("unroll") for (int k_ = 0; k_ < DPT; k_ += 2) {                   \
    const float2 r_ = FN##_w2(make_float2(X[k_], X[k_ + 1]));               \
    Y[k_] = r_.x;                                                           \
    Y[k_ + 1] = r_.y;                                                       \
  }
#define SR_MAP2(FN, Y, X, Z)                                                \
  _Pragma("unroll") for (int k_ = 0; k_ < DPT; k_ += 2) {                   \
    const float2 r_ = FN##_w2(make_float2(X[k_], X[k_ + 1]),                \
                              make_float2(Z[k_], Z[k_ + 1]));               \
    Y[k_] = r_.x;                                                           \
    Y[k_ + 1] = r_.y;                                                       \
  }
#else
#define SR_MAP1(FN, Y, X)                                                   \
  _Pragma("unroll") for (int h_ = 0; h_ < DPT / 4; ++h_)                    \
      unquad<DPT>(Y, h_, FN##_w4(quad<DPT>(X, h_)));
#define SR_MAP2(FN, Y, X, Z)                                                \
  _Pragma("unroll") for (int h_ = 0; h_ < DPT / 4; ++h_)                    \
      unquad<DPT>(Y, h_, FN##_w4(quad<DPT>(X, h_), quad<DPT>(Z, h_)));
#endif

template <int DPT>
__device__ __forceinline__ float4 quad(const float (&v)[DPT], int h) {
  return make_float4(v[4 * h + 0], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}
template <int DPT>
__device__ __forceinline__ void unquad(float (&v)[DPT], int h, float4 q) {
  v[4 * h + 0] = q.x;
  v[4 * h + 1] = q.y;
  v[4 * h + 2] = q.z;
  v[4 * h + 3] = q.w;
}

// T = leaf; kind and payload are warp-uniform.  CACHE = false compiles out
// the cached-subtree kind (programs compiled without cache hints have none),
// which keeps the dispatch code compact.
template <int DPT, bool CACHE = true>
__device__ __forceinline__ void load_leaf(uint32_t kind, uint32_t payload, float (&T)[DPT],
                                          const float *xs, int xrs, int lane,
                                          const float *cache, int64_t ldc, int64_t dp0) {
  if (kind == kLeafX) {
    lds_vec<DPT>(xs + payload * xrs, lane, T);
  } else if (!CACHE || kind == kLeafC) {
    const float c = __uint_as_float(payload);
#pragma unroll
    for (int k = 0; k < DPT; ++k) T[k] = c;
  } else {
    ldg_vec<DPT>(cache + static_cast<int64_t>(payload) * ldc + dp0, lane, T);
  }
}

// b = operand; kind and payload are warp-uniform, kind != kBNone.
// Spill stack of one warp: slots below s_smem in shared memory (ss), the
// rest in global scratch (gs) written and read by the same warp only.
struct SpillStack {
  float *ss;
  float *gs;
  int s_smem;
};

// Slots in global scratch are rare (deep expressions only): their copies
// run out of line, through stack copies of the lane's values, to keep the
// dispatch code compact.
template <int DPT>
__device__ __noinline__ void spill_store_global(float *dst, int lane, const float *src) {
  float v[DPT];
#pragma unroll
  for (int k = 0; k < DPT; ++k) v[k] = src[k];
  stg_vec<DPT>(dst, lane, v);
}

template <int DPT>
__device__ __noinline__ void spill_load_global(const float *src, int lane, float *dst) {
  // Plain (coherent) loads: the data was written by this warp in this kernel.
#pragma unroll
  for (int h = 0; h < DPT / 4; ++h) {
    const float4 q = *reinterpret_cast<const float4 *>(src + h * 128 + lane * 4);
    dst[4 * h + 0] = q.x;
    dst[4 * h + 1] = q.y;
    dst[4 * h + 2] = q.z;
    dst[4 * h + 3] = q.w;
  }
}

template <int DPT>
__device__ __forceinline__ void spill_store(const SpillStack &st, uint32_t slot, int lane,
                                            const float (&T)[DPT]) {
  constexpr int TILE = 32 * DPT;
  if (static_cast<int>(slot) < st.s_smem) {
    sts_vec<DPT>(st.ss + slot * TILE, lane, T);
  } else {
    float t[DPT];
#pragma unroll
    for (int k = 0; k < DPT; ++k) t[k] = T[k];
    spill_store_global<DPT>(st.gs + (slot - st.s_smem) * TILE, lane, t);
  }
}

template <int DPT>
__device__ __forceinline__ void spill_load(const SpillStack &st, uint32_t slot, int lane,
                                           float (&v)[DPT]) {
  constexpr int TILE = 32 * DPT;
  if (static_cast<int>(slot) < st.s_smem) {
    lds_vec<DPT>(st.ss + slot * TILE, lane, v);
  } else {
    float t[DPT];
    spill_load_global<DPT>(st.gs + (slot - st.s_smem) * TILE, lane, t);
#pragma unroll
    for (int k = 0; k < DPT; ++k) v[k] = t[k];
  }
}

// b = operand; kind and payload are warp-uniform, kind != kBNone.
template <int DPT, bool CACHE = true>
__device__ __forceinline__ void load_operand(uint32_t kind, uint32_t payload, float (&b)[DPT],
                                             const float *xs, int xrs, const SpillStack &st,
                                             int lane, const float *cache, int64_t ldc,
                                             int64_t dp0) {
  if (kind == kBX) {
    lds_vec<DPT>(xs + payload * xrs, lane, b);
  } else if (kind == kBS) {
    spill_load<DPT>(st, payload, lane, b);
  } else if (!CACHE || kind == kBC) {
    const float c = __uint_as_float(payload);
#pragma unroll
    for (int k = 0; k < DPT; ++k) b[k] = c;
  } else {
    ldg_vec<DPT>(cache + static_cast<int64_t>(payload) * ldc + dp0, lane, b);
  }
}

#define SR_EACH(STMT)                                            \
  {                                                              \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) { STMT; }   \
  }                                                              \
  break;
#define SR_CALL1(FN) \
  { SR_MAP1(FN, T, T) } \
  break;
#define SR_CALL2(FN, X, Y) \
  { SR_MAP2(FN, T, X, Y) } \
  break;

// One switch case per device opcode: T = op(T, b) (T = op(T) for unary
// operators) for the DPT datapoints of a lane.  Semantics: sr_ops.cuh.
#define SR_C_NONE case 0: break;
// + - * two datapoints at a time in the paired FP32 instructions of sm_100
// (add.rn.f32x2, mul.rn.f32x2): each half is the same correctly rounded
// operation, and a - b is a + (-b) exactly, so results are those of the
// scalar forms (batched subset 12.91 -> 12.70 ms).
#define SR_PAIRED(EXPR)                                                        \
  {                                                                            \
    _Pragma("unroll") for (int k = 0; k < DPT; k += 2) {                       \
      const float2 t_ = make_float2(T[k], T[k + 1]);                           \
      const float2 u_ = make_float2(b[k], b[k + 1]);                           \
      const float2 r_ = (EXPR);                                                \
      T[k] = r_.x;                                                             \
      T[k + 1] = r_.y;                                                         \
    }                                                                          \
  }                                                                            \
  break;
#define SR_C_ADD case 1: SR_PAIRED(__fadd2_rn(t_, u_))
#define SR_C_SUB case 2: SR_PAIRED(__fadd2_rn(t_, make_float2(-u_.x, -u_.y)))
#define SR_C_RSUB case 42: SR_PAIRED(__fadd2_rn(u_, make_float2(-t_.x, -t_.y)))
#define SR_C_MUL case 3: SR_PAIRED(__fmul2_rn(t_, u_))
#define SR_C_DIV /* NaN when the divisor is 0 */                              \
  case 4: {                                                                    \
    SR_MAP2(v_div, T, T, b)                                                    \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = (b[k] == 0.0f) ? qnan() : T[k]; \
  } break;
#define SR_C_RDIV /* b / T */                                                 \
  case 44: {                                                                   \
    float den[DPT];                                                            \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) den[k] = T[k];             \
    SR_MAP2(v_div, T, b, den)                                                  \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = (den[k] == 0.0f) ? qnan() : T[k]; \
  } break;
#define SR_C_POW case 5: SR_CALL2(v_pow, T, b)
#define SR_C_RPOW case 45: SR_CALL2(v_pow, b, T)
#define SR_C_MIN case 6: SR_EACH(T[k] = fminf(T[k], b[k]))
#define SR_C_RMIN case 46: SR_EACH(T[k] = fminf(b[k], T[k]))
#define SR_C_MAX case 7: SR_EACH(T[k] = fmaxf(T[k], b[k]))
#define SR_C_RMAX case 47: SR_EACH(T[k] = fmaxf(b[k], T[k]))
#define SR_C_LDIV /* T / protected(b) */                                      \
  case 8: {                                                                    \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) b[k] = loose_denom(b[k]);  \
  }                                                                            \
    SR_CALL2(v_div, T, b)
#define SR_C_RLDIV /* b / protected(T) */                                     \
  case 48: {                                                                   \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = loose_denom(T[k]);  \
  }                                                                            \
    SR_CALL2(v_div, b, T)
#define SR_C_LPOW /* 0^0 = 0, else |T|^b */                                   \
  case 9: {                                                                    \
    bool z[DPT];                                                               \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) {                          \
      z[k] = (T[k] == 0.0f && b[k] == 0.0f);                                   \
      T[k] = fabsf(T[k]);                                                      \
    }                                                                          \
    SR_MAP2(v_pow, T, T, b)                                                    \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = z[k] ? 0.0f : T[k]; \
  } break;
#define SR_C_RLPOW /* 0^0 = 0, else |b|^T */                                  \
  case 49: {                                                                   \
    bool z[DPT];                                                               \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) {                          \
      z[k] = (T[k] == 0.0f && b[k] == 0.0f);                                   \
      b[k] = fabsf(b[k]);                                                      \
    }                                                                          \
    SR_MAP2(v_pow, T, b, T)                                                    \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = z[k] ? 0.0f : T[k]; \
  } break;
#define SR_C_SIN case 10: SR_CALL1(v_sin)
#define SR_C_COS case 11: SR_CALL1(v_cos)
#define SR_C_TAN case 12: SR_CALL1(v_tan)
#define SR_C_SINH case 13: SR_CALL1(v_sinh)
#define SR_C_COSH case 14: SR_CALL1(v_cosh)
#define SR_C_TANH case 15: SR_CALL1(v_tanh)
#define SR_C_EXP case 16: SR_CALL1(v_exp)
#define SR_C_LOG case 17: SR_CALL1(v_log)
#define SR_C_INV case 18: SR_CALL1(v_rcp)
#define SR_C_ASIN case 19: SR_CALL1(v_asin)
#define SR_C_ACOS case 20: SR_CALL1(v_acos)
#define SR_C_ATAN case 21: SR_CALL1(v_atan)
#define SR_C_LLOG /* -1e9 at 0, else log|T| */                                \
  case 22: {                                                                   \
    bool z[DPT];                                                               \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) {                          \
      z[k] = (T[k] == 0.0f);                                                   \
      T[k] = fabsf(T[k]);                                                      \
    }                                                                          \
    SR_MAP1(v_log, T, T)                                                       \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = z[k] ? -1e9f : T[k]; \
  } break;
#define SR_C_LINV /* 1 / protected(T) */                                      \
  case 23: {                                                                   \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = loose_denom(T[k]);  \
  }                                                                            \
    SR_CALL1(v_rcp)
#define SR_C_ABS case 24: SR_EACH(T[k] = fabsf(T[k]))
#define SR_C_NEG case 25: SR_EACH(T[k] = -T[k])
#define SR_C_SQRT case 26: SR_CALL1(v_sqrt)
#define SR_C_LSQRT /* sqrt|T| */                                              \
  case 27: {                                                                   \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = fabsf(T[k]);        \
  }                                                                            \
    SR_CALL1(v_sqrt)
#define SR_C_EXPC /* exp clamped at 80 (extension) */                         \
  case 32: {                                                                   \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = fminf(T[k], 80.0f); \
  }                                                                            \
    SR_CALL1(v_exp)

// Inline forms of exp (a few instructions around ex2), sqrt and the IEEE
// division: the same functions expanded at their case instead of called two
// datapoints at a time, for the switches of the protected profile and of its
// out-of-line path, in launches of at most 8 datapoints per thread.  There a
// call cost more than these bodies (batched population forward 78.7 -> 73.7
// ms, subtree-cache population 44.9 -> 42.0 ms, results bit-identical); at 16
// datapoints per thread the copies cost more than the calls (36.8 -> 40.6 ms).
// sin / cos / log stay out of line (inlined, the instruction cache overflows:
// 100.6 ms with sin and cos inline), and so do all of them in the
// every-operator switch (kOpsAll), which inlining made slower (150.1 -> 162.3
// ms on a population that uses every operator).
constexpr int kInlineMaxDpt = 8;  // wider launches call them (16 copies overflow the I-cache)
#define SR_C_INL_OR(CASE, INLINE_STMT, CALLED)                                 \
  case CASE:                                                                   \
    if constexpr (DPT <= kInlineMaxDpt) {                                      \
      _Pragma("unroll") for (int k = 0; k < DPT; ++k) { INLINE_STMT; }         \
    } else {                                                                   \
      CALLED                                                                   \
    }                                                                          \
    break;
#define SR_C_EXPC_INL                                                          \
  SR_C_INL_OR(32, T[k] = expf(fminf(T[k], 80.0f)),                             \
              _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = fminf(T[k], 80.0f); \
              SR_MAP1(v_exp, T, T))
#define SR_C_LSQRT_INL                                                         \
  SR_C_INL_OR(27, T[k] = __fsqrt_rn(fabsf(T[k])),                              \
              _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = fabsf(T[k]); \
              SR_MAP1(v_sqrt, T, T))
#define SR_C_LDIV_INL                                                          \
  SR_C_INL_OR(8, T[k] = __fdiv_rn(T[k], loose_denom(b[k])),                    \
              _Pragma("unroll") for (int k = 0; k < DPT; ++k) b[k] = loose_denom(b[k]); \
              SR_MAP2(v_div, T, T, b))
#define SR_C_RLDIV_INL                                                         \
  SR_C_INL_OR(48, T[k] = __fdiv_rn(b[k], loose_denom(T[k])),                   \
              _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = loose_denom(T[k]); \
              SR_MAP2(v_div, T, b, T))

// sin / cos / protected log (this library's own, sr_math.cuh) expanded at
// their case in the protected profile's switch at up to 8 datapoints per
// thread.  sin and cos take their fast path for every datapoint of the lane;
// a lane holding an argument beyond the fast range (|x| > 32768, inf, NaN)
// evaluates its datapoints through sincos_cold instead (out of line, rare).
template <int DPT>
__device__ __noinline__ void sincos_cold(float *T, int q_offset) {
#pragma unroll
  for (int k = 0; k < DPT; ++k) T[k] = q_offset ? sr_cosf(T[k]) : sr_sinf(T[k]);
}
#define SR_C_SINCOS_INL(CASE, QOFF, NAME)                                      \
  case CASE:                                                                   \
    if constexpr (DPT <= kInlineMaxDpt) {                                      \
      bool slow_ = false;                                                      \
      _Pragma("unroll") for (int k = 0; k < DPT; ++k) slow_ |= !sincos_fast_ok(T[k]); \
      if (slow_) {                                                             \
        float t_[DPT];                                                         \
        _Pragma("unroll") for (int k = 0; k < DPT; ++k) t_[k] = T[k];          \
        sincos_cold<DPT>(t_, QOFF);                                            \
        _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = t_[k];          \
      } else {                                                                 \
        _Pragma("unroll") for (int k = 0; k < DPT; k += 2) {                   \
          SinCosParts p0_, p1_;                                                \
          sincos_parts2(make_float2(T[k], T[k + 1]), p0_, p1_);                \
          const float y0_ = sincos_pick(p0_, QOFF), y1_ = sincos_pick(p1_, QOFF); \
          T[k] = (QOFF == 0 && T[k] == 0.0f) ? T[k] : y0_;                     \
          T[k + 1] = (QOFF == 0 && T[k + 1] == 0.0f) ? T[k + 1] : y1_;         \
        }                                                                      \
      }                                                                        \
    } else {                                                                   \
      SR_MAP1(NAME, T, T)                                                      \
    }                                                                          \
    break;
#define SR_C_SIN_INL SR_C_SINCOS_INL(10, 0, v_sin)
#define SR_C_COS_INL SR_C_SINCOS_INL(11, 1, v_cos)
#define SR_C_LLOG_INL                                                          \
  SR_C_INL_OR(22, if ((k & 1) == 0) {                                          \
                const float2 l_ = sr_log_nonneg2(fabsf(T[k]), fabsf(T[k + 1])); \
                T[k] = T[k] == 0.0f ? -1e9f : l_.x;                            \
                T[k + 1] = T[k + 1] == 0.0f ? -1e9f : l_.y;                    \
              },                                                               \
              {                                                                \
                bool z_[DPT];                                                  \
                _Pragma("unroll") for (int k = 0; k < DPT; ++k) {              \
                  z_[k] = (T[k] == 0.0f);                                      \
                  T[k] = fabsf(T[k]);                                          \
                }                                                              \
                SR_MAP1(v_log, T, T)                                           \
                _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = z_[k] ? -1e9f : T[k]; \
              })

// Operator profiles (kOpsAll / kOpsProtected and the host-side membership
// test live in sr_internal.hpp).  kOpsAll dispatches every operator inline;
// kOpsProtected dispatches + - *, protected division, sin, cos, exp clamped
// at 80, protected log and sqrt|x| (the evolution workloads' set) inline and
// every other operator through apply_op_cold, one out-of-line routine with
// the complete switch.  Keeping cases out of the inline switch keeps the
// interpreter's hot code compact (instruction-cache pressure): on the batched
// population, whose operators are kOpsProtected's, the forward launch took
// 95.6 ms with every case inline and 82.9 ms with kOpsProtected's inline set;
// a population that uses every operator (the reference generator's) runs
// faster with all of them inline.

template <int DPT>
__device__ __forceinline__ void apply_op_any(uint32_t op, float (&T)[DPT], float (&b)[DPT]) {
  switch (op) {
    SR_C_NONE SR_C_ADD SR_C_SUB SR_C_RSUB SR_C_MUL SR_C_DIV SR_C_RDIV SR_C_POW SR_C_RPOW
    SR_C_MIN SR_C_RMIN SR_C_MAX SR_C_RMAX SR_C_LDIV SR_C_RLDIV SR_C_LPOW SR_C_RLPOW
    SR_C_SIN SR_C_COS SR_C_TAN SR_C_SINH SR_C_COSH SR_C_TANH SR_C_EXP SR_C_LOG SR_C_INV
    SR_C_ASIN SR_C_ACOS SR_C_ATAN SR_C_LLOG SR_C_LINV SR_C_ABS SR_C_NEG SR_C_SQRT SR_C_LSQRT
    SR_C_EXPC
    default: SR_EACH(T[k] = 0.0f)
  }
}

// Out-of-line entry of the operators outside a profile; T and b travel
// through the caller's stack (copies, so the caller's arrays stay in
// registers).
// The complete switch of the out-of-line path (apply_op_cold), with the
// inline forms above.
template <int DPT>
__device__ __forceinline__ void apply_op_cold_switch(uint32_t op, float (&T)[DPT],
                                                     float (&b)[DPT]) {
  switch (op) {
    SR_C_NONE SR_C_ADD SR_C_SUB SR_C_RSUB SR_C_MUL SR_C_DIV SR_C_RDIV SR_C_POW SR_C_RPOW
    SR_C_MIN SR_C_RMIN SR_C_MAX SR_C_RMAX SR_C_LDIV_INL SR_C_RLDIV_INL SR_C_LPOW SR_C_RLPOW
    SR_C_SIN SR_C_COS SR_C_TAN SR_C_SINH SR_C_COSH SR_C_TANH SR_C_EXP SR_C_LOG SR_C_INV
    SR_C_ASIN SR_C_ACOS SR_C_ATAN SR_C_LLOG SR_C_LINV SR_C_ABS SR_C_NEG SR_C_SQRT SR_C_LSQRT_INL
    SR_C_EXPC_INL
    default: SR_EACH(T[k] = 0.0f)
  }
}

template <int DPT>
__device__ __noinline__ void apply_op_cold(uint32_t op, float *T, float *b) {
  float t[DPT], bb[DPT];
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    t[k] = T[k];
    bb[k] = b[k];
  }
  apply_op_cold_switch<DPT>(op, t, bb);
#pragma unroll
  for (int k = 0; k < DPT; ++k) T[k] = t[k];
}

#define SR_C_COLD                                                              \
  default: {                                                                   \
    float t_[DPT], b_[DPT];                                                    \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) {                          \
      t_[k] = T[k];                                                            \
      b_[k] = b[k];                                                            \
    }                                                                          \
    apply_op_cold<DPT>(op, t_, b_);                                            \
    _Pragma("unroll") for (int k = 0; k < DPT; ++k) T[k] = t_[k];              \
  } break;

template <int DPT, int OPS>
__device__ __forceinline__ void apply_op(uint32_t op, float (&T)[DPT], float (&b)[DPT]) {
  if constexpr (OPS == kOpsProtected) {
    switch (op) {
      SR_C_NONE SR_C_ADD SR_C_SUB SR_C_RSUB SR_C_MUL SR_C_LDIV_INL SR_C_RLDIV_INL SR_C_SIN_INL
      SR_C_COS_INL SR_C_EXPC_INL SR_C_LLOG_INL SR_C_LSQRT_INL
      SR_C_COLD
    }
  } else {
    apply_op_any<DPT>(op, T, b);
  }
}

#undef SR_EACH
#undef SR_CALL1
#undef SR_CALL2
#undef SR_C_COLD

// Run one compiled program over the warp's DPT x 32 datapoints of a tile.
// xs points at the tile's first datapoint of X row 0; rows are xrs floats
// apart.
template <int DPT, int OPS, bool CACHE>
__device__ __forceinline__ void run_program(const Instr *__restrict__ code,
                                            int len, const float *xs, int xrs,
                                            const SpillStack &st, int lane,
                                            const float *cache, int64_t ldc, int64_t dp0,
                                            float (&T)[DPT]) {
  // Every program starts with an instruction that loads T.
  uint4 ins = ldg_instr(code);
  for (int i = 0; i < len; ++i) {
    // The code buffer ends with a padding instruction, so this prefetch of
    // the next word is always in bounds.
    const uint4 nxt = ldg_instr(code + i + 1);
    const uint32_t w = ins.x;
    if (w & (kLoadBit | kSpillBit)) {
      if (instr_spill(w)) spill_store<DPT>(st, instr_spill_slot(w), lane, T);
      if (instr_load(w))
        load_leaf<DPT, CACHE>(instr_leaf_kind(w), ins.y, T, xs, xrs, lane, cache, ldc, dp0);
    }
    float b[DPT];
    const uint32_t bk = instr_b_kind(w);
    if (bk != kBNone) load_operand<DPT, CACHE>(bk, ins.z, b, xs, xrs, st, lane, cache, ldc, dp0);
    apply_op<DPT, OPS>(instr_op(w), T, b);
    ins = nxt;
  }
}

// Sum of the valid squared errors of a lane's DPT datapoints in FP64: the
// fallback when the FP32 Kahan sum overflowed (or a square is infinite); exact
// for DPT finite squares and +Inf when one is infinite, like the reference's
// double sum.  Out of line: it almost never runs.
template <int DPT>
__device__ __noinline__ double tile_sum_fp64(const float *T, const float *y, bool full,
                                             int64_t dp0, int lane, int64_t N) {
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    const bool valid = (full || dp0 + (k / 4) * 128 + lane * 4 + (k % 4) < N) && isfinite(T[k]);
    const float df = __fsub_rn(T[k], y[k]);
    sum += valid ? static_cast<double>(__fmul_rn(df, df)) : 0.0;
  }
  return sum;
}

// Per-span result of one expression of a work item, written by the warp that
// evaluated it (shared memory, one slot per buffer and group position).
struct SpanPart {
  double sum;   // sum of the valid squared errors over the span
  int32_t cnt;  // valid datapoints
  int32_t e;    // expression
};

// Per-item accumulator of one expression (producer thread only): the span
// sums added in span order as a double-double (hi + lo, Knuth's two-sum), so
// that the result does not depend on how many spans an item covers.
struct GroupAcc {
  double hi, lo, cnt;
  int32_t e, pad;
};

__device__ __forceinline__ void dd_add(double &hi, double &lo, double x) {
  const double s = __dadd_rn(hi, x);
  if (isfinite(s)) {
    const double bb = __dsub_rn(s, hi);
    lo = __dadd_rn(lo, __dadd_rn(__dsub_rn(hi, __dsub_rn(s, bb)), __dsub_rn(x, bb)));
  } else {
    lo = 0.0;  // an infinite sum stays infinite
  }
  hi = s;
}

// What the producer of an MSE launch folds: the span slots, its accumulators
// and where a finished item's sums go ([span group][E] entries of two
// double2: (hi, lo) and (count, 0)).  n_valid: expressions in the launch's
// group table (groups are padded at their end only).  Gradient launches
// (K > 0) also fold each expression's constant gradients: K doubles per span
// slot, added in span order into K doubles per expression, written out to
// gout[span group][C] at the expression's constant offset.
struct FoldArgs {
  SpanPart *part;  // [kBufs][G]
  GroupAcc *acc;   // [G]
  double2 *out;
  int G, E, n_valid;
  int K;
  const double *gpart;       // [kBufs][G][K]
  double *gacc;              // [G][K]
  double *gout;              // [span groups][C]
  const int64_t *const_off;  // [E]
  const int32_t *const_cnt;  // [E]
  int64_t C;
};

// The producer thread of a block: claims work items from the global counter
// (item = span group x expression group; single-span items are numbered
// span-major, so concurrent blocks share X spans in L2; multi-span items
// expression-group-major, so the most expensive groups, which come first in
// the cost-sorted group table, are claimed first and the last items are the
// cheapest), and copies each of the item's spans
// (k_spans consecutive spans, the last group shorter) with every row of X
// into one of kBufs shared-memory buffers with the bulk-copy engine;
// publishes item -1 when the work runs out.  With FOLD (MSE launches) it also
// folds, once the warps have released a buffer, the span slots written for it
// into the item's accumulators (in span order) and writes each finished
// item's sums out.  Every wait is bounded.
template <bool FOLD>
__device__ __noinline__ void run_producer(int n_groups, int n_items, int k_spans, int n_spans,
                                          int32_t *work_counter, int32_t *error, const float *X,
                                          int64_t ldx, int rows, int span, float *xbuf,
                                          ItemDesc *desc, uint64_t *full, uint64_t *empty,
                                          FoldArgs fa) {
  uint32_t buf = 0, phase = 0;
  uint32_t armed = 0;  // buffers with a copy in flight
  uint32_t fill_phase[kBufs] = {0, 0};
  bool held[kBufs] = {false, false};  // a span whose slots are still to fold
  int held_item[kBufs] = {0, 0}, held_group[kBufs] = {0, 0};
  int acc_item = -1, acc_sg = 0, acc_n = 0;
  const uint32_t row_bytes = static_cast<uint32_t>(span) * sizeof(float);

  auto flush = [&]() {
    if constexpr (FOLD) {
      if (acc_item < 0) return;
      for (int j = 0; j < acc_n; ++j) {
        const GroupAcc a = fa.acc[j];
        double2 *o = fa.out + 2 * (static_cast<int64_t>(acc_sg) * fa.E + a.e);
        o[0] = make_double2(a.hi, a.lo);
        o[1] = make_double2(a.cnt, 0.0);
        if (fa.K > 0) {
          const int nc = min(fa.const_cnt[a.e], fa.K);
          double *g = fa.gout + static_cast<int64_t>(acc_sg) * fa.C + fa.const_off[a.e];
          for (int c = 0; c < nc; ++c) g[c] = fa.gacc[j * fa.K + c];
        }
      }
      acc_item = -1;
    }
  };
  auto fold = [&](uint32_t b) {
    if constexpr (FOLD) {
      const int it = held_item[b];
      if (it != acc_item) {
        flush();
        acc_item = it;
        acc_sg = k_spans > 1 ? it % ((n_spans + k_spans - 1) / k_spans) : it / n_groups;
        const int g = held_group[b];
        acc_n = min(fa.G, fa.n_valid - g * fa.G);  // groups are padded at their end only
        for (int j = 0; j < acc_n; ++j) fa.acc[j] = GroupAcc{0.0, 0.0, 0.0, 0, 0};
        for (int j = 0; j < acc_n * fa.K; ++j) fa.gacc[j] = 0.0;
      }
      const SpanPart *q = fa.part + static_cast<size_t>(b) * fa.G;
      for (int j = 0; j < acc_n; ++j) {
        const SpanPart v = q[j];
        dd_add(fa.acc[j].hi, fa.acc[j].lo, v.sum);
        fa.acc[j].cnt += static_cast<double>(v.cnt);
        fa.acc[j].e = v.e;
      }
      if (fa.K > 0) {
        const double *gq = fa.gpart + static_cast<size_t>(b) * fa.G * fa.K;
        for (int j = 0; j < acc_n * fa.K; ++j) fa.gacc[j] += gq[j];
      }
      held[b] = false;
    }
  };
  auto drain = [&]() {
    // Let copies already issued land before the block exits.
    if (armed & 1u) mbar_drain(&full[0], fill_phase[0]);
    if (armed & 2u) mbar_drain(&full[1], fill_phase[1]);
  };

  for (;;) {
    const int item = atomicAdd(work_counter, 1);
    const bool last = item >= n_items;
    const int n_sg = (n_spans + k_spans - 1) / k_spans;
    const int group = last ? 0 : (k_spans > 1 ? item / n_sg : item % n_groups);
    const int sgi = last ? 0 : (k_spans > 1 ? item % n_sg : item / n_groups);
    const int s_begin = sgi * k_spans;
    const int s_end = last ? 1 : min(n_spans, s_begin + k_spans);
    for (int sp = s_begin; sp < s_end; ++sp) {
      if (!mbar_wait(&empty[buf], phase ^ 1u, error)) {
        drain();
        return;
      }
      // The consumers released this buffer, so its previous copy landed and
      // its span slots are complete.
      armed &= ~(1u << buf);
      if (held[buf]) fold(buf);
      if (last) {
        desc[buf] = ItemDesc{-1, 0, 0, 0};
        mbar_arrive(&full[buf]);
        if (FOLD) {
          const uint32_t other = buf ^ 1u;
          if (held[other]) {
            if (!mbar_wait(&empty[other], fill_phase[other], error)) {
              drain();
              return;
            }
            fold(other);
          }
          flush();
        }
        return;
      }
      desc[buf] = ItemDesc{item, group, sp, 0};
      mbar_arrive_expect_tx(&full[buf], row_bytes * rows);
      const float *src = X + static_cast<int64_t>(sp) * span;
      float *dst = xbuf + static_cast<size_t>(buf) * rows * span;
      for (int v = 0; v < rows; ++v)
        bulk_g2s(dst + static_cast<size_t>(v) * span, src + v * ldx, row_bytes, &full[buf]);
      armed |= 1u << buf;
      fill_phase[buf] = phase;
      held[buf] = FOLD;
      held_item[buf] = item;
      held_group[buf] = group;
      if (++buf == kBufs) {
        buf = 0;
        phase ^= 1u;
      }
    }
  }
}

}  // namespace
}  // namespace sr
