// sr_math.cuh — the evaluator's own single-precision sin, cos and log.
//
// CUDA's accurate sinf / cosf / logf are general-purpose routines (each with
// a slow path for arguments its fast path cannot reduce) that cost 30+
// instructions a datapoint and, DPT times inlined into the interpreter's
// dispatch switch, overflow the instruction cache, so the interpreter had to
// call them out of line.  These versions are short enough to be expanded at
// their switch case:
//
//   * sin / cos: Cody and Waite's argument reduction (W. J. Cody, W. Waite,
//     Software Manual for the Elementary Functions, 1980) by pi/2, with a
//     three-part float constant applied by fused multiply-adds, and minimax
//     polynomials on [-pi/4, pi/4] (Remez exchange algorithm, coefficients
//     derived by csrc/gen_minimax.py): sin r = r + r^3 S(r^2), cos r = 1 +
//     r^2 (-1/2 + r^2 C(r^2)), S and C of degree 2; the quadrant picks the
//     polynomial and the sign.  Arguments with |x| > 32768 and non-finite
//     ones go to CUDA's sinf / cosf, out of line.
//   * log: x = 2^e m with m in [sqrt(1/2), sqrt(2)), f = m - 1 (exact),
//     log x = e ln2 + f - f^2/2 + f^3 R(f) (R of degree 7, minimax, same
//     script), ln2 split in two so that e * ln2_hi is exact; subnormal
//     arguments are scaled by 2^23 first.
//
// The interpreter evaluates two datapoints at once with the paired FP32
// instructions of sm_100 (fma.rn.f32x2 and friends: sincos_parts2,
// sr_log_nonneg2); each half is the same correctly rounded operation as the
// scalar form, so both forms give identical results.
//
// Their accuracy is measured on every float argument against the correctly
// rounded value (sr_check_math, tests/test_gpu_math.py) and is the device
// column of the parity rule's error table.  Every kernel of this library that
// evaluates these operators calls these functions, so results do not depend
// on which kernel or dispatch path evaluates an operator.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace sr {
namespace {  // one copy per kernel translation unit

// pi/2 = kPio2Hi + kPio2Mid + kPio2Lo to about 1e-23.
constexpr float kTwoOverPi = 0.636619772f;
constexpr float kPio2Hi = 1.57079637f;
constexpr float kPio2Mid = -4.37113883e-08f;
constexpr float kPio2Lo = -1.71512451e-15f;
constexpr float kSinCosFastMax = 32768.0f;  // larger |x|: CUDA's sinf / cosf
// 1.5 * 2^23: adding it rounds a float of magnitude below 2^22 to an integer
// held in the low mantissa bits.
constexpr float kRoundMagic = 12582912.0f;

// sin r = r + r^3 (kS0 + z (kS1 + z kS2)), z = r^2
constexpr float kS0 = -0.166666546743f;
constexpr float kS1 = 0.00833210095313f;
constexpr float kS2 = -0.000195039631257f;
// cos r = 1 + z (-1/2 + z (kC0 + z (kC1 + z kC2)))
constexpr float kC0 = 0.0416666546518f;
constexpr float kC1 = -0.00138876543845f;
constexpr float kC2 = 2.4463837439e-05f;

// Reduced argument, quadrant and both polynomials of x (|x| <= 32768).
struct SinCosParts {
  float s, c;  // sin r, cos r
  int q;       // quadrant (x = q pi/2 + r)
};

__device__ __forceinline__ SinCosParts sincos_parts(float x) {
  const float t = fmaf(x, kTwoOverPi, kRoundMagic);
  const float j = __fsub_rn(t, kRoundMagic);
  SinCosParts p;
  p.q = __float_as_int(t);  // low bits: j mod 2^22
  float r = fmaf(-j, kPio2Hi, x);
  r = fmaf(-j, kPio2Mid, r);
  r = fmaf(-j, kPio2Lo, r);
  const float z = __fmul_rn(r, r);
  float ps = fmaf(kS2, z, kS1);
  ps = fmaf(ps, z, kS0);
  p.s = fmaf(__fmul_rn(r, z), ps, r);
  float pc = fmaf(kC2, z, kC1);
  pc = fmaf(pc, z, kC0);
  pc = fmaf(pc, z, -0.5f);
  p.c = fmaf(z, pc, 1.0f);
  return p;
}

// sin (q_offset 0) or cos (q_offset 1) from the parts.
__device__ __forceinline__ float sincos_pick(const SinCosParts &p, int q_offset) {
  const int q = p.q + q_offset;
  const float y = (q & 1) ? p.c : p.s;
  return __int_as_float(__float_as_int(y) ^ ((q & 2) << 30));
}

__device__ __forceinline__ bool sincos_fast_ok(float x) { return fabsf(x) <= kSinCosFastMax; }

__device__ __noinline__ float sincos_slow(float x, int q_offset) {
  return q_offset ? cosf(x) : sinf(x);
}

__device__ __forceinline__ float sr_sinf(float x) {
  if (!sincos_fast_ok(x)) return sincos_slow(x, 0);
  const float y = sincos_pick(sincos_parts(x), 0);
  return x == 0.0f ? x : y;  // sin(-0) = -0
}

__device__ __forceinline__ float sr_cosf(float x) {
  if (!sincos_fast_ok(x)) return sincos_slow(x, 1);
  return sincos_pick(sincos_parts(x), 1);
}

// sin and cos of the same argument (one reduction): the values sr_sinf and
// sr_cosf return.
__device__ __forceinline__ void sr_sincosf(float x, float *s, float *c) {
  if (!sincos_fast_ok(x)) {
    *s = sincos_slow(x, 0);
    *c = sincos_slow(x, 1);
    return;
  }
  const SinCosParts p = sincos_parts(x);
  const float sv = sincos_pick(p, 0);
  *s = x == 0.0f ? x : sv;
  *c = sincos_pick(p, 1);
}

// Two arguments at once in paired FP32 operations (fma.rn.f32x2 and friends:
// each half is the same correctly rounded operation as the scalar form, so
// the results are those of sincos_parts).
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ void sincos_parts2(float2 x, SinCosParts &p0, SinCosParts &p1) {
  const float2 t = __ffma2_rn(x, f2(kTwoOverPi), f2(kRoundMagic));
  const float2 j = __fadd2_rn(t, f2(-kRoundMagic));
  p0.q = __float_as_int(t.x);
  p1.q = __float_as_int(t.y);
  float2 r = __ffma2_rn(j, f2(-kPio2Hi), x);
  r = __ffma2_rn(j, f2(-kPio2Mid), r);
  r = __ffma2_rn(j, f2(-kPio2Lo), r);
  const float2 z = __fmul2_rn(r, r);
  float2 ps = __ffma2_rn(f2(kS2), z, f2(kS1));
  ps = __ffma2_rn(ps, z, f2(kS0));
  const float2 s = __ffma2_rn(__fmul2_rn(r, z), ps, r);
  float2 pc = __ffma2_rn(f2(kC2), z, f2(kC1));
  pc = __ffma2_rn(pc, z, f2(kC0));
  pc = __ffma2_rn(pc, z, f2(-0.5f));
  const float2 c = __ffma2_rn(z, pc, f2(1.0f));
  p0.s = s.x; p1.s = s.y; p0.c = c.x; p1.c = c.y;
}

// log(1 + f) = f + f^2 (-1/2 + f R(f)), R(f) = kR0 + f (kR1 + ... f kR7)
constexpr float kR0 = 0.333333317078f;
constexpr float kR1 = -0.250008210321f;
constexpr float kR2 = 0.20001226863f;
constexpr float kR3 = -0.166233574103f;
constexpr float kR4 = 0.142017583522f;
constexpr float kR5 = -0.13160182163f;
constexpr float kR6 = 0.127615745496f;
constexpr float kR7 = -0.0763449398631f;
// ln 2 = kLn2Hi + kLn2Lo; kLn2Hi has 10 trailing zero bits, so e * kLn2Hi
// is exact for every exponent e.
constexpr float kLn2Hi = 0.693115234f;
constexpr float kLn2Lo = 3.19461833e-05f;

// log(a) for a >= 0 (+inf and NaN pass through, log(0) = -inf).
__device__ __forceinline__ float sr_log_nonneg(float a) {
  const bool sub = a < 1.17549435e-38f;
  const float as = sub ? __fmul_rn(a, 8388608.0f) : a;
  const int ia = __float_as_int(as);
  // e such that as / 2^e lies in [sqrt(1/2), sqrt(2)); 0x3f3504f3 is
  // sqrt(1/2) rounded to float.
  const int e = (ia - 0x3f3504f3) >> 23;
  const float m = __int_as_float(ia - (e << 23));
  const float f = __fsub_rn(m, 1.0f);
  const float ef = static_cast<float>(sub ? e - 23 : e);
  float p = fmaf(kR7, f, kR6);
  p = fmaf(p, f, kR5);
  p = fmaf(p, f, kR4);
  p = fmaf(p, f, kR3);
  p = fmaf(p, f, kR2);
  p = fmaf(p, f, kR1);
  p = fmaf(p, f, kR0);
  p = fmaf(p, f, -0.5f);
  const float y = fmaf(__fmul_rn(f, f), p, f);
  const float r = fmaf(ef, kLn2Hi, fmaf(ef, kLn2Lo, y));
  return (a == 0.0f) ? __int_as_float(0xff800000) : (a < INFINITY ? r : a);
}

// sr_log_nonneg of two arguments, the polynomial in paired operations.
__device__ __forceinline__ float2 sr_log_nonneg2(float a0, float a1) {
  const bool sub0 = a0 < 1.17549435e-38f, sub1 = a1 < 1.17549435e-38f;
  const float as0 = sub0 ? __fmul_rn(a0, 8388608.0f) : a0;
  const float as1 = sub1 ? __fmul_rn(a1, 8388608.0f) : a1;
  const int ia0 = __float_as_int(as0), ia1 = __float_as_int(as1);
  const int e0 = (ia0 - 0x3f3504f3) >> 23, e1 = (ia1 - 0x3f3504f3) >> 23;
  const float2 m = make_float2(__int_as_float(ia0 - (e0 << 23)), __int_as_float(ia1 - (e1 << 23)));
  const float2 f = __fadd2_rn(m, f2(-1.0f));
  const float2 ef = make_float2(static_cast<float>(sub0 ? e0 - 23 : e0),
                                static_cast<float>(sub1 ? e1 - 23 : e1));
  float2 p = __ffma2_rn(f2(kR7), f, f2(kR6));
  p = __ffma2_rn(p, f, f2(kR5));
  p = __ffma2_rn(p, f, f2(kR4));
  p = __ffma2_rn(p, f, f2(kR3));
  p = __ffma2_rn(p, f, f2(kR2));
  p = __ffma2_rn(p, f, f2(kR1));
  p = __ffma2_rn(p, f, f2(kR0));
  p = __ffma2_rn(p, f, f2(-0.5f));
  const float2 y = __ffma2_rn(__fmul2_rn(f, f), p, f);
  const float2 r = __ffma2_rn(ef, f2(kLn2Hi), __ffma2_rn(ef, f2(kLn2Lo), y));
  return make_float2(
      (a0 == 0.0f) ? __int_as_float(0xff800000) : (a0 < INFINITY ? r.x : a0),
      (a1 == 0.0f) ? __int_as_float(0xff800000) : (a1 < INFINITY ? r.y : a1));
}

// logf semantics: NaN for negative arguments.
__device__ __forceinline__ float sr_logf(float x) {
  return x < 0.0f ? __int_as_float(0x7fc00000) : sr_log_nonneg(x);
}

// Protected log (reference LOOSE_LOG): -1e9 at 0, else log|x|.
__device__ __forceinline__ float sr_loose_logf(float x) {
  return x == 0.0f ? -1e9f : sr_log_nonneg(fabsf(x));
}

}  // namespace
}  // namespace sr
