// sr_ops.cuh — FP32 operator semantics on the device.
//
// One definition per reference operator, following eval_op_cpu
// (src/cleaned/cl_cpu_eval.cpp:16-56), which is identical to the reference
// device version eval_op_gpu_state (src/cleaned/cl_gpu_eval.cu:14-54):
// x is the first popped (left) operand, y the second.  sin, cos and log are
// this library's own (sr_math.cuh); the other functions are the CUDA math
// library's, called as they are; IEEE-rounded intrinsics are spelled out for
// the basic operations so no contraction into FMA can change a result.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "sr_math.cuh"

namespace sr {

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fc00000); }

// Protected denominator of LOOSE_DIV / LOOSE_INV: |d| <= 1e-9 becomes +-1e-9
// (sign of d; -0 and +0 both give +1e-9), NaN stays NaN.
__device__ __forceinline__ float loose_denom(float d) {
  const float kDelta = 1e-9f;
  return fabsf(d) <= kDelta ? (d < 0.0f ? -kDelta : kDelta) : d;
}

__device__ __forceinline__ float op_binary(int op, float x, float y) {
  switch (op) {
    case 1: return __fadd_rn(x, y);
    case 2: return __fsub_rn(x, y);
    case 3: return __fmul_rn(x, y);
    case 4: return (y == 0.0f) ? qnan() : __fdiv_rn(x, y);
    case 5: return powf(x, y);
    case 6: return fminf(x, y);
    case 7: return fmaxf(x, y);
    case 8: return __fdiv_rn(x, loose_denom(y));
    case 9: return (x == 0.0f && y == 0.0f) ? 0.0f : powf(fabsf(x), y);
    default: return 0.0f;
  }
}

__device__ __forceinline__ float op_unary(int op, float x) {
  switch (op) {
    case 0: return x;  // MOV (bytecode only)
    case 10: return sr_sinf(x);
    case 11: return sr_cosf(x);
    case 12: return tanf(x);
    case 13: return sinhf(x);
    case 14: return coshf(x);
    case 15: return tanhf(x);
    case 16: return expf(x);
    case 17: return sr_logf(x);
    case 18: return __frcp_rn(x);
    case 19: return asinf(x);
    case 20: return acosf(x);
    case 21: return atanf(x);
    case 22: return sr_loose_logf(x);
    case 23: return __frcp_rn(loose_denom(x));
    case 24: return fabsf(x);
    case 25: return -x;
    case 26: return __fsqrt_rn(x);
    case 27: return __fsqrt_rn(fabsf(x));
    case 32: return expf(fminf(x, 80.0f));
    default: return 0.0f;
  }
}

__device__ __forceinline__ float op_apply(int op, float x, float y) {
  return (op >= 1 && op <= 9) ? op_binary(op, x, y) : op_unary(op, x);
}

// The same operators evaluated in double: the FP64 reference of the accuracy
// report (MIN / MAX as fmin / fmax like the float path; the protected regions
// at 1e-9; LOOSE_LOG -1e9 at 0).
__device__ __forceinline__ double op_apply_f64(int op, double x, double y) {
  const double kDelta = 1e-9;
  switch (op) {
    case 1: return x + y;
    case 2: return x - y;
    case 3: return x * y;
    case 4: return (y == 0.0) ? __longlong_as_double(0x7ff8000000000000ll) : x / y;
    case 5: return pow(x, y);
    case 6: return fmin(x, y);
    case 7: return fmax(x, y);
    case 8: return x / (fabs(y) <= kDelta ? (y < 0.0 ? -kDelta : kDelta) : y);
    case 9: return (x == 0.0 && y == 0.0) ? 0.0 : pow(fabs(x), y);
    case 10: return sin(x);
    case 11: return cos(x);
    case 12: return tan(x);
    case 13: return sinh(x);
    case 14: return cosh(x);
    case 15: return tanh(x);
    case 16: return exp(x);
    case 17: return log(x);
    case 18: return 1.0 / x;
    case 19: return asin(x);
    case 20: return acos(x);
    case 21: return atan(x);
    case 22: return (x == 0.0) ? -1e9 : log(fabs(x));
    case 23: return 1.0 / (fabs(x) <= kDelta ? (x < 0.0 ? -kDelta : kDelta) : x);
    case 24: return fabs(x);
    case 25: return -x;
    case 26: return sqrt(x);
    case 27: return sqrt(fabs(x));
    case 32: return exp(fmin(x, 80.0));
    default: return 0.0;
  }
}

}  // namespace sr
