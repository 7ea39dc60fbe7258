// sr_mathcheck.cu — accuracy of the library's own sin / cos / log
// (sr_math.cuh), measured on the device over ranges of float arguments
// against the correctly rounded value, for the tests and the parity rule's
// table of device errors.  No counterpart in the reference.
//
// The reference value is the double-precision function of the argument
// (CUDA's sin / cos / log in double, within 2 ulps of double: about 2^-52
// relative, far below a float ulp).  The error of a result is
// |result - reference| in units of the float spacing at the reference
// (2^-149 below 2^-126), so 0.5 means correctly rounded.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sr_eval.h"
#include "sr_math.cuh"

namespace sr {
namespace {

__device__ __forceinline__ double ulp32_of(double r) {
  const double a = fabs(r);
  if (a < 1.1754943508222875e-38) return 1.401298464324817e-45;
  return ldexp(1.0, ilogb(a) - 23);
}

// fn: 10 sin, 11 cos, 17 log (this library's); 110, 111, 117: CUDA's sinf,
// cosf, logf for comparison.  Arguments whose result or reference is not
// finite are skipped for sin / cos; for log the special results (0 -> -inf,
// negative -> NaN, inf -> inf) are checked for exact agreement instead.
__global__ void math_check_kernel(int fn, uint32_t begin, uint64_t count,
                                  unsigned long long *worst, unsigned long long *counts) {
  unsigned long long best = 0, over_half = 0, over_one = 0, checked = 0;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += stride) {
    const uint32_t bits = begin + static_cast<uint32_t>(i);
    const float x = __uint_as_float(bits);
    float got;
    double ref;
    switch (fn) {
      case 10: got = sr_sinf(x); ref = sin(static_cast<double>(x)); break;
      case 11: got = sr_cosf(x); ref = cos(static_cast<double>(x)); break;
      case 17: got = sr_logf(x); ref = log(static_cast<double>(x)); break;
      case 110: got = sinf(x); ref = sin(static_cast<double>(x)); break;
      case 111: got = cosf(x); ref = cos(static_cast<double>(x)); break;
      default: got = logf(x); ref = log(static_cast<double>(x)); break;
    }
    double err;
    const bool fin_g = isfinite(got), fin_r = isfinite(ref);
    if (!fin_g || !fin_r) {
      if (isnan(x)) continue;
      const float rf = static_cast<float>(ref);
      const bool same = (isnan(got) && isnan(rf)) || got == rf;
      err = same ? 0.0 : 1e30;
      if (!isfinite(x) && (fn == 10 || fn == 11 || fn == 110 || fn == 111)) continue;
    } else {
      err = fabs(static_cast<double>(got) - ref) / ulp32_of(ref);
    }
    ++checked;
    over_half += err > 0.5 ? 1 : 0;
    over_one += err > 1.0 ? 1 : 0;
    const float ef = static_cast<float>(err);
    const unsigned long long key =
        (static_cast<unsigned long long>(__float_as_uint(ef)) << 32) | bits;
    best = key > best ? key : best;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long b2 = __shfl_xor_sync(0xffffffffu, best, o);
    best = b2 > best ? b2 : best;
    over_half += __shfl_xor_sync(0xffffffffu, over_half, o);
    over_one += __shfl_xor_sync(0xffffffffu, over_one, o);
    checked += __shfl_xor_sync(0xffffffffu, checked, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(worst, best);
    atomicAdd(&counts[0], checked);
    atomicAdd(&counts[1], over_half);
    atomicAdd(&counts[2], over_one);
  }
}

}  // namespace
}  // namespace sr

extern "C" sr_status sr_check_math(int32_t fn, uint32_t begin, uint64_t count, double *max_ulp,
                                   uint32_t *argmax_bits, uint64_t *checked,
                                   uint64_t *over_half_ulp, uint64_t *over_one_ulp) {
  if (!(fn == 10 || fn == 11 || fn == 17 || fn == 110 || fn == 111 || fn == 117))
    return SR_ERR_INVALID_ARGUMENT;
  if (!max_ulp || !argmax_bits || !checked || !over_half_ulp || !over_one_ulp)
    return SR_ERR_INVALID_ARGUMENT;
  if (count > (1ull << 32) - begin) return SR_ERR_INVALID_ARGUMENT;
  unsigned long long *d = nullptr;
  if (cudaMalloc(&d, 4 * sizeof(unsigned long long)) != cudaSuccess) return SR_ERR_OUT_OF_MEMORY;
  sr_status st = SR_OK;
  unsigned long long h[4] = {0, 0, 0, 0};
  if (cudaMemset(d, 0, sizeof(h)) != cudaSuccess) st = SR_ERR_CUDA;
  if (st == SR_OK && count > 0) {
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sr::math_check_kernel<<<sms * 8, 256>>>(fn, begin, count, d, d + 1);
    if (cudaGetLastError() != cudaSuccess) st = SR_ERR_CUDA;
  }
  if (st == SR_OK && cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = SR_ERR_CUDA;
  cudaFree(d);
  if (st != SR_OK) return st;
  const uint32_t ebits = static_cast<uint32_t>(h[0] >> 32);
  float e;
  memcpy(&e, &ebits, sizeof e);
  *max_ulp = e;
  *argmax_bits = static_cast<uint32_t>(h[0] & 0xffffffffu);
  *checked = h[1];
  *over_half_ulp = h[2];
  *over_one_ulp = h[3];
  return SR_OK;
}
