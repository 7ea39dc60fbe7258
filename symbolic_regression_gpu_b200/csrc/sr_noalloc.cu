// sr_noalloc.cu — population MSE for callers that cannot allocate device
// memory.
//
// Who needs this: code that keeps its whole population on the GPU and must
// not call cudaMalloc while it runs — a GA loop that breeds and evaluates on
// the device and has handed all device memory to its own pool or budget, a
// host framework that owns the device allocator (a custom or pooled
// allocator that this library cannot call into), or a caller that records
// its work into a stream it does not want to synchronise for an allocation.
// Such callers pass device pointers for everything they own (tokens,
// values, offsets, the dataset and the output vector); the only working
// memory this entry point needs — per-block partial sums and an error word —
// lives in one fixed array compiled into the library, so nothing is
// allocated by any call.
//
// Costs of that choice:
//   * the array (SR_NOALLOC_SCRATCH_BYTES, 4 MiB) is resident on every GPU
//     that loads the library, until the process exits;
//   * it bounds the population size (SR_NOALLOC_MAX_EXPRS expressions);
//   * all calls share it: two calls whose kernels overlap on the GPU (on
//     different streams, or from different host threads) race on it and
//     both results are undefined.  Serialise such calls on one stream.
//
// The kernel is a variant of the plain per-expression kernel (sr_kernels.cu)
// that also validates the tokens it reads, because tokens that live on the
// device cannot be checked by the host compiler first.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "sr_eval.h"
#include "sr_kernels.hpp"
#include "sr_ops.cuh"

namespace sr {
namespace {

// Layout of the fixed scratch: [error word | pad to 256 B | partial sums].
constexpr size_t kScratchBytes = SR_NOALLOC_SCRATCH_BYTES;
constexpr size_t kPartialOffset = 256;
constexpr size_t kPartialCapacity = (kScratchBytes - kPartialOffset) / sizeof(double2);

static __device__ __align__(256) unsigned char noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
// Per device: the device address of noalloc_scratch and the id of the CUDA
// context it belongs to.  A device reset (cudaDeviceReset) makes a new
// context in which the array has a new address, so the address is looked up
// again whenever the current context is not the one it was looked up in.
void *g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (the
// library does not link the driver library itself).
typedef int (*ctx_get_current_fn)(void **ctx);
typedef int (*ctx_get_id_fn)(void *ctx, unsigned long long *id);

bool current_context_id(unsigned long long *id) {
  static ctx_get_current_fn get_current = nullptr;
  static ctx_get_id_fn get_id = nullptr;
  if (!get_current || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) !=
            cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !f1)
      return false;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) !=
            cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f2)
      return false;
    get_current = reinterpret_cast<ctx_get_current_fn>(f1);
    get_id = reinterpret_cast<ctx_get_id_fn>(f2);
  }
  void *ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx) return false;
  return get_id(ctx, id) == 0;
}

// Set-up per device (and per context of that device), with that device
// current: the host-side name of a __device__ array is only a stand-in, the
// kernel needs its device address.  Called by every call (under a mutex);
// it looks the address up only on the first call in a context.
sr_status scratch_address(int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices) return SR_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long ctx_id = 0;
  if (!current_context_id(&ctx_id)) return SR_ERR_CUDA;
  if (!g_scratch_addr[device] || g_scratch_ctx[device] != ctx_id) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, noalloc_scratch);
    if (e != cudaSuccess || !ptr) return SR_ERR_CUDA;
    g_scratch_addr[device] = ptr;
    g_scratch_ctx[device] = ctx_id;
  }
  *out = static_cast<unsigned char *>(g_scratch_addr[device]);
  return SR_OK;
}

// Structural check of expression e, made before anything of it is read for
// evaluation: its offsets lie in [off[0], off[E]] (off[0] >= 0, and the
// caller's contract is that off[E] is the length of the token and value
// buffers), it has 1..SR_MAX_TOKENS tokens, every token is known, the
// right-to-left evaluation never pops an empty stack or holds more than
// kPlainStack values, and exactly one value is left at the end.
__device__ bool expr_well_formed(const int32_t *__restrict__ tok,
                                 const int64_t *__restrict__ off, int e, int E) {
  const int64_t lo = off[0], hi = off[E];
  const int64_t o = off[e], o1 = off[e + 1];
  if (!(lo >= 0 && lo <= o && o <= o1 && o1 <= hi)) return false;
  const int64_t len = o1 - o;
  if (len < 1 || len > SR_MAX_TOKENS) return false;
  int sp = 0;
  for (int64_t i = len - 1; i >= 0; --i) {
    const int t = tok[o + i];
    if (t == SR_TOK_CONST || t == SR_TOK_VAR) {
      if (++sp > kPlainStack) return false;
    } else if (t >= 1 && t <= 9) {
      if (sp < 2) return false;
      --sp;
    } else if ((t >= 10 && t <= 27) || t == SR_OP_EXP_CLAMP) {
      if (sp < 1) return false;
    } else {
      return false;
    }
  }
  return sp == 1;
}

// Plain-kernel variant over device-resident tokens: 4 expressions x 128
// datapoints per block, token stack in local memory, squared errors reduced
// in FP64 per block into partial[blockIdx.y][e].  Every block first checks
// the structure of its 4 expressions (expr_well_formed); a malformed one is
// never evaluated, contributes no valid datapoint (NaN MSE) and, in the
// blocks of row blockIdx.y == 0, sets error bit 1.  The grid has at least
// one row, so the check also runs when there are no datapoints.
__global__ void __launch_bounds__(128)
    plain_checked_kernel(const int32_t *__restrict__ tok, const float *__restrict__ val,
                         const int64_t *__restrict__ off, const float *__restrict__ X,
                         int64_t ldx, int V, int64_t N, int E, double2 *__restrict__ partial,
                         int32_t *__restrict__ error) {
  __shared__ double red_s[4][4];
  __shared__ int red_c[4][4];
  __shared__ bool well_formed[4];
  const int e0 = blockIdx.x * 4;
  if (threadIdx.x < 4) {
    const int e = e0 + static_cast<int>(threadIdx.x);
    const bool ok = e < E && expr_well_formed(tok, off, e, E);
    well_formed[threadIdx.x] = ok;
    if (e < E && !ok && blockIdx.y == 0) atomicOr(error, 1);
  }
  __syncthreads();
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int cnt[4] = {0, 0, 0, 0};
  for (int64_t dp = static_cast<int64_t>(blockIdx.y) * 128 + threadIdx.x; dp < N;
       dp += static_cast<int64_t>(gridDim.y) * 128) {
    float xc[SR_MAX_VARS + 1];
    for (int v = 0; v <= V; ++v) xc[v] = X[v * ldx + dp];
    const float yv = xc[V];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (!well_formed[j]) continue;  // also every e >= E
      const int e = e0 + j;
      const int64_t o = off[e];
      const int64_t len = off[e + 1] - o;
      // Well-formed: the stack stays within [1, kPlainStack] and one value
      // is left at the end.
      float stk[kPlainStack];
      int sp = 0;
      for (int64_t i = len - 1; i >= 0; --i) {
        const int t = tok[o + i];
        if (t == SR_TOK_CONST) {
          stk[sp++] = val[o + i];
        } else if (t == SR_TOK_VAR) {
          const float fv = val[o + i];
          const int vi = (fv > -2147483648.0f && fv < 2147483648.0f) ? static_cast<int>(fv) : -1;
          stk[sp++] = (vi >= 0 && vi < V) ? xc[vi] : 0.0f;
        } else if (t >= 1 && t <= 9) {
          const float v1 = stk[--sp];
          const float v2 = stk[--sp];
          stk[sp++] = op_binary(t, v1, v2);
        } else {
          stk[sp - 1] = op_unary(t, stk[sp - 1]);
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
      partial[static_cast<int64_t>(blockIdx.y) * E + e] = make_double2(s, static_cast<double>(c));
    }
  }
}

}  // namespace
}  // namespace sr

extern "C" sr_status sr_eval_mse_device_noalloc(const int32_t *tokens, const float *values,
                                                const int64_t *offsets, int32_t num_exprs,
                                                const float *X, int64_t ld, int32_t num_vars,
                                                int64_t num_dps, float *mse_out, void *stream) {
  if (num_exprs < 0 || num_vars < 0 || num_dps < 0 || ld < num_dps) return SR_ERR_INVALID_ARGUMENT;
  if (num_exprs == 0) return SR_OK;
  if (!tokens || !values || !offsets || !mse_out || (num_dps > 0 && !X))
    return SR_ERR_INVALID_ARGUMENT;
  if (num_vars > SR_MAX_VARS) return SR_ERR_TOO_MANY_VARS;
  if (num_exprs > SR_NOALLOC_MAX_EXPRS) return SR_ERR_UNSUPPORTED;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) return SR_ERR_NO_DEVICE;
  unsigned char *scratch = nullptr;
  const sr_status st = sr::scratch_address(device, &scratch);
  if (st != SR_OK) return st;
  int32_t *d_error = reinterpret_cast<int32_t *>(scratch);
  double2 *partial = reinterpret_cast<double2 *>(scratch + sr::kPartialOffset);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);

  // Datapoint blocks: up to 256, fewer when the partial sums of all
  // expressions would not fit the fixed scratch (E <= capacity keeps at
  // least one), and at least one, so that the structural check of the
  // expressions also runs when there are no datapoints.
  int64_t dpblocks = (num_dps + 127) / 128;
  dpblocks = dpblocks < 256 ? dpblocks : 256;
  const int64_t fit = static_cast<int64_t>(sr::kPartialCapacity) / num_exprs;
  if (dpblocks > fit) dpblocks = fit;
  if (dpblocks < 1) dpblocks = 1;

  // The error word must start at zero; the partial sums are fully
  // overwritten by every launch that reads them.
  if (cudaMemsetAsync(d_error, 0, sizeof(int32_t), s) != cudaSuccess) return SR_ERR_CUDA;
  const dim3 grid(static_cast<unsigned>((num_exprs + 3) / 4), static_cast<unsigned>(dpblocks));
  sr::plain_checked_kernel<<<grid, 128, 0, s>>>(tokens, values, offsets, X, ld, num_vars,
                                                 num_dps, num_exprs, partial, d_error);
  if (cudaGetLastError() != cudaSuccess) return SR_ERR_CUDA;
  if (sr::launch_finalize(partial, static_cast<int>(dpblocks), num_exprs, mse_out, s) !=
      cudaSuccess)
    return SR_ERR_CUDA;
  int32_t h_error = 0;
  if (cudaMemcpyAsync(&h_error, d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
      cudaSuccess)
    return SR_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return SR_ERR_CUDA;
  return h_error ? SR_ERR_MALFORMED_EXPRESSION : SR_OK;
}
