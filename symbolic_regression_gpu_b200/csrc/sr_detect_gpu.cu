// sr_detect_gpu.cu — common-subtree detection on the device (reference
// detect_common_subtrees, src/utils/detect.cpp:120-387; host restatement in
// csrc/sr_detect.cpp).  Same candidates, same grouping, same verification,
// same statistics:
//
//   merkle_kernel        one thread per expression: the reverse pass giving
//                        every position its subtree size and Merkle hash
//                        (detect.cpp:97-118) and the candidate flag
//                        (size >= min_size).
//   cub select / sort    candidates compacted and sorted by hash (stable, so
//                        equal hashes keep (expression, position) order, the
//                        host's tie order).
//   cub run-length       runs of equal hashes = hash groups.
//   verify_kernel        one thread per group of >= min_freq candidates: every
//                        member compared with the first (size, tokens and
//                        value bits, detect.cpp:239-248); groups with >=
//                        min_freq verified members are the common subtrees,
//                        and their verified members are flagged in place.
//   cover_kernel         one thread per expression: the greedy
//                        non-overlapping cover of the reference (groups
//                        largest first, an occurrence taken when none of its
//                        tokens is covered) equals "every flagged occurrence
//                        with no flagged ancestor", because subtrees are
//                        nested or disjoint and an ancestor is strictly larger;
//                        a pre-order walk counts those tokens.
// The host orders the (few) common subtrees by size, largest first, stable
// in hash order, exactly as the host detector does.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "sr_detect_gpu.hpp"

namespace sr {
namespace {

constexpr uint64_t kOffset = 14695981039346656037ull;
constexpr uint64_t kPrime = 1099511628211ull;

__device__ __forceinline__ uint64_t node_hash(int32_t tok, double val, const uint64_t *ch,
                                              int nch) {
  uint64_t h = kOffset;
  h ^= static_cast<uint64_t>(static_cast<int64_t>(tok));
  h *= kPrime;
  h ^= static_cast<uint64_t>(__double_as_longlong(val));
  h *= kPrime;
  for (int k = 0; k < nch; ++k) h = h ^ (ch[k] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2));
  return h;
}

__global__ void merkle_kernel(const int32_t *__restrict__ tok, const double *__restrict__ val,
                              const int64_t *__restrict__ off, int E, int min_size,
                              int32_t *__restrict__ size, uint64_t *__restrict__ hash,
                              uint8_t *__restrict__ cand) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= E) return;
  const int64_t o = off[x] - off[0];
  const int len = static_cast<int>(off[x + 1] - off[x]);
  for (int i = len - 1; i >= 0; --i) {
    const int64_t g = o + i;
    const int t = tok[g];
    int s = 1;
    uint64_t ch[2];
    int nch = 0;
    if (t > 0) {  // detect.cpp simple_op_arity: 1..9 binary, >= 10 unary
      const int arity = t < 10 ? 2 : 1;
      int pos = i + 1;
      for (int k = 0; k < arity && pos < len; ++k) {
        const int cs = size[o + pos];
        s += cs;
        ch[nch++] = hash[o + pos];
        pos += cs;
      }
    }
    size[g] = s;
    hash[g] = node_hash(t, val[g], ch, nch);
    cand[g] = s >= min_size ? 1 : 0;
  }
}

__global__ void gather_hash_kernel(const uint64_t *__restrict__ hash, const int32_t *__restrict__ pos,
                                   int M, uint64_t *__restrict__ key) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < M) key[k] = hash[pos[k]];
}

// One thread per run of equal hashes.  run_start is the exclusive prefix of
// run_count.  Writes rep[r] (first member's position), gsize[r] and
// vcount[r] (verified members; 0 when the run is too small), and flags the
// verified members of common subtrees in mark[].
__global__ void verify_kernel(const int32_t *__restrict__ tok, const double *__restrict__ val,
                              const int32_t *__restrict__ size, const int32_t *__restrict__ pos,
                              const int32_t *__restrict__ run_count, int n_runs, int min_freq,
                              int32_t *__restrict__ run_start, int32_t *__restrict__ rep,
                              int32_t *__restrict__ gsize, int32_t *__restrict__ vcount,
                              uint8_t *__restrict__ rflag, uint8_t *__restrict__ mark) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_runs) return;
  const int start = run_start[r];
  const int cnt = run_count[r];
  const int p0 = pos[start];
  const int s0 = size[p0];
  rep[r] = p0;
  gsize[r] = s0;
  if (cnt < min_freq) {
    vcount[r] = 0;
    rflag[r] = 0;
    return;
  }
  int v = 0;
  for (int k = start; k < start + cnt; ++k) {
    const int p = pos[k];
    if (size[p] != s0) continue;
    bool same = true;
    for (int q = 0; q < s0 && same; ++q)
      same = tok[p + q] == tok[p0 + q] && val[p + q] == val[p0 + q];
    v += same ? 1 : 0;
  }
  vcount[r] = v >= min_freq ? v : 0;
  rflag[r] = v >= min_freq ? 1 : 0;
  if (v < min_freq) return;
  for (int k = start; k < start + cnt; ++k) {
    const int p = pos[k];
    if (size[p] != s0) continue;
    bool same = true;
    for (int q = 0; q < s0 && same; ++q)
      same = tok[p + q] == tok[p0 + q] && val[p + q] == val[p0 + q];
    if (same) mark[p] = 1;
  }
}

__global__ void cover_kernel(const int64_t *__restrict__ off, int E, const int32_t *__restrict__ size,
                             const uint8_t *__restrict__ mark,
                             unsigned long long *__restrict__ covered) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= E) return;
  const int64_t o = off[x] - off[0];
  const int len = static_cast<int>(off[x + 1] - off[x]);
  unsigned long long c = 0;
  for (int i = 0; i < len;) {
    if (mark[o + i]) {
      const int s = size[o + i];
      c += static_cast<unsigned long long>(s);
      i += s;
    } else {
      ++i;
    }
  }
  if (c) atomicAdd(covered, c);
}

__global__ void iota_kernel(int32_t *__restrict__ out, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = static_cast<int32_t>(i);
}

inline unsigned grid_for(int64_t n, int block) {
  return static_cast<unsigned>((n + block - 1) / block);
}

}  // namespace

DetectScratchSizes detect_scratch_sizes(int64_t T) {
  DetectScratchSizes z{};
  const int n = static_cast<int>(T);
  size_t a = 0, b = 0, c = 0;
  cub::DeviceSelect::Flagged(nullptr, a, static_cast<const int32_t *>(nullptr),
                             static_cast<const uint8_t *>(nullptr), static_cast<int32_t *>(nullptr),
                             static_cast<int32_t *>(nullptr), n);
  cub::DeviceRadixSort::SortPairs(nullptr, b, static_cast<const uint64_t *>(nullptr),
                                  static_cast<uint64_t *>(nullptr),
                                  static_cast<const int32_t *>(nullptr),
                                  static_cast<int32_t *>(nullptr), n);
  cub::DeviceRunLengthEncode::Encode(nullptr, c, static_cast<const uint64_t *>(nullptr),
                                     static_cast<uint64_t *>(nullptr),
                                     static_cast<int32_t *>(nullptr),
                                     static_cast<int32_t *>(nullptr), n);
  z.temp_bytes = std::max(a, std::max(b, c));
  return z;
}

cudaError_t detect_candidates(const DetectArgs &a, cudaStream_t s) {
  merkle_kernel<<<grid_for(a.E, 64), 64, 0, s>>>(a.tok, a.val, a.off, a.E, a.min_size, a.size,
                                                a.hash, a.cand);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  // positions 0..T-1 (in pos_out as scratch), kept where cand != 0
  iota_kernel<<<grid_for(a.T, 256), 256, 0, s>>>(a.pos_out, a.T);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  size_t tb = a.temp_bytes;
  err = cub::DeviceSelect::Flagged(a.temp, tb, static_cast<const int32_t *>(a.pos_out), a.cand,
                                   a.pos_in, a.n_sel, static_cast<int>(a.T), s);
  return err;
}

cudaError_t detect_groups(const DetectArgs &a, int M, cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  gather_hash_kernel<<<grid_for(M, 256), 256, 0, s>>>(a.hash, a.pos_in, M, a.key_in);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  size_t tb = a.temp_bytes;
  err = cub::DeviceRadixSort::SortPairs(a.temp, tb, a.key_in, a.key_out, a.pos_in, a.pos_out, M, 0,
                                        64, s);
  if (err != cudaSuccess) return err;
  tb = a.temp_bytes;
  return cub::DeviceRunLengthEncode::Encode(a.temp, tb, a.key_out, a.run_key, a.run_count,
                                            a.n_runs, M, s);
}

cudaError_t detect_verify(const DetectArgs &a, int n_runs, cudaStream_t s) {
  // nothing covered when there is no run (the counter is reused across calls)
  cudaError_t err = cudaMemsetAsync(a.covered, 0, sizeof(unsigned long long), s);
  if (err != cudaSuccess || n_runs <= 0) return err;
  // run starts: exclusive prefix sum of the counts
  size_t tb = a.temp_bytes;
  err = cub::DeviceScan::ExclusiveSum(a.temp, tb, a.run_count, a.run_start, n_runs, s);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(a.mark, 0, static_cast<size_t>(a.T), s);
  if (err != cudaSuccess) return err;
  // a.cand (no longer needed after the selection) holds the run flags
  verify_kernel<<<grid_for(n_runs, 128), 128, 0, s>>>(a.tok, a.val, a.size, a.pos_out, a.run_count,
                                                      n_runs, a.min_freq, a.run_start, a.rep,
                                                      a.gsize, a.vcount, a.cand, a.mark);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  cover_kernel<<<grid_for(a.E, 128), 128, 0, s>>>(a.off, a.E, a.size, a.mark, a.covered);
  return cudaGetLastError();
}

__global__ void gather_runs_kernel(const int32_t *__restrict__ ids, const int32_t *__restrict__ n,
                                   const int32_t *__restrict__ rep,
                                   const int32_t *__restrict__ gsize,
                                   const int32_t *__restrict__ vcount, int32_t *__restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *n) return;
  const int r = ids[k];
  out[3 * k + 0] = rep[r];
  out[3 * k + 1] = gsize[r];
  out[3 * k + 2] = vcount[r];
}

cudaError_t detect_frequent(const DetectArgs &a, int n_runs, int32_t *out, cudaStream_t s) {
  if (n_runs <= 0) return cudaMemsetAsync(a.n_sel, 0, sizeof(int32_t), s);
  iota_kernel<<<grid_for(n_runs, 256), 256, 0, s>>>(a.run_start, n_runs);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  size_t tb = a.temp_bytes;
  // selected run ids (in hash order) into pos_in, their count into n_sel
  err = cub::DeviceSelect::Flagged(a.temp, tb, static_cast<const int32_t *>(a.run_start), a.cand,
                                   a.pos_in, a.n_sel, n_runs, s);
  if (err != cudaSuccess) return err;
  gather_runs_kernel<<<grid_for(n_runs, 256), 256, 0, s>>>(a.pos_in, a.n_sel, a.rep, a.gsize,
                                                           a.vcount, out);
  return cudaGetLastError();
}

size_t detect_scan_temp_bytes(int n) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, static_cast<const int32_t *>(nullptr),
                                static_cast<int32_t *>(nullptr), n);
  return b;
}

}  // namespace sr
