// sr_detect_gpu.hpp — device common-subtree detection (sr_detect_gpu.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace sr {

// Buffers of one detection; positions are token indices relative to the
// population's first token (T tokens, E expressions).
struct DetectArgs {
  const int32_t *tok;        // [T]
  const double *val;         // [T]
  const int64_t *off;        // [E + 1] (absolute, off[0] may be non-zero)
  int E;
  int64_t T;
  int min_size, min_freq;
  int32_t *size;             // [T] subtree size of every position
  uint64_t *hash;            // [T] Merkle hash of every position
  uint8_t *cand;             // [T] size >= min_size
  uint8_t *mark;             // [T] verified occurrence of a common subtree
  int32_t *pos_in, *pos_out; // [T] candidate positions (selected / sorted)
  uint64_t *key_in, *key_out;// [T] candidate hashes (gathered / sorted)
  uint64_t *run_key;         // [T] distinct hashes
  int32_t *run_count;        // [T] candidates per distinct hash
  int32_t *run_start;        // [T]
  int32_t *rep, *gsize, *vcount;  // [T] per run: first member, size, verified count
  int32_t *n_sel;            // [1] candidates
  int32_t *n_runs;           // [1] distinct hashes
  unsigned long long *covered;  // [1] tokens under the cover
  void *temp;
  size_t temp_bytes;
};

struct DetectScratchSizes {
  size_t temp_bytes;
};
DetectScratchSizes detect_scratch_sizes(int64_t T);
size_t detect_scan_temp_bytes(int n);

// Stage 1: hashes, sizes, candidate selection (*n_sel).
cudaError_t detect_candidates(const DetectArgs &a, cudaStream_t s);
// Stage 2: sort the M candidates by hash, run-length encode (*n_runs).
cudaError_t detect_groups(const DetectArgs &a, int M, cudaStream_t s);
// Stage 3: verify the runs, flag verified members, count covered tokens.
cudaError_t detect_verify(const DetectArgs &a, int n_runs, cudaStream_t s);
// Stage 4: the common subtrees in hash order: *n_sel of them, out[3k..3k+2] =
// (first member's position, size, verified members); out holds 3 * n_runs.
cudaError_t detect_frequent(const DetectArgs &a, int n_runs, int32_t *out, cudaStream_t s);

}  // namespace sr
