// sr_detect.hpp — common-subtree detection and the cross-generation subtree
// cache (host side).  Keys are bit-identical to the reference's.
#pragma once
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace sr {

constexpr uint64_t kFnvOffset = 14695981039346656037ull;
constexpr uint64_t kFnvPrime = 1099511628211ull;

// Flat cache key of a token/value run (reference compute_subtree_hash_gpu,
// src/cleaned/cl_gpu_eval.cu:259-272, = compute_hash, src/utils/detect.cpp:50-68):
// h = O; for each token: h ^= (uint64)(int64)tok; h *= P; h ^= bits(double);
// h *= P.
uint64_t flat_key(const int32_t *tok, const double *val, int len);

// Merkle hash of one node given its children's hashes in prefix order
// (reference hash_node / combine_hashes, src/utils/detect.cpp:97-118).
uint64_t merkle_node(int32_t tok, double val, const uint64_t *child, int nchild);

// Per-position subtree sizes and Merkle hashes of one expression (one reverse
// pass, reference detect.cpp:169-191).
void merkle_hashes(const int32_t *tok, const double *val, int len,
                   int32_t *sizes, uint64_t *hashes);

// Outcome of one detection pass (reference SubtreeDetectionResult,
// src/utils/detect.h:13-40), groups ordered by subtree size, largest first.
struct Detection {
  struct Group {
    int32_t expr, pos, size;   // representative occurrence
    int32_t occurrences;       // verified occurrences
  };
  std::vector<Group> groups;
  int64_t total_tokens = 0;
  int64_t covered_tokens = 0;  // tokens under the greedy non-overlapping cover
  double avg_subtree_size = 0.0;
  double coverage = 0.0;
};

// Reference detect_common_subtrees (src/utils/detect.cpp:120-387): candidates
// are subtrees of >= min_size tokens; they are grouped by Merkle hash, each
// group verified token-by-token against its first member, groups with >=
// min_freq verified members kept, ordered by size descending, and covered
// greedily without overlap.  Ties are ordered deterministically (hash, then
// expression, then position; stable size sort) where the reference's
// std::sort leaves them unspecified.
void detect_common_subtrees(int E, const int32_t *tok, const double *val,
                            const int64_t *off, int min_size, int min_freq,
                            int threads, Detection &out);

// Persistent key -> slot map (reference GPUSubtreeStateContext::hash_to_idx,
// src/cleaned/cl_gpu_common.h:26-31): slots are handed out in insertion order
// until the capacity is reached.
struct SubtreeCache {
  std::unordered_map<uint64_t, int32_t> slot_of;
  int32_t used = 0;
  int32_t capacity = 2048;
  // Keys inserted by a prepare whose launch has not been enqueued yet: their
  // values exist only once that launch runs, so they are taken out again if
  // the prepared launch is dropped (or its prepare fails) before that.
  std::vector<uint64_t> pending;
  int32_t pending_base = 0;
  void clear() {
    slot_of.clear();
    used = 0;
    pending.clear();
    pending_base = 0;
  }
  void begin_pending() {
    pending.clear();
    pending_base = used;
  }
  void commit() { pending.clear(); }
  void rollback() {
    if (pending.empty()) return;
    for (uint64_t k : pending) slot_of.erase(k);
    used = pending_base;
    pending.clear();
  }
};

// Reference mark_cached_subtrees_from_state (src/cleaned/cl_gpu_eval.cu:294-329):
// pre-order scan of every expression; a position of an unmarked subtree of
// >= 3 tokens whose flat key is cached becomes a root (hint = slot) and its
// body is marked -2; everything else is -1.  hints has off[E] entries.
// Returns the number of tokens removed from the skeletons.
int64_t mark_cached_subtrees(int E, const int32_t *tok, const double *val,
                             const int64_t *off, const SubtreeCache &cache,
                             int threads, int32_t *hints);

// Run fn(begin, end) over [0, n) split into contiguous chunks on `threads`
// host threads (1 = inline).
template <class F>
void parallel_for(int64_t n, int threads, F &&fn);

}  // namespace sr

#include "sr_parallel.hpp"
