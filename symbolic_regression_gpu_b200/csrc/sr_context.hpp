// sr_context.hpp — evaluator context: device-resident dataset, compiled
// programs, launch plans and the subtree cache (reference
// GPUSubtreeStateContext / SimpleGPUContext, src/cleaned/cl_gpu_common.h:26-212).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "sr_detect.hpp"
#include "sr_eval.h"
#include "sr_internal.hpp"
#include "sr_program.hpp"

namespace sr {

// Host-side fault injection for tests (sr_inject_allocation_failure): when the
// countdown is n > 0, the n-th following DevBuf / PinnedBuf allocation fails
// with cudaErrorMemoryAllocation without reaching the allocator (once).
inline std::atomic<int64_t> &alloc_fault_countdown() {
  static std::atomic<int64_t> countdown{0};
  return countdown;
}
inline bool alloc_fault_fires() {
  std::atomic<int64_t> &c = alloc_fault_countdown();
  int64_t v = c.load(std::memory_order_relaxed);
  while (v > 0)
    if (c.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return v == 1;
  return false;
}

// Grow-only device buffer.  Callers synchronise the stream before growing.
// A failed growth leaves the buffer empty (p == nullptr, cap == 0).
template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  cudaError_t ensure(size_t n) {
    if (p && n <= cap) return cudaSuccess;
    const size_t want = std::max<size_t>(n + n / 4, 64);
    release();
    if (alloc_fault_fires()) return cudaErrorMemoryAllocation;
    const cudaError_t e = cudaMalloc(&p, want * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
};

// Grow-only pinned host buffer used as the staging area of async copies.
template <class T>
struct PinnedBuf {
  T *p = nullptr;
  size_t cap = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf &) = delete;
  PinnedBuf &operator=(const PinnedBuf &) = delete;
  ~PinnedBuf() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
  cudaError_t ensure(size_t n) {
    if (p && n <= cap) return cudaSuccess;
    const size_t want = std::max<size_t>(n + n / 4, 64);
    release();
    if (alloc_fault_fires()) return cudaErrorMemoryAllocation;
    const cudaError_t e = cudaMallocHost(&p, want * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
};

// Launch shape of one interpreter launch.
struct Plan {
  int dpt = 8;
  int W = 8;           // evaluating warps per block
  int ops = 0;         // operator profile dispatched inline (kOpsAll / kOpsProtected)
  bool cache = false;  // programs read cached subtrees (cached-operand paths compiled in)
  int smax = 0;        // spill slots per warp
  int s_smem = 0;      // of which in shared memory
  int G = 0;           // expressions per group
  int n_groups = 0;
  int span = 0;        // datapoints per span
  int n_spans = 0;
  int k_spans = 1;     // spans per work item (EvalArgs::span_per_item)
  int blocks = 0;
  size_t smem = 0;
  int n_span_groups() const { return (n_spans + k_spans - 1) / k_spans; }
  int64_t items() const { return static_cast<int64_t>(n_groups) * n_span_groups(); }
};

// A compiled population resident on the device.
struct ProgramSet {
  DevBuf<Instr> code;
  DevBuf<int64_t> off;
  DevBuf<int32_t> len;
  DevBuf<int32_t> group;
  DevBuf<int32_t> row;
  PinnedBuf<Instr> h_code;
  PinnedBuf<int64_t> h_off;
  PinnedBuf<int32_t> h_len;
  PinnedBuf<int32_t> h_group;
  PinnedBuf<int32_t> h_row;
  std::vector<float> cost;  // per expression
  std::vector<int32_t> n_const;  // constants per expression
  int E = 0;
  int smax = 0;
  int64_t n_instr = 0;
  int64_t n_instr_protected = 0;  // instructions whose opcode kOpsProtected dispatches inline
  bool cache_refs = false;        // some instruction reads a cached subtree
  int64_t n_tokens = 0;      // tokens represented (skeleton-equivalent)
  double sfu_per_dp = 0.0;   // declared work, summed over expressions
  double fp32_per_dp = 0.0;
  Plan plan;
};

// Buffers of the plain baseline kernel.
struct PlainSet {
  DevBuf<int32_t> tok;
  DevBuf<float> val;
  DevBuf<int64_t> off;
  DevBuf<int32_t> len;
  PinnedBuf<int32_t> h_tok;
  PinnedBuf<float> h_val;
  PinnedBuf<int64_t> h_off;
  PinnedBuf<int32_t> h_len;
  int E = 0;
  int n_dpblocks = 0;
};

// One launch of the forward+adjoint kernel: expressions whose programs fit
// the class's tape length.
struct AdjClass {
  int tape_len = 0;
  int gmax = 0;
  bool global_tape = false;  // tape in per-warp global scratch instead of shared memory
  int seg_cap = 0;           // recompute mode: segment-tape entries
  int64_t group_off = 0;     // into the concatenated group table
  Plan plan;
};

// Buffers of the device common-subtree detection (sr_detect_gpu.cu), per
// token of the population unless noted.
struct DetectBufs {
  DevBuf<int32_t> tok;
  DevBuf<double> val;
  DevBuf<int64_t> off;      // [E + 1]
  DevBuf<int32_t> size, pos_in, pos_out, run_count, run_start, rep, gsize, vcount, out3;
  DevBuf<uint64_t> hash, key_in, key_out, run_key;
  DevBuf<uint8_t> cand, mark;
  DevBuf<int32_t> counters;               // [2]: candidates, runs
  DevBuf<unsigned long long> covered;     // [1]
  DevBuf<unsigned char> temp;
  PinnedBuf<int32_t> h_counters;
  PinnedBuf<unsigned long long> h_covered;
  PinnedBuf<int32_t> h_out3;
};

// Device state of a gradient / constant-optimisation call.
// A forward-mode (tangent) gradient launch: the expressions with at most K
// constants (and more than the previous width's).
struct TanSet {
  int K = 0;
  int n_exprs = 0;
  int64_t group_off = 0;  // into the concatenated group table
  int64_t expr_off = 0;   // into the expression lists
  int64_t part_off = 0;   // double2 offset of its MSE sums in tan_partial
  int64_t gout_off = 0;   // double offset of its gradient sums in tan_gout
  Plan plan;
};

struct GradSet {
  DevBuf<int64_t> const_off;
  DevBuf<int32_t> const_cnt;
  DevBuf<int64_t> const_loc;  // (instruction << 1) | (operand b)
  DevBuf<double> grad_acc;
  DevBuf<float> grad;
  DevBuf<float> consts;
  DevBuf<float> m, v;
  DevBuf<int32_t> groups;
  DevBuf<int32_t> bwd_lo;     // [E] lowest instruction holding a constant
  DevBuf<float> gtape;        // global tapes of classes that do not fit shared memory
  PinnedBuf<int32_t> h_bwd_lo;
  PinnedBuf<int64_t> h_const_off;
  PinnedBuf<int32_t> h_const_cnt;
  PinnedBuf<int64_t> h_const_loc;
  PinnedBuf<float> h_consts;
  PinnedBuf<int32_t> h_groups;
  std::vector<AdjClass> classes;
  // Forward-mode launches, their mask words ([instructions + 1], aligned with
  // the code) and span-group sums; the expression lists (tangent sets first,
  // then the reverse-mode expressions) that the finalize kernels walk.
  std::vector<TanSet> tsets;
  DevBuf<uint32_t> tmask;
  PinnedBuf<uint32_t> h_tmask;
  DevBuf<double2> tan_partial;
  DevBuf<double> tan_gout;
  DevBuf<int32_t> exprs;
  PinnedBuf<int32_t> h_exprs;
  int64_t rev_expr_off = 0;
  int n_rev = 0;  // expressions evaluated in reverse mode
  int64_t C = 0;
  int span = 0;
  int n_spans = 0;
  bool recompute = false;
};

enum class Mode { kNone, kBatched, kCached, kPlain, kGrad };

}  // namespace sr

struct sr_context {
  sr_options opts{};
  int device = 0;
  int num_sms = 0;
  size_t device_memory = 0;  // bytes of device memory (cudaDeviceProp::totalGlobalMem)
  std::string device_name;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;

  // dataset
  sr::DevBuf<float> X;
  int64_t ldx = 0;
  int32_t V = -1;
  int64_t N = 0;

  // compiled work
  sr::ProgramSet main;   // expressions (or skeletons)
  sr::ProgramSet sub;    // new cached subtrees of this call
  sr::PlainSet plain;
  sr::Mode mode = sr::Mode::kNone;
  int E = 0;

  // reduction / control
  sr::DevBuf<double2> partial;
  sr::DevBuf<float> mse;
  sr::PinnedBuf<float> h_mse;
  int32_t *d_counter = nullptr;   // [2]: main and subtree launches
  int32_t *d_error = nullptr;
  int32_t *h_error = nullptr;     // pinned

  // subtree cache
  sr::SubtreeCache cache;
  sr::DevBuf<float> cache_vals;   // [capacity][ldx]
  std::vector<int32_t> hints;     // per token of the last cached population

  // predictions
  sr::DevBuf<float> pred;
  // spill slots beyond the shared-memory ones (per resident warp)
  sr::DevBuf<float> spill;
  // gradients / constant optimisation
  sr::GradSet grad;
  // FP64 accuracy report
  sr::DevBuf<double> mse64;
  sr::PinnedBuf<double> h_mse64;
  sr::DevBuf<double2> sums;  // (sum, count) per expression for datapoint sharding
  sr::PinnedBuf<double2> h_sums;
  // device common-subtree detection
  sr::DetectBufs det;
  // device-side evolution: ranking scratch and the device-compile summary
  sr::DevBuf<unsigned char> evo_temp;
  sr::DevBuf<uint32_t> evo_keys;   // [2E]
  sr::DevBuf<int32_t> evo_idx;     // [E]
  sr::DevBuf<int32_t> evo_order;   // [E]
  sr::DevBuf<float> evo_fit;       // [E] fitness in rank order
  sr::DevBuf<int32_t> evo_summary; // [8] see launch_compile_device
  sr::PinnedBuf<int32_t> h_evo_summary;

  // timing
  cudaEvent_t ev[6] = {};
  // use_graphs: the prepared launch sequence as an instantiated CUDA graph,
  // captured on the first sr_launch after a prepare and replayed until the
  // next prepare / set_data (which destroy it: buffers may move).
  cudaGraphExec_t graph_exec = nullptr;
  int graph_launches = 0;
  bool capturing = false;  // sr_launch is capturing graph_exec
  bool timing_valid = false;

  // statistics of the prepared population
  sr_stats prep_stats{};

  // tuned launch shapes: key -> (dpt, W, spill slots in shared memory (-1 =
  // the default for the dpt), expressions per group and warp)
  struct TunedShape {
    int dpt, W, split, per_warp;
  };
  std::map<std::string, TunedShape> tuned;
  bool tune_loaded = false;

  sr_status fail(sr_status s, const std::string &msg) {
    last_error = msg;
    return s;
  }
};
