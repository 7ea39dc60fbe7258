// sr_capi.cpp — the C ABI (sr_eval.h): context lifecycle, dataset upload,
// population compilation / planning / upload, launches and read-back
// (gradients and Adam: sr_capi_grad.cpp; the FP64 reference, the device
// generation loop, microbenchmarks, detection and host-only helpers:
// sr_capi_tools.cpp; shared helpers: sr_capi_internal.hpp).
//
// Reference counterpart: evaluate_gpu_mse (src/cleaned/cl_gpu_eval.cu:332-564)
// and evaluate_gpu_simple (src/cleaned/cl_gpu_simple.cu:187-310).  Where the
// reference synchronises after every copy and kernel and exits the process
// on a CUDA error, this runtime compiles on host threads, issues pinned
// asynchronous copies and all kernels back to back on one stream, waits once,
// and reports failures as status codes.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <thread>

#include "sr_adjoint.hpp"
#include "sr_capi_internal.hpp"
#include "sr_context.hpp"
#include "sr_detect_gpu.hpp"
#include "sr_evolve.hpp"
#include "sr_kernels.hpp"
#include "sr_trace.hpp"

using sr::Instr;
using sr::ProgramSet;
using namespace sr::capi;

namespace sr {
namespace capi {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Milliseconds between two events, 0 when either was never recorded (the
// device-resident paths skip the upload pair).  cudaEventElapsedTime reports
// that case as an error that would otherwise stay as the thread's last error
// and surface at the next launch check, so it is consumed here.
float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

sr_status cuda_fail(sr_context *ctx, cudaError_t e, const char *what) {
  const sr_status s = (e == cudaErrorMemoryAllocation) ? SR_ERR_OUT_OF_MEMORY : SR_ERR_CUDA;
  cudaGetLastError();  // reported here; a non-sticky error must not fail the next call's launch check
  return ctx->fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

int host_threads(const sr_context *ctx) {
  int t = ctx->opts.host_threads;
  if (t <= 0) t = static_cast<int>(std::thread::hardware_concurrency());
  return std::max(1, std::min(t, 64));
}

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

sr_status check_population(sr_context *ctx, const sr_population *pop) {
  if (!pop) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "population is NULL");
  if (pop->num_exprs < 0) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "num_exprs < 0");
  if (pop->num_exprs == 0) return SR_OK;
  if (!pop->tokens || !pop->values || !pop->offsets)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "population arrays must not be NULL");
  if (pop->offsets[0] != 0) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
  for (int i = 0; i < pop->num_exprs; ++i) {
    const int64_t len = pop->offsets[i + 1] - pop->offsets[i];
    if (len <= 0)
      return ctx->fail(SR_ERR_MALFORMED_EXPRESSION,
                       "expression " + std::to_string(i) + " is empty");
    if (len > SR_MAX_TOKENS)
      return ctx->fail(SR_ERR_EXPRESSION_TOO_LONG,
                       "expression " + std::to_string(i) + " has " + std::to_string(len) +
                           " tokens (max " + std::to_string(SR_MAX_TOKENS) + ")");
  }
  return SR_OK;
}

// Compile expressions [0, E) of a CSR population into ps (pinned staging).
sr_status compile_set(sr_context *ctx, int E, const int32_t *tok, const double *val,
                      const int64_t *off, const int32_t *hints, ProgramSet &ps) {
  SR_TRACE("sr: compile");
  ps.E = E;
  ps.cost.assign(static_cast<size_t>(E), 0.f);
  ps.n_const.assign(static_cast<size_t>(E), 0);
  ps.smax = 0;
  ps.n_instr = 0;
  ps.n_tokens = 0;
  ps.sfu_per_dp = ps.fp32_per_dp = 0.0;
  const int nt = std::max(1, std::min(host_threads(ctx), std::max(1, E / 32)));
  std::vector<std::vector<Instr>> codes(static_cast<size_t>(nt));
  std::vector<sr::ExprInfo> infos(static_cast<size_t>(E));
  std::vector<sr_status> st(static_cast<size_t>(nt), SR_OK);
  std::vector<std::string> msg(static_cast<size_t>(nt));
  std::vector<int64_t> bad(static_cast<size_t>(nt), -1);
  sr::parallel_for(nt, nt, [&](int64_t b, int64_t e) {
    for (int64_t c = b; c < e; ++c) {
      const int64_t x0 = static_cast<int64_t>(E) * c / nt, x1 = static_cast<int64_t>(E) * (c + 1) / nt;
      auto &code = codes[static_cast<size_t>(c)];
      code.reserve(static_cast<size_t>((off[x1] - off[x0]) / 2 + 8));
      for (int64_t x = x0; x < x1; ++x) {
        std::string err;
        const sr_status s = sr::compile_expression(
            tok + off[x], val + off[x], static_cast<int>(off[x + 1] - off[x]), ctx->V,
            hints ? hints + off[x] : nullptr, code, infos[static_cast<size_t>(x)], &err);
        if (s != SR_OK) {
          st[static_cast<size_t>(c)] = s;
          msg[static_cast<size_t>(c)] = err;
          bad[static_cast<size_t>(c)] = x;
          return;
        }
      }
    }
  });
  for (int c = 0; c < nt; ++c)
    if (st[static_cast<size_t>(c)] != SR_OK)
      return ctx->fail(st[static_cast<size_t>(c)],
                       "expression " + std::to_string(bad[static_cast<size_t>(c)]) + ": " +
                           msg[static_cast<size_t>(c)]);
  int64_t total = 0;
  for (auto &c : codes) total += static_cast<int64_t>(c.size());
  SR_TRY_CUDA(ctx, ps.h_code.ensure(static_cast<size_t>(total + 1)));
  SR_TRY_CUDA(ctx, ps.h_off.ensure(static_cast<size_t>(std::max(E, 1))));
  SR_TRY_CUDA(ctx, ps.h_len.ensure(static_cast<size_t>(std::max(E, 1))));
  int64_t pos = 0;
  for (auto &c : codes) {
    std::memcpy(ps.h_code.p + pos, c.data(), c.size() * sizeof(Instr));
    pos += static_cast<int64_t>(c.size());
  }
  ps.h_code.p[total] = Instr{0, 0, 0, 0};  // prefetch padding
  int64_t in_profile = 0;
  bool cache_refs = false;
  for (int64_t i = 0; i < total; ++i) {
    const uint32_t w = ps.h_code.p[i].w;
    in_profile += sr::in_protected_profile(sr::instr_op(w)) ? 1 : 0;
    cache_refs = cache_refs || (sr::instr_load(w) && sr::instr_leaf_kind(w) == sr::kLeafR) ||
                 sr::instr_b_kind(w) == sr::kBR;
  }
  ps.n_instr_protected = in_profile;
  ps.cache_refs = cache_refs;
  int64_t o = 0;
  for (int x = 0; x < E; ++x) {
    const auto &in = infos[static_cast<size_t>(x)];
    ps.h_off.p[x] = o;
    ps.h_len.p[x] = in.n_instr;
    o += in.n_instr;
    ps.cost[static_cast<size_t>(x)] = in.cost;
    ps.n_const[static_cast<size_t>(x)] = in.n_const;
    ps.smax = std::max(ps.smax, in.need);
    ps.n_tokens += in.n_tokens;
    ps.sfu_per_dp += in.sfu_ops;
    ps.fp32_per_dp += in.fp32_ops;
  }
  ps.n_instr = total;
  return SR_OK;
}

// Operator profile of a compiled set (the evaluation launches; prediction
// launches always use kOpsAll).
// Shortest datapoint span the planner shrinks to for occupancy.
constexpr int64_t kMinSpan = 256;

bool protected_profile(const ProgramSet &ps) {
  return ps.n_instr > 0 &&
         static_cast<double>(ps.n_instr_protected) >= sr::kProtectedShare * ps.n_instr;
}

// Launch shape: groups of G cost-sorted expressions x spans of datapoints.
// `split`: spill slots per warp kept in shared memory (-1 = the default for
// the dpt); the deeper slots live in per-warp global scratch.  `per_warp`:
// expressions per group and evaluating warp (a group of G = W x per_warp
// expressions shares each staged X span).
sr_status plan_set(sr_context *ctx, ProgramSet &ps, bool pred, int dpt, int W, int split,
                   int per_warp, int span_target) {
  sr::Plan p;
  p.dpt = dpt;
  p.W = W;
  p.ops = (!pred && protected_profile(ps)) ? sr::kOpsProtected : sr::kOpsAll;
  p.cache = !pred && ps.cache_refs;
  p.smax = std::max(ps.smax, 0);
  p.s_smem = std::min(p.smax, split < 0 ? sr::smem_spill_slots(dpt) : split);
  const int64_t tile = 32 * dpt;
  const int E = ps.E;
  p.G = std::max(1, W * per_warp);
  p.n_groups = (E + p.G - 1) / p.G;
  int dev_max_smem = 0;
  cudaDeviceGetAttribute(&dev_max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  // Span: the target, shrunk to the data and to the shared-memory budget.
  int64_t span = std::min<int64_t>(span_target, std::max<int64_t>(tile, round_up(ctx->N, tile)));
  while (span > tile &&
         sr::interp_smem_bytes(dpt, W, ctx->V, p.s_smem, static_cast<int>(span), p.G, pred) >
             static_cast<size_t>(dev_max_smem))
    span = std::max<int64_t>(tile, (span / 2) / tile * tile);
  // Then, while the span's shared memory (the X buffers grow with the
  // variable count) rather than the registers limits the resident blocks,
  // halve it: more resident warps pay for more, shorter work items
  // (9 variables, 8 datapoints x 8 warps: 2 -> 3 blocks per SM at 512).
  if (span_target > 0) {
    int bps_now = 0;
    SR_TRY_CUDA(ctx, sr::interp_configure(dpt, pred, p.ops, p.cache,
                                          sr::interp_smem_bytes(dpt, W, ctx->V, p.s_smem,
                                                                static_cast<int>(span), p.G,
                                                                pred),
                                          W, &bps_now));
    while (span / 2 >= std::max<int64_t>(tile, kMinSpan) && (span / 2) % tile == 0) {
      int bps_half = 0;
      SR_TRY_CUDA(ctx, sr::interp_configure(dpt, pred, p.ops, p.cache,
                                            sr::interp_smem_bytes(dpt, W, ctx->V, p.s_smem,
                                                                  static_cast<int>(span / 2),
                                                                  p.G, pred),
                                            W, &bps_half));
      if (bps_half <= bps_now) break;
      span /= 2;
      bps_now = bps_half;
    }
  }
  // The kernel walks a span tile by tile: it must hold whole tiles.
  if (span % tile != 0) return ctx->fail(SR_ERR_UNSUPPORTED, "span is not a multiple of the tile");
  p.span = static_cast<int>(span);
  p.smem = sr::interp_smem_bytes(dpt, W, ctx->V, p.s_smem, p.span, p.G, pred);
  if (p.smem > static_cast<size_t>(dev_max_smem))
    return ctx->fail(SR_ERR_UNSUPPORTED, "launch shape needs " + std::to_string(p.smem) +
                                             " bytes of shared memory");
  p.n_spans = (ctx->N == 0 || E == 0) ? 0 : static_cast<int>((ctx->N + span - 1) / span);
  // Spans per work item: as many as keep about 32 items of 32 expressions
  // per SM (up to 32 spans), so the per-(span group, expression) entries stay
  // small while the items still balance over the SMs; counted in units of 32
  // expressions, so that larger groups (more warps per block) do not cut the
  // span range into more span groups.  The result does not depend on this
  // choice (the spans' sums are added as double-doubles).
  p.k_spans = 1;
  if (!pred && p.n_spans > 0) {
    const int64_t units = (static_cast<int64_t>(E) + 31) / 32;
    const int64_t per_sm = static_cast<int64_t>(p.n_spans) * units /
                           (32 * static_cast<int64_t>(std::max(ctx->num_sms, 1)));
    p.k_spans = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(32, per_sm)));
  }
  // One FP64 (sum as hi + lo, count) per (span group, expression): 32 B x E
  // x span groups.  It is sized against the device's memory (the allocation
  // itself reports SR_ERR_OUT_OF_MEMORY when the free memory is short).
  if (!pred) {
    const double need = static_cast<double>(p.n_span_groups()) * E * 32.0;
    if (need > 0.9 * static_cast<double>(ctx->device_memory))
      return ctx->fail(SR_ERR_UNSUPPORTED,
                       "partial-sum buffer (" + std::to_string(static_cast<int64_t>(need)) +
                           " bytes) exceeds the device memory; split the population or the "
                           "datapoints");
  }
  int bps = 0;
  SR_TRY_CUDA(ctx, sr::interp_configure(dpt, pred, p.ops, p.cache, p.smem, W, &bps));
  if (bps <= 0) return ctx->fail(SR_ERR_UNSUPPORTED, "launch shape does not fit on an SM");
  const int64_t resident = static_cast<int64_t>(bps) * ctx->num_sms;
  // Few single-span items per resident block (a small population over few
  // datapoints): shorter spans give more, smaller items and a shorter tail.
  if (!pred && p.k_spans == 1) {
    while (p.items() < 16 * resident && p.span / 2 >= std::max<int64_t>(tile, 256) &&
           (p.span / 2) % tile == 0) {
      p.span /= 2;
      p.n_spans = static_cast<int>((ctx->N + p.span - 1) / p.span);
    }
    p.smem = sr::interp_smem_bytes(dpt, W, ctx->V, p.s_smem, p.span, p.G, pred);
  }
  p.blocks = static_cast<int>(std::min<int64_t>(resident, std::max<int64_t>(p.items(), 1)));
  // Global scratch for the spill slots that do not fit in shared memory.
  const size_t spill_floats = static_cast<size_t>(p.blocks) * W *
                              static_cast<size_t>(p.smax - p.s_smem) * static_cast<size_t>(tile);
  if (spill_floats > 0) SR_TRY_CUDA(ctx, ctx->spill.ensure(spill_floats));
  // Group table: expressions in decreasing modelled cost, G per group, so
  // every group holds similar work and hands out its largest first.
  SR_TRY_CUDA(ctx, ps.h_group.ensure(static_cast<size_t>(std::max(p.n_groups * p.G, 1))));
  std::vector<int32_t> order(static_cast<size_t>(E));
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return ps.cost[static_cast<size_t>(a)] > ps.cost[static_cast<size_t>(b)];
  });
  for (int64_t k = 0; k < static_cast<int64_t>(p.n_groups) * p.G; ++k)
    ps.h_group.p[k] = k < E ? order[static_cast<size_t>(k)] : -1;
  ps.plan = p;
  return SR_OK;
}

sr_status upload_groups(sr_context *ctx, ProgramSet &ps) {
  SR_TRACE("sr: upload groups");
  const size_t ng = static_cast<size_t>(std::max(ps.plan.n_groups * ps.plan.G, 1));
  ctx->prep_stats.h2d_bytes += static_cast<int64_t>(ng * sizeof(int32_t));
  SR_TRY_CUDA(ctx, ps.group.ensure(ng));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.group.p, ps.h_group.p, ng * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, ctx->stream));
  return SR_OK;
}

sr_status upload_code(sr_context *ctx, ProgramSet &ps) {
  SR_TRACE("sr: upload code");
  const int E = ps.E;
  SR_TRY_CUDA(ctx, ps.code.ensure(static_cast<size_t>(ps.n_instr + 1)));
  SR_TRY_CUDA(ctx, ps.off.ensure(static_cast<size_t>(std::max(E, 1))));
  SR_TRY_CUDA(ctx, ps.len.ensure(static_cast<size_t>(std::max(E, 1))));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.code.p, ps.h_code.p, (ps.n_instr + 1) * sizeof(Instr),
                                   cudaMemcpyHostToDevice, ctx->stream));
  ctx->prep_stats.h2d_bytes += static_cast<int64_t>((ps.n_instr + 1) * sizeof(Instr)) +
                               static_cast<int64_t>(E) * (sizeof(int64_t) + sizeof(int32_t));
  if (E > 0) {
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.off.p, ps.h_off.p, E * sizeof(int64_t),
                                     cudaMemcpyHostToDevice, ctx->stream));
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.len.p, ps.h_len.p, E * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, ctx->stream));
  }
  return SR_OK;
}

sr::EvalArgs make_args(sr_context *ctx, ProgramSet &ps, int32_t *counter) {
  sr::EvalArgs a{};
  a.X = ctx->X.p;
  a.ldx = ctx->ldx;
  a.N = ctx->N;
  a.code = ps.code.p;
  a.code_off = ps.off.p;
  a.code_len = ps.len.p;
  a.group_expr = ps.group.p;
  a.partial = ctx->partial.p;
  a.work_counter = counter;
  a.error = ctx->d_error;
  a.cache = ctx->cache_vals.p;
  a.ldc = ctx->ldx;
  a.V = ctx->V;
  a.E = ps.E;
  a.W = ps.plan.W;
  a.smax = ps.plan.smax;
  a.G = ps.plan.G;
  a.n_groups = ps.plan.n_groups;
  a.span = ps.plan.span;
  a.n_spans = ps.plan.n_spans;
  a.spill = ctx->spill.p;
  a.s_smem = ps.plan.s_smem;
  a.span_per_item = ps.plan.k_spans;
  return a;
}

sr_status launch_set(sr_context *ctx, ProgramSet &ps, bool pred, int32_t *counter,
                     float *pred_out, int64_t ldp, const int32_t *pred_row) {
  if (ps.plan.items() == 0) return SR_OK;
  sr::EvalArgs a = make_args(ctx, ps, counter);
  a.pred = pred_out;
  a.ldp = ldp;
  a.pred_row = pred_row;
  SR_TRY_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(int32_t), ctx->stream));
  SR_TRY_CUDA(ctx, sr::launch_interp(ps.plan.dpt, pred, ps.plan.ops, ps.plan.cache, a,
                                     ps.plan.blocks, ps.plan.smem,
                                     ctx->stream));
  return SR_OK;
}

// ---- launch-shape tuning ---------------------------------------------------

std::string tune_key(const sr_context *ctx, const ProgramSet &ps) {
  const int lg_n = ctx->N > 0 ? static_cast<int>(std::log2(static_cast<double>(ctx->N))) : 0;
  const int lg_e = ps.E > 0 ? static_cast<int>(std::log2(static_cast<double>(ps.E))) : 0;
  const double mean_instr = ps.E > 0 ? static_cast<double>(ps.n_instr) / ps.E : 0.0;
  std::ostringstream k;
  const bool prot = protected_profile(ps);
  k << ctx->device_name << "|V" << ctx->V << "|N" << lg_n << "|E" << lg_e << "|I"
    << static_cast<int>(std::lround(std::log2(1.0 + mean_instr) * 4.0)) << "|S" << ps.smax
    << "|P" << (prot ? sr::kOpsProtected : sr::kOpsAll);
  return k.str();
}

void load_tune_cache(sr_context *ctx) {
  ctx->tune_loaded = true;
  if (!ctx->opts.tune_cache_path) return;
  std::ifstream f(ctx->opts.tune_cache_path);
  if (!f) return;
  // Format: one entry per line:  "key": [dpt, W, split, per_warp],  (the last
  // two optional)
  std::string line;
  while (std::getline(f, line)) {
    const size_t q0 = line.find('"'), q1 = line.find('"', q0 + 1);
    const size_t b0 = line.find('[', q1), b1 = line.find(']', b0);
    if (q0 == std::string::npos || q1 == std::string::npos || b0 == std::string::npos ||
        b1 == std::string::npos)
      continue;
    int dpt = 0, w = 0, split = -1, per_warp = 4;
    const int n = std::sscanf(line.c_str() + b0, "[%d, %d, %d, %d]", &dpt, &w, &split, &per_warp);
    if (n >= 2 && (dpt == 4 || dpt == 8 || dpt == 16) && w >= 1 && w <= sr::kMaxInterpWarps &&
        split >= -1 && split <= sr::kMaxSpillSlots && per_warp >= 1 && per_warp <= 16)
      ctx->tuned[line.substr(q0 + 1, q1 - q0 - 1)] = {dpt, w, n >= 3 ? split : -1,
                                                       n >= 4 ? per_warp : 4};
  }
}

void save_tune_cache(const sr_context *ctx) {
  if (!ctx->opts.tune_cache_path) return;
  std::ofstream f(ctx->opts.tune_cache_path, std::ios::trunc);
  if (!f) return;
  f << "{\n";
  size_t i = 0;
  for (const auto &kv : ctx->tuned) {
    f << "  \"" << kv.first << "\": [" << kv.second.dpt << ", " << kv.second.W << ", "
      << kv.second.split << ", " << kv.second.per_warp << "]"
      << (++i < ctx->tuned.size() ? "," : "") << "\n";
  }
  f << "}\n";
}

// Milliseconds of two launches of the prepared main set in the given shape
// (after one warm-up launch); a negative value when the shape does not fit.
static sr_status time_shape(sr_context *ctx, int dpt, int W, int split, int per_warp,
                            float *ms_out) {
  *ms_out = -1.f;
  if (plan_set(ctx, ctx->main, false, dpt, W, split, per_warp) != SR_OK) {
    ctx->last_error.clear();
    return SR_OK;
  }
  SR_TRY(upload_groups(ctx, ctx->main));
  SR_TRY_CUDA(ctx, ctx->partial.ensure(static_cast<size_t>(std::max<int64_t>(
                       2 * static_cast<int64_t>(ctx->main.plan.n_span_groups()) * ctx->main.E,
                       1))));
  cudaEvent_t a = ctx->ev[4], b = ctx->ev[5];
  float t_sum = 0.f;
  for (int rep = 0; rep < 3; ++rep) {
    SR_TRY_CUDA(ctx, cudaEventRecord(a, ctx->stream));
    SR_TRY(launch_set(ctx, ctx->main, false, ctx->d_counter, nullptr, 0, nullptr));
    SR_TRY_CUDA(ctx, cudaEventRecord(b, ctx->stream));
    SR_TRY_CUDA(ctx, cudaEventSynchronize(b));
    const float ms = elapsed_ms(a, b);
    if (rep > 0) t_sum += ms;  // the first run warms up
  }
  *ms_out = t_sum;
  return SR_OK;
}

// Times candidate shapes on the prepared population and keeps the fastest:
// first datapoints per thread x warps per block with the default spill split,
// then, for programs that spill, other splits of the spill slots between
// shared memory and global scratch for the winning shape (fewer slots in
// shared memory can fit more blocks per SM; more keep the deeper slots out
// of L2), then the expressions per group (2, 4 or 8 per warp: larger groups
// reuse each staged X span more, smaller ones balance better).
sr_status autotune_main(sr_context *ctx, const std::string &key) {
  SR_TRACE("sr: autotune");
  static const int kCand[][2] = {{16, 8}, {16, 16}, {8, 8}, {8, 15}, {8, 31}, {4, 8}, {4, 16}};
  float best = 1e30f;
  sr_context::TunedShape win{8, 8, -1, 4};
  for (const auto &c : kCand) {
    float ms = 0.f;
    SR_TRY(time_shape(ctx, c[0], c[1], -1, 4, &ms));
    if (ms >= 0.f && ms < best) {
      best = ms;
      win = {c[0], c[1], -1, 4};
    }
  }
  const int smax = ctx->main.smax;
  if (smax > 0) {
    const int rule = std::min(smax, sr::smem_spill_slots(win.dpt));
    int tried[4] = {rule, -1, -1, -1};
    int n_tried = 1;
    for (const int split : {0, rule / 2, smax}) {
      if (split > sr::kMaxSpillSlots || std::find(tried, tried + n_tried, split) != tried + n_tried)
        continue;
      tried[n_tried++] = split;
      float ms = 0.f;
      SR_TRY(time_shape(ctx, win.dpt, win.W, split, 4, &ms));
      if (ms >= 0.f && ms < best) {
        best = ms;
        win.split = split;
      }
    }
  }
  for (const int per_warp : {2, 8}) {
    float ms = 0.f;
    SR_TRY(time_shape(ctx, win.dpt, win.W, win.split, per_warp, &ms));
    if (ms >= 0.f && ms < best) {
      best = ms;
      win.per_warp = per_warp;
    }
  }
  ctx->tuned[key] = win;
  save_tune_cache(ctx);
  return SR_OK;
}

sr_status prepare_main_shape(sr_context *ctx, bool allow_tune) {
  ProgramSet &ps = ctx->main;
  int dpt = ctx->opts.dpt, W = ctx->opts.warps_per_block, split = -1, per_warp = 4;
  if (dpt == 0 || W == 0) {
    if (!ctx->tune_loaded) load_tune_cache(ctx);
    const std::string key = tune_key(ctx, ps);
    auto it = ctx->tuned.find(key);
    if (it == ctx->tuned.end() && allow_tune && ctx->opts.autotune && ps.E > 0 && ctx->N > 0) {
      SR_TRY(autotune_main(ctx, key));
      it = ctx->tuned.find(key);
    }
    // Untuned defaults: 8 datapoints x 31 warps (one 1,024-thread block per
    // SM) for the protected profile, 8 x 8 (3 blocks per SM) where the wide
    // block's shared memory would not fit even at the shortest span (many
    // variables); 4 x 16 for populations over every operator, whose larger
    // dispatch switch fits the instruction cache better at 4 datapoints
    // (150 -> 82 ms on 4,000 all-operator expressions x 1M datapoints).
    const bool prot = protected_profile(ps);
    const bool have = it != ctx->tuned.end();
    int wide = 8;
    if (prot) {
      int dev_max_smem = 0;
      cudaDeviceGetAttribute(&dev_max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
      const int s_smem = std::min(std::max(ps.smax, 0), sr::smem_spill_slots(8));
      const int W = sr::kMaxInterpWarps;
      if (sr::interp_smem_bytes(8, W, ctx->V, s_smem, 32 * 8 * 2, W * per_warp, false) <=
          static_cast<size_t>(dev_max_smem))
        wide = W;
    }
    const int tdpt = have ? it->second.dpt : (prot ? 8 : 4);
    const int tw = have ? it->second.W : (prot ? wide : 16);
    // the tuned split belongs to the tuned shape only
    if (have && (dpt == 0 || dpt == tdpt) && (W == 0 || W == tw)) {
      split = it->second.split;
      per_warp = it->second.per_warp;
    }
    if (dpt == 0) dpt = W > sr::kMaxWarps ? 8 : tdpt;
    if (W == 0) W = tw;
  }
  if (ctx->opts.smem_spill_slots >= 0) split = ctx->opts.smem_spill_slots;
  SR_TRY(plan_set(ctx, ps, false, dpt, W, split, per_warp));
  SR_TRY(upload_groups(ctx, ps));
  SR_TRY_CUDA(ctx, ctx->partial.ensure(static_cast<size_t>(std::max<int64_t>(
                       2 * static_cast<int64_t>(ps.plan.n_span_groups()) * ps.E, 1))));
  return SR_OK;
}

}  // namespace capi
}  // namespace sr

// ============================================================================
// Record timing event k on the context stream.  While sr_launch captures a
// graph the event is recorded as an external event, which makes it an
// event-record node of the graph (a plain record would only mark a capture
// dependency); outside capture that flag is not accepted.
cudaError_t sr::capi::record_event(sr_context *ctx, int k) {
  return ctx->capturing ? cudaEventRecordWithFlags(ctx->ev[k], ctx->stream, cudaEventRecordExternal)
                        : cudaEventRecord(ctx->ev[k], ctx->stream);
}

// Forget the prepared launch (and its captured graph, whose kernel arguments
// point into buffers that the next prepare / set_data may move).
void sr::capi::reset_prepared(sr_context *ctx) {
  ctx->mode = sr::Mode::kNone;
  ctx->cache.rollback();  // subtrees of a launch that never ran hold no values
  if (ctx->graph_exec) {
    cudaGraphExecDestroy(ctx->graph_exec);
    ctx->graph_exec = nullptr;
  }
  ctx->graph_launches = 0;
}

// Drop the dataset, the cache built on it and every prepared launch.
void sr::capi::invalidate_data(sr_context *ctx) {
  reset_prepared(ctx);
  ctx->cache.clear();  // cached subtree values belong to the old data
  ctx->V = -1;
  ctx->N = 0;
}

extern "C" {

int32_t sr_abi_version(void) { return SR_ABI_VERSION; }

sr_status sr_inject_allocation_failure(int64_t n) {
  if (n < 0) return SR_ERR_INVALID_ARGUMENT;
  sr::alloc_fault_countdown().store(n);
  return SR_OK;
}

const char *sr_status_string(sr_status s) {
  switch (s) {
    case SR_OK: return "ok";
    case SR_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SR_ERR_BAD_TOKEN: return "unknown token";
    case SR_ERR_MALFORMED_EXPRESSION: return "malformed expression";
    case SR_ERR_EXPRESSION_TOO_LONG: return "expression too long";
    case SR_ERR_NO_DATA: return "no dataset on the device";
    case SR_ERR_CUDA: return "CUDA error";
    case SR_ERR_OUT_OF_MEMORY: return "out of memory";
    case SR_ERR_DEVICE_TIMEOUT: return "device wait timed out";
    case SR_ERR_DEVICE_CHECK: return "device bounds check failed";
    case SR_ERR_UNSUPPORTED: return "unsupported";
    case SR_ERR_NO_DEVICE: return "no CUDA device";
    case SR_ERR_TOO_MANY_VARS: return "too many variables";
  }
  return "unknown status";
}

const char *sr_last_error(const sr_context *ctx) {
  return ctx ? ctx->last_error.c_str() : "";
}

sr_status sr_options_init(sr_options *o) {
  if (!o) return SR_ERR_INVALID_ARGUMENT;
  std::memset(o, 0, sizeof *o);
  o->device = -1;
  o->cache_capacity = 2048;
  o->min_subtree_size = 3;
  o->min_subtree_freq = 10;
  o->dpt = 0;
  o->warps_per_block = 0;
  o->autotune = 0;
  o->use_graphs = 0;
  o->host_threads = 0;
  o->tune_cache_path = nullptr;
  o->stream = nullptr;
  o->smem_spill_slots = -1;
  return SR_OK;
}

sr_status sr_create(const sr_options *opts, sr_context **out) {
  if (!out) return SR_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  sr_options o;
  if (opts) o = *opts;
  else sr_options_init(&o);
  if (o.dpt != 0 && o.dpt != 4 && o.dpt != 8 && o.dpt != 16) return SR_ERR_INVALID_ARGUMENT;
  if (o.warps_per_block < 0 || o.warps_per_block > sr::kMaxInterpWarps) return SR_ERR_INVALID_ARGUMENT;
  // More than 16 warps per block exist only at 8 datapoints per thread.
  if (o.warps_per_block > sr::kMaxWarps && o.dpt != 0 && o.dpt != 8) return SR_ERR_INVALID_ARGUMENT;
  if (o.smem_spill_slots < -1 || o.smem_spill_slots > sr::kMaxSpillSlots)
    return SR_ERR_INVALID_ARGUMENT;
  if (o.cache_capacity < 0 || o.min_subtree_size < 1 || o.min_subtree_freq < 1)
    return SR_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return SR_ERR_NO_DEVICE;
  }
  int dev = o.device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return SR_ERR_NO_DEVICE;
  if (dev >= ndev) return SR_ERR_INVALID_ARGUMENT;
  auto *ctx = new sr_context();
  ctx->opts = o;
  ctx->device = dev;
  DeviceScope scope(dev);
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major < 10) {
    delete ctx;
    return SR_ERR_NO_DEVICE;  // this build carries sm_100a code only
  }
  ctx->num_sms = prop.multiProcessorCount;
  ctx->device_memory = prop.totalGlobalMem;
  ctx->device_name = prop.name;
  ctx->cache.capacity = o.cache_capacity;
  cudaError_t e = cudaSuccess;
  if (o.stream) {
    ctx->stream = static_cast<cudaStream_t>(o.stream);
  } else {
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    ctx->own_stream = (e == cudaSuccess);
  }
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counter, 2 * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_error, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_error, 0, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_error, sizeof(int32_t));
  for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&ctx->ev[i]);
  if (e != cudaSuccess) {
    sr_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? SR_ERR_OUT_OF_MEMORY : SR_ERR_CUDA;
  }
  *out = ctx;
  return SR_OK;
}

sr_status sr_destroy(sr_context *ctx) {
  if (!ctx) return SR_OK;
  DeviceScope scope(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  reset_prepared(ctx);
  for (auto &ev : ctx->ev)
    if (ev) cudaEventDestroy(ev);
  if (ctx->d_counter) cudaFree(ctx->d_counter);
  if (ctx->d_error) cudaFree(ctx->d_error);
  if (ctx->h_error) cudaFreeHost(ctx->h_error);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;  // device and pinned buffers are released by their owners
  return SR_OK;
}

sr_status sr_set_data_device(sr_context *ctx, const float *X_dev, int64_t ld, int32_t num_vars,
                             int64_t num_dps) {
  SR_TRACE("sr_set_data_device");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (num_vars < 0 || num_dps < 0 || (num_dps > 0 && !X_dev) || ld < num_dps)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad dataset arguments");
  if (num_vars > SR_MAX_VARS)
    return ctx->fail(SR_ERR_TOO_MANY_VARS, "num_vars " + std::to_string(num_vars) +
                                               " exceeds " + std::to_string(SR_MAX_VARS));
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // Done before X is touched: a failure below (allocation, copy) leaves the
  // context without data instead of holding launches that point into a
  // released or half-written X.
  invalidate_data(ctx);
  const int64_t ldx = std::max<int64_t>(sr::kDataAlign, round_up(num_dps, sr::kDataAlign));
  const size_t rows = static_cast<size_t>(num_vars) + 1;
  SR_TRY_CUDA(ctx, ctx->X.ensure(rows * static_cast<size_t>(ldx)));
  SR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->X.p, 0, rows * ldx * sizeof(float), ctx->stream));
  if (num_dps > 0)
    SR_TRY_CUDA(ctx, cudaMemcpy2DAsync(ctx->X.p, ldx * sizeof(float), X_dev, ld * sizeof(float),
                                       num_dps * sizeof(float), rows, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ldx = ldx;
  ctx->V = num_vars;
  ctx->N = num_dps;
  return SR_OK;
}

static sr_status set_data_host(sr_context *ctx, const float *X, const float *const *rows_ptr,
                               int32_t num_vars, int64_t num_dps) {
  SR_TRACE("sr_set_data");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (num_vars < 0 || num_dps < 0 || (num_dps > 0 && !X && !rows_ptr))
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad dataset arguments");
  if (num_vars > SR_MAX_VARS)
    return ctx->fail(SR_ERR_TOO_MANY_VARS, "num_vars " + std::to_string(num_vars) +
                                               " exceeds " + std::to_string(SR_MAX_VARS));
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // Done before X is touched: a failure below (allocation, copy) leaves the
  // context without data instead of holding launches that point into a
  // released or half-written X.
  invalidate_data(ctx);
  const int64_t ldx = std::max<int64_t>(sr::kDataAlign, round_up(num_dps, sr::kDataAlign));
  const size_t rows = static_cast<size_t>(num_vars) + 1;
  SR_TRY_CUDA(ctx, ctx->X.ensure(rows * static_cast<size_t>(ldx)));
  SR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->X.p, 0, rows * ldx * sizeof(float), ctx->stream));
  if (num_dps > 0) {
    if (X) {
      SR_TRY_CUDA(ctx, cudaMemcpy2DAsync(ctx->X.p, ldx * sizeof(float), X,
                                         num_dps * sizeof(float), num_dps * sizeof(float), rows,
                                         cudaMemcpyHostToDevice, ctx->stream));
    } else {
      for (size_t v = 0; v < rows; ++v) {
        if (!rows_ptr[v]) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "data row is NULL");
        SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->X.p + v * ldx, rows_ptr[v], num_dps * sizeof(float),
                                         cudaMemcpyHostToDevice, ctx->stream));
      }
    }
  }
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ldx = ldx;
  ctx->V = num_vars;
  ctx->N = num_dps;
  return SR_OK;
}

sr_status sr_set_data(sr_context *ctx, const float *X, int32_t num_vars, int64_t num_dps) {
  return set_data_host(ctx, X, nullptr, num_vars, num_dps);
}

sr_status sr_set_data_rows(sr_context *ctx, const float *const *rows, int32_t num_vars,
                           int64_t num_dps) {
  if (ctx && num_dps > 0 && !rows) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "rows is NULL");
  return set_data_host(ctx, nullptr, rows, num_vars, num_dps);
}

}  // extern "C"

namespace sr {
namespace capi {

// ---- prepare --------------------------------------------------------------

sr_status prepare_plain(sr_context *ctx, const sr_population *pop) {
  SR_TRACE("sr: prepare plain");
  sr::PlainSet &ps = ctx->plain;
  const int E = pop->num_exprs;
  const int64_t T = pop->offsets[E];
  // Validate through the compiler (same rules as the batched path) and check
  // the raw stack depth against the plain kernel's local stack.
  std::vector<Instr> scratch;
  for (int x = 0; x < E; ++x) {
    const int64_t o = pop->offsets[x];
    const int len = static_cast<int>(pop->offsets[x + 1] - o);
    sr::ExprInfo info;
    std::string err;
    scratch.clear();
    const sr_status s = sr::compile_expression(pop->tokens + o, pop->values + o, len, ctx->V,
                                               nullptr, scratch, info, &err);
    if (s != SR_OK) return ctx->fail(s, "expression " + std::to_string(x) + ": " + err);
    int depth = 0, maxd = 0;
    for (int i = len - 1; i >= 0; --i) {
      const int t = pop->tokens[o + i];
      if (t <= 0) ++depth;
      else if (sr::is_binary_token(t)) --depth;
      maxd = std::max(maxd, depth);
    }
    if (maxd > sr::kPlainStack)
      return ctx->fail(SR_ERR_UNSUPPORTED, "expression " + std::to_string(x) +
                                               " exceeds the plain kernel's stack");
  }
  SR_TRY_CUDA(ctx, ps.h_tok.ensure(static_cast<size_t>(T)));
  SR_TRY_CUDA(ctx, ps.h_val.ensure(static_cast<size_t>(T)));
  SR_TRY_CUDA(ctx, ps.h_off.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ps.h_len.ensure(static_cast<size_t>(E)));
  for (int64_t i = 0; i < T; ++i) {
    const int t = pop->tokens[i];
    const double v = pop->values[i];
    ps.h_tok.p[i] = t;
    if (t == SR_TOK_VAR) {
      const bool ok = v > -2147483648.0 && v < 2147483648.0;
      const int vi = ok ? static_cast<int>(v) : -1;
      ps.h_val.p[i] = static_cast<float>((vi >= 0 && vi < ctx->V) ? vi : -1);
    } else {
      ps.h_val.p[i] = static_cast<float>(v);
    }
  }
  for (int x = 0; x < E; ++x) {
    ps.h_off.p[x] = pop->offsets[x];
    ps.h_len.p[x] = static_cast<int32_t>(pop->offsets[x + 1] - pop->offsets[x]);
  }
  SR_TRY_CUDA(ctx, ps.tok.ensure(static_cast<size_t>(T)));
  SR_TRY_CUDA(ctx, ps.val.ensure(static_cast<size_t>(T)));
  SR_TRY_CUDA(ctx, ps.off.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ps.len.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.tok.p, ps.h_tok.p, T * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.val.p, ps.h_val.p, T * sizeof(float),
                                   cudaMemcpyHostToDevice, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.off.p, ps.h_off.p, E * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ps.len.p, ps.h_len.p, E * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, ctx->stream));
  ps.E = E;
  ctx->prep_stats.h2d_bytes += T * static_cast<int64_t>(sizeof(int32_t) + sizeof(float)) +
                               static_cast<int64_t>(E) * (sizeof(int64_t) + sizeof(int32_t));
  ps.n_dpblocks = static_cast<int>(std::min<int64_t>((ctx->N + 127) / 128, 256));
  SR_TRY_CUDA(ctx, ctx->partial.ensure(static_cast<size_t>(
                       std::max<int64_t>(static_cast<int64_t>(ps.n_dpblocks) * E, 1))));
  ctx->prep_stats.node_evals = T * ctx->N;
  ctx->prep_stats.node_evals_executed = T * ctx->N;
  return SR_OK;
}

// Common-subtree detection on the context's GPU: the same Detection as
// sr::detect_common_subtrees (groups largest first, stable in hash order).
sr_status detect_on_device(sr_context *ctx, int E, const int32_t *tok, const double *val,
                                  const int64_t *off, int min_size, int min_freq,
                                  sr::Detection &out) {
  SR_TRACE("sr: detect (device)");
  out = sr::Detection{};
  out.total_tokens = E > 0 ? off[E] - off[0] : 0;
  const int64_t T = out.total_tokens;
  if (E <= 0 || T <= 0) return SR_OK;
  if (T >= (1ll << 31)) return ctx->fail(SR_ERR_UNSUPPORTED, "population too large for device detection");
  sr::DetectBufs &b = ctx->det;
  cudaStream_t s = ctx->stream;
  const size_t n = static_cast<size_t>(T);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(s));  // buffers may grow
  SR_TRY_CUDA(ctx, b.tok.ensure(n));
  SR_TRY_CUDA(ctx, b.val.ensure(n));
  SR_TRY_CUDA(ctx, b.off.ensure(static_cast<size_t>(E) + 1));
  for (auto *buf : {&b.size, &b.pos_in, &b.pos_out, &b.run_count, &b.run_start, &b.rep, &b.gsize,
                    &b.vcount})
    SR_TRY_CUDA(ctx, buf->ensure(n));
  SR_TRY_CUDA(ctx, b.out3.ensure(3 * n));
  for (auto *buf : {&b.hash, &b.key_in, &b.key_out, &b.run_key}) SR_TRY_CUDA(ctx, buf->ensure(n));
  SR_TRY_CUDA(ctx, b.cand.ensure(n));
  SR_TRY_CUDA(ctx, b.mark.ensure(n));
  SR_TRY_CUDA(ctx, b.counters.ensure(2));
  SR_TRY_CUDA(ctx, b.covered.ensure(1));
  SR_TRY_CUDA(ctx, b.h_counters.ensure(2));
  SR_TRY_CUDA(ctx, b.h_covered.ensure(1));
  const size_t temp = std::max(sr::detect_scratch_sizes(T).temp_bytes,
                               sr::detect_scan_temp_bytes(static_cast<int>(T)));
  SR_TRY_CUDA(ctx, b.temp.ensure(std::max<size_t>(temp, 1)));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(b.tok.p, tok + off[0], n * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(b.val.p, val + off[0], n * sizeof(double),
                                   cudaMemcpyHostToDevice, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(b.off.p, off, (static_cast<size_t>(E) + 1) * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, s));
  sr::DetectArgs a{};
  a.tok = b.tok.p;
  a.val = b.val.p;
  a.off = b.off.p;
  a.E = E;
  a.T = T;
  a.min_size = min_size;
  a.min_freq = min_freq;
  a.size = b.size.p;
  a.hash = b.hash.p;
  a.cand = b.cand.p;
  a.mark = b.mark.p;
  a.pos_in = b.pos_in.p;
  a.pos_out = b.pos_out.p;
  a.key_in = b.key_in.p;
  a.key_out = b.key_out.p;
  a.run_key = b.run_key.p;
  a.run_count = b.run_count.p;
  a.run_start = b.run_start.p;
  a.rep = b.rep.p;
  a.gsize = b.gsize.p;
  a.vcount = b.vcount.p;
  a.n_sel = b.counters.p;
  a.n_runs = b.counters.p + 1;
  a.covered = b.covered.p;
  a.temp = b.temp.p;
  a.temp_bytes = b.temp.cap;
  auto read_counters = [&]() -> sr_status {
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(b.h_counters.p, b.counters.p, 2 * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, s));
    SR_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    return SR_OK;
  };
  SR_TRY_CUDA(ctx, cudaMemsetAsync(b.counters.p, 0, 2 * sizeof(int32_t), s));
  SR_TRY_CUDA(ctx, sr::detect_candidates(a, s));
  SR_TRY(read_counters());
  const int M = b.h_counters.p[0];
  SR_TRY_CUDA(ctx, sr::detect_groups(a, M, s));
  SR_TRY(read_counters());
  const int R = M > 0 ? b.h_counters.p[1] : 0;
  SR_TRY_CUDA(ctx, sr::detect_verify(a, R, s));
  SR_TRY_CUDA(ctx, sr::detect_frequent(a, R, b.out3.p, s));
  SR_TRY(read_counters());
  const int F = R > 0 ? b.h_counters.p[0] : 0;
  SR_TRY_CUDA(ctx, b.h_out3.ensure(static_cast<size_t>(3 * std::max(F, 1))));
  if (F > 0)
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(b.h_out3.p, b.out3.p, 3 * static_cast<size_t>(F) * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(b.h_covered.p, b.covered.p, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, s));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(s));
  // Groups in hash order -> size descending, stable.
  std::vector<int> order(static_cast<size_t>(F));
  std::iota(order.begin(), order.end(), 0);
  const int32_t *o3 = b.h_out3.p;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return o3[3 * x + 1] > o3[3 * y + 1]; });
  int64_t size_sum = 0;
  out.groups.reserve(static_cast<size_t>(F));
  for (int k : order) {
    const int64_t g = o3[3 * k] + off[0];  // absolute token index
    const int64_t *it = std::upper_bound(off, off + E + 1, g) - 1;
    const int32_t x = static_cast<int32_t>(it - off);
    out.groups.push_back(sr::Detection::Group{x, static_cast<int32_t>(g - off[x]), o3[3 * k + 1],
                                              o3[3 * k + 2]});
    size_sum += o3[3 * k + 1];
  }
  out.covered_tokens = static_cast<int64_t>(*b.h_covered.p);
  out.avg_subtree_size = F > 0 ? static_cast<double>(size_sum) / F : 0.0;
  out.coverage = T > 0 ? static_cast<double>(out.covered_tokens) / T : 0.0;
  return SR_OK;
}

sr_status prepare_cached(sr_context *ctx, const sr_population *pop, uint32_t flags) {
  SR_TRACE("sr: prepare cached");
  const int E = pop->num_exprs;
  const int64_t T = pop->offsets[E];
  // Validate first so that malformed input never reaches the cache.
  {
    std::vector<Instr> scratch;
    for (int x = 0; x < E; ++x) {
      const int64_t o = pop->offsets[x];
      sr::ExprInfo info;
      std::string err;
      scratch.clear();
      const sr_status s = sr::compile_expression(pop->tokens + o, pop->values + o,
                                                 static_cast<int>(pop->offsets[x + 1] - o), ctx->V,
                                                 nullptr, scratch, info, &err);
      if (s != SR_OK) return ctx->fail(s, "expression " + std::to_string(x) + ": " + err);
    }
  }
  if (flags & SR_EVAL_CLEAR_CACHE) ctx->cache.clear();
  const int threads = host_threads(ctx);
  const double t0 = now_ms();
  sr::Detection det;
  if (ctx->opts.device_detect) {
    SR_TRY(detect_on_device(ctx, E, pop->tokens, pop->values, pop->offsets,
                            ctx->opts.min_subtree_size, ctx->opts.min_subtree_freq, det));
  } else {
    SR_TRACE("sr: detect (host)");
    sr::detect_common_subtrees(E, pop->tokens, pop->values, pop->offsets,
                               ctx->opts.min_subtree_size, ctx->opts.min_subtree_freq, threads,
                               det);
  }
  ctx->prep_stats.detect_time_ms = now_ms() - t0;
  ctx->prep_stats.num_subtrees = static_cast<int32_t>(det.groups.size());
  ctx->prep_stats.avg_subtree_size = det.avg_subtree_size;
  ctx->prep_stats.coverage = det.coverage;

  // Cache update (reference cl_gpu_eval.cu:384-396): new keys get the next
  // free slot until the capacity is reached.  They stay pending until this
  // prepare's launch is enqueued (sr_launch commits them).
  ctx->cache.begin_pending();
  std::vector<int32_t> sub_tok;
  std::vector<double> sub_val;
  std::vector<int64_t> sub_off{0};
  std::vector<int32_t> sub_slot;
  for (const auto &g : det.groups) {
    const int32_t *t = pop->tokens + pop->offsets[g.expr] + g.pos;
    const double *v = pop->values + pop->offsets[g.expr] + g.pos;
    const uint64_t key = sr::flat_key(t, v, g.size);
    if (ctx->cache.slot_of.count(key)) continue;
    if (ctx->cache.used >= ctx->cache.capacity) continue;
    const int32_t slot = ctx->cache.used++;
    ctx->cache.slot_of.emplace(key, slot);
    ctx->cache.pending.push_back(key);
    sub_tok.insert(sub_tok.end(), t, t + g.size);
    sub_val.insert(sub_val.end(), v, v + g.size);
    sub_off.push_back(static_cast<int64_t>(sub_tok.size()));
    sub_slot.push_back(slot);
  }
  const int n_new = static_cast<int>(sub_slot.size());
  ctx->prep_stats.new_subtrees = n_new;
  ctx->prep_stats.cache_slots_used = ctx->cache.used;

  // Cache values live in [capacity][ldx]; allocated on first use.
  if (ctx->cache.capacity > 0)
    SR_TRY_CUDA(ctx, ctx->cache_vals.ensure(static_cast<size_t>(ctx->cache.capacity) * ctx->ldx));

  // Subtrees to evaluate into the cache this call.
  const double tc0 = now_ms();
  SR_TRY(compile_set(ctx, n_new, sub_tok.data(), sub_val.data(), sub_off.data(), nullptr, ctx->sub));
  SR_TRY_CUDA(ctx, ctx->sub.h_row.ensure(static_cast<size_t>(std::max(n_new, 1))));
  for (int k = 0; k < n_new; ++k) ctx->sub.h_row.p[k] = sub_slot[static_cast<size_t>(k)];
  if (n_new > 0) {
    SR_TRY(plan_set(ctx, ctx->sub, true, 8, sr::kMaxWarps));
    SR_TRY(upload_code(ctx, ctx->sub));
    SR_TRY(upload_groups(ctx, ctx->sub));
    SR_TRY_CUDA(ctx, ctx->sub.row.ensure(static_cast<size_t>(n_new)));
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->sub.row.p, ctx->sub.h_row.p, n_new * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, ctx->stream));
    ctx->prep_stats.h2d_bytes += static_cast<int64_t>(n_new) * sizeof(int32_t);
  } else {
    ctx->sub.plan = sr::Plan{};
  }

  // Skeletons (reference mark_cached_subtrees_from_state + skeleton rewrite,
  // cl_gpu_eval.cu:294-329, 433-459).
  ctx->hints.resize(static_cast<size_t>(T));
  const int64_t removed = sr::mark_cached_subtrees(E, pop->tokens, pop->values, pop->offsets,
                                                   ctx->cache, threads, ctx->hints.data());
  SR_TRY(compile_set(ctx, E, pop->tokens, pop->values, pop->offsets, ctx->hints.data(), ctx->main));
  ctx->prep_stats.host_compile_time_ms = now_ms() - tc0;
  SR_TRY(upload_code(ctx, ctx->main));
  SR_TRY(prepare_main_shape(ctx, false));
  ctx->prep_stats.node_evals = T * ctx->N;
  ctx->prep_stats.node_evals_executed = (T - removed + static_cast<int64_t>(sub_tok.size())) * ctx->N;
  return SR_OK;
}

}  // namespace capi
}  // namespace sr

extern "C" {

sr_status sr_prepare(sr_context *ctx, const sr_population *pop, uint32_t flags) {
  SR_TRACE("sr_prepare");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  SR_TRY(check_population(ctx, pop));
  if (ctx->V < 0) return ctx->fail(SR_ERR_NO_DATA, "no dataset: call sr_set_data first");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  reset_prepared(ctx);
  ctx->prep_stats = sr_stats{};
  const int E = pop->num_exprs;
  ctx->E = E;
  if (E == 0) return SR_OK;
  SR_TRY_CUDA(ctx, ctx->mse.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->h_mse.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
  if (flags & SR_EVAL_GRADIENT) {
    SR_TRY(prepare_grad(ctx, pop, (flags & SR_EVAL_GRAD_RECOMPUTE) != 0,
                        (flags & SR_EVAL_GRAD_REVERSE) != 0));
    ctx->mode = sr::Mode::kGrad;
  } else if (flags & SR_EVAL_PLAIN) {
    SR_TRY(prepare_plain(ctx, pop));
    ctx->mode = sr::Mode::kPlain;
  } else if (flags & SR_EVAL_SUBTREE_CACHE) {
    SR_TRY(prepare_cached(ctx, pop, flags));
    ctx->mode = sr::Mode::kCached;
  } else {
    const double tc0 = now_ms();
    SR_TRY(compile_set(ctx, E, pop->tokens, pop->values, pop->offsets, nullptr, ctx->main));
    ctx->prep_stats.host_compile_time_ms = now_ms() - tc0;
    SR_TRY(upload_code(ctx, ctx->main));
    SR_TRY(prepare_main_shape(ctx, true));
    ctx->prep_stats.node_evals = ctx->main.n_tokens * ctx->N;
    ctx->prep_stats.node_evals_executed = ctx->prep_stats.node_evals;
    ctx->mode = sr::Mode::kBatched;
  }
  SR_TRY_CUDA(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
  return SR_OK;
}

// Enqueue the prepared launch sequence on the context stream.
static sr_status enqueue_launch(sr_context *ctx, int *launches_out) {
  cudaStream_t s = ctx->stream;
  SR_TRY_CUDA(ctx, record_event(ctx, 0));
  int launches = 0;
  if (ctx->mode == sr::Mode::kGrad) {
    SR_TRY(launch_grad(ctx));
    launches = grad_launch_count(ctx->grad);
  } else if (ctx->mode == sr::Mode::kPlain) {
    SR_TRY_CUDA(ctx, record_event(ctx, 1));
    SR_TRY_CUDA(ctx, sr::launch_plain(ctx->plain.tok.p, ctx->plain.val.p, ctx->plain.off.p,
                                      ctx->plain.len.p, ctx->X.p, ctx->ldx, ctx->V, ctx->N,
                                      ctx->plain.E, ctx->partial.p, ctx->plain.n_dpblocks, s));
    launches += ctx->N > 0 ? 1 : 0;
    SR_TRY_CUDA(ctx, record_event(ctx, 2));
    SR_TRY_CUDA(ctx, sr::launch_finalize(ctx->partial.p, ctx->N > 0 ? ctx->plain.n_dpblocks : 0,
                                         ctx->E, ctx->mse.p, s));
    ++launches;
  } else {
    if (ctx->mode == sr::Mode::kCached && ctx->sub.plan.items() > 0) {
      SR_TRY(launch_set(ctx, ctx->sub, true, ctx->d_counter + 1, ctx->cache_vals.p, ctx->ldx,
                        ctx->sub.row.p));
      ++launches;
    }
    SR_TRY_CUDA(ctx, record_event(ctx, 1));
    if (ctx->main.plan.items() > 0) {
      SR_TRY(launch_set(ctx, ctx->main, false, ctx->d_counter, nullptr, 0, nullptr));
      ++launches;
    }
    SR_TRY_CUDA(ctx, record_event(ctx, 2));
    SR_TRY_CUDA(ctx, sr::launch_finalize_groups(ctx->partial.p, ctx->main.plan.n_span_groups(),
                                                ctx->E, ctx->mse.p, nullptr, s));
    ++launches;
  }
  SR_TRY_CUDA(ctx, record_event(ctx, 3));
  *launches_out = launches;
  return SR_OK;
}

static sr_status launch_prepared(sr_context *ctx, bool allow_graph);

sr_status sr_launch(sr_context *ctx) { return launch_prepared(ctx, true); }

// allow_graph = false for one-shot evaluations (a graph pays off only when the
// prepared launch is replayed).
static sr_status launch_prepared(sr_context *ctx, bool allow_graph) {
  SR_TRACE("sr_launch");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (ctx->E == 0) return SR_OK;
  if (ctx->mode == sr::Mode::kNone) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "nothing prepared");
  DeviceScope scope(ctx->device);
  cudaStream_t s = ctx->stream;
  int launches = 0;
  if (ctx->opts.use_graphs && (allow_graph || ctx->graph_exec)) {
    if (!ctx->graph_exec) {
      // Relaxed mode: the launchers set kernel attributes while capturing.
      SR_TRY_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
      ctx->capturing = true;
      const sr_status st = enqueue_launch(ctx, &launches);
      ctx->capturing = false;
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (st != SR_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
      }
      SR_TRY_CUDA(ctx, ce);
      const cudaError_t ie = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) ctx->graph_exec = nullptr;
      SR_TRY_CUDA(ctx, ie);
      ctx->graph_launches = launches;
    }
    SR_TRY_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, s));
    launches = ctx->graph_launches;
  } else {
    SR_TRY(enqueue_launch(ctx, &launches));
  }
  ctx->cache.commit();  // the subtree launch that writes the new cached values is enqueued
  ctx->timing_valid = true;
  ctx->prep_stats.kernel_launches = launches;
  return SR_OK;
}

}  // extern "C"

namespace sr {
namespace capi {

sr_status check_device_error(sr_context *ctx) {
  if (*ctx->h_error == 0) return SR_OK;
  const int32_t code = *ctx->h_error;
  *ctx->h_error = 0;
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  ctx->cache.clear();  // the failed launch may have left cached values unwritten
  if (code & sr::kDevErrTimeout)
    return ctx->fail(SR_ERR_DEVICE_TIMEOUT, "a device-side wait exceeded its time limit");
  return ctx->fail(SR_ERR_DEVICE_CHECK, "device bounds check failed");
}

void fill_stats(sr_context *ctx, sr_stats *st) {
  if (!st) return;
  *st = ctx->prep_stats;
  if (ctx->timing_valid) {
    st->gpu_kernel_time_ms = elapsed_ms(ctx->ev[0], ctx->ev[3]);
    st->eval_kernel_time_ms = elapsed_ms(ctx->ev[1], ctx->ev[2]);
    st->data_transfer_time_ms = elapsed_ms(ctx->ev[4], ctx->ev[5]);
  }
  if (ctx->mode == sr::Mode::kBatched || ctx->mode == sr::Mode::kCached) {
    st->declared_sfu_ops = ctx->main.sfu_per_dp * static_cast<double>(ctx->N);
    st->declared_fp32_ops = ctx->main.fp32_per_dp * static_cast<double>(ctx->N);
  }
  st->d2h_bytes += static_cast<int64_t>(ctx->E) * static_cast<int64_t>(sizeof(float)) +
                   static_cast<int64_t>(sizeof(int32_t));
  const sr::Plan &p = ctx->main.plan;
  st->dpt = p.dpt;
  st->warps_per_block = p.W;
  st->blocks = p.blocks;
  st->work_items = static_cast<int32_t>(p.items());
}

}  // namespace capi
}  // namespace sr

extern "C" {

sr_status sr_read_mse(sr_context *ctx, float *mse_out, sr_stats *stats) {
  SR_TRACE("sr_read_mse");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (ctx->E == 0) return SR_OK;
  if (ctx->mode == sr::Mode::kNone) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "nothing launched");
  if (!mse_out) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "mse_out is NULL");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_mse.p, ctx->mse.p, ctx->E * sizeof(float),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  SR_TRY(check_device_error(ctx));
  std::memcpy(mse_out, ctx->h_mse.p, ctx->E * sizeof(float));
  fill_stats(ctx, stats);
  return SR_OK;
}

sr_status sr_read_sums(sr_context *ctx, double *sum_out, double *count_out) {
  SR_TRACE("sr_read_sums");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (ctx->E == 0) return SR_OK;
  if (ctx->mode == sr::Mode::kNone) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "nothing launched");
  if (!sum_out || !count_out)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "sum_out / count_out is NULL");
  int n_spans = 0;
  switch (ctx->mode) {
    case sr::Mode::kPlain: n_spans = ctx->N > 0 ? ctx->plain.n_dpblocks : 0; break;
    case sr::Mode::kGrad: n_spans = ctx->grad.n_spans; break;
    default: n_spans = ctx->main.plan.n_span_groups(); break;
  }
  const int E = ctx->E;
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the buffers may grow
  SR_TRY_CUDA(ctx, ctx->sums.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->h_sums.ensure(static_cast<size_t>(E)));
  if (ctx->mode == sr::Mode::kPlain)
    SR_TRY_CUDA(ctx, sr::launch_sums(ctx->partial.p, n_spans, E, ctx->sums.p, ctx->stream));
  else if (ctx->mode == sr::Mode::kGrad)
    ;  // the gradient finalize kernels wrote ctx->sums
  else
    SR_TRY_CUDA(ctx, sr::launch_finalize_groups(ctx->partial.p, n_spans, E, nullptr,
                                                ctx->sums.p, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_sums.p, ctx->sums.p, E * sizeof(double2),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  SR_TRY(check_device_error(ctx));
  for (int e = 0; e < E; ++e) {
    sum_out[e] = ctx->h_sums.p[e].x;
    count_out[e] = ctx->h_sums.p[e].y;
  }
  return SR_OK;
}

sr_status sr_read_grad_sums(sr_context *ctx, double *grad_sum_out) {
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (ctx->E == 0) return SR_OK;
  if (ctx->mode != sr::Mode::kGrad)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "no gradient prepared (SR_EVAL_GRADIENT)");
  const int64_t C = ctx->grad.C;
  if (C == 0) return SR_OK;
  if (!grad_sum_out) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "grad_sum_out is NULL");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(grad_sum_out, ctx->grad.grad_acc.p, C * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SR_OK;
}

sr_status sr_read_grad(sr_context *ctx, float *grad_out) {
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (ctx->E == 0) return SR_OK;
  if (ctx->mode != sr::Mode::kGrad)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "no gradient prepared (SR_EVAL_GRADIENT)");
  const int64_t C = ctx->grad.C;
  if (C == 0) return SR_OK;
  if (!grad_out) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "grad_out is NULL");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(grad_out, ctx->grad.grad.p, C * sizeof(float),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  SR_TRY(check_device_error(ctx));
  ctx->prep_stats.d2h_bytes += C * static_cast<int64_t>(sizeof(float));
  return SR_OK;
}

sr_status sr_last_launch_times(sr_context *ctx, float *launch_ms, float *eval_kernel_ms) {
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (!ctx->timing_valid) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "no launch recorded");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
  float a = 0.f, b = 0.f;
  SR_TRY_CUDA(ctx, cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[3]));
  SR_TRY_CUDA(ctx, cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]));
  if (launch_ms) *launch_ms = a;
  if (eval_kernel_ms) *eval_kernel_ms = b;
  return SR_OK;
}

sr_status sr_device_mse(sr_context *ctx, float **mse_dev) {
  if (!ctx || !mse_dev) return SR_ERR_INVALID_ARGUMENT;
  *mse_dev = ctx->mse.p;
  return SR_OK;
}

sr_status sr_eval_mse(sr_context *ctx, const sr_population *pop, uint32_t flags, float *mse_out,
                      sr_stats *stats) {
  SR_TRACE("sr_eval_mse");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  const double t0 = now_ms();
  SR_TRY(sr_prepare(ctx, pop, flags));
  if (pop->num_exprs == 0) {
    if (stats) *stats = sr_stats{};
    return SR_OK;
  }
  SR_TRY(launch_prepared(ctx, false));
  SR_TRY(sr_read_mse(ctx, mse_out, stats));
  if (stats) stats->total_eval_time_ms = now_ms() - t0;
  return SR_OK;
}

sr_status sr_eval_predictions(sr_context *ctx, const sr_population *pop, int64_t dp_begin,
                              int64_t dp_count, float *pred_out) {
  SR_TRACE("sr_eval_predictions");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  SR_TRY(check_population(ctx, pop));
  if (ctx->V < 0) return ctx->fail(SR_ERR_NO_DATA, "no dataset: call sr_set_data first");
  if (dp_begin < 0 || dp_count < 0 || dp_begin + dp_count > ctx->N)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "datapoint range outside the dataset");
  if (pop->num_exprs == 0 || dp_count == 0) return SR_OK;
  if (!pred_out) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "pred_out is NULL");
  const int E = pop->num_exprs;
  const double bytes = static_cast<double>(E) * ctx->ldx * sizeof(float);
  if (bytes > 16.0 * (1ull << 30))
    return ctx->fail(SR_ERR_UNSUPPORTED, "prediction buffer would exceed 16 GiB");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  reset_prepared(ctx);
  SR_TRY(compile_set(ctx, E, pop->tokens, pop->values, pop->offsets, nullptr, ctx->main));
  SR_TRY_CUDA(ctx, ctx->main.h_row.ensure(static_cast<size_t>(E)));
  for (int x = 0; x < E; ++x) ctx->main.h_row.p[x] = x;
  int dpt = ctx->opts.dpt ? ctx->opts.dpt : 8;
  int W = ctx->opts.warps_per_block ? std::min(ctx->opts.warps_per_block, sr::kMaxWarps)
                                     : sr::kMaxWarps;
  SR_TRY(plan_set(ctx, ctx->main, true, dpt, W));
  SR_TRY(upload_code(ctx, ctx->main));
  SR_TRY(upload_groups(ctx, ctx->main));
  SR_TRY_CUDA(ctx, ctx->main.row.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->main.row.p, ctx->main.h_row.p, E * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, ctx->stream));
  SR_TRY_CUDA(ctx, ctx->pred.ensure(static_cast<size_t>(E) * ctx->ldx));
  SR_TRY(launch_set(ctx, ctx->main, true, ctx->d_counter, ctx->pred.p, ctx->ldx, ctx->main.row.p));
  SR_TRY_CUDA(ctx, cudaMemcpy2DAsync(pred_out, dp_count * sizeof(float), ctx->pred.p + dp_begin,
                                     ctx->ldx * sizeof(float), dp_count * sizeof(float), E,
                                     cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  SR_TRY(check_device_error(ctx));
  return SR_OK;
}

sr_status sr_count_constants(const sr_population *pop, int64_t *const_offsets) {
  if (!pop || !const_offsets || pop->num_exprs < 0) return SR_ERR_INVALID_ARGUMENT;
  int64_t acc = 0;
  for (int x = 0; x < pop->num_exprs; ++x) {
    const_offsets[x] = acc;
    for (int64_t i = pop->offsets[x]; i < pop->offsets[x + 1]; ++i)
      acc += pop->tokens[i] == SR_TOK_CONST ? 1 : 0;
  }
  const_offsets[pop->num_exprs] = acc;
  return SR_OK;
}

}  // extern "C"
