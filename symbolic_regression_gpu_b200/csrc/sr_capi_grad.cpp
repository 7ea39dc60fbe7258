// sr_capi_grad.cpp — the C ABI of the fused forward + adjoint (sr_eval_grad,
// gradient launches prepared by sr_prepare) and of on-device Adam
// (sr_optimize_constants).  No reference counterpart: the reference
// evaluates MSE only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sr_adjoint.hpp"
#include "sr_capi_internal.hpp"
#include "sr_context.hpp"
#include "sr_kernels.hpp"
#include "sr_trace.hpp"

using sr::Instr;
using sr::ProgramSet;
using namespace sr::capi;

// ---- forward + adjoint ------------------------------------------------------

namespace sr {
namespace capi {

constexpr int kMaxAdjConsts = 64;  // constants per expression with a gradient

// Forward-mode widths (tangent rows per warp): an expression goes to the
// first launch whose width holds its constants; expressions with more than
// the widest are differentiated in reverse mode.
constexpr int kTanWidths[] = {4, sr::kMaxTangentConsts};
constexpr int kNumTanWidths = 2;

// Mask words of one program for the forward-mode kernel (TanArgs::tmask):
// the constants (token-order indices, all below kMaxTangentConsts here) under
// the accumulator before each operator (A) and under its operand b (B), and
// the constant-load flag.
void tangent_masks(const Instr *code, int len, uint32_t *out) {
  uint32_t mT = 0;
  uint32_t mS[32] = {};
  for (int i = 0; i < len; ++i) {
    const Instr &in = code[i];
    if (sr::instr_spill(in.w)) mS[sr::instr_spill_slot(in.w) & 31u] = mT;
    uint32_t A = mT, L = 0;
    if (sr::instr_load(in.w)) {
      const uint32_t ca = in.c & 0x3FFu;
      const bool cl = sr::instr_leaf_kind(in.w) == sr::kLeafC && ca < 8u;
      A = cl ? (1u << ca) : 0u;
      L = cl ? sr::kTanLoadConst : 0u;
    }
    uint32_t B = 0;
    const uint32_t bk = sr::instr_b_kind(in.w);
    const uint32_t cb = (in.c >> 10) & 0x3FFu;
    if (bk == sr::kBC && cb < 8u) B = 1u << cb;
    if (bk == sr::kBS) B = mS[in.b & 31u];
    mT = A | B;
    out[i] = A | (B << 8) | L;
  }
}

// Kernel launches of one gradient evaluation (forward-mode launches, reverse
// classes, finalize kernels).
int grad_launch_count(const sr::GradSet &g) {
  int n = 0;
  for (const sr::TanSet &t : g.tsets) n += (t.plan.items() > 0 ? 1 : 0) + 1;
  for (const sr::AdjClass &cl : g.classes) n += cl.plan.items() > 0 ? 1 : 0;
  return n + (g.n_rev > 0 ? 1 : 0);
}

// Compile, lay out constants, split expressions into tape-length classes and
// upload everything the adjoint launches need.
sr_status prepare_grad(sr_context *ctx, const sr_population *pop, bool recompute,
                       bool reverse_only) {
  sr::GradSet &g = ctx->grad;
  g.recompute = recompute;
  ProgramSet &ps = ctx->main;
  const int E = pop->num_exprs;
  SR_TRY(compile_set(ctx, E, pop->tokens, pop->values, pop->offsets, nullptr, ps));
  SR_TRY(upload_code(ctx, ps));
  // Constants: CSR offsets and the bytecode word that holds each one.
  SR_TRY_CUDA(ctx, g.h_const_off.ensure(static_cast<size_t>(E) + 1));
  SR_TRY_CUDA(ctx, g.h_const_cnt.ensure(static_cast<size_t>(std::max(E, 1))));
  int64_t C = 0;
  int gmax = 0;
  for (int x = 0; x < E; ++x) {
    const int nc = ps.n_const[static_cast<size_t>(x)];
    if (nc > kMaxAdjConsts)
      return ctx->fail(SR_ERR_UNSUPPORTED, "expression " + std::to_string(x) + " has " +
                                               std::to_string(nc) + " constants (gradient limit " +
                                               std::to_string(kMaxAdjConsts) + ")");
    g.h_const_off.p[x] = C;
    g.h_const_cnt.p[x] = nc;
    C += nc;
    gmax = std::max(gmax, nc);
  }
  g.h_const_off.p[E] = C;
  g.C = C;
  SR_TRY_CUDA(ctx, g.h_const_loc.ensure(static_cast<size_t>(std::max<int64_t>(C, 1))));
  SR_TRY_CUDA(ctx, g.h_consts.ensure(static_cast<size_t>(std::max<int64_t>(C, 1))));
  for (int x = 0; x < E; ++x) {
    const int64_t i0 = ps.h_off.p[x];
    const int64_t base = g.h_const_off.p[x];
    for (int i = 0; i < ps.h_len.p[x]; ++i) {
      const Instr &in = ps.h_code.p[i0 + i];
      const uint32_t ca = in.c & 0x3FFu, cb = (in.c >> 10) & 0x3FFu;
      if (sr::instr_load(in.w) && sr::instr_leaf_kind(in.w) == sr::kLeafC && ca != sr::kNoConst) {
        g.h_const_loc.p[base + ca] = ((i0 + i) << 1);
        std::memcpy(&g.h_consts.p[base + ca], &in.a, sizeof(float));
      }
      if (sr::instr_b_kind(in.w) == sr::kBC && cb != sr::kNoConst) {
        g.h_const_loc.p[base + cb] = ((i0 + i) << 1) | 1;
        std::memcpy(&g.h_consts.p[base + cb], &in.b, sizeof(float));
      }
    }
  }
  // Forward mode for the expressions with at most kMaxTangentConsts
  // constants, reverse mode for the others (for all with reverse_only).
  std::vector<std::vector<int32_t>> tan_members(kNumTanWidths);
  std::vector<int32_t> rev_members;
  for (int x = 0; x < E; ++x) {
    const int nc = ps.n_const[static_cast<size_t>(x)];
    int k = 0;
    while (k < kNumTanWidths && nc > kTanWidths[k]) ++k;
    if (reverse_only) k = kNumTanWidths;
    if (k < kNumTanWidths)
      tan_members[static_cast<size_t>(k)].push_back(x);
    else
      rev_members.push_back(x);
  }
  g.n_rev = static_cast<int>(rev_members.size());
  SR_TRY_CUDA(ctx, g.h_tmask.ensure(static_cast<size_t>(ps.n_instr) + 1));
  std::memset(g.h_tmask.p, 0, (static_cast<size_t>(ps.n_instr) + 1) * sizeof(uint32_t));
  for (const auto &mem : tan_members)
    for (int32_t x : mem)
      tangent_masks(ps.h_code.p + ps.h_off.p[x], ps.h_len.p[x], g.h_tmask.p + ps.h_off.p[x]);

  // Backward range and Jacobian-tape length of each reverse-mode program:
  // the sweep runs from the last instruction down to the lowest one holding
  // a constant (lo); the tape holds d out / d T of [lo, len) and d out / d b
  // of the instructions in that range whose operand b is a constant or a
  // spilled subtree.
  SR_TRY_CUDA(ctx, g.h_bwd_lo.ensure(static_cast<size_t>(std::max(E, 1))));
  std::vector<int32_t> tape_need(static_cast<size_t>(E));
  for (int x = 0; x < E; ++x) {
    const Instr *code = ps.h_code.p + ps.h_off.p[x];
    const int len = ps.h_len.p[x];
    int lo = len;
    for (int i = 0; i < len; ++i) {
      const Instr &in = code[i];
      const bool leaf_c = sr::instr_load(in.w) && sr::instr_leaf_kind(in.w) == sr::kLeafC &&
                          (in.c & 0x3FFu) != sr::kNoConst;
      const bool b_c = sr::instr_b_kind(in.w) == sr::kBC && ((in.c >> 10) & 0x3FFu) != sr::kNoConst;
      if (leaf_c || b_c) {
        lo = i;
        break;
      }
    }
    int nb = 0;
    for (int i = lo; i < len; ++i) {
      const uint32_t bk = sr::instr_b_kind(code[i].w);
      nb += (bk == sr::kBC || bk == sr::kBS) ? 1 : 0;
    }
    g.h_bwd_lo.p[x] = lo;
    if (recompute) {
      // Segment tape, adjoint spill slots, checkpoints.
      const int seg = sr::adj_segment();
      const int nseg = (len + seg - 1) / seg;
      tape_need[static_cast<size_t>(x)] =
          2 * std::min(seg, len) + ps.smax + std::max(nseg - 1, 0) * (1 + ps.smax);
    } else {
      tape_need[static_cast<size_t>(x)] = (len - lo) + nb;
    }
  }
  // Tape-length classes, each a separate launch with its own tape size.
  static const int kTapeClasses[] = {8, 16, 32, 64, 128, 256, 512, 2048};
  constexpr int kNumClasses = 8;
  std::vector<std::vector<int32_t>> members(kNumClasses);
  for (int32_t x : rev_members) {
    const int need = tape_need[static_cast<size_t>(x)];
    int k = 0;
    while (k < kNumClasses - 1 && need > kTapeClasses[k]) ++k;
    members[static_cast<size_t>(k)].push_back(x);
  }
  const int dpt = sr::adj_dpt();
  const int64_t tile = 32 * dpt;
  int dev_max_smem = 0;
  cudaDeviceGetAttribute(&dev_max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  // One span for every class (the MSE partials are laid out per span): the
  // largest of 1024 / 512 / 256 / 128 datapoints whose double-buffered X
  // stage fits in 48 KB.
  int span = 1024;
  while (span > tile && 2 * static_cast<int64_t>(ctx->V + 1) * span * 4 > 48 * 1024) span /= 2;
  g.span = static_cast<int>(std::min<int64_t>(span, std::max<int64_t>(tile, round_up(ctx->N, tile))));
  g.n_spans = (ctx->N == 0) ? 0 : static_cast<int>((ctx->N + g.span - 1) / g.span);
  g.classes.clear();
  std::vector<int32_t> table;
  int64_t spill_floats = 0, gtape_floats = 0;
  const int s_smem = std::min(ps.smax, sr::smem_spill_slots(dpt));
  for (int k = 0; k < kNumClasses; ++k) {
    auto &mem = members[static_cast<size_t>(k)];
    if (mem.empty()) continue;
    sr::AdjClass cl;
    int tape_len = 1, cg = 0;
    int maxlen = 1;
    for (int32_t x : mem) {
      tape_len = std::max(tape_len, tape_need[static_cast<size_t>(x)]);
      cg = std::max(cg, ps.n_const[static_cast<size_t>(x)]);
      maxlen = std::max(maxlen, static_cast<int>(ps.h_len.p[x]));
    }
    cl.seg_cap = std::min(sr::adj_segment(), maxlen);
    cl.tape_len = tape_len;
    cl.gmax = std::max(cg, 1);
    // Most resident evaluating warps per SM.  A shared-memory tape costs
    // occupancy (every warp holds its whole tape), a global one costs L2
    // traffic (each tape entry is written and read back once per tile, by the
    // same warp, so it stays in L2 while the resident tapes fit there): the
    // global tape is taken only when it gives strictly more resident warps
    // and the resident tapes stay within kL2TapeBytes.
    constexpr int64_t kL2TapeBytes = 64ll << 20;
    int best_w = 0, best_res = 0;
    size_t best_smem = 0;
    for (int pass = 0; pass < 2; ++pass) {
      const bool gt = (pass == 1);
      for (int W = sr::kMaxWarps; W >= 1; --W) {
        const size_t smem =
            sr::adj_smem_bytes(W, ctx->V, s_smem, g.span, cl.tape_len, cl.gmax, gt);
        if (smem > static_cast<size_t>(dev_max_smem)) continue;
        int bps = 0;
        SR_TRY_CUDA(ctx, sr::adj_configure(smem, W, gt, recompute, &bps));
        if (bps <= 0) continue;
        const int64_t resident_tape =
            static_cast<int64_t>(W) * bps * ctx->num_sms * cl.tape_len * tile * 4;
        if (gt && best_w != 0 && resident_tape > kL2TapeBytes) continue;
        if (W * bps > best_res) {
          best_res = W * bps;
          best_w = W;
          best_smem = smem;
          cl.global_tape = gt;
        }
      }
    }
    if (best_w == 0)
      return ctx->fail(SR_ERR_UNSUPPORTED, "no adjoint launch shape fits " +
                                               std::to_string(cl.tape_len) + " tape entries");
    sr::Plan &p = cl.plan;
    p.dpt = dpt;
    p.W = best_w;
    p.smax = ps.smax;
    p.s_smem = s_smem;
    p.G = best_w * 4;
    p.n_groups = static_cast<int>((mem.size() + p.G - 1) / p.G);
    p.span = g.span;
    p.n_spans = g.n_spans;
    p.smem = best_smem;
    p.blocks = static_cast<int>(std::min<int64_t>(
        static_cast<int64_t>(best_res / best_w) * ctx->num_sms, std::max<int64_t>(p.items(), 1)));
    spill_floats = std::max<int64_t>(spill_floats, static_cast<int64_t>(p.blocks) * p.W *
                                                       (p.smax - p.s_smem) * tile);
    if (cl.global_tape)
      gtape_floats = std::max<int64_t>(gtape_floats, static_cast<int64_t>(p.blocks) * p.W *
                                                         cl.tape_len * tile);
    std::stable_sort(mem.begin(), mem.end(), [&](int32_t a, int32_t b) {
      return ps.cost[static_cast<size_t>(a)] > ps.cost[static_cast<size_t>(b)];
    });
    cl.group_off = static_cast<int64_t>(table.size());
    for (int64_t q = 0; q < static_cast<int64_t>(p.n_groups) * p.G; ++q)
      table.push_back(q < static_cast<int64_t>(mem.size()) ? mem[static_cast<size_t>(q)] : -1);
    g.classes.push_back(cl);
  }
  // Forward-mode launches: the interpreter's shape (span groups folded by
  // each block's producer).
  g.tsets.clear();
  std::vector<int32_t> expr_list;
  int64_t tan_part = 0, tan_gout = 0;
  for (int k = 0; k < kNumTanWidths; ++k) {
    auto &mem = tan_members[static_cast<size_t>(k)];
    if (mem.empty()) continue;
    sr::TanSet ts;
    ts.K = 1;
    for (int32_t x : mem) ts.K = std::max(ts.K, ps.n_const[static_cast<size_t>(x)]);
    sr::Plan &p = ts.plan;
    p.dpt = sr::tan_dpt();
    const int64_t ttile = 32 * p.dpt;
    p.W = sr::tan_warps(ts.K);
    p.smax = ps.smax;
    // Wider sets keep one spill slot per warp in shared memory (the others in
    // per-warp global scratch): the tangent rows need the room.
    p.s_smem = std::min(ps.smax, ts.K > 4 ? 1 : sr::smem_spill_slots(p.dpt));
    int64_t tspan = 1024;
    while (tspan > ttile && 2 * static_cast<int64_t>(ctx->V + 1) * tspan * 4 > 48 * 1024)
      tspan /= 2;
    tspan = std::min<int64_t>(tspan, std::max<int64_t>(ttile, round_up(ctx->N, ttile)));
    // One block per SM: shorter spans (down to 512 datapoints) while the
    // block's shared memory does not fit, then fewer evaluating warps.
    const size_t budget = static_cast<size_t>(dev_max_smem);
    while (tspan / 2 >= std::max<int64_t>(ttile, 512) && (tspan / 2) % ttile == 0 &&
           sr::tan_smem_bytes(ts.K, p.W, ctx->V, p.s_smem, static_cast<int>(tspan), p.W * 4) >
               budget)
      tspan /= 2;
    while (p.W > 4 && sr::tan_smem_bytes(ts.K, p.W, ctx->V, p.s_smem, static_cast<int>(tspan),
                                         p.W * 4) > budget)
      --p.W;
    p.G = p.W * 4;
    p.n_groups = static_cast<int>((mem.size() + p.G - 1) / p.G);
    p.span = static_cast<int>(tspan);
    p.n_spans = (ctx->N == 0) ? 0 : static_cast<int>((ctx->N + tspan - 1) / tspan);
    p.smem = sr::tan_smem_bytes(ts.K, p.W, ctx->V, p.s_smem, p.span, p.G);
    if (p.smem > static_cast<size_t>(dev_max_smem))
      return ctx->fail(SR_ERR_UNSUPPORTED, "forward-mode launch needs " +
                                               std::to_string(p.smem) + " bytes of shared memory");
    p.k_spans = 1;
    if (p.n_spans > 0) {
      const int64_t per_sm = static_cast<int64_t>(p.n_spans) * p.n_groups /
                             (32 * static_cast<int64_t>(std::max(ctx->num_sms, 1)));
      p.k_spans = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(32, per_sm)));
    }
    int bps = 0;
    SR_TRY_CUDA(ctx, sr::tan_configure(ts.K, p.smem, p.W, &bps));
    if (bps <= 0) return ctx->fail(SR_ERR_UNSUPPORTED, "forward-mode launch does not fit on an SM");
    p.blocks = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(bps) * ctx->num_sms,
                                                  std::max<int64_t>(p.items(), 1)));
    spill_floats = std::max<int64_t>(spill_floats, static_cast<int64_t>(p.blocks) * p.W *
                                                       (p.smax - p.s_smem) * ttile);
    std::stable_sort(mem.begin(), mem.end(), [&](int32_t a, int32_t b) {
      return ps.cost[static_cast<size_t>(a)] > ps.cost[static_cast<size_t>(b)];
    });
    ts.group_off = static_cast<int64_t>(table.size());
    for (int64_t q = 0; q < static_cast<int64_t>(p.n_groups) * p.G; ++q)
      table.push_back(q < static_cast<int64_t>(mem.size()) ? mem[static_cast<size_t>(q)] : -1);
    ts.n_exprs = static_cast<int>(mem.size());
    ts.expr_off = static_cast<int64_t>(expr_list.size());
    expr_list.insert(expr_list.end(), mem.begin(), mem.end());
    ts.part_off = tan_part;
    tan_part += 2 * static_cast<int64_t>(p.n_span_groups()) * E;
    ts.gout_off = tan_gout;
    tan_gout += static_cast<int64_t>(p.n_span_groups()) * C;
    g.tsets.push_back(ts);
  }
  g.rev_expr_off = static_cast<int64_t>(expr_list.size());
  expr_list.insert(expr_list.end(), rev_members.begin(), rev_members.end());
  {
    const double need = static_cast<double>(tan_part) * sizeof(double2) +
                        static_cast<double>(tan_gout) * sizeof(double);
    if (need > 0.9 * static_cast<double>(ctx->device_memory))
      return ctx->fail(SR_ERR_UNSUPPORTED,
                       "forward-mode span sums (" + std::to_string(static_cast<int64_t>(need)) +
                           " bytes) exceed the device memory; split the population or the "
                           "datapoints");
  }
  // Uploads.
  const size_t Cs = static_cast<size_t>(std::max<int64_t>(C, 1));
  SR_TRY_CUDA(ctx, g.h_groups.ensure(std::max<size_t>(table.size(), 1)));
  if (!table.empty()) std::memcpy(g.h_groups.p, table.data(), table.size() * sizeof(int32_t));
  SR_TRY_CUDA(ctx, g.groups.ensure(std::max<size_t>(table.size(), 1)));
  SR_TRY_CUDA(ctx, g.const_off.ensure(static_cast<size_t>(E) + 1));
  SR_TRY_CUDA(ctx, g.const_cnt.ensure(static_cast<size_t>(std::max(E, 1))));
  SR_TRY_CUDA(ctx, g.bwd_lo.ensure(static_cast<size_t>(std::max(E, 1))));
  if (gtape_floats > 0) SR_TRY_CUDA(ctx, g.gtape.ensure(static_cast<size_t>(gtape_floats)));
  SR_TRY_CUDA(ctx, g.const_loc.ensure(Cs));
  SR_TRY_CUDA(ctx, g.grad_acc.ensure(Cs));
  SR_TRY_CUDA(ctx, g.grad.ensure(Cs));
  SR_TRY_CUDA(ctx, g.consts.ensure(Cs));
  SR_TRY_CUDA(ctx, g.m.ensure(Cs));
  SR_TRY_CUDA(ctx, g.v.ensure(Cs));
  if (spill_floats > 0) SR_TRY_CUDA(ctx, ctx->spill.ensure(static_cast<size_t>(spill_floats)));
  if (tan_part > 0) SR_TRY_CUDA(ctx, g.tan_partial.ensure(static_cast<size_t>(tan_part)));
  if (tan_gout > 0) SR_TRY_CUDA(ctx, g.tan_gout.ensure(static_cast<size_t>(tan_gout)));
  if (g.n_rev > 0)
    SR_TRY_CUDA(ctx, ctx->partial.ensure(static_cast<size_t>(
                         std::max<int64_t>(static_cast<int64_t>(g.n_spans) * E, 1))));
  SR_TRY_CUDA(ctx, g.tmask.ensure(static_cast<size_t>(ps.n_instr) + 1));
  SR_TRY_CUDA(ctx, g.h_exprs.ensure(std::max<size_t>(expr_list.size(), 1)));
  if (!expr_list.empty())
    std::memcpy(g.h_exprs.p, expr_list.data(), expr_list.size() * sizeof(int32_t));
  SR_TRY_CUDA(ctx, g.exprs.ensure(std::max<size_t>(expr_list.size(), 1)));
  SR_TRY_CUDA(ctx, ctx->sums.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->mse.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->h_mse.ensure(static_cast<size_t>(E)));
  cudaStream_t s = ctx->stream;
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.tmask.p, g.h_tmask.p,
                                   (static_cast<size_t>(ps.n_instr) + 1) * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, s));
  if (!expr_list.empty())
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.exprs.p, g.h_exprs.p, expr_list.size() * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, s));
  if (!table.empty())
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.groups.p, g.h_groups.p, table.size() * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.const_off.p, g.h_const_off.p, (E + 1) * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.const_cnt.p, g.h_const_cnt.p, E * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.bwd_lo.p, g.h_bwd_lo.p, E * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, s));
  if (C > 0) {
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.const_loc.p, g.h_const_loc.p, C * sizeof(int64_t),
                                     cudaMemcpyHostToDevice, s));
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(g.consts.p, g.h_consts.p, C * sizeof(float),
                                     cudaMemcpyHostToDevice, s));
  }
  ctx->prep_stats.node_evals = ps.n_tokens * ctx->N;
  ctx->prep_stats.node_evals_executed = ctx->prep_stats.node_evals;
  return SR_OK;
}

// Forward-mode launches, the reverse-mode classes, then mse / grad (and the
// FP64 sums the datapoint-sharding reads return).
sr_status launch_grad(sr_context *ctx) {
  sr::GradSet &g = ctx->grad;
  ProgramSet &ps = ctx->main;
  cudaStream_t s = ctx->stream;
  if (g.C > 0) SR_TRY_CUDA(ctx, cudaMemsetAsync(g.grad_acc.p, 0, g.C * sizeof(double), s));
  // One shared-memory limit per kernel, the largest its launches here need
  // (forward-mode sets of the same width class share a kernel, and so do the
  // reverse classes with the same tape placement).
  {
    size_t tan_max[2] = {0, 0}, adj_max[2] = {0, 0};
    for (const sr::TanSet &ts : g.tsets)
      if (ts.plan.items() > 0) {
        size_t &m = tan_max[ts.K > 4 ? 1 : 0];
        m = std::max(m, ts.plan.smem);
      }
    for (const sr::AdjClass &cl : g.classes)
      if (cl.plan.items() > 0) {
        size_t &m = adj_max[cl.global_tape ? 1 : 0];
        m = std::max(m, cl.plan.smem);
      }
    if (tan_max[0] > 0) SR_TRY_CUDA(ctx, sr::tan_set_smem_limit(4, tan_max[0]));
    if (tan_max[1] > 0) SR_TRY_CUDA(ctx, sr::tan_set_smem_limit(8, tan_max[1]));
    for (int gt = 0; gt < 2; ++gt)
      if (adj_max[gt] > 0)
        SR_TRY_CUDA(ctx, sr::adj_set_smem_limit(gt == 1, g.recompute, adj_max[gt]));
  }
  SR_TRY_CUDA(ctx, record_event(ctx, 1));
  for (const sr::TanSet &ts : g.tsets) {
    if (ts.plan.items() == 0) continue;
    sr::TanArgs a{};
    a.e = make_args(ctx, ps, ctx->d_counter);
    a.e.W = ts.plan.W;
    a.e.smax = ts.plan.smax;
    a.e.s_smem = ts.plan.s_smem;
    a.e.G = ts.plan.G;
    a.e.n_groups = ts.plan.n_groups;
    a.e.span = ts.plan.span;
    a.e.n_spans = ts.plan.n_spans;
    a.e.span_per_item = ts.plan.k_spans;
    a.e.group_expr = g.groups.p + ts.group_off;
    a.e.partial = g.tan_partial.p + ts.part_off;
    a.tmask = g.tmask.p;
    a.const_off = g.const_off.p;
    a.const_cnt = g.const_cnt.p;
    a.gout = g.tan_gout.p + ts.gout_off;
    a.C = g.C;
    a.n_valid = ts.n_exprs;
    a.K = ts.K;
    SR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
    SR_TRY_CUDA(ctx, sr::launch_tangent(a, ts.plan.blocks, ts.plan.smem, s));
  }
  for (const sr::AdjClass &cl : g.classes) {
    if (cl.plan.items() == 0) continue;
    sr::AdjArgs a{};
    a.e = make_args(ctx, ps, ctx->d_counter);
    a.e.W = cl.plan.W;
    a.e.smax = cl.plan.smax;
    a.e.s_smem = cl.plan.s_smem;
    a.e.G = cl.plan.G;
    a.e.n_groups = cl.plan.n_groups;
    a.e.span = cl.plan.span;
    a.e.n_spans = cl.plan.n_spans;
    a.e.group_expr = g.groups.p + cl.group_off;
    a.const_off = g.const_off.p;
    a.const_cnt = g.const_cnt.p;
    a.bwd_lo = g.bwd_lo.p;
    a.grad_acc = g.grad_acc.p;
    a.gtape = cl.global_tape ? g.gtape.p : nullptr;
    a.tape_len = cl.tape_len;
    a.seg_cap = cl.seg_cap;
    a.gmax = cl.gmax;
    SR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
    SR_TRY_CUDA(ctx, sr::launch_adjoint(a, g.recompute, cl.plan.blocks, cl.plan.smem, s));
  }
  SR_TRY_CUDA(ctx, record_event(ctx, 2));
  for (const sr::TanSet &ts : g.tsets)
    SR_TRY_CUDA(ctx, sr::launch_tan_finalize(
                         g.tan_partial.p + ts.part_off, g.tan_gout.p + ts.gout_off,
                         ts.plan.n_span_groups(), ps.E, g.C, g.exprs.p + ts.expr_off, ts.n_exprs,
                         g.const_off.p, g.const_cnt.p, ts.K, ctx->mse.p, g.grad.p, g.grad_acc.p,
                         ctx->sums.p, s));
  if (g.n_rev > 0)
    SR_TRY_CUDA(ctx, sr::launch_grad_finalize(ctx->partial.p, g.n_spans, ps.E,
                                              g.exprs.p + g.rev_expr_off, g.n_rev, g.const_off.p,
                                              g.const_cnt.p, g.grad_acc.p, ctx->mse.p, g.grad.p,
                                              ctx->sums.p, s));
  return SR_OK;
}

}  // namespace capi
}  // namespace sr

extern "C" {

sr_status sr_eval_grad(sr_context *ctx, const sr_population *pop, int32_t mode, float *mse_out,
                       float *grad_out, sr_stats *stats) {
  SR_TRACE("sr_eval_grad");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  const int32_t store = mode & ~SR_GRAD_REVERSE_ONLY;
  if (store != SR_GRAD_CHECKPOINT && store != SR_GRAD_RECOMPUTE)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "unknown gradient mode");
  const double t0 = now_ms();
  const uint32_t flags = SR_EVAL_GRADIENT |
                         (store == SR_GRAD_RECOMPUTE ? SR_EVAL_GRAD_RECOMPUTE : 0u) |
                         ((mode & SR_GRAD_REVERSE_ONLY) ? SR_EVAL_GRAD_REVERSE : 0u);
  SR_TRY(sr_prepare(ctx, pop, flags));
  if (pop->num_exprs == 0) {
    if (stats) *stats = sr_stats{};
    return SR_OK;
  }
  SR_TRY(sr_launch(ctx));
  SR_TRY(sr_read_mse(ctx, mse_out, nullptr));
  if (grad_out) SR_TRY(sr_read_grad(ctx, grad_out));
  if (stats) {
    fill_stats(ctx, stats);
    stats->total_eval_time_ms = now_ms() - t0;
  }
  return SR_OK;
}

sr_status sr_optimize_constants(sr_context *ctx, const sr_population *pop,
                                const sr_adam_options *adam, float *const_out, float *mse_out,
                                sr_stats *stats) {
  SR_TRACE("sr_optimize_constants");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  if (!adam || adam->steps < 0) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad Adam options");
  const int32_t store = adam->mode & ~SR_GRAD_REVERSE_ONLY;
  if (store != SR_GRAD_CHECKPOINT && store != SR_GRAD_RECOMPUTE)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "unknown gradient mode");
  SR_TRY(check_population(ctx, pop));
  if (ctx->V < 0) return ctx->fail(SR_ERR_NO_DATA, "no dataset: call sr_set_data first");
  if (pop->num_exprs == 0) return SR_OK;
  if (!mse_out) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "mse_out is NULL");
  DeviceScope scope(ctx->device);
  const double t0 = now_ms();
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  reset_prepared(ctx);
  ctx->prep_stats = sr_stats{};
  ctx->E = pop->num_exprs;
  SR_TRY(prepare_grad(ctx, pop, store == SR_GRAD_RECOMPUTE,
                      (adam->mode & SR_GRAD_REVERSE_ONLY) != 0));
  ctx->mode = sr::Mode::kGrad;
  sr::GradSet &g = ctx->grad;
  cudaStream_t s = ctx->stream;
  if (g.C > 0) {
    SR_TRY_CUDA(ctx, cudaMemsetAsync(g.m.p, 0, g.C * sizeof(float), s));
    SR_TRY_CUDA(ctx, cudaMemsetAsync(g.v.p, 0, g.C * sizeof(float), s));
  }
  SR_TRY_CUDA(ctx, cudaEventRecord(ctx->ev[0], s));
  int launches = 0;
  for (int step = 1; step <= adam->steps; ++step) {
    SR_TRY(launch_grad(ctx));
    SR_TRY_CUDA(ctx, sr::launch_adam(g.C, g.grad.p, g.m.p, g.v.p, g.consts.p, g.const_loc.p,
                                     ctx->main.code.p, step, adam->lr, adam->beta1, adam->beta2,
                                     adam->eps, s));
    launches += grad_launch_count(g) + 1;
  }
  SR_TRY(launch_grad(ctx));  // MSE at the final constants
  launches += grad_launch_count(g);
  SR_TRY_CUDA(ctx, cudaEventRecord(ctx->ev[3], s));
  ctx->timing_valid = true;
  const int E = pop->num_exprs;
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_mse.p, ctx->mse.p, E * sizeof(float),
                                   cudaMemcpyDeviceToHost, s));
  if (g.C > 0 && const_out)
    SR_TRY_CUDA(ctx, cudaMemcpyAsync(const_out, g.consts.p, g.C * sizeof(float),
                                     cudaMemcpyDeviceToHost, s));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, s));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(s));
  SR_TRY(check_device_error(ctx));
  std::memcpy(mse_out, ctx->h_mse.p, E * sizeof(float));
  ctx->prep_stats.kernel_launches = launches;
  if (stats) {
    fill_stats(ctx, stats);
    stats->total_eval_time_ms = now_ms() - t0;
  }
  return SR_OK;
}

}  // extern "C"
