// sr_capi_tools.cpp — the rest of the C ABI: the FP64 device reference of the
// accuracy report, the generation loop on the device (sr_evolve_*,
// sr_prepare_device_population), stream access, the device microbenchmarks,
// subtree detection (host and device) and the host-only helpers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sr_capi_internal.hpp"
#include "sr_context.hpp"
#include "sr_detect_gpu.hpp"
#include "sr_evolve.hpp"
#include "sr_kernels.hpp"
#include "sr_trace.hpp"

using sr::Instr;
using sr::ProgramSet;
using namespace sr::capi;

extern "C" {

sr_status sr_eval_mse_fp64(sr_context *ctx, const sr_population *pop, double *mse64_out) {
  SR_TRACE("sr_eval_mse_fp64");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  SR_TRY(check_population(ctx, pop));
  if (ctx->V < 0) return ctx->fail(SR_ERR_NO_DATA, "no dataset: call sr_set_data first");
  const int E = pop->num_exprs;
  if (E == 0) return SR_OK;
  if (!mse64_out) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "mse64_out is NULL");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  reset_prepared(ctx);
  ctx->prep_stats = sr_stats{};
  for (int x = 0; x < E; ++x) {  // the FP64 kernel's stack is shallower than the plain one's
    int depth = 0, maxd = 0;
    for (int64_t i = pop->offsets[x + 1] - 1; i >= pop->offsets[x]; --i) {
      const int t = pop->tokens[i];
      if (t <= 0) ++depth;
      else if (sr::is_binary_token(t)) --depth;
      maxd = std::max(maxd, depth);
    }
    if (maxd > sr::kFp64Stack)
      return ctx->fail(SR_ERR_UNSUPPORTED, "expression " + std::to_string(x) +
                                               " is deeper than the FP64 reference stack (" +
                                               std::to_string(sr::kFp64Stack) + ")");
  }
  SR_TRY(prepare_plain(ctx, pop));  // raw tokens on the device, as the plain kernel reads them
  SR_TRY_CUDA(ctx, ctx->mse64.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->h_mse64.ensure(static_cast<size_t>(E)));
  sr::PlainSet &ps = ctx->plain;
  SR_TRY_CUDA(ctx, sr::launch_fp64(ps.tok.p, ps.val.p, ps.off.p, ps.len.p, ctx->X.p, ctx->ldx,
                                   ctx->V, ctx->N, E, ctx->partial.p, ps.n_dpblocks,
                                   ctx->mse64.p, ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_mse64.p, ctx->mse64.p, E * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(mse64_out, ctx->h_mse64.p, E * sizeof(double));
  return SR_OK;
}

// ---- the generation loop on the device ------------------------------------------

sr_status sr_evolve_options_init(sr_evolve_options *o, int32_t num_vars) {
  if (!o) return SR_ERR_INVALID_ARGUMENT;
  *o = sr_evolve_options{};
  // Reference EvolutionParams defaults (src/utils/utils.h:178-187) and loop
  // constants (src/cleaned/cl_sr_system.cpp:293-309).
  o->num_vars = num_vars;
  o->max_tokens = 64;
  o->max_depth = 5;
  o->tournament = 3;
  o->const_min = -5.0f;
  o->const_max = 5.0f;
  o->prob_leaf = 0.1f;
  o->prob_const_leaf = 0.5f;
  o->prob_unary = 0.35f;
  o->elite_frac = 0.05f;
  o->mutation_prob = 0.2f;
  o->n_unary = 18;  // SIN .. LOOSE_SQRT (utils.cpp:939-943)
  for (int k = 0; k < 18; ++k) o->unary_ops[k] = 10 + k;
  o->n_binary = 9;  // ADD .. LOOSE_POW (utils.cpp:945-948)
  for (int k = 0; k < 9; ++k) o->binary_ops[k] = 1 + k;
  o->seed = 0x5EED5EEDull;
  return SR_OK;
}

}  // extern "C"

namespace {

sr_status evolve_params(sr_context *ctx, const sr_evolve_options *o, int E, int stride,
                        sr::EvolveParams *p) {
  if (!o) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "evolve options are NULL");
  if (E < 0) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "negative population size");
  if (o->num_vars < 0 || o->num_vars > SR_MAX_VARS)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "num_vars out of range");
  if (o->max_tokens < 1 || o->max_depth < 0 || o->max_depth > 62 || o->tournament < 1)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad max_tokens / max_depth / tournament");
  if (stride < o->max_tokens || stride > SR_EVOLVE_MAX_STRIDE)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT,
                     "stride must lie in [max_tokens, " + std::to_string(SR_EVOLVE_MAX_STRIDE) +
                         "]");
  if (o->n_unary < 1 || o->n_unary > 32 || o->n_binary < 1 || o->n_binary > 16)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "operator tables must be non-empty");
  for (int k = 0; k < o->n_unary; ++k)
    if (!sr::is_unary_token(o->unary_ops[k]))
      return ctx->fail(SR_ERR_BAD_TOKEN, "unary_ops[" + std::to_string(k) + "] is not unary");
  for (int k = 0; k < o->n_binary; ++k)
    if (!sr::is_binary_token(o->binary_ops[k]))
      return ctx->fail(SR_ERR_BAD_TOKEN, "binary_ops[" + std::to_string(k) + "] is not binary");
  const float probs[] = {o->prob_leaf, o->prob_const_leaf, o->prob_unary, o->elite_frac,
                         o->mutation_prob};
  for (float q : probs)
    if (!(q >= 0.0f && q <= 1.0f)) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "probability outside [0, 1]");
  if (!(o->const_min <= o->const_max)) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "const_min > const_max");
  sr::EvolveParams q{};
  q.num_vars = o->num_vars;
  q.max_tokens = o->max_tokens;
  q.max_depth = o->max_depth;
  q.tournament = o->tournament;
  q.const_min = o->const_min;
  q.const_max = o->const_max;
  q.prob_leaf = o->prob_leaf;
  q.prob_const_leaf = o->prob_const_leaf;
  q.prob_unary = o->prob_unary;
  q.mutation_prob = o->mutation_prob;
  q.n_unary = o->n_unary;
  q.n_binary = o->n_binary;
  std::memcpy(q.unary_ops, o->unary_ops, sizeof q.unary_ops);
  std::memcpy(q.binary_ops, o->binary_ops, sizeof q.binary_ops);
  q.seed = o->seed;
  *p = q;
  return SR_OK;
}

}  // namespace

extern "C" {

sr_status sr_evolve_init(sr_context *ctx, const sr_evolve_options *opts, int32_t num_exprs,
                         int32_t stride, int32_t *tokens, float *values, int32_t *lengths) {
  SR_TRACE("sr_evolve_init");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  sr::EvolveParams p;
  SR_TRY(evolve_params(ctx, opts, num_exprs, stride, &p));
  if (num_exprs == 0) return SR_OK;
  if (!tokens || !values || !lengths) return ctx->fail(SR_ERR_INVALID_ARGUMENT, "NULL buffer");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, sr::launch_evolve_init(p, num_exprs, stride, tokens, values, lengths,
                                          ctx->stream));
  return SR_OK;
}

sr_status sr_evolve_step(sr_context *ctx, const sr_evolve_options *opts, int32_t generation,
                         int32_t num_exprs, int32_t stride, const float *fitness,
                         const int32_t *tokens, const float *values, const int32_t *lengths,
                         int32_t *tokens_out, float *values_out, int32_t *lengths_out) {
  SR_TRACE("sr_evolve_step");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  sr::EvolveParams p;
  SR_TRY(evolve_params(ctx, opts, num_exprs, stride, &p));
  const int E = num_exprs;
  if (E == 0) return SR_OK;
  if (!fitness || !tokens || !values || !lengths || !tokens_out || !values_out || !lengths_out)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "NULL buffer");
  const size_t slots = static_cast<size_t>(E) * static_cast<size_t>(stride);
  auto overlaps = [&](const void *a, const void *b, size_t bytes) {
    const char *x = static_cast<const char *>(a), *y = static_cast<const char *>(b);
    return x < y + bytes && y < x + bytes;
  };
  if (overlaps(tokens, tokens_out, slots * sizeof(int32_t)) ||
      overlaps(values, values_out, slots * sizeof(float)) ||
      overlaps(lengths, lengths_out, static_cast<size_t>(E) * sizeof(int32_t)))
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "output buffers overlap the inputs");
  DeviceScope scope(ctx->device);
  const size_t temp = sr::rank_temp_bytes(E);
  const bool grow = ctx->evo_temp.cap < std::max<size_t>(temp, 1) ||
                    ctx->evo_keys.cap < 2 * static_cast<size_t>(E) ||
                    ctx->evo_order.cap < static_cast<size_t>(E);
  if (grow) SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  SR_TRY_CUDA(ctx, ctx->evo_temp.ensure(std::max<size_t>(temp, 1)));
  SR_TRY_CUDA(ctx, ctx->evo_keys.ensure(2 * static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->evo_idx.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->evo_order.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->evo_fit.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, sr::launch_rank(fitness, E, ctx->evo_temp.p, ctx->evo_temp.cap,
                                   ctx->evo_keys.p, ctx->evo_idx.p, ctx->evo_order.p,
                                   ctx->evo_fit.p, ctx->stream));
  int elites = static_cast<int>(static_cast<double>(E) * static_cast<double>(opts->elite_frac));
  elites = std::min(std::max(elites, 1), E);
  SR_TRY_CUDA(ctx, sr::launch_evolve_step(p, generation, E, stride, elites, ctx->evo_order.p,
                                          ctx->evo_fit.p, tokens, values, lengths, tokens_out,
                                          values_out, lengths_out, ctx->stream));
  return SR_OK;
}

sr_status sr_prepare_device_population(sr_context *ctx, const int32_t *tokens,
                                       const float *values, const int32_t *lengths,
                                       int32_t num_exprs, int32_t stride) {
  SR_TRACE("sr_prepare_device_population");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  if (num_exprs < 0 || stride < 1 || stride > SR_EVOLVE_MAX_STRIDE)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad population size or stride");
  if (num_exprs > 0 && (!tokens || !values || !lengths))
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "NULL buffer");
  if (ctx->V < 0) return ctx->fail(SR_ERR_NO_DATA, "no dataset: call sr_set_data first");
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  reset_prepared(ctx);
  ctx->prep_stats = sr_stats{};
  const int E = num_exprs;
  ctx->E = E;
  if (E == 0) return SR_OK;
  const double t0 = now_ms();
  ProgramSet &ps = ctx->main;
  ps.E = E;
  const size_t n_code = static_cast<size_t>(E) * (static_cast<size_t>(stride) + 1) + 1;
  SR_TRY_CUDA(ctx, ps.code.ensure(n_code));
  SR_TRY_CUDA(ctx, ps.off.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ps.len.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->evo_summary.ensure(8));
  SR_TRY_CUDA(ctx, ctx->h_evo_summary.ensure(8));
  SR_TRY_CUDA(ctx, ctx->mse.ensure(static_cast<size_t>(E)));
  SR_TRY_CUDA(ctx, ctx->h_mse.ensure(static_cast<size_t>(E)));
  // The interpreter prefetches one instruction past a program: keep the
  // padding word defined.
  SR_TRY_CUDA(ctx, cudaMemsetAsync(ps.code.p + (n_code - 1), 0, sizeof(Instr), ctx->stream));
  SR_TRY_CUDA(ctx, sr::launch_compile_device(tokens, values, lengths, E, stride, ctx->V,
                                             ps.code.p, ps.off.p, ps.len.p, ctx->evo_summary.p,
                                             ctx->stream));
  SR_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_evo_summary.p, ctx->evo_summary.p, 8 * sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int32_t *sm = ctx->h_evo_summary.p;
  if (sm[1] != 0)
    return ctx->fail(SR_ERR_MALFORMED_EXPRESSION,
                     "the device population holds an invalid expression (or one longer than "
                     "the stride)");
  int64_t n_tok = 0, n_ins = 0;
  std::memcpy(&n_tok, sm + 2, sizeof n_tok);
  std::memcpy(&n_ins, sm + 4, sizeof n_ins);
  ps.smax = sm[0];
  ps.n_tokens = n_tok;
  ps.n_instr = n_ins;
  ps.n_instr_protected = sm[6];
  ps.cache_refs = false;  // compiled without cache hints
  ps.cost.assign(static_cast<size_t>(E), 0.0f);  // groups in population order
  ps.n_const.assign(static_cast<size_t>(E), 0);
  ps.sfu_per_dp = 0.0;
  ps.fp32_per_dp = 0.0;
  ctx->prep_stats.host_compile_time_ms = now_ms() - t0;
  // No timing here: a generation loop would re-tune whenever its populations
  // move to another shape class; the tuned shape of a class is used when the
  // context has one, else the profile's default.
  SR_TRY(prepare_main_shape(ctx, false));
  ctx->prep_stats.node_evals = n_tok * ctx->N;
  ctx->prep_stats.node_evals_executed = ctx->prep_stats.node_evals;
  ctx->mode = sr::Mode::kBatched;
  return SR_OK;
}

sr_status sr_get_stream(sr_context *ctx, void **stream) {
  if (!ctx || !stream) return SR_ERR_INVALID_ARGUMENT;
  *stream = ctx->stream;
  return SR_OK;
}

sr_status sr_synchronize(sr_context *ctx) {
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  DeviceScope scope(ctx->device);
  SR_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SR_OK;
}

sr_status sr_measure_pipes(sr_context *ctx, double *fp32_ops_per_s, double *sfu_ops_per_s,
                           int32_t *num_sms) {
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  DeviceScope scope(ctx->device);
  float *dummy = nullptr;
  SR_TRY_CUDA(ctx, cudaMalloc(&dummy, 1024 * sizeof(float)));
  const int blocks = ctx->num_sms * 8, threads = 256, iters = 8192;
  double rates[2] = {0, 0};
  for (int m = 0; m < 2; ++m) {
    const bool mufu = (m == 1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(ctx->ev[4], ctx->stream);
      const cudaError_t e = sr::launch_pipe_bench(mufu, dummy, blocks, threads, iters, ctx->stream);
      cudaEventRecord(ctx->ev[5], ctx->stream);
      if (e != cudaSuccess || cudaEventSynchronize(ctx->ev[5]) != cudaSuccess) {
        cudaFree(dummy);
        return cuda_fail(ctx, e != cudaSuccess ? e : cudaGetLastError(), "pipe benchmark");
      }
      const float ms = elapsed_ms(ctx->ev[4], ctx->ev[5]);
      if (rep > 0) best = std::min(best, ms);
    }
    rates[m] = static_cast<double>(blocks) * threads * iters * 8.0 / (best * 1e-3);
  }
  cudaFree(dummy);
  if (fp32_ops_per_s) *fp32_ops_per_s = rates[0];
  if (sfu_ops_per_s) *sfu_ops_per_s = rates[1];
  if (num_sms) *num_sms = ctx->num_sms;
  return SR_OK;
}

sr_status sr_measure_operator_rates(sr_context *ctx, const int32_t *ops, int32_t n_ops,
                                   double *evals_per_s) {
  SR_TRACE("sr_measure_operator_rates");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  if (n_ops < 0 || (n_ops > 0 && (!ops || !evals_per_s)))
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad operator list");
  for (int32_t i = 0; i < n_ops; ++i)
    if (!(ops[i] >= 0 && ops[i] <= 27) && ops[i] != static_cast<int32_t>(sr::kOpExpClamp))
      return ctx->fail(SR_ERR_BAD_TOKEN, "operator " + std::to_string(ops[i]) + " has no rate kernel");
  DeviceScope scope(ctx->device);
  float *dummy = nullptr;
  SR_TRY_CUDA(ctx, cudaMalloc(&dummy, 1024 * sizeof(float)));
  const int blocks = ctx->num_sms * 8, threads = 256, iters = 256;
  for (int32_t i = 0; i < n_ops; ++i) {
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(ctx->ev[4], ctx->stream);
      const cudaError_t e = sr::launch_op_rate(ops[i], dummy, blocks, threads, iters, ctx->stream);
      cudaEventRecord(ctx->ev[5], ctx->stream);
      if (e != cudaSuccess || cudaEventSynchronize(ctx->ev[5]) != cudaSuccess) {
        cudaFree(dummy);
        return cuda_fail(ctx, e != cudaSuccess ? e : cudaGetLastError(), "operator rate");
      }
      const float ms = elapsed_ms(ctx->ev[4], ctx->ev[5]);
      if (rep > 0) best = std::min(best, ms);
    }
    evals_per_s[i] = static_cast<double>(blocks) * threads * iters * 8.0 / (best * 1e-3);
  }
  cudaFree(dummy);
  return SR_OK;
}

}  // extern "C"

// ---- host-only helpers ------------------------------------------------------
extern "C" {

uint64_t sr_subtree_key(const int32_t *tokens, const double *values, int32_t len) {
  if (!tokens || !values || len <= 0) return sr::kFnvOffset;
  return sr::flat_key(tokens, values, len);
}

sr_status sr_subtree_hashes(const int32_t *tokens, const double *values, int32_t len,
                            int32_t *sizes, uint64_t *hashes) {
  if (!tokens || !values || !sizes || !hashes || len < 0) return SR_ERR_INVALID_ARGUMENT;
  sr::merkle_hashes(tokens, values, len, sizes, hashes);
  return SR_OK;
}

sr_status sr_detect_subtrees(const sr_population *pop, int32_t min_size, int32_t min_freq,
                             int32_t max_groups, sr_detect_result *res, int32_t *group_expr,
                             int32_t *group_pos, int32_t *group_size, int32_t *group_count,
                             uint64_t *group_key) {
  SR_TRACE("sr_detect_subtrees");
  if (!pop || !res || pop->num_exprs < 0 || min_size < 1 || min_freq < 1)
    return SR_ERR_INVALID_ARGUMENT;
  if (pop->num_exprs > 0 && (!pop->tokens || !pop->values || !pop->offsets))
    return SR_ERR_INVALID_ARGUMENT;
  sr::Detection det;
  sr::detect_common_subtrees(pop->num_exprs, pop->tokens, pop->values, pop->offsets, min_size,
                             min_freq, static_cast<int>(std::thread::hardware_concurrency()), det);
  res->num_subtrees = static_cast<int32_t>(det.groups.size());
  res->total_tokens = det.total_tokens;
  res->covered_tokens = det.covered_tokens;
  res->avg_subtree_size = det.avg_subtree_size;
  res->coverage = det.coverage;
  const int n = std::min<int>(std::max(max_groups, 0), static_cast<int>(det.groups.size()));
  for (int g = 0; g < n; ++g) {
    const auto &G = det.groups[static_cast<size_t>(g)];
    if (group_expr) group_expr[g] = G.expr;
    if (group_pos) group_pos[g] = G.pos;
    if (group_size) group_size[g] = G.size;
    if (group_count) group_count[g] = G.occurrences;
    if (group_key)
      group_key[g] = sr::flat_key(pop->tokens + pop->offsets[G.expr] + G.pos,
                                  pop->values + pop->offsets[G.expr] + G.pos, G.size);
  }
  return SR_OK;
}

sr_status sr_detect_subtrees_device(sr_context *ctx, const sr_population *pop, int32_t min_size,
                                    int32_t min_freq, int32_t max_groups, sr_detect_result *res,
                                    int32_t *group_expr, int32_t *group_pos, int32_t *group_size,
                                    int32_t *group_count, uint64_t *group_key) {
  SR_TRACE("sr_detect_subtrees_device");
  if (!ctx) return SR_ERR_INVALID_ARGUMENT;
  ctx->last_error.clear();
  if (!pop || !res || pop->num_exprs < 0 || min_size < 1 || min_freq < 1)
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "bad detection arguments");
  if (pop->num_exprs > 0 && (!pop->tokens || !pop->values || !pop->offsets))
    return ctx->fail(SR_ERR_INVALID_ARGUMENT, "NULL population arrays");
  DeviceScope scope(ctx->device);
  sr::Detection det;
  SR_TRY(detect_on_device(ctx, pop->num_exprs, pop->tokens, pop->values, pop->offsets, min_size,
                          min_freq, det));
  res->num_subtrees = static_cast<int32_t>(det.groups.size());
  res->total_tokens = det.total_tokens;
  res->covered_tokens = det.covered_tokens;
  res->avg_subtree_size = det.avg_subtree_size;
  res->coverage = det.coverage;
  const int n = std::min<int>(std::max(max_groups, 0), static_cast<int>(det.groups.size()));
  for (int g = 0; g < n; ++g) {
    const auto &G = det.groups[static_cast<size_t>(g)];
    if (group_expr) group_expr[g] = G.expr;
    if (group_pos) group_pos[g] = G.pos;
    if (group_size) group_size[g] = G.size;
    if (group_count) group_count[g] = G.occurrences;
    if (group_key)
      group_key[g] = sr::flat_key(pop->tokens + pop->offsets[G.expr] + G.pos,
                                  pop->values + pop->offsets[G.expr] + G.pos, G.size);
  }
  return SR_OK;
}

sr_status sr_mark_cached(const sr_population *pop, const uint64_t *keys, const int32_t *slots,
                         int32_t n_keys, int32_t *hints) {
  if (!pop || pop->num_exprs < 0 || n_keys < 0 || (n_keys > 0 && (!keys || !slots)))
    return SR_ERR_INVALID_ARGUMENT;
  if (pop->num_exprs == 0) return SR_OK;
  if (!pop->tokens || !pop->values || !pop->offsets || !hints) return SR_ERR_INVALID_ARGUMENT;
  sr::SubtreeCache cache;
  cache.capacity = n_keys;
  for (int32_t k = 0; k < n_keys; ++k) cache.slot_of.emplace(keys[k], slots[k]);
  cache.used = n_keys;
  sr::mark_cached_subtrees(pop->num_exprs, pop->tokens, pop->values, pop->offsets, cache,
                           static_cast<int>(std::thread::hardware_concurrency()), hints);
  return SR_OK;
}

sr_status sr_validate_population(const sr_population *pop, int32_t num_vars, int32_t *n_instr,
                                 int32_t *spill_slots, int32_t *bad_expr) {
  if (bad_expr) *bad_expr = -1;
  if (!pop || pop->num_exprs < 0 || num_vars < 0) return SR_ERR_INVALID_ARGUMENT;
  if (pop->num_exprs == 0) return SR_OK;
  if (!pop->tokens || !pop->values || !pop->offsets || pop->offsets[0] != 0)
    return SR_ERR_INVALID_ARGUMENT;
  std::vector<sr::Instr> scratch;
  for (int x = 0; x < pop->num_exprs; ++x) {
    const int64_t o = pop->offsets[x];
    const int64_t len = pop->offsets[x + 1] - o;
    sr::ExprInfo info;
    sr_status s;
    if (len <= 0) {
      s = SR_ERR_MALFORMED_EXPRESSION;
    } else if (len > SR_MAX_TOKENS) {
      s = SR_ERR_EXPRESSION_TOO_LONG;
    } else {
      scratch.clear();
      s = sr::compile_expression(pop->tokens + o, pop->values + o, static_cast<int>(len),
                                 num_vars, nullptr, scratch, info, nullptr);
    }
    if (s != SR_OK) {
      if (bad_expr) *bad_expr = x;
      return s;
    }
    if (n_instr) n_instr[x] = info.n_instr;
    if (spill_slots) spill_slots[x] = info.need;
  }
  return SR_OK;
}

}  // extern "C"

extern "C" sr_status sr_compile_population(const sr_population *pop, int32_t num_vars,
                                           uint32_t *code, int64_t code_capacity,
                                           int64_t *instr_offsets, int32_t *spill_slots) {
  if (!pop || pop->num_exprs < 0 || num_vars < 0 || !instr_offsets || code_capacity < 0)
    return SR_ERR_INVALID_ARGUMENT;
  instr_offsets[0] = 0;
  if (pop->num_exprs == 0) return SR_OK;
  if (!pop->tokens || !pop->values || !pop->offsets || pop->offsets[0] != 0)
    return SR_ERR_INVALID_ARGUMENT;
  std::vector<sr::Instr> out;
  for (int x = 0; x < pop->num_exprs; ++x) {
    const int64_t o = pop->offsets[x];
    const int64_t len = pop->offsets[x + 1] - o;
    if (len <= 0) return SR_ERR_MALFORMED_EXPRESSION;
    if (len > SR_MAX_TOKENS) return SR_ERR_EXPRESSION_TOO_LONG;
    sr::ExprInfo info;
    const sr_status s = sr::compile_expression(pop->tokens + o, pop->values + o,
                                               static_cast<int>(len), num_vars, nullptr, out,
                                               info, nullptr);
    if (s != SR_OK) return s;
    instr_offsets[x + 1] = static_cast<int64_t>(out.size());
    if (spill_slots) spill_slots[x] = info.need;
  }
  if (code) {
    if (static_cast<int64_t>(out.size()) > code_capacity) return SR_ERR_INVALID_ARGUMENT;
    std::memcpy(code, out.data(), out.size() * sizeof(sr::Instr));
  }
  return SR_OK;
}
