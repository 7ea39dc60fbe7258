/*
 * sr_eval.h — C ABI of the B200 population evaluator.
 *
 * The hot path is fitness evaluation of a whole GP population: every
 * prefix-encoded expression is evaluated on every datapoint of one shared
 * dataset and reduced to its mean squared error.  In the reference
 * (phi-jkim/symbolic_regression_gpu) this is evaluate_gpu_mse_wrapper
 * (src/cleaned/cl_gpu_eval.cu:578-592), evaluate_gpu_simple_wrapper
 * (src/cleaned/cl_gpu_simple.cu:324-336) and the CPU evaluator
 * evaluate_cpu_mse (src/cleaned/cl_cpu_eval.cpp:94-168).  Those are C++
 * functions taking InputInfo& / std::vector<float>&; the same entry points
 * with their exact C++ signatures are exported by this library too (see
 * sr_reference_abi.h).  This header is the language-neutral boundary: plain
 * pointers and sizes, status codes instead of exit(), no C++ or torch types.
 *
 * Token encoding (reference src/utils/opcodes.h:10-40): a population is a
 * set of prefix token arrays.  Token 0 = constant (value = the constant),
 * token -1 = variable (value = variable index as a number), tokens 1..9 are
 * binary operators, 10..27 unary operators.  Expressions are evaluated right
 * to left with a stack; for a binary operator the first value popped is the
 * LEFT operand (reference cl_gpu_eval.cu:98-101).  Token 32 is an extension
 * of this library (exp with its argument clamped at 80); the reference has no
 * such opcode.
 *
 * Data layout: X is column-major, X[v * num_dps + dp] for v in [0, num_vars],
 * with the target y in row num_vars (reference flatten_X_col_major_full,
 * cl_gpu_eval.cu:249-257).
 *
 * Threading: a context is used from one host thread at a time.  Every
 * sr_eval_* call is synchronous: results are valid on return.
 */
#ifndef SR_EVAL_H
#define SR_EVAL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SR_ABI_VERSION 2

/* ---- token encoding (reference src/utils/opcodes.h:10-40) ---------------- */
#define SR_TOK_CONST 0
#define SR_TOK_VAR (-1)
#define SR_OP_ADD 1
#define SR_OP_SUB 2
#define SR_OP_MUL 3
#define SR_OP_DIV 4
#define SR_OP_POW 5
#define SR_OP_MIN 6
#define SR_OP_MAX 7
#define SR_OP_LOOSE_DIV 8
#define SR_OP_LOOSE_POW 9
#define SR_OP_SIN 10
#define SR_OP_COS 11
#define SR_OP_TAN 12
#define SR_OP_SINH 13
#define SR_OP_COSH 14
#define SR_OP_TANH 15
#define SR_OP_EXP 16
#define SR_OP_LOG 17
#define SR_OP_INV 18
#define SR_OP_ASIN 19
#define SR_OP_ACOS 20
#define SR_OP_ATAN 21
#define SR_OP_LOOSE_LOG 22
#define SR_OP_LOOSE_INV 23
#define SR_OP_ABS 24
#define SR_OP_NEG 25
#define SR_OP_SQRT 26
#define SR_OP_LOOSE_SQRT 27
/* Extension (no reference counterpart): expf(fminf(x, 80.0f)). */
#define SR_OP_EXP_CLAMP 32

/* Longest expression accepted (tokens).  The reference caps generated
 * expressions at MAX_TOKEN_NUM = 64 (src/utils/utils.h:20); this library
 * accepts longer ones. */
#define SR_MAX_TOKENS 1024
/* Largest number of input variables (reference MAX_NUM_FEATURES = 32 incl. y,
 * src/cleaned/cl_gpu_common.h:9-11). */
#define SR_MAX_VARS 31

typedef enum sr_status {
  SR_OK = 0,
  SR_ERR_INVALID_ARGUMENT = 1,   /* null pointer, negative size, ...          */
  SR_ERR_BAD_TOKEN = 2,          /* token outside the encoding above          */
  SR_ERR_MALFORMED_EXPRESSION = 3, /* stack underflow or != 1 result value    */
  SR_ERR_EXPRESSION_TOO_LONG = 4,  /* more than SR_MAX_TOKENS tokens          */
  SR_ERR_NO_DATA = 5,            /* no dataset resident on the device          */
  SR_ERR_CUDA = 6,               /* a CUDA runtime call failed                 */
  SR_ERR_OUT_OF_MEMORY = 7,      /* device or pinned host allocation failed    */
  SR_ERR_DEVICE_TIMEOUT = 8,     /* a bounded device-side wait gave up         */
  SR_ERR_DEVICE_CHECK = 9,       /* a device-side bounds check fired           */
  SR_ERR_UNSUPPORTED = 10,       /* option or size this build does not handle  */
  SR_ERR_NO_DEVICE = 11,         /* no CUDA device / extension unusable        */
  SR_ERR_TOO_MANY_VARS = 12      /* num_vars > SR_MAX_VARS                     */
} sr_status;

/* Evaluation flags. */
#define SR_EVAL_SUBTREE_CACHE 0x1u /* use the cross-generation subtree cache  */
#define SR_EVAL_CLEAR_CACHE 0x2u   /* drop the cache first (reference clear_cache) */
#define SR_EVAL_PLAIN 0x4u         /* plain per-expression kernel (baseline)   */
#define SR_EVAL_GRADIENT 0x8u      /* sr_prepare: fused forward + adjoint (MSE and
                                      d MSE / d constants; read with sr_read_grad) */
#define SR_EVAL_GRAD_RECOMPUTE 0x10u /* with SR_EVAL_GRADIENT: recompute mode      */
#define SR_EVAL_GRAD_REVERSE 0x20u   /* with SR_EVAL_GRADIENT: reverse mode for every
                                        expression (see SR_GRAD_REVERSE_ONLY)     */

typedef struct sr_context sr_context;

typedef struct sr_options {
  int32_t device;           /* CUDA device ordinal; -1 = the current device   */
  int32_t cache_capacity;   /* subtree-cache slots; reference: 2048
                               (MAX_CACHED_SUBTREES, cl_gpu_common.h:13)       */
  int32_t min_subtree_size; /* detection min size; reference 3 (cl_gpu_eval.cu:373) */
  int32_t min_subtree_freq; /* detection min frequency; reference 10 (same line) */
  int32_t dpt;              /* datapoints per thread: 0 = tuned, 4, 8 or 16   */
  int32_t warps_per_block;  /* evaluating warps per block: 0 = tuned, 1..31
                               (above 16 only with dpt 8, or dpt 0, which
                               then means 8; predictions use at most 16)   */
  int32_t autotune;         /* 1 = time candidate launch shapes on first use  */
  int32_t use_graphs;       /* 1 = sr_launch captures the prepared launch
                               sequence (memsets, kernels, timing events) in
                               a CUDA graph on first use and replays it until
                               the next sr_prepare / sr_set_data            */
  int32_t host_threads;     /* host compile threads; 0 = hardware concurrency  */
  int32_t device_detect;    /* 1 = the subtree-cache path detects common
                               subtrees on the device (same result)           */
  const char *tune_cache_path; /* JSON file for tuned shapes; NULL = none      */
  void *stream;             /* cudaStream_t to run on; NULL = own stream      */
  int32_t smem_spill_slots; /* spill slots per warp kept in shared memory (the
                               deeper ones live in per-warp global scratch):
                               -1 = tuned / the default for the datapoints per
                               thread, 0..16 = fixed                          */
  int32_t reserved1;
} sr_options;

/* A population in CSR form: expression i is tokens/values[offsets[i] ..
 * offsets[i+1]).  values are doubles as in the reference InputInfo.values
 * (src/utils/utils.h:31); constants are used as (float)value and variable
 * indices as (int)value, exactly as the reference evaluators do. */
typedef struct sr_population {
  int32_t num_exprs;
  int32_t reserved0;
  const int32_t *tokens;
  const double *values;
  const int64_t *offsets; /* num_exprs + 1 entries, offsets[0] == 0 */
} sr_population;

/* Per-call statistics; the first block mirrors the reference RunStats
 * (src/utils/utils.h:103-114). */
typedef struct sr_stats {
  double total_eval_time_ms;    /* wall time of the call                       */
  double detect_time_ms;        /* host subtree detection (RunStats.drift_detect_time_ms) */
  double data_transfer_time_ms; /* host<->device copies (device-timed)        */
  double gpu_kernel_time_ms;    /* all kernels of the call (device-timed)     */
  int32_t num_subtrees;         /* common subtrees detected this call         */
  int32_t new_subtrees;         /* of which newly evaluated into the cache    */
  double avg_subtree_size;
  double coverage;              /* covered tokens / total tokens (detection)  */
  /* additions */
  double host_compile_time_ms;  /* token validation + bytecode compilation    */
  double eval_kernel_time_ms;   /* main interpreter kernel only               */
  int64_t node_evals;           /* sum(tokens) * num_dps (original expressions) */
  int64_t node_evals_executed;  /* node-evals actually computed (cache skips some) */
  int32_t kernel_launches;      /* launches of this library's kernels         */
  int32_t cache_slots_used;
  int32_t dpt;                  /* launch shape used                          */
  int32_t warps_per_block;
  int32_t blocks;
  int32_t work_items;
  /* Declared work of one launch of the main kernel (roofline model: operator
   * counts per datapoint summed over expressions, times num_dps). */
  double declared_sfu_ops;
  double declared_fp32_ops;
  /* Bytes copied host->device / device->host by the call. */
  int64_t h2d_bytes;
  int64_t d2h_bytes;
} sr_stats;

/* ---- lifecycle (reference create_gpu_context / destroy_gpu_context,
 *      cl_gpu_eval.cu:569-575; create/destroy_gpu_simple_context,
 *      cl_gpu_simple.cu:315-321) ------------------------------------------- */
sr_status sr_options_init(sr_options *opts);
sr_status sr_create(const sr_options *opts, sr_context **out);
sr_status sr_destroy(sr_context *ctx);
const char *sr_status_string(sr_status s);
/* Message of the last failed call on ctx ("" if none). */
const char *sr_last_error(const sr_context *ctx);
int32_t sr_abi_version(void);
/* Fault injection for tests (process-wide): with n > 0 the n-th following
 * device or pinned-host allocation made by the library fails as if the
 * memory were exhausted (the call returns SR_ERR_OUT_OF_MEMORY and the
 * context stays usable); n = 0 disables it.  The reference has no
 * counterpart (its CUDA_CHECK exits the process on any failure,
 * cl_gpu_common.h:15-23). */
sr_status sr_inject_allocation_failure(int64_t n);

/* ---- dataset (reference upload_X branch, cl_gpu_eval.cu:474-489) --------
 * X: host pointer, column-major [(num_vars+1) x num_dps], y in the last row.
 * The data stays on the device until replaced.  A new dataset drops the
 * prepared launch and the subtree cache; a call that fails after its
 * arguments were accepted (allocation, copy) leaves the context with no
 * dataset (SR_ERR_NO_DATA until the next successful call). */
sr_status sr_set_data(sr_context *ctx, const float *X, int32_t num_vars,
                      int64_t num_dps);
/* Same from the reference's row-pointer form all_vars[0][v][dp] (v <= num_vars). */
sr_status sr_set_data_rows(sr_context *ctx, const float *const *rows,
                           int32_t num_vars, int64_t num_dps);
/* Same from a device pointer (row stride ld >= num_dps floats). */
sr_status sr_set_data_device(sr_context *ctx, const float *X_dev, int64_t ld,
                             int32_t num_vars, int64_t num_dps);

/* ---- forward MSE (reference evaluate_gpu_mse, cl_gpu_eval.cu:332-564;
 *      evaluate_gpu_simple, cl_gpu_simple.cu:187-310) -----------------------
 * mse_out[i] = sum over valid dps of (pred - y)^2 / count, valid = pred is
 * neither NaN nor +-Inf; NaN when no datapoint is valid.  num_exprs == 0
 * returns SR_OK without touching mse_out (reference cl_gpu_eval.cu:342). */
sr_status sr_eval_mse(sr_context *ctx, const sr_population *pop,
                      uint32_t flags, float *mse_out, sr_stats *stats);

/* Two-phase form of sr_eval_mse for callers that evaluate the same compiled
 * population repeatedly: sr_prepare validates, compiles and uploads;
 * sr_launch enqueues the device work on the context stream (asynchronous);
 * sr_read_mse waits and copies the result. */
sr_status sr_prepare(sr_context *ctx, const sr_population *pop, uint32_t flags);
sr_status sr_launch(sr_context *ctx);
sr_status sr_read_mse(sr_context *ctx, float *mse_out, sr_stats *stats);
/* Device times of the most recent sr_launch, after it completed: the whole
 * launch sequence and the main interpreter kernel alone (CUDA events on the
 * context stream). */
sr_status sr_last_launch_times(sr_context *ctx, float *launch_ms, float *eval_kernel_ms);
/* Device pointer of the MSE vector written by sr_launch (num_exprs floats). */
sr_status sr_device_mse(sr_context *ctx, float **mse_dev);
/* Datapoint sharding: after sr_launch (or sr_eval_mse / sr_eval_grad), the
 * FP64 sum of the valid squared errors and the valid-datapoint count of every
 * expression (sum_out[i] / count_out[i] is the MSE before its rounding to
 * float; count 0 = no valid datapoint).  A caller that splits the datapoints
 * over several contexts (one per GPU, each holding its columns of X) adds the
 * shards' sums and counts and divides.  No reference counterpart (the
 * reference evaluates every datapoint on one GPU, cl_gpu_eval.cu:332-564). */
sr_status sr_read_sums(sr_context *ctx, double *sum_out, double *count_out);

/* Per-datapoint predictions of every expression for dps [dp_begin,
 * dp_begin+dp_count): pred_out[i * dp_count + j].  Predictions are the raw
 * FP32 stack result, NaN/Inf included (reference evaluate_single_expr,
 * cl_cpu_eval.cpp:59-90). */
sr_status sr_eval_predictions(sr_context *ctx, const sr_population *pop,
                              int64_t dp_begin, int64_t dp_count,
                              float *pred_out);

/* ---- gradients with respect to the constants (no reference counterpart) --
 * Constants are the SR_TOK_CONST tokens of each expression, in token order;
 * grad_out uses the same CSR layout as the constants themselves: for
 * expression i its constants are numbered from const_offsets[i], where
 * const_offsets is the exclusive prefix sum of the per-expression constant
 * counts (sr_count_constants).  grad_out[k] = d mse_i / d c_k. */
/* Expressions with at most 8 constants are differentiated in forward mode:
 * one launch runs each program once per tile of datapoints with a tangent per
 * constant beside every value (no tape, no second pass).  Expressions with
 * more constants are differentiated in reverse mode, forward and backward
 * fused per tile, in one launch per tape-size class, with the tape kept as
 * the mode says:
 *   SR_GRAD_CHECKPOINT keeps every instruction's local partials (the Jacobian
 *     tape) for the tile, in shared memory, or in per-warp global scratch
 *     (L2-resident) when that keeps more warps resident; the backward sweep
 *     reads them.
 *   SR_GRAD_RECOMPUTE keeps only the forward state at segment boundaries and
 *     recomputes each segment's values and partials during the backward sweep
 *     (about one more forward pass, a much smaller tape).
 * SR_GRAD_REVERSE_ONLY, or-ed into the mode, sends every expression through
 * reverse mode.  Both modes multiply the same local partials along each
 * constant's path, in opposite orders, so their gradients agree to rounding
 * (an intermediate product can overflow in one order and not the other). */
#define SR_GRAD_RECOMPUTE 0
#define SR_GRAD_CHECKPOINT 1
#define SR_GRAD_REVERSE_ONLY 2
sr_status sr_count_constants(const sr_population *pop, int64_t *const_offsets);
sr_status sr_eval_grad(sr_context *ctx, const sr_population *pop, int32_t mode,
                       float *mse_out, float *grad_out, sr_stats *stats);
/* After sr_prepare(..., SR_EVAL_GRADIENT) and sr_launch: the gradient of the
 * last launch (CSR layout above); sr_read_mse gives its MSE. */
sr_status sr_read_grad(sr_context *ctx, float *grad_out);
/* Datapoint sharding of the gradient: the FP64 sum over valid datapoints of
 * d (squared error) / d constant (CSR layout above); the gradient is this sum
 * divided by the expression's valid count (sr_read_sums). */
sr_status sr_read_grad_sums(sr_context *ctx, double *grad_sum_out);

/* On-device Adam over every expression's constants (steps iterations of
 * fused forward+adjoint then an Adam update); const_out receives the final
 * constants (CSR as above), mse_out the MSE at those constants. */
typedef struct sr_adam_options {
  int32_t steps;
  int32_t mode; /* SR_GRAD_RECOMPUTE or SR_GRAD_CHECKPOINT, | SR_GRAD_REVERSE_ONLY */
  float lr, beta1, beta2, eps;
} sr_adam_options;
sr_status sr_optimize_constants(sr_context *ctx, const sr_population *pop,
                                const sr_adam_options *adam, float *const_out,
                                float *mse_out, sr_stats *stats);

/* ---- host-side subtree keys and detection (no device needed) -------------- */
/* Flat cache key of a token/value run: h = 14695981039346656037; per token
 * h ^= (uint64)(int64)token; h *= 1099511628211; h ^= bits(double value);
 * h *= 1099511628211 (reference compute_subtree_hash_gpu,
 * src/cleaned/cl_gpu_eval.cu:259-272 = compute_hash, src/utils/detect.cpp:50-68). */
uint64_t sr_subtree_key(const int32_t *tokens, const double *values, int32_t len);
/* Per-position subtree sizes and Merkle hashes of one expression (reference
 * detect_common_subtrees reverse pass, src/utils/detect.cpp:169-191, with
 * hash_node / combine_hashes, detect.cpp:97-118). */
sr_status sr_subtree_hashes(const int32_t *tokens, const double *values, int32_t len,
                            int32_t *sizes, uint64_t *hashes);

typedef struct sr_detect_result {
  int32_t num_subtrees;     /* groups found                                 */
  int32_t reserved0;
  int64_t total_tokens;
  int64_t covered_tokens;   /* tokens under the greedy non-overlapping cover */
  double avg_subtree_size;
  double coverage;          /* covered_tokens / total_tokens                */
} sr_detect_result;

/* Common-subtree detection (reference detect_common_subtrees,
 * src/utils/detect.cpp:120-387).  Groups come out largest first; for group g
 * (g < max_groups) the optional arrays receive its representative occurrence
 * (expression, position), size, verified occurrence count and flat key. */
sr_status sr_detect_subtrees(const sr_population *pop, int32_t min_size, int32_t min_freq,
                             int32_t max_groups, sr_detect_result *res, int32_t *group_expr,
                             int32_t *group_pos, int32_t *group_size, int32_t *group_count,
                             uint64_t *group_key);

/* The same detection on the context's GPU (csrc/sr_detect_gpu.cu): Merkle
 * hashes per expression, candidates sorted and grouped by hash, groups
 * verified member by member, cover counted per expression; identical
 * groups, order and statistics.  Synchronous. */
sr_status sr_detect_subtrees_device(sr_context *ctx, const sr_population *pop, int32_t min_size,
                                    int32_t min_freq, int32_t max_groups, sr_detect_result *res,
                                    int32_t *group_expr, int32_t *group_pos, int32_t *group_size,
                                    int32_t *group_count, uint64_t *group_key);

/* Cache marking (reference mark_cached_subtrees_from_state,
 * src/cleaned/cl_gpu_eval.cu:294-329): given cached keys and their slots,
 * hints[t] for every token t of pop is the slot at the root of a cached
 * subtree, -2 on its body, -1 elsewhere (outermost subtree of >= 3 tokens wins). */
sr_status sr_mark_cached(const sr_population *pop, const uint64_t *keys, const int32_t *slots,
                         int32_t n_keys, int32_t *hints);

/* Validate a population and report per-expression bytecode size and spill
 * slots (either output may be NULL).  First error wins; sr_last_error is not
 * available here, so the failing expression index goes to *bad_expr. */
sr_status sr_validate_population(const sr_population *pop, int32_t num_vars,
                                 int32_t *n_instr, int32_t *spill_slots, int32_t *bad_expr);

/* The interpreter bytecode of a population, as sr_prepare compiles it (for
 * inspection and host-side verification of the compiler).  Each instruction
 * is 4 uint32 words {w, a, b, c} and executes
 *     [spill T -> S[slot]]  [T = leaf a]  [b = operand b]  T = op(T, b):
 *   w bits 0..5 opcode: reference token 1..9 (T = f(T, b)), 10..27 (T = f(T)),
 *     32 = exp clamped at 80, 40 + k = reversed binary k (T = f_k(b, T)),
 *     0 = none; bit 6 load leaf a into T, bits 7..8 its kind (0 = variable,
 *     1 = constant, 2 = cached subtree); bits 9..11 kind of operand b
 *     (0 = none, 1 = spill slot, 2 = variable, 3 = constant, 4 = cached
 *     subtree); bit 12 spill T into slot bits 13..17 first;
 *   a, b payloads (variable index / float bits / slot);
 *   c bits 0..9 / 10..19 constant index of leaf a / operand b (0x3FF = none).
 * code may be NULL to query sizes: instr_offsets (num_exprs+1) always
 * receives the per-expression instruction offsets. */
sr_status sr_compile_population(const sr_population *pop, int32_t num_vars, uint32_t *code,
                                int64_t code_capacity, int64_t *instr_offsets,
                                int32_t *spill_slots);

/* ---- evaluation without any device allocation (no counterpart in the
 *      reference) ------------------------------------------------------------
 * For callers that keep their population on the GPU and cannot let a library
 * call cudaMalloc: a GA loop that breeds and evaluates on the device inside a
 * fixed memory budget, or a host framework whose own pooled allocator owns
 * all device memory.  Every argument is a device pointer the caller owns:
 * tokens / values (float: the constant, or the variable index as a number) /
 * offsets (num_exprs + 1, int64) describe the population in the layout of
 * sr_population, X is column-major with row stride ld (y in row num_vars),
 * mse_out receives num_exprs floats.  The plain per-expression kernel does
 * the work; its partial sums live in one fixed array built into the
 * library (SR_NOALLOC_SCRATCH_BYTES, resident on every GPU that loads the
 * library until exit), so no call allocates.  The first call on a device
 * looks up that array's device address (one-time set-up, repeated only if
 * the device's context was reset in between; make that first call before
 * any stream capture).  The call runs on `stream` (NULL = the default
 * stream) and waits for it before returning.  Calls share the array: calls
 * whose kernels overlap on the GPU race and their results are undefined.
 * offsets: off[0] >= 0 and off[num_exprs] must be the length of the tokens
 * and values buffers (the kernel reads only tokens in [off[0],
 * off[num_exprs]) and checks every expression's offsets against those two).
 * Expressions are validated on the device before they are evaluated, also
 * when num_dps is 0: one whose offsets are inconsistent, with no token or
 * more than SR_MAX_TOKENS, an unknown token, or a stack that underflows or
 * does not end with exactly one value gets a NaN MSE and the call returns
 * SR_ERR_MALFORMED_EXPRESSION.  num_exprs > SR_NOALLOC_MAX_EXPRS returns
 * SR_ERR_UNSUPPORTED. */
#define SR_NOALLOC_SCRATCH_BYTES (4u << 20)
#define SR_NOALLOC_MAX_EXPRS ((int32_t)((SR_NOALLOC_SCRATCH_BYTES - 256u) / 16u))
sr_status sr_eval_mse_device_noalloc(const int32_t *tokens, const float *values,
                                     const int64_t *offsets, int32_t num_exprs, const float *X,
                                     int64_t ld, int32_t num_vars, int64_t num_dps,
                                     float *mse_out, void *stream);

/* ---- misc ------------------------------------------------------------------ */
/* FP64 reference MSE of every expression, evaluated on the device: the same
 * operators in double, constants as (double)(float)value, the FP32 dataset,
 * a datapoint counted when its FP64 prediction would be a finite float.
 * The accuracy report of the FP32 results: |mse - mse_fp64| / |mse_fp64|
 * per expression.  No reference counterpart (the reference reports FP32
 * results only).  Synchronous; clears the prepared launch. */
sr_status sr_eval_mse_fp64(sr_context *ctx, const sr_population *pop, double *mse64_out);

/* ---- the generation loop on the device ---------------------------------------
 * The reference runs its evolution loop on the host (src/cleaned/cl_sr_system.cpp:
 * 150-330: evaluate, sort by fitness with NaN last, keep the top 5 %, fill the rest
 * by size-3 tournaments with 20 % subtree mutation / 80 % subtree crossover,
 * utils.cpp:1163-1273), packing every generation into InputInfo for the
 * evaluator.  These calls run the same steps on the device, on a population held
 * in device memory in a slot layout: expression i has lengths[i] tokens at
 * tokens[i * stride ...] (int32) with values at values[i * stride ...] (float).
 * Every call is enqueued on the context stream.  Random numbers come from a
 * counter-based stream per (seed, generation, child): results are deterministic
 * for a seed, with the reference's distributions but not its samples. */
#define SR_EVOLVE_MAX_STRIDE 256
typedef struct sr_evolve_options {
  int32_t num_vars;       /* variables of generated leaves (EvolutionParams.num_vars) */
  int32_t max_tokens;     /* 64 (EvolutionParams.max_tokens = MAX_TOKEN_NUM)          */
  int32_t max_depth;      /* 5                                                         */
  int32_t tournament;     /* 3 (cl_sr_system.cpp:301)                                  */
  float const_min;        /* -5                                                        */
  float const_max;        /* 5                                                         */
  float prob_leaf;        /* 0.1                                                       */
  float prob_const_leaf;  /* 0.5                                                       */
  float prob_unary;       /* 0.35                                                      */
  float elite_frac;       /* 0.05: elites = max(1, (int)(num_exprs * elite_frac))     */
  float mutation_prob;    /* 0.2 (the rest is crossover)                               */
  int32_t n_unary;        /* operator tables (reference kUnaryOps / kBinaryOps,        */
  int32_t n_binary;       /*  utils.cpp:939-948: tokens 10..27 and 1..9)               */
  int32_t unary_ops[32];
  int32_t binary_ops[16];
  uint64_t seed;
} sr_evolve_options;
/* The reference's parameters for `num_vars` input variables. */
sr_status sr_evolve_options_init(sr_evolve_options *opts, int32_t num_vars);
/* Generation 0: one random expression per slot (reference
 * generate_random_expression, utils.cpp:1156-1161).  stride in
 * [max_tokens, SR_EVOLVE_MAX_STRIDE]; 2 * max_tokens + 2 leaves room for the
 * generator's budget-exhausted leaves (utils.cpp:1072-1078), below that a
 * child that does not fit keeps its parent. */
sr_status sr_evolve_init(sr_context *ctx, const sr_evolve_options *opts, int32_t num_exprs,
                         int32_t stride, int32_t *tokens, float *values, int32_t *lengths);
/* One breeding step from device fitness (for instance sr_device_mse after an
 * evaluation on the same context).  The *_out buffers must not overlap the
 * inputs. */
sr_status sr_evolve_step(sr_context *ctx, const sr_evolve_options *opts, int32_t generation,
                         int32_t num_exprs, int32_t stride, const float *fitness,
                         const int32_t *tokens, const float *values, const int32_t *lengths,
                         int32_t *tokens_out, float *values_out, int32_t *lengths_out);
/* sr_prepare for a device-resident population in the slot layout: the
 * programs are compiled on the device (the same bytecode the host compiler
 * emits; constants and variable indices read from the float values), then
 * sr_launch / sr_read_mse / sr_device_mse work as after sr_prepare.  Waits
 * for the compile (one small device-to-host read: the spill-slot count and
 * the validity flag); an invalid expression fails with
 * SR_ERR_MALFORMED_EXPRESSION. */
sr_status sr_prepare_device_population(sr_context *ctx, const int32_t *tokens,
                                       const float *values, const int32_t *lengths,
                                       int32_t num_exprs, int32_t stride);

/* ---- file loaders (host, no device needed) ------------------------------------
 * Parallel readers of the reference's text files: the file is memory-mapped,
 * cut into line-aligned chunks and parsed by `threads` host threads (0 = all
 * cores).  Numbers are parsed correctly rounded (as strtod) into doubles;
 * dataset values are narrowed to float exactly like the reference loop
 * (cl_sr_system.cpp:98-104).  Unlike the reference's stream readers they
 * expect the files' line structure: one datapoint per line, four lines per
 * expression.  Call with the output pointers NULL to get the sizes first. */
/* shared_data.txt (reference load_data_file, utils.cpp:235-300): X[v * ld + j]
 * = column v (x0 .. x_{num_vars-1}, y) of datapoint j, for the first
 * min(lines, max_dps) datapoints (max_dps < 0: all); *num_dps receives that
 * count.  SR_ERR_MALFORMED_EXPRESSION if a line does not hold num_vars + 1
 * numbers. */
sr_status sr_load_shared_data(const char *path, int32_t num_vars, int64_t max_dps, float *X,
                              int64_t ld, int64_t *num_dps, int32_t threads);
/* gen_N.txt (reference parse_input_info, utils.cpp:122-233): the population in
 * CSR form (offsets[num_exprs + 1]), each expression's num_vars / num_dps
 * (nullable) and the first expression's data file name (nullable). */
sr_status sr_load_population(const char *path, int32_t *num_exprs, int64_t *num_tokens,
                             int32_t *tokens, double *values, int64_t *offsets,
                             int32_t *num_vars, int32_t *num_dps, char *data_file,
                             int32_t data_file_cap, int32_t threads);

sr_status sr_get_stream(sr_context *ctx, void **stream);
sr_status sr_synchronize(sr_context *ctx);
/* Measured device-wide pipe peaks (FP32 FMA and MUFU rsqrt thread-operations
 * per second) from two short microbenchmarks, plus the SM count. */
sr_status sr_measure_pipes(sr_context *ctx, double *fp32_ops_per_s,
                           double *sfu_ops_per_s, int32_t *num_sms);
/* Measured throughput (evaluations per second, whole device) of each listed
 * operator's FP32 semantics alone: 8 independent evaluations per thread per
 * iteration, each added into an accumulator, first operand in [-3, 3] moving
 * by 1e-6 per iteration, second operand in [0.5, 3].  Operator 0 times the
 * harness alone (two adds per evaluation).  The accurate-operator bound of a population is the sum over
 * its operator tokens of 1 / rate (less the harness), times the datapoints.
 * Operators: 0-27 and 32.  No reference counterpart. */
sr_status sr_measure_operator_rates(sr_context *ctx, const int32_t *ops, int32_t n_ops,
                                   double *evals_per_s);
/* Accuracy of this library's own single-precision sin / cos / log (the
 * operators' implementation in every kernel) over the float arguments whose
 * bit patterns are [begin, begin + count): the largest error in ulps of the
 * float result against the double-precision function (0.5 = correctly
 * rounded), the argument where it occurs, and how many checked arguments
 * were off by more than 0.5 and more than 1 ulp.  fn: 10 sin, 11 cos,
 * 17 log; 110, 111, 117: CUDA's sinf, cosf, logf for comparison.  Runs on
 * the current device, synchronous.  No reference counterpart. */
sr_status sr_check_math(int32_t fn, uint32_t begin, uint64_t count, double *max_ulp,
                        uint32_t *argmax_bits, uint64_t *checked, uint64_t *over_half_ulp,
                        uint64_t *over_one_ulp);

#ifdef __cplusplus
}
#endif

#endif /* SR_EVAL_H */
