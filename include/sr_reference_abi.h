/*
 * sr_reference_abi.h — the reference's own C++ entry points, exported by
 * libsr_eval.so with their exact signatures so that the reference evolution
 * loop (src/cleaned/cl_sr_system.cpp) and benchmark driver
 * (src/cleaned/cl_main.cpp) link against this library unchanged.
 *
 * The two structs must be layout- and name-identical to the reference's
 * InputInfo (src/utils/utils.h:25-47) and RunStats (src/utils/utils.h:103-114):
 * they are part of the C++ linkage (mangled names) and of the memory layout
 * the caller hands over.  A translation unit must include either this header
 * or the reference utils.h, never both.
 */
#ifndef SR_REFERENCE_ABI_H
#define SR_REFERENCE_ABI_H

#ifndef __cplusplus
#error "sr_reference_abi.h declares C++ entry points; C callers use sr_eval.h"
#endif

#include <string>
#include <vector>

/* Same members, order and types as the reference InputInfo. */
typedef struct {
  int num_exprs;
  int *num_vars;
  int *num_dps;
  int *num_tokens;
  int **tokens;
  double **values;
  std::string *data_filenames;
  int max_tokens;
  int max_num_dps;
  int max_num_features;
  int **tokens_packed;
  float **values_packed_f32;
  float **X_packed_f32;
  bool has_shared_data;
} InputInfo;

/* Same members, order and defaults as the reference RunStats. */
struct RunStats {
  double total_eval_time_ms = 0.0;
  double drift_detect_time_ms = 0.0;
  double data_transfer_time_ms = 0.0;
  double gpu_kernel_time_ms = 0.0;
  double jit_compile_time_ms = 0.0;
  int num_subtrees = 0;
  double avg_subtree_size = 0.0;
  double coverage = 0.0;
};

/* Subtree-cache evaluator: replaces create_gpu_context / destroy_gpu_context /
 * evaluate_gpu_mse_wrapper (src/cleaned/cl_gpu_eval.cu:569-592). */
void *create_gpu_context();
void destroy_gpu_context(void *ctx);
void evaluate_gpu_mse_wrapper(InputInfo &input_info, float ***all_vars,
                              std::vector<float> &mses, void *ctx,
                              bool upload_X, bool clear_cache, RunStats &stats);

/* Evaluator without the cache: replaces create_gpu_simple_context /
 * destroy_gpu_simple_context / evaluate_gpu_simple_wrapper
 * (src/cleaned/cl_gpu_simple.cu:315-336). */
void *create_gpu_simple_context();
void destroy_gpu_simple_context(void *ctx);
void evaluate_gpu_simple_wrapper(InputInfo &input_info, float ***all_vars,
                                 std::vector<float> &mses, void *ctx,
                                 bool upload_X, RunStats &stats);

#endif /* SR_REFERENCE_ABI_H */
