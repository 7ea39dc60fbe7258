/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference CPU evaluator and of the subtree
 * keys, used as the checker of the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the
 * product (libsr_eval.so, the symbolic_regression_gpu_b200 package) never
 * does.  Its results are pinned against the reference itself: the golden
 * vectors under tests/golden/ were produced by the reference sources compiled
 * unchanged (oracle/ref_cpu_shim.cpp, oracle/ref_gpu_shim.cu, tests/golden/
 * make_golden.py), and tests/test_oracle.py checks this file against them.
 *
 * Each function names the reference code it restates.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SRO_STACK 1024
#define SRO_MAX_VARS 64

/* Operator semantics, float path (reference eval_op_cpu,
 * src/cleaned/cl_cpu_eval.cpp:16-56; v1 = first popped = left operand).
 * Opcode 32 is this project's extension: expf(fminf(v1, 80)). */
float sro_op_f32(int op, float v1, float v2) {
  const float DELTA = 1e-9f;
  const float MAX_VAL = 1e9f;
  switch (op) {
    case 1: return v1 + v2;
    case 2: return v1 - v2;
    case 3: return v1 * v2;
    case 4: return (v2 == 0.0f) ? NAN : v1 / v2;
    case 5: return powf(v1, v2);
    case 6: return fminf(v1, v2);
    case 7: return fmaxf(v1, v2);
    case 8: {
      const float d = fabsf(v2) <= DELTA ? (v2 < 0.0f ? -DELTA : DELTA) : v2;
      return v1 / d;
    }
    case 9: return (v1 == 0.0f && v2 == 0.0f) ? 0.0f : powf(fabsf(v1), v2);
    case 10: return sinf(v1);
    case 11: return cosf(v1);
    case 12: return tanf(v1);
    case 13: return sinhf(v1);
    case 14: return coshf(v1);
    case 15: return tanhf(v1);
    case 16: return expf(v1);
    case 17: return logf(v1);
    case 18: return 1.0f / v1;
    case 19: return asinf(v1);
    case 20: return acosf(v1);
    case 21: return atanf(v1);
    case 22: return (v1 == 0.0f) ? -MAX_VAL : logf(fabsf(v1));
    case 23: {
      const float d = fabsf(v1) <= DELTA ? (v1 < 0.0f ? -DELTA : DELTA) : v1;
      return 1.0f / d;
    }
    case 24: return fabsf(v1);
    case 25: return -v1;
    case 26: return sqrtf(v1);
    case 27: return sqrtf(fabsf(v1));
    case 32: return expf(fminf(v1, 80.0f));
    default: return 0.0f;
  }
}

/* The same semantics evaluated in double (FP64 oracle).  MIN/MAX use
 * fmin/fmax like the float path (not the <=/>= of the reference's double
 * evaluators, src/eval/cpu_simple_multi.cpp:29-32, which treat NaN
 * differently); constants enter as (double)(float)value like the float path. */
double sro_op_f64(int op, double v1, double v2) {
  const double DELTA = 1e-9;
  const double MAX_VAL = 1e9;
  switch (op) {
    case 1: return v1 + v2;
    case 2: return v1 - v2;
    case 3: return v1 * v2;
    case 4: return (v2 == 0.0) ? NAN : v1 / v2;
    case 5: return pow(v1, v2);
    case 6: return fmin(v1, v2);
    case 7: return fmax(v1, v2);
    case 8: {
      const double d = fabs(v2) <= DELTA ? (v2 < 0.0 ? -DELTA : DELTA) : v2;
      return v1 / d;
    }
    case 9: return (v1 == 0.0 && v2 == 0.0) ? 0.0 : pow(fabs(v1), v2);
    case 10: return sin(v1);
    case 11: return cos(v1);
    case 12: return tan(v1);
    case 13: return sinh(v1);
    case 14: return cosh(v1);
    case 15: return tanh(v1);
    case 16: return exp(v1);
    case 17: return log(v1);
    case 18: return 1.0 / v1;
    case 19: return asin(v1);
    case 20: return acos(v1);
    case 21: return atan(v1);
    case 22: return (v1 == 0.0) ? -MAX_VAL : log(fabs(v1));
    case 23: {
      const double d = fabs(v1) <= DELTA ? (v1 < 0.0 ? -DELTA : DELTA) : v1;
      return 1.0 / d;
    }
    case 24: return fabs(v1);
    case 25: return -v1;
    case 26: return sqrt(v1);
    case 27: return sqrt(fabs(v1));
    case 32: return exp(fmin(v1, 80.0));
    default: return 0.0;
  }
}

static int var_index(double v) {
  if (!(v > -2147483648.0 && v < 2147483648.0)) return -1;
  return (int)v;
}

/* One expression at one datapoint, float path (reference evaluate_single_expr,
 * src/cleaned/cl_cpu_eval.cpp:59-90): right to left; constants push
 * (float)value; variables push vars[(int)value] or 0 when the index is not an
 * input variable; binary iff 1 <= token <= 9. */
float sro_eval_f32(const int32_t *tok, const double *val, int len, const float *vars,
                   int num_vars) {
  float stack[SRO_STACK];
  int sp = 0;
  for (int i = len - 1; i >= 0; --i) {
    const int t = tok[i];
    if (t == 0) {
      stack[sp++] = (float)val[i];
    } else if (t == -1) {
      const int vi = var_index(val[i]);
      stack[sp++] = (vi >= 0 && vi < num_vars) ? vars[vi] : 0.0f;
    } else {
      const float v1 = stack[--sp];
      float v2 = 0.0f;
      if (t >= 1 && t <= 9) v2 = stack[--sp];
      stack[sp++] = sro_op_f32(t, v1, v2);
    }
  }
  return stack[0];
}

double sro_eval_f64(const int32_t *tok, const double *val, int len, const double *vars,
                    int num_vars) {
  double stack[SRO_STACK];
  int sp = 0;
  for (int i = len - 1; i >= 0; --i) {
    const int t = tok[i];
    if (t == 0) {
      stack[sp++] = (double)(float)val[i];
    } else if (t == -1) {
      const int vi = var_index(val[i]);
      stack[sp++] = (vi >= 0 && vi < num_vars) ? vars[vi] : 0.0;
    } else {
      const double v1 = stack[--sp];
      double v2 = 0.0;
      if (t >= 1 && t <= 9) v2 = stack[--sp];
      stack[sp++] = sro_op_f64(t, v1, v2);
    }
  }
  return stack[0];
}

/* ---- population-level passes (threads over contiguous expression ranges,
 *      as reference evaluate_cpu_mse, cl_cpu_eval.cpp:101-165) ----------- */
typedef struct {
  int kind; /* 0 preds f32, 1 mse f32, 2 mse f64 */
  int e0, e1;
  const int32_t *tok;
  const double *val;
  const int64_t *off;
  int num_vars;
  int64_t N;
  const float *X; /* column-major [(V+1)][N], y = row V */
  float *out_f32;
  double *out_f64;
  int64_t *out_count;
} sro_job;

static void *sro_worker(void *arg) {
  sro_job *j = (sro_job *)arg;
  const int V = j->num_vars;
  const float *y = j->X + (int64_t)V * j->N;
  float xf[SRO_MAX_VARS];
  double xd[SRO_MAX_VARS];
  for (int e = j->e0; e < j->e1; ++e) {
    const int32_t *t = j->tok + j->off[e];
    const double *v = j->val + j->off[e];
    const int len = (int)(j->off[e + 1] - j->off[e]);
    double sum = 0.0;
    int64_t valid = 0;
    for (int64_t dp = 0; dp < j->N; ++dp) {
      if (j->kind == 2) {
        for (int k = 0; k < V; ++k) xd[k] = (double)j->X[(int64_t)k * j->N + dp];
        const double p = sro_eval_f64(t, v, len, xd, V);
        /* Valid when the value would be a finite float (the float path's mask). */
        if (!isnan(p) && !isinf((float)p)) {
          const double d = p - (double)y[dp];
          sum += d * d;
          ++valid;
        }
      } else {
        for (int k = 0; k < V; ++k) xf[k] = j->X[(int64_t)k * j->N + dp];
        const float p = sro_eval_f32(t, v, len, xf, V);
        if (j->kind == 0) {
          j->out_f32[(int64_t)e * j->N + dp] = p;
        } else if (!isnan(p) && !isinf(p)) {
          /* Reference: float diff, float square, double sum (cl_cpu_eval.cpp:147-151). */
          const float d = p - y[dp];
          const float sq = d * d;
          sum += sq;
          ++valid;
        }
      }
    }
    if (j->kind == 1) {
      j->out_f32[e] = valid > 0 ? (float)(sum / (double)valid) : NAN;
    } else if (j->kind == 2) {
      j->out_f64[e] = valid > 0 ? sum / (double)valid : NAN;
      if (j->out_count) j->out_count[e] = valid;
    }
  }
  return NULL;
}

static void sro_run(sro_job proto, int E, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (threads > E) threads = E > 0 ? E : 1;
  pthread_t th[256];
  sro_job jobs[256];
  for (int k = 0; k < threads; ++k) {
    jobs[k] = proto;
    jobs[k].e0 = (int)((int64_t)E * k / threads);
    jobs[k].e1 = (int)((int64_t)E * (k + 1) / threads);
  }
  for (int k = 1; k < threads; ++k) pthread_create(&th[k], NULL, sro_worker, &jobs[k]);
  sro_worker(&jobs[0]);
  for (int k = 1; k < threads; ++k) pthread_join(th[k], NULL);
}

/* Per-datapoint float predictions, out[e*N + dp]. */
void sro_predict_f32(int E, const int32_t *tok, const double *val, const int64_t *off,
                     int num_vars, int64_t N, const float *X, float *out, int threads) {
  sro_job j = {0, 0, 0, tok, val, off, num_vars, N, X, out, NULL, NULL};
  sro_run(j, E, threads);
}

/* Reference float-path MSE (reference evaluate_cpu_mse, cl_cpu_eval.cpp:94-168). */
void sro_mse_f32(int E, const int32_t *tok, const double *val, const int64_t *off,
                 int num_vars, int64_t N, const float *X, float *mse, int threads) {
  sro_job j = {1, 0, 0, tok, val, off, num_vars, N, X, mse, NULL, NULL};
  sro_run(j, E, threads);
}

/* FP64 evaluation and FP64 accumulation. */
void sro_mse_f64(int E, const int32_t *tok, const double *val, const int64_t *off,
                 int num_vars, int64_t N, const float *X, double *mse, int64_t *count,
                 int threads) {
  sro_job j = {2, 0, 0, tok, val, off, num_vars, N, X, NULL, mse, count};
  sro_run(j, E, threads);
}

/* ---- keys (reference compute_hash, src/utils/detect.cpp:50-68, =
 *      compute_subtree_hash_gpu, src/cleaned/cl_gpu_eval.cu:259-272) ------ */
uint64_t sro_flat_key(const int32_t *tok, const double *val, int len) {
  uint64_t h = 14695981039346656037ull;
  const uint64_t P = 1099511628211ull;
  for (int i = 0; i < len; ++i) {
    uint64_t b;
    memcpy(&b, &val[i], sizeof b);
    h ^= (uint64_t)(int64_t)tok[i];
    h *= P;
    h ^= b;
    h *= P;
  }
  return h;
}

/* Merkle node hashes (reference hash_node / combine_hashes, detect.cpp:97-118;
 * reverse pass of detect_common_subtrees, detect.cpp:169-191). */
void sro_merkle(const int32_t *tok, const double *val, int len, int32_t *sizes,
                uint64_t *hashes) {
  const uint64_t P = 1099511628211ull;
  for (int i = len - 1; i >= 0; --i) {
    uint64_t b;
    memcpy(&b, &val[i], sizeof b);
    uint64_t h = 14695981039346656037ull;
    h ^= (uint64_t)(int64_t)tok[i];
    h *= P;
    h ^= b;
    h *= P;
    int size = 1;
    if (tok[i] > 0) {
      const int arity = tok[i] < 10 ? 2 : 1;
      int pos = i + 1;
      for (int k = 0; k < arity && pos < len; ++k) {
        h = h ^ (hashes[pos] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2));
        size += sizes[pos];
        pos += sizes[pos];
      }
    }
    sizes[i] = size;
    hashes[i] = h;
  }
}

/* ---- FP64 gradient of the MSE with respect to the constants --------------
 * No reference counterpart (the reference has no gradient).  Reverse mode on
 * the expression tree in double: values bottom-up, adjoints top-down in
 * prefix order (a parent precedes its children).  Derivative conventions at
 * non-smooth points match the device adjoint: |x|, sqrt|x|, LOOSE_LOG have
 * derivative 0 at 0; the protected regions of LOOSE_DIV / LOOSE_INV and the
 * exp clamp (x >= 80) have derivative 0; MIN / MAX route to the returned
 * operand (the first on ties, the non-NaN one); 0^0 of LOOSE_POW has
 * derivative 0; a zero adjoint times any partial is zero.  A datapoint
 * counts when its FP64 prediction would be a finite float. */
static double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
static double strong(double g, double d) { return g == 0.0 ? 0.0 : g * d; }

typedef struct {
  int E, V;
  int64_t N;
  const int32_t *tok;
  const double *val;
  const int64_t *off;
  const float *X;
  double *mse;
  double *grad;
  double *gabs;
  int e0, e1;
} sro_gjob;

static void *sro_grad_worker(void *arg) {
  sro_gjob *j = (sro_gjob *)arg;
  const int V = j->V;
  const float *y = j->X + (int64_t)V * j->N;
  for (int e = j->e0; e < j->e1; ++e) {
    const int32_t *t = j->tok + j->off[e];
    const double *vl = j->val + j->off[e];
    const int L = (int)(j->off[e + 1] - j->off[e]);
    int size[SRO_STACK], cidx[SRO_STACK];
    double v[SRO_STACK], adj[SRO_STACK];
    int nc = 0;
    for (int i = 0; i < L; ++i) cidx[i] = (t[i] == 0) ? nc++ : -1;
    /* constants of this expression start at its CSR offset */
    int64_t cbase = 0;
    for (int64_t q = 0; q < j->off[e]; ++q) cbase += (j->tok[q] == 0);
    double *g = j->grad + cbase;
    double *ga = j->gabs ? j->gabs + cbase : NULL;
    for (int c = 0; c < nc; ++c) g[c] = 0.0;
    if (ga)
      for (int c = 0; c < nc; ++c) ga[c] = 0.0;
    for (int i = L - 1; i >= 0; --i) {
      if (t[i] <= 0) { size[i] = 1; continue; }
      int s = 1, pos = i + 1, ar = (t[i] >= 1 && t[i] <= 9) ? 2 : 1;
      for (int k = 0; k < ar && pos < L; ++k) { s += size[pos]; pos += size[pos]; }
      size[i] = s;
    }
    double sum = 0.0;
    int64_t count = 0;
    for (int pass = 0; pass < 2; ++pass) {
      for (int64_t dp = 0; dp < j->N; ++dp) {
        for (int i = L - 1; i >= 0; --i) {
          const int tk = t[i];
          if (tk == 0) { v[i] = (double)(float)vl[i]; continue; }
          if (tk == -1) {
            const int vi = var_index(vl[i]);
            v[i] = (vi >= 0 && vi < V) ? (double)j->X[(int64_t)vi * j->N + dp] : 0.0;
            continue;
          }
          const double a = v[i + 1];
          const double b = (tk >= 1 && tk <= 9) ? v[i + 1 + size[i + 1]] : 0.0;
          v[i] = sro_op_f64(tk, a, b);
        }
        const double p = v[0];
        if (isnan(p) || isinf((float)p)) continue;
        const double d = p - (double)y[dp];
        if (pass == 0) { sum += d * d; ++count; continue; }
        for (int i = 0; i < L; ++i) adj[i] = 0.0;
        adj[0] = 2.0 * d;
        for (int i = 0; i < L; ++i) {
          const int tk = t[i];
          const double gi = adj[i];
          if (tk == 0) {
            g[cidx[i]] += gi;
            if (ga) ga[cidx[i]] += fabs(gi);
            continue;
          }
          if (tk == -1) continue;
          const int l = i + 1;
          const double a = v[l], out = v[i];
          if (tk >= 1 && tk <= 9) {
            const int r = l + size[l];
            const double b = v[r];
            double da = 0, db = 0;
            switch (tk) {
              case 1: da = 1; db = 1; break;
              case 2: da = 1; db = -1; break;
              case 3: da = b; db = a; break;
              case 4: da = 1.0 / b; db = -out / b; break;
              case 5: da = b * pow(a, b - 1.0); db = out * log(a); break;
              case 6: { const int first = isnan(b) || (!isnan(a) && a <= b); da = first; db = !first; } break;
              case 7: { const int first = isnan(b) || (!isnan(a) && a >= b); da = first; db = !first; } break;
              case 8: {
                const double den = fabs(b) <= 1e-9 ? (b < 0 ? -1e-9 : 1e-9) : b;
                da = 1.0 / den;
                db = fabs(b) <= 1e-9 ? 0.0 : -out / den;
              } break;
              case 9: {
                const int z = (a == 0.0 && b == 0.0);
                da = z ? 0.0 : b * pow(fabs(a), b - 1.0) * sgn(a);
                db = z ? 0.0 : out * log(fabs(a));
              } break;
            }
            adj[l] += strong(gi, da);
            adj[r] += strong(gi, db);
          } else {
            double da = 0;
            switch (tk) {
              case 10: da = cos(a); break;
              case 11: da = -sin(a); break;
              case 12: da = 1.0 + out * out; break;
              case 13: da = cosh(a); break;
              case 14: da = sinh(a); break;
              case 15: da = 1.0 - out * out; break;
              case 16: da = out; break;
              case 17: da = 1.0 / a; break;
              case 18: da = -out * out; break;
              case 19: da = 1.0 / sqrt(1.0 - a * a); break;
              case 20: da = -1.0 / sqrt(1.0 - a * a); break;
              case 21: da = 1.0 / (1.0 + a * a); break;
              case 22: da = (a == 0.0) ? 0.0 : 1.0 / a; break;
              case 23: da = fabs(a) <= 1e-9 ? 0.0 : -out * out; break;
              case 24: da = sgn(a); break;
              case 25: da = -1; break;
              case 26: da = 0.5 / out; break;
              case 27: da = (a == 0.0) ? 0.0 : sgn(a) * 0.5 / out; break;
              case 32: da = (a < 80.0) ? out : 0.0; break;
            }
            adj[l] += strong(gi, da);
          }
        }
      }
    }
    j->mse[e] = count > 0 ? sum / (double)count : NAN;
    for (int c = 0; c < nc; ++c) g[c] = count > 0 ? g[c] / (double)count : NAN;
    if (ga)
      for (int c = 0; c < nc; ++c) ga[c] = count > 0 ? ga[c] / (double)count : NAN;
  }
  return NULL;
}

/* mse [E] and grad [C] (constants in token order, CSR over expressions);
 * gabs [C] (may be NULL) = mean over valid datapoints of |adjoint reaching
 * each constant occurrence|, the scale of the summation's rounding error. */
void sro_grad_f64(int E, const int32_t *tok, const double *val, const int64_t *off,
                  int num_vars, int64_t N, const float *X, double *mse, double *grad,
                  double *gabs, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (threads > E) threads = E > 0 ? E : 1;
  pthread_t th[256];
  sro_gjob jobs[256];
  for (int k = 0; k < threads; ++k) {
    sro_gjob jb = {E, num_vars, N, tok, val, off, X, mse, grad, gabs,
                   (int)((int64_t)E * k / threads), (int)((int64_t)E * (k + 1) / threads)};
    jobs[k] = jb;
  }
  for (int k = 1; k < threads; ++k) pthread_create(&th[k], NULL, sro_grad_worker, &jobs[k]);
  sro_grad_worker(&jobs[0]);
  for (int k = 1; k < threads; ++k) pthread_join(th[k], NULL);
}
