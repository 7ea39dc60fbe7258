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

/* ---- condition-aware allowance ---------------------------------------------
 * Test infrastructure for the parity bar "within 4 ulp per datapoint / 1e-6
 * on the MSE, except where the expression's conditioning amplifies the
 * permitted per-operator differences".  No reference counterpart: the
 * reference states no tolerance.
 *
 * Two FP32 evaluations of one expression at one datapoint, A (the device
 * evaluator) and B (the reference's evaluate_single_expr, glibc functions;
 * or, in mode 1, the exact value, approximated by the FP64 evaluation), see
 * identical leaves.  They can differ only where an operator's result is
 * rounded differently: the IEEE operators (+ - * / sqrt, reciprocal, the
 * protected forms) are correctly rounded in both, so they agree on equal
 * operands; a transcendental function f has at most u_A(f) and u_B(f) ulps of
 * error in the two implementations (their documented maxima, passed in by the
 * caller).  A running forward error bound (the node-by-node forward analysis
 * of Wilkinson, Rounding Errors in Algebraic Processes, 1963, with exact
 * interval deviations in place of first-order derivatives) bounds |A - B| at
 * every node, in postfix order of the prefix tree (right to left):
 *
 *   D(leaf) = 0;
 *   D(f(a, b)) = dev_f(a, D(a), b, D(b)) + r_f * ulp32(|f(a, b)| + dev_f),
 *
 * dev_f = max |f(x, y) - f(a, b)| over |x - a| <= D(a), |y - b| <= D(b)
 * (exact: at the interval ends for the operators that are monotone in each
 * operand on the box, convex cosh, Lipschitz bounds for sin and cos, Da + Db
 * for + and -, |a| Db + |b| Da + Da Db for *, max(Da, Db) for min / max),
 * r_f = u_A + u_B for a transcendental f, and for an IEEE operator 1 when an
 * operand may differ (two correctly rounded results of different exact
 * values), else 0; in mode 1 (A against the exact value) r_f = u_A for a
 * transcendental f and 0.5 for every IEEE operator.  The centre values are
 * B's own: the FP32 evaluation (mode 0) or the FP64 one (mode 1).
 *
 * A datapoint is FLAGGED (no bound is claimed; its expression is exempt from
 * the MSE bar too) when the box of some node touches a point where the
 * operator is discontinuous, singular or changes domain: a zero divisor (/,
 * reciprocal), the protected boundary |d| = 1e-9 or its sign change
 * (protected / and reciprocal), 0 for log, protected log, sqrt and pow's
 * base, a pole of tan, +-1 for asin / acos; when a value could overflow (or
 * overflowed where the other evaluation might not); and when a non-finite
 * value meets an operand that may differ.  Non-finite values reached with
 * no perturbed operand are deterministic (IEEE special values) and carry
 * D = 0.  The squared error of a datapoint adds the two float operations of
 * the reference's MSE rule (d = pred - y, d * d) the same way.
 */
#include <float.h>

static double ulp32(double x) {
  x = fabs(x);
  if (!(x < 3.5e38)) x = FLT_MAX;
  if (x < 1.1754943508222875e-38) return 1.401298464324817e-45;
  int e;
  frexp(x, &e); /* x = m * 2^e, m in [0.5, 1) */
  return ldexp(1.0, e - 24);
}

static int is_ieee_op(int op) {
  switch (op) {
    case 1: case 2: case 3: case 4: case 6: case 7: case 8: case 18: case 23: case 24:
    case 25: case 26: case 27:
      return 1;
    default:
      return 0;
  }
}

static int finite32(double v) { return !isnan(v) && fabs(v) <= FLT_MAX; }

#define DELTA_P 1e-9 /* the protected operators' threshold (as float: 1e-9f) */

/* max |f(x) - f(a)| over |x - a| <= r for f = sro_op_f64(op, ., b) monotone
 * (or convex) on the interval: at its ends. */
static double dev_ends1(int op, double a, double r, double fa) {
  const double lo = sro_op_f64(op, a - r, 0.0), hi = sro_op_f64(op, a + r, 0.0);
  double d = fabs(lo - fa);
  if (fabs(hi - fa) > d) d = fabs(hi - fa);
  return d;
}

/* ... over the box |x - a| <= ra, |y - b| <= rb at its corners (operators
 * monotone in each operand on the box). */
static double dev_corners2(int op, double a, double ra, double b, double rb, double fab) {
  double d = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double x = (i & 1) ? a + ra : a - ra;
    const double y = (i & 2) ? b + rb : b - rb;
    const double v = sro_op_f64(op, x, y);
    if (isnan(v)) return INFINITY;
    if (fabs(v - fab) > d) d = fabs(v - fab);
  }
  return d;
}

/* The protected denominator's branch is fixed on [x - r, x + r]: either
 * every point has |x| > 1e-9 on one side of zero, or every point has
 * |x| <= 1e-9 with one sign (zero and -0 count as positive). */
static int protected_branch_stable(double x, double r) {
  if (fabs(x) > DELTA_P) return fabs(x) - r > DELTA_P;
  if (r == 0.0) return 1;
  if (x < 0.0) return x + r < 0.0 && x - r >= -DELTA_P;
  return x - r >= 0.0 && x + r <= DELTA_P;
}

/* Results that C99 Annex F fixes exactly and both implementations return:
 * sin, tan, sinh, tanh, asin, atan of +-0 are +-0; cos, cosh, exp (and exp
 * clamped) of +-0 are 1; log of 1 is +0; pow(x, +-0) and pow(1, y) are 1. */
static int exact_special_value(int op, double a, double b) {
  switch (op) {
    case 10: case 12: case 13: case 15: case 19: case 21:
    case 11: case 14: case 16: case 32:
      return a == 0.0;
    case 17: return a == 1.0;
    case 22: return fabs(a) == 1.0;
    case 5: return b == 0.0 || a == 1.0;
    case 9: return b == 0.0 || fabs(a) == 1.0;
    default: return 0;
  }
}

/* One node.  a, b: centre values of the operands (b unused for unary
 * operators), Da, Db their bounds; fab: the centre value of the node as the
 * exact function of the centre operands (FP64).  Returns 1 to flag,
 * else 0 with *Dout set. */
static int node_bound(int op, double a, double Da, double b, double Db, double fab,
                      double uA, double uB, int mode, double *Dout) {
  const int binary = (op >= 1 && op <= 9);
  const double db_ = binary ? Db : 0.0;
  const int perturbed = (Da > 0.0) || (db_ > 0.0);
  const int ieee = is_ieee_op(op);
  const int in_finite = finite32(a) && (!binary || finite32(b));
  double dev = 0.0;
  const int known = (op >= 1 && op <= 27) || op == 32;
  if (!in_finite) {
    /* Special operands (inf, NaN): nothing is claimed when an operand may
     * differ.  Otherwise an IEEE or unknown operator is deterministic, and
     * a function's finite result (atan(inf), tanh(-inf), exp clamped of
     * NaN ...) carries the two implementations' error allowance; an
     * infinite or NaN result of a function of a special operand is an
     * exact special value. */
    if (perturbed) return 1;
    const double r0 = mode == 1 ? uA : uA + uB;
    *Dout = (ieee || !known || !finite32(fab)) ? 0.0 : r0 * ulp32(2.0 * fabs(fab));
    return 0;
  }
  if (perturbed) {
    switch (op) {
      case 1: case 2: dev = Da + Db; break;
      case 3: dev = fabs(a) * Db + fabs(b) * Da + Da * Db; break;
      case 6: case 7: dev = Da > Db ? Da : Db; break;
      case 4:
        if (fabs(b) - Db <= 0.0) return 1;
        dev = dev_corners2(op, a, Da, b, Db, fab);
        break;
      case 8:
        if (!protected_branch_stable(b, Db)) return 1;
        dev = (fabs(b) > DELTA_P) ? dev_corners2(op, a, Da, b, Db, fab) : Da / DELTA_P;
        break;
      case 5:
        if (a - Da <= 0.0) return 1;
        dev = dev_corners2(op, a, Da, b, Db, fab);
        break;
      case 9:
        if (fabs(a) - Da <= 0.0) return 1;
        dev = dev_corners2(op, fabs(a), Da, b, Db, fab);
        break;
      case 10: { const double c = fabs(cos(a)) + Da; dev = Da * (c < 1.0 ? c : 1.0); } break;
      case 11: { const double s = fabs(sin(a)) + Da; dev = Da * (s < 1.0 ? s : 1.0); } break;
      case 12:
        if (fabs(cos(a)) <= Da || Da >= 1.0) return 1;
        dev = dev_ends1(op, a, Da, fab);
        break;
      case 13: case 14: case 15: case 16: case 21: case 32:
        dev = dev_ends1(op, a, Da, fab);
        break;
      case 17:
        if (a - Da <= 0.0) {
          if (a + Da < 0.0) { *Dout = 0.0; return 0; } /* NaN on the whole interval */
          return 1;
        }
        dev = dev_ends1(op, a, Da, fab);
        break;
      case 19: case 20:
        if (fabs(a) + Da >= 1.0) {
          if (fabs(a) - Da > 1.0) { *Dout = 0.0; return 0; } /* NaN on the whole interval */
          return 1;
        }
        dev = dev_ends1(op, a, Da, fab);
        break;
      case 18:
        if (fabs(a) - Da <= 0.0) return 1;
        dev = dev_ends1(op, a, Da, fab);
        break;
      case 23:
        if (!protected_branch_stable(a, Da)) return 1;
        dev = (fabs(a) > DELTA_P) ? dev_ends1(op, a, Da, fab) : 0.0;
        break;
      case 22:
        if (fabs(a) - Da <= 0.0) return 1;
        dev = dev_ends1(17, fabs(a), Da, fab);
        break;
      case 24: case 25: dev = Da; break;
      case 26:
        if (a < 0.0) {
          if (a + Da < 0.0) { *Dout = 0.0; return 0; }
          return 1;
        }
        if (a - Da < 0.0) return 1;
        dev = dev_ends1(op, a, Da, fab);
        break;
      case 27: {
        const double lo = fabs(a) - Da > 0.0 ? fabs(a) - Da : 0.0;
        const double s = sqrt(fabs(a));
        dev = sqrt(fabs(a) + Da) - s;
        if (s - sqrt(lo) > dev) dev = s - sqrt(lo);
      } break;
      default: dev = 0.0; break; /* unknown operators give 0 */
    }
    if (!(dev < INFINITY)) return 1;
  }
  /* Mode 0: an IEEE operator on operands that cannot differ gives the same
   * correctly rounded result in both evaluations, whatever it is (an
   * overflow or a NaN included).  Unknown operators give 0 in both, and so
   * do the constant branches of protected log (-1e9 at 0) and protected pow
   * (0 at 0^0). */
  const int constant_branch =
      !perturbed && ((op == 22 && a == 0.0) || (op == 9 && a == 0.0 && b == 0.0) ||
                     exact_special_value(op, a, b));
  if (constant_branch || (mode == 0 && (!known || (ieee && !perturbed)))) {
    *Dout = 0.0;
    return 0;
  }
  /* A NaN centre (a domain error reached without perturbation, e.g. log of
   * a negative constant) is deterministic. */
  if (isnan(fab)) {
    if (perturbed) return 1;
    *Dout = 0.0;
    return 0;
  }
  double r;
  if (mode == 1) r = !known ? 0.0 : (ieee ? 0.5 : uA);
  else r = ieee ? 1.0 : uA + uB;
  /* ulps counted at the largest magnitude the result can reach (a result
   * near a power of two may land in the binade above, with twice the ulp). */
  const double top0 = fabs(fab) + dev;
  const double top = top0 + (r + 1.0) * ulp32(top0);
  const double err = dev + r * ulp32(top) + 1e-12 * fabs(fab);
  if (!finite32(fab)) {
    /* Overflowed at the centre.  Mode 0: robust only when even the smallest
     * value on the box lies beyond FLT_MAX by more than the rounding
     * allowance (both evaluations then hold inf).  Mode 1: the FP32
     * evaluation overflows where the exact value does not: no claim. */
    if (mode == 0 && fabs(fab) - dev > (double)FLT_MAX * (1.0 + (r + 1.0) * 1.2e-7)) {
      *Dout = 0.0;
      return 0;
    }
    return 1;
  }
  if (top + r * ulp32(top) >= (double)FLT_MAX) return 1; /* may overflow */
  *Dout = err;
  return 0;
}

/* Per-datapoint pass over one expression.  Mode 0: centre = B's FP32
 * values (float path, sro_op_f32); mode 1: centre = FP64 values.  Returns the
 * centre prediction (as double), its bound in *D and the flag. */
static int expr_bound(const int32_t *tok, const double *val, int len, const float *xf,
                      int num_vars, const double *uA, const double *uB, int mode,
                      double *pred, double *D) {
  double sv[SRO_STACK], sd[SRO_STACK];
  int sp = 0, flag = 0;
  for (int i = len - 1; i >= 0; --i) {
    const int t = tok[i];
    if (t == 0) {
      sv[sp] = (double)(float)val[i];
      sd[sp++] = 0.0;
    } else if (t == -1) {
      const int vi = var_index(val[i]);
      sv[sp] = (vi >= 0 && vi < num_vars) ? (double)xf[vi] : 0.0;
      sd[sp++] = 0.0;
    } else {
      const double a = sv[--sp], Da = sd[sp];
      double b = 0.0, Db = 0.0;
      if (t >= 1 && t <= 9) { b = sv[--sp]; Db = sd[sp]; }
      const double fab = sro_op_f64(t, a, b);
      double Dn = 0.0;
      const int u = (t >= 0 && t < 64) ? t : 0;
      if (!flag && node_bound(t, a, Da, b, Db, fab, uA[u], uB[u], mode, &Dn)) flag = 1;
      /* Mode 0 continues from B's own FP32 value, mode 1 from the FP64 one. */
      sv[sp] = (mode == 0) ? (double)sro_op_f32(t, (float)a, (float)b) : fab;
      sd[sp++] = flag ? 0.0 : Dn;
    }
  }
  *pred = sv[0];
  *D = sd[0];
  return flag;
}

typedef struct {
  int e0, e1, mode;
  const int32_t *tok;
  const double *val;
  const int64_t *off;
  int num_vars;
  int64_t N;
  const float *X;
  const double *uA, *uB;
  /* per datapoint (optional, [E][N]) */
  double *pred_out, *bound_out;
  uint8_t *flag_out;
  /* per expression (optional) */
  double *mse_out, *mse_bound_out;
  int64_t *flagged_out, *valid_out;
} sro_bjob;

static void *sro_bound_worker(void *arg) {
  sro_bjob *j = (sro_bjob *)arg;
  const int V = j->num_vars;
  const float *y = j->X + (int64_t)V * j->N;
  float xf[SRO_MAX_VARS];
  for (int e = j->e0; e < j->e1; ++e) {
    const int32_t *t = j->tok + j->off[e];
    const double *v = j->val + j->off[e];
    const int len = (int)(j->off[e + 1] - j->off[e]);
    double sum = 0.0, dsum = 0.0;
    int64_t valid = 0, flagged = 0;
    for (int64_t dp = 0; dp < j->N; ++dp) {
      for (int k = 0; k < V; ++k) xf[k] = j->X[(int64_t)k * j->N + dp];
      double p, D;
      int flag = expr_bound(t, v, len, xf, V, j->uA, j->uB, j->mode, &p, &D);
      const double yv = (double)y[dp];
      double dsq = 0.0;
      const int ok = j->mode == 0 ? finite32(p) : (!isnan(p) && fabs(p) <= FLT_MAX);
      if (ok) {
        /* The centre squared error counts for every valid datapoint.  In
         * mode 0 it is B's own: float difference, float square (the
         * reference MSE rule, cl_cpu_eval.cpp:147-151); mode 1: FP64. */
        const float d32 = (float)p - y[dp];
        const float sq32 = d32 * d32;
        const double d = p - yv;
        sum += (j->mode == 0) ? (double)sq32 : d * d;
        ++valid;
        if (!flag) {
          /* d = pred - y and d * d, each an IEEE float operation (0.5 ulp
           * each against the exact value in mode 1; 1 ulp when the
           * prediction may differ in mode 0). */
          const double rr = j->mode == 1 ? 0.5 : (D > 0.0 ? 1.0 : 0.0);
          const double Dd = D + rr * ulp32((fabs(d) + D) * (1.0 + 2.4e-7));
          const double top = (fabs(d) + Dd) * (fabs(d) + Dd) * (1.0 + 2.4e-7);
          const double low = fabs(d) > Dd ? (fabs(d) - Dd) * (fabs(d) - Dd) * (1.0 - 2.4e-7) : 0.0;
          if (low > (double)FLT_MAX) {
            /* Mode 0: the square overflows in both (+inf, the MSE is +inf
             * in both).  Mode 1: the FP32 square overflows where the FP64
             * one does not: no claim. */
            if (j->mode == 1) flag = 1;
          } else if (top + ulp32(top) >= (double)FLT_MAX) {
            flag = 1; /* the square may overflow in one evaluation only */
          } else {
            dsq = (2.0 * fabs(d) + Dd) * Dd + rr * ulp32(top);
            dsum += dsq;
          }
        }
      }
      if (flag) ++flagged;
      if (j->pred_out) {
        const int64_t k = (int64_t)e * j->N + dp;
        j->pred_out[k] = p;
        j->bound_out[k] = D;
        j->flag_out[k] = (uint8_t)flag;
      }
    }
    if (j->mse_out) {
      j->mse_out[e] = valid > 0 ? sum / (double)valid : NAN;
      j->mse_bound_out[e] = valid > 0 ? dsum / (double)valid : 0.0;
      j->flagged_out[e] = flagged;
      j->valid_out[e] = valid;
    }
  }
  return NULL;
}

/* Per-datapoint centre predictions, bounds and flags ([E][N] each; any of
 * the per-expression outputs may be NULL) and, per expression, the centre
 * MSE (FP64 sum of B's squared errors over B's valid datapoints / count), the
 * bound on |MSE_A - MSE_B| from the prediction bounds (sum of the squared
 * errors' bounds / count; the caller adds the summation and final rounding
 * allowances), the number of flagged datapoints and of valid ones.
 * uA, uB: per opcode (64 entries), the maximum error in ulps of each
 * implementation's function (used for non-IEEE operators only). */
void sro_error_bound(int E, const int32_t *tok, const double *val, const int64_t *off,
                     int num_vars, int64_t N, const float *X, const double *uA,
                     const double *uB, int mode, double *pred_out, double *bound_out,
                     uint8_t *flag_out, double *mse_out, double *mse_bound_out,
                     int64_t *flagged_out, int64_t *valid_out, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (threads > E) threads = E > 0 ? E : 1;
  pthread_t th[256];
  sro_bjob jobs[256];
  for (int k = 0; k < threads; ++k) {
    sro_bjob jb = {(int)((int64_t)E * k / threads), (int)((int64_t)E * (k + 1) / threads), mode,
                   tok, val, off, num_vars, N, X, uA, uB, pred_out, bound_out, flag_out,
                   mse_out, mse_bound_out, flagged_out, valid_out};
    jobs[k] = jb;
  }
  for (int k = 1; k < threads; ++k) pthread_create(&th[k], NULL, sro_bound_worker, &jobs[k]);
  sro_bound_worker(&jobs[0]);
  for (int k = 1; k < threads; ++k) pthread_join(th[k], NULL);
}

/* ---- a perturbed FP32 evaluator (tests of the allowance itself) -----------
 * The float path with every transcendental operator's result moved by a
 * pseudo-random whole number of ulps in [-k(op), k(op)] (a hash of seed,
 * expression, datapoint and node), except the results C99 Annex F fixes
 * exactly: an evaluator whose functions differ from glibc's by up to k ulps.  tests/ check that sro_error_bound covers its
 * differences from the float path with k = uA, and that it does not cover a
 * planted operator mistake. */
static float step_ulps(float x, int k) {
  if (k == 0 || !(fabsf(x) <= FLT_MAX)) return x;
  for (int i = 0; i < (k > 0 ? k : -k); ++i) x = nextafterf(x, k > 0 ? INFINITY : -INFINITY);
  return x;
}

static uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

void sro_predict_f32_perturbed(int E, const int32_t *tok, const double *val, const int64_t *off,
                               int num_vars, int64_t N, const float *X, const double *k_ulps,
                               uint64_t seed, int swap_sin_cos, float *out) {
  float stack[SRO_STACK];
  for (int e = 0; e < E; ++e) {
    const int32_t *t = tok + off[e];
    const double *v = val + off[e];
    const int len = (int)(off[e + 1] - off[e]);
    for (int64_t dp = 0; dp < N; ++dp) {
      int sp = 0;
      for (int i = len - 1; i >= 0; --i) {
        const int op = t[i];
        if (op == 0) {
          stack[sp++] = (float)v[i];
        } else if (op == -1) {
          const int vi = var_index(v[i]);
          stack[sp++] = (vi >= 0 && vi < num_vars) ? X[(int64_t)vi * N + dp] : 0.0f;
        } else {
          const float v1 = stack[--sp];
          float v2 = 0.0f;
          if (op >= 1 && op <= 9) v2 = stack[--sp];
          int o = op;
          if (swap_sin_cos && (o == 10 || o == 11)) o = 21 - o; /* a planted mistake */
          float r = sro_op_f32(o, v1, v2);
          const int u = (op >= 0 && op < 64) ? op : 0;
          const int kmax = (int)k_ulps[u];
          const int exact = exact_special_value(op, v1, v2) || (op == 22 && v1 == 0.0f) ||
                            (op == 9 && v1 == 0.0f && v2 == 0.0f);
          if (kmax > 0 && !is_ieee_op(op) && !exact) {
            const uint64_t h = mix64(seed ^ mix64(((uint64_t)e << 40) ^ ((uint64_t)dp << 8) ^ (uint64_t)i));
            const int k = (int)(h % (uint64_t)(2 * kmax + 1)) - kmax;
            r = step_ulps(r, k);
          }
          stack[sp++] = r;
        }
      }
      out[(int64_t)e * N + dp] = stack[0];
    }
  }
}
