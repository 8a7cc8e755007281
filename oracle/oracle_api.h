/*
 * oracle_api.h -- C interface shared by the two CPU checkers of this repository.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library under
 * lbfgsb-gpu_b200/) includes, links or calls anything under oracle/.  Only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use it.
 *
 * Two implementations sit behind this one interface:
 *   - liboracle.so          : lbfgsb_oracle.c, a plain-C restatement of the reference's
 *                              CPU L-BFGS-B (culbfgsb/lbfgsbcpu.cpp, L-BFGS-B 2.1) that also
 *                              emits a per-iteration trace (free-set hash, breakpoints passed,
 *                              col/head/theta/stp ...).
 *   - _ref/libref_lbfgsb.so : the reference's own culbfgsb/lbfgsbcpu.cpp + ap.cpp compiled
 *                              from the reference sources with ref_shim.cpp (Makefile here).
 *                              It is the pin for the restatement.
 *
 * Arrays are 0-based host arrays of length n.  The callbacks mirror the std::function
 * callbacks of culbfgsb.h:55-67 with a void* user pointer added.
 */
#ifndef LBFGSB_ORACLE_API_H_
#define LBFGSB_ORACLE_API_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double residual_g, residual_f, residual_x;
  int num_iteration, info;
} orc_summary_f64;

typedef struct {
  float residual_g, residual_f, residual_x;
  int num_iteration, info;
} orc_summary_f32;

/* culbfgsb.h:33-44 field for field (mode is implied: this is the CPU path). */
typedef struct {
  double machine_epsilon, machine_maximum, step_scaling, eps_g, eps_f, eps_x;
  int hessian_approximate_dimension, max_iteration;
} orc_option_f64;

typedef struct {
  float machine_epsilon, machine_maximum, step_scaling, eps_g, eps_f, eps_x;
  int hessian_approximate_dimension, max_iteration;
} orc_option_f32;

typedef int (*orc_cb_f64)(void* user, double* x, double* f, double* g,
                          const orc_summary_f64* summary);
typedef int (*orc_cb_f32)(void* user, float* x, float* f, float* g,
                          const orc_summary_f32* summary);

/* One record per outer iteration of the restatement (not available from the reference
 * build, which has no such hook).  Emitted right after the line search of iteration
 * `iter` (1-based, the value summary.num_iteration takes), before the stopping tests. */
typedef struct {
  int iter;          /* iteration number after the increment */
  int nint;          /* GCP segments explored (1 + breakpoints passed); 0 if GCP skipped */
  int nbreak;        /* breakpoints found by the GCP scan */
  int nfree;         /* |free set| after freev */
  int nenter, nleave;/* entering / leaving variables of freev */
  int col, head;     /* ring state when the step was computed */
  int nfgv;          /* function evaluations so far */
  int ifun;          /* evaluations in this line search */
  int iword;         /* subsm: 1 if the subspace step was truncated */
  int reset;         /* 1 if this iteration followed a memory reset */
  unsigned long long free_hash; /* sum over free i of mix64(i) (order-free hash) */
  unsigned long long at_lower, at_upper; /* counts of iwhere==1 / iwhere==2 after GCP */
  double f, theta, stp, dtm, tsum, gd, gdold, dtd, stpmx;
  double f1_0, f2_0; /* Cauchy f' and f'' before the first breakpoint */
  double dbg[8];     /* p(1), p(col+1), c(1), c(col+1), (Mc)(1), (Mc)(col+1), sy(1,1), wt(1,1) */
} orc_trace_rec;

typedef void (*orc_trace_cb)(void* user, const orc_trace_rec* rec);

/* The restatement (liboracle.so). */
void orc_lbfgsb_minimize_f64(int n, double* x, const int* nbd, const double* l,
                             const double* u, const orc_option_f64* opt,
                             orc_cb_f64 funcgrad, orc_cb_f64 after_iter,
                             orc_cb_f64 custom_stop, void* user,
                             orc_trace_cb trace, void* trace_user,
                             orc_summary_f64* summary);
void orc_lbfgsb_minimize_f32(int n, float* x, const int* nbd, const float* l,
                             const float* u, const orc_option_f32* opt,
                             orc_cb_f32 funcgrad, orc_cb_f32 after_iter,
                             orc_cb_f32 custom_stop, void* user,
                             orc_trace_cb trace, void* trace_user,
                             orc_summary_f32* summary);
/* 1: subsm takes the L-BFGS-B 3.0 step (the projection of the subspace minimizer onto the
 * box when that is a descent direction, else the 2.1 truncated step); 0 (default): the
 * reference's 2.1 step.  Process-wide, for tests. */
void orc_set_subsm_projection(int on);
void orc_default_option_f64(orc_option_f64* opt);
void orc_default_option_f32(orc_option_f32* opt);

/* Synthetic objective used by every parity case (objective.c).  fields = kappa, w, t, b,
 * each of length s*s, index k = j*s + i with i fast; h = 1/(s+1). */
void orc_synth_eval_f64(int s, const double* kappa, const double* w, const double* t,
                        const double* b, const double* x, double* f, double* g);
void orc_synth_eval_f32(int s, const double* kappa, const double* w, const double* t,
                        const double* b, const float* x, float* f, float* g);
/* The same with f0 subtracted from the double sum before f is rounded. */
void orc_synth_eval_off_f64(int s, const double* kappa, const double* w, const double* t,
                            const double* b, double f0, const double* x, double* f, double* g);
void orc_synth_eval_off_f32(int s, const double* kappa, const double* w, const double* t,
                            const double* b, double f0, const float* x, float* f, float* g);

/* dsscfg, the reference example's steady-state combustion objective (objective.c): start
 * point and f, g on an nx x ny grid; g may be NULL.  The ref_ variants run the
 * reference's own examples/dsscfg/dsscfg_cpu.cpp (in _ref/libref_lbfgsb.so only). */
void orc_dsscfg_start_f64(int nx, int ny, double lam, double* x);
void orc_dsscfg_start_f32(int nx, int ny, float lam, float* x);
void orc_dsscfg_eval_f64(int nx, int ny, double lam, const double* x, double* f, double* g);
void orc_dsscfg_eval_f32(int nx, int ny, float lam, const float* x, float* f, float* g);
void ref_dsscfg_start_f64(int nx, int ny, double lam, double* x);
void ref_dsscfg_start_f32(int nx, int ny, float lam, float* x);
void ref_dsscfg_eval_f64(int nx, int ny, double lam, double* x, double* f, double* g);
void ref_dsscfg_eval_f32(int nx, int ny, float lam, float* x, float* f, float* g);

/* Separable quadratic sum_k 0.5*a_k*(x_k - c_k)^2 (objective.c), for ties and zero
 * gradients. */
void orc_quad_eval_f64(int n, const double* a, const double* c, const double* x, double* f,
                       double* g);
void orc_quad_eval_f32(int n, const double* a, const double* c, const float* x, float* f,
                       float* g);

/* The reference build (_ref/libref_lbfgsb.so): same signatures without the trace. */
void ref_lbfgsb_minimize_f64(int n, double* x, const int* nbd, const double* l,
                             const double* u, const orc_option_f64* opt,
                             orc_cb_f64 funcgrad, orc_cb_f64 after_iter,
                             orc_cb_f64 custom_stop, void* user,
                             orc_summary_f64* summary);
void ref_lbfgsb_minimize_f32(int n, float* x, const int* nbd, const float* l,
                             const float* u, const orc_option_f32* opt,
                             orc_cb_f32 funcgrad, orc_cb_f32 after_iter,
                             orc_cb_f32 custom_stop, void* user,
                             orc_summary_f32* summary);

#ifdef __cplusplus
}
#endif
#endif /* LBFGSB_ORACLE_API_H_ */
