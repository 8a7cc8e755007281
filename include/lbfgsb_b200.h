/*
 * lbfgsb_b200.h -- C ABI of the B200 (sm_100a) L-BFGS-B library (liblbfgsb_b200.so).
 *
 * The entry points take plain pointers and sizes.  Vectors x, l, u and the int array nbd
 * are DEVICE pointers of length n, as in the reference's LCM_CUDA mode (README "Usage";
 * culbfgsb.h:157-163).  Streams are passed as void* (a cudaStream_t; NULL is the legacy
 * default stream, which is what the reference uses).  The C++ drop-in surface of the
 * reference (culbfgsb.h: LBFGSB_CUDA_OPTION/STATE/SUMMARY, lbfgsbcuda::lbfgsbminimize,
 * lbfgsbdefaultoption) is include/culbfgsb.h, a header-only adapter over these calls.
 *
 * Return value of every lbfgsb_b200_* call: an LBFGSB_B200_* status.  The optimisation
 * outcome is summary->info with the reference's codes (culbfgsb.h:131-138):
 *   -2 abnormal termination in the line search, -1 wrong parameters (also: mode
 *   LCM_NO_ACCELERATION, which this GPU-only library does not provide), 0 stopped by the
 *   user's stopping callback, 1 relative decrease of f <= eps_f, 2 step <= eps_x,
 *   4 projected gradient <= eps_g, 5 iteration limit.
 * Unlike the reference's GPU driver (lbfgsbcuda.cpp:393, which forces info = 0), info
 * reports the real reason the solve stopped, as the reference's CPU driver does.
 */
#ifndef LBFGSB_B200_H_
#define LBFGSB_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBFGSB_B200_OK 0
#define LBFGSB_B200_ERR_ARGUMENT 1   /* null pointer or unsupported mode */
#define LBFGSB_B200_ERR_CUDA 2       /* a CUDA call failed; see lbfgsb_b200_last_error() */
#define LBFGSB_B200_ERR_CALLBACK 3   /* a sharded solve's allgather returned nonzero */

/* culbfgsb.h:31 */
#define LBFGSB_B200_MODE_NO_ACCELERATION 0
#define LBFGSB_B200_MODE_CUDA 1

/* LBFGSB_CUDA_OPTION<double> (culbfgsb.h:33-44), same field order and layout. */
typedef struct {
  double machine_epsilon;
  double machine_maximum;
  double step_scaling;
  double eps_g;
  double eps_f;
  double eps_x;
  int hessian_approximate_dimension;
  int max_iteration;
  int mode;
} lbfgsb_b200_option_f64;

typedef struct {
  float machine_epsilon;
  float machine_maximum;
  float step_scaling;
  float eps_g;
  float eps_f;
  float eps_x;
  int hessian_approximate_dimension;
  int max_iteration;
  int mode;
} lbfgsb_b200_option_f32;

/* LBFGSB_CUDA_SUMMARY<real> (culbfgsb.h:46-53). */
typedef struct {
  double residual_g;
  double residual_f;
  double residual_x;
  int num_iteration;
  int info;
} lbfgsb_b200_summary_f64;

typedef struct {
  float residual_g;
  float residual_f;
  float residual_x;
  int num_iteration;
  int info;
} lbfgsb_b200_summary_f32;

/* The callbacks of LBFGSB_CUDA_STATE (culbfgsb.h:55-67) with a user pointer: x and g are
 * device pointers of length n, f is a host scalar, stream is the solver's stream.
 * funcgrad fills *f and g at x; its return value is ignored, as in the reference.
 * customized_stopping returning nonzero stops the solve with info = 0.  Callbacks other
 * than funcgrad must not modify x or g. */
typedef int (*lbfgsb_b200_callback_f64)(void* user, double* x, double* f, double* g,
                                        void* stream, const lbfgsb_b200_summary_f64* summary);
typedef int (*lbfgsb_b200_callback_f32)(void* user, float* x, float* f, float* g,
                                        void* stream, const lbfgsb_b200_summary_f32* summary);

/* lbfgsbdefaultoption (culbfgsb/lbfgsb.cpp:43-66). */
void lbfgsb_b200_default_option_f64(lbfgsb_b200_option_f64* option);
void lbfgsb_b200_default_option_f32(lbfgsb_b200_option_f32* option);

/* lbfgsbcuda::lbfgsbminimize<double|float> with mode LCM_CUDA (culbfgsb.h:157-163,
 * dispatch lbfgsb.cpp:24-42, driver lbfgsbcuda.cpp:39-441).  The iteration follows the
 * reference's L-BFGS-B 2.1 algorithm as implemented in lbfgsbcpu.cpp:117-465 (full
 * breakpoint walk for the Cauchy point, subspace step truncated at the first bound).
 * x is updated in place with the final iterate.  after_iteration and
 * customized_stopping may be NULL.  The workspace (about 6 vectors of n reals, 18 of n
 * history elements, n bytes + n bits) is taken on `stream` from the library's per-device
 * memory pool for the duration of the call (see lbfgsb_b200_trim_memory). */
int lbfgsb_b200_minimize_f64(int n, double* x, const int* nbd, const double* l,
                             const double* u, const lbfgsb_b200_option_f64* option,
                             lbfgsb_b200_callback_f64 funcgrad,
                             lbfgsb_b200_callback_f64 after_iteration,
                             lbfgsb_b200_callback_f64 customized_stopping, void* user,
                             void* stream, lbfgsb_b200_summary_f64* summary);
int lbfgsb_b200_minimize_f32(int n, float* x, const int* nbd, const float* l, const float* u,
                             const lbfgsb_b200_option_f32* option,
                             lbfgsb_b200_callback_f32 funcgrad,
                             lbfgsb_b200_callback_f32 after_iteration,
                             lbfgsb_b200_callback_f32 customized_stopping, void* user,
                             void* stream, lbfgsb_b200_summary_f32* summary);

/* ---- extensions (no counterpart in the reference) ---------------------------------- */

/* Batched independent solves (the reference solves one problem per call): `count`
 * instances of possibly different sizes n[k], each with its own device arrays x[k] (in /
 * out), nbd[k], l[k], u[k] and funcgrad user pointer user[k], one option set for all.
 * `concurrency` host workers (0: 16), each on its own non-blocking stream on the calling
 * thread's device, run the plain solve on instances in turn, so small solves overlap on
 * the GPU; funcgrad is called from those workers (at most one call per instance at a
 * time).  Instance k's summary, x and status equal what its solo lbfgsb_b200_minimize
 * call gives.  status[k]: its return code; seconds[k] (may be NULL): its wall time. */
int lbfgsb_b200_minimize_batch_f64(int count, const int* n, double* const* x,
                                   const int* const* nbd, const double* const* l,
                                   const double* const* u, const lbfgsb_b200_option_f64* option,
                                   lbfgsb_b200_callback_f64 funcgrad, void* const* user,
                                   int concurrency, lbfgsb_b200_summary_f64* summary,
                                   int* status, double* seconds);
int lbfgsb_b200_minimize_batch_f32(int count, const int* n, float* const* x,
                                   const int* const* nbd, const float* const* l,
                                   const float* const* u, const lbfgsb_b200_option_f32* option,
                                   lbfgsb_b200_callback_f32 funcgrad, void* const* user,
                                   int concurrency, lbfgsb_b200_summary_f32* summary,
                                   int* status, double* seconds);


/* An upper bound on the device bytes one solve of n elements takes from the workspace pool
 * (real_size 8: the f64 entry points; 4: the f32 ones with `form` as in lbfgsb_b200_ext).
 * Host-only arithmetic; 0 for a bad argument. */
unsigned long long lbfgsb_b200_workspace_bytes(int n, int real_size, int form);

/* Serving front end (the reference has none: it solves one problem per call).  A server
 * owns `workers` host threads (0: 16), each with its own non-blocking stream on the device
 * that is current when it is created.  lbfgsb_b200_server_submit_f32 queues one whole FP32
 * solve on the caller's device arrays (x in / out, nbd, l, u; they must stay valid until
 * the request is waited on) and returns at once with its id.  Requests are admitted in
 * arrival order, each when its workspace bound (lbfgsb_b200_workspace_bytes) fits beside
 * the solves already running within `hbm_budget_bytes`; a request that does not fit holds
 * back the ones behind it.  A request larger than the whole budget is refused at submit
 * (LBFGSB_B200_ERR_ARGUMENT).  `form` is the precision form of every request
 * (LBFGSB_B200_FORM_MIXED: FP32 vectors with FP64 small-matrix steps).  funcgrad is
 * called from the worker that runs the request, with that worker's stream.
 * lbfgsb_b200_server_wait blocks until request `id` has finished and gives its summary,
 * its solve's return code, the seconds from submit to result and the seconds it waited
 * for admission; a request's result equals what the same solve gives through
 * lbfgsb_b200_minimize_ext_f32 with that form.  lbfgsb_b200_server_peak reports the most
 * workspace bytes and the most solves that were admitted at once.
 * lbfgsb_b200_server_destroy finishes every queued request, then stops the workers and
 * frees the server: no other call on the server may overlap it or follow it.  Submit, wait
 * and peak may be called from any threads. */
typedef struct lbfgsb_b200_server lbfgsb_b200_server;
int lbfgsb_b200_server_create(int workers, unsigned long long hbm_budget_bytes, int form,
                              lbfgsb_b200_server** server);
int lbfgsb_b200_server_submit_f32(lbfgsb_b200_server* server, int n, float* x, const int* nbd,
                                  const float* l, const float* u,
                                  const lbfgsb_b200_option_f32* option,
                                  lbfgsb_b200_callback_f32 funcgrad, void* user, long long* id);
int lbfgsb_b200_server_wait(lbfgsb_b200_server* server, long long id,
                            lbfgsb_b200_summary_f32* summary, int* status, double* latency_s,
                            double* queue_s);
int lbfgsb_b200_server_peak(lbfgsb_b200_server* server, unsigned long long* peak_bytes,
                            int* peak_running);
int lbfgsb_b200_server_destroy(lbfgsb_b200_server* server);

/* One record per accepted iteration, mirroring the CPU oracle's trace: the state the step
 * was computed from (col, head, theta, Cauchy-point and free-set statistics) and the
 * line-search outcome. */
typedef struct {
  int iter, nint, nbreak, nfree, nenter, nleave, col, head, nfgv, ifun, iword, reset;
  unsigned long long free_hash, at_lower, at_upper;
  double f, theta, stp, dtm, tsum, gd, gdold, dtd, stpmx;
  double f1_0, f2_0;  /* Cauchy f' and f'' before the first breakpoint */
  double dbg[8];      /* p(1), p(col+1), c(1), c(col+1), (Mc)(1), (Mc)(col+1), sy(1,1), wt(1,1) */
} lbfgsb_b200_trace_record;
typedef void (*lbfgsb_b200_trace_callback)(void* user, const lbfgsb_b200_trace_record* rec);

/* Precision forms of the f32 entry point:
 *   0 plain f32 (vectors, history and scalars in float, like the reference's float path)
 *   1 mixed: f32 vectors and history, f64 small-matrix, Cauchy and line-search scalars
 *   2 mixed with bf16 history storage */
#define LBFGSB_B200_FORM_PLAIN 0
#define LBFGSB_B200_FORM_MIXED 1
#define LBFGSB_B200_FORM_MIXED_BF16 2

typedef struct {
  int form;                           /* f32 entry point only */
  int profile;                        /* 1: time every kernel with CUDA events */
  lbfgsb_b200_trace_callback trace;   /* may be NULL */
  void* trace_user;
  /* 1: the L-BFGS-B 3.0 subspace step (Morales and Nocedal, ACM TOMS 38(1), 2011): the
   * subspace minimizer projected onto the box when that gives a descent direction, else
   * the 2.1 step truncated at the first bound.  0 (default): the reference's 2.1 step. */
  int subsm_projection;
} lbfgsb_b200_ext;

int lbfgsb_b200_minimize_ext_f64(int n, double* x, const int* nbd, const double* l,
                                 const double* u, const lbfgsb_b200_option_f64* option,
                                 lbfgsb_b200_callback_f64 funcgrad,
                                 lbfgsb_b200_callback_f64 after_iteration,
                                 lbfgsb_b200_callback_f64 customized_stopping, void* user,
                                 void* stream, const lbfgsb_b200_ext* ext,
                                 lbfgsb_b200_summary_f64* summary);
int lbfgsb_b200_minimize_ext_f32(int n, float* x, const int* nbd, const float* l,
                                 const float* u, const lbfgsb_b200_option_f32* option,
                                 lbfgsb_b200_callback_f32 funcgrad,
                                 lbfgsb_b200_callback_f32 after_iteration,
                                 lbfgsb_b200_callback_f32 customized_stopping, void* user,
                                 void* stream, const lbfgsb_b200_ext* ext,
                                 lbfgsb_b200_summary_f32* summary);

/* ---- sharded solves: one problem over several GPUs (no counterpart in the reference) --
 * The reference solves one problem on one GPU (lbfgsbcuda.cpp:39-441).  Here a problem of
 * n_global variables can be split by index range over `world` ranks, one process (or
 * thread) per GPU: rank r holds the n_local variables offset .. offset + n_local - 1 (its
 * slices of x, nbd, l and u, and its rows of the S/Y history).  Every pass of an iteration
 * sweeps only the local variables; its small reductions (about 200 doubles) are combined
 * over the ranks through `allgather`, and every rank then runs the same scalar steps, so
 * every rank keeps the same solver state and takes the same decisions.
 *
 * allgather(user, send, recv, count, stream): every rank passes `count` doubles at send
 * (device memory); when the work the call enqueues on `stream` completes, recv (device
 * memory, world * count doubles) holds rank r's values at recv[r * count].  It may enqueue
 * the exchange (an NCCL all-gather on `stream`) or complete it before returning; it
 * returns 0 on success.  Every rank makes the same calls in the same order.
 *
 * funcgrad evaluates this rank's part: it receives the local x (n_local values), writes
 * the local g, and returns in *f this rank's share of f (the solver adds the shares of the
 * ranks in rank order; a rank may return the whole f and the others 0).  after_iteration and
 * customized_stopping receive the local x and g and the whole f.  ext->trace reports the
 * whole problem's counts (the free-set hash over global indices).  If one rank fails, the
 * others wait in their next allgather: the allgather should carry a timeout.  Sharded
 * solves are host-driven (this callback API); the device-driven and batched forms run on
 * one GPU each. */
typedef int (*lbfgsb_b200_allgather_fn)(void* user, const double* send, double* recv, int count,
                                        void* stream);
typedef struct {
  int rank;
  int world;
  int n_global;   /* variables of the whole problem */
  int offset;     /* global index of this rank's first variable */
  lbfgsb_b200_allgather_fn allgather;
  void* allgather_user;
} lbfgsb_b200_shard;

int lbfgsb_b200_minimize_sharded_f64(const lbfgsb_b200_shard* shard, int n_local, double* x,
                                     const int* nbd, const double* l, const double* u,
                                     const lbfgsb_b200_option_f64* option,
                                     lbfgsb_b200_callback_f64 funcgrad,
                                     lbfgsb_b200_callback_f64 after_iteration,
                                     lbfgsb_b200_callback_f64 customized_stopping, void* user,
                                     void* stream, const lbfgsb_b200_ext* ext,
                                     lbfgsb_b200_summary_f64* summary);
int lbfgsb_b200_minimize_sharded_f32(const lbfgsb_b200_shard* shard, int n_local, float* x,
                                     const int* nbd, const float* l, const float* u,
                                     const lbfgsb_b200_option_f32* option,
                                     lbfgsb_b200_callback_f32 funcgrad,
                                     lbfgsb_b200_callback_f32 after_iteration,
                                     lbfgsb_b200_callback_f32 customized_stopping, void* user,
                                     void* stream, const lbfgsb_b200_ext* ext,
                                     lbfgsb_b200_summary_f32* summary);

/* ---- device-driven solves (no counterpart in the reference) ------------------------
 * The reference's funcgrad returns f on the host, so every evaluation costs the solver a
 * device-to-host synchronisation and the host must steer each step.  An objective that
 * leaves f in device memory lets the whole outer loop run on the device: one round of
 * launches (the loop top, the Cauchy point and the subspace step, the trial point, one
 * evaluation, the line-search decision and the stopping tests) is captured once into a
 * CUDA graph and relaunched; the host reads the solver's state before the first iteration
 * and then only every few rounds.
 *
 * The objective is called once to evaluate at x0 and once while the round is captured, so
 * it must only enqueue work on `stream` (no synchronisation, no allocation, nothing a
 * stream capture rejects).  Its arguments are DEVICE addresses: *x (the pointer to the n
 * values of x to evaluate at) and *g (the pointer to the n values of g to write) are read
 * by the objective's kernels on the device, because the solver rotates its buffers without
 * the host; f receives f(x) as a double; *active is 0 when the result of this round's
 * evaluation is not used (the objective may then skip its work, e.g. return at once from
 * its kernels).  The solve gives the same iterates and summary as lbfgsb_b200_minimize_ext
 * with a funcgrad that computes the same f and g.  Not supported in this mode: the
 * after_iteration / customized_stopping callbacks and ext->trace / ext->profile (ignored);
 * ext->form and ext->subsm_projection apply. */
typedef int (*lbfgsb_b200_device_objective_f64)(void* user, const double* const* x,
                                                double* const* g, double* f, const int* active,
                                                void* stream);
typedef int (*lbfgsb_b200_device_objective_f32)(void* user, const float* const* x,
                                                float* const* g, double* f, const int* active,
                                                void* stream);
int lbfgsb_b200_minimize_device_f64(int n, double* x, const int* nbd, const double* l,
                                    const double* u, const lbfgsb_b200_option_f64* option,
                                    lbfgsb_b200_device_objective_f64 objective, void* user,
                                    void* stream, const lbfgsb_b200_ext* ext,
                                    lbfgsb_b200_summary_f64* summary);
int lbfgsb_b200_minimize_device_f32(int n, float* x, const int* nbd, const float* l,
                                    const float* u, const lbfgsb_b200_option_f32* option,
                                    lbfgsb_b200_device_objective_f32 objective, void* user,
                                    void* stream, const lbfgsb_b200_ext* ext,
                                    lbfgsb_b200_summary_f32* summary);

/* ---- batched device-driven solves (no counterpart in the reference) -----------------
 * `count` independent instances of possibly different sizes n[k] (device arrays x[k] in /
 * out, nbd[k], l[k], u[k]; one option set; ids[k] the id the objective sees for instance k,
 * or ids = NULL for 0..count-1) solved together: every pass of a round is one launch for
 * all live instances (instance k gets its own contiguous range of CTAs, sized by its n from
 * a tuned table), the rounds are captured into a CUDA graph, converged instances are
 * retired and the launches shrink to the rest.  Each instance's workspace is one segment of
 * the library's pool.  An instance's results do not depend on the other instances of the
 * batch (it runs the same launches on its own reduction rows); status[k] is its return
 * code.  ext->form, ext->subsm_projection apply; the other ext fields are ignored.
 *
 * The objective evaluates a list of instances at once, enqueued on `stream` with nothing
 * synchronised (it is captured with the round): `count` entries, entry j being instance
 * ids[j]; x[j] (device) holds the pointer to that instance's x, g[j] the pointer to its
 * gradient, f[j] receives its f (double), and active[j] = 0 marks an entry whose result is
 * not used this round.  ids, x, g, f and active are device arrays of `count` entries.
 * first (device, count + 1 entries) is a suggested launch shape: entry j may use CTAs
 * first[j] .. first[j+1]-1 of a launch of `ctas` CTAs of 256 threads (at most 64 each). */
typedef int (*lbfgsb_b200_batch_objective_f64)(void* user, int count, const int* ids,
                                               const int* first, int ctas,
                                               const double* const* x, double* const* g,
                                               double* f, const int* active, void* stream);
typedef int (*lbfgsb_b200_batch_objective_f32)(void* user, int count, const int* ids,
                                               const int* first, int ctas,
                                               const float* const* x, float* const* g,
                                               double* f, const int* active, void* stream);
int lbfgsb_b200_minimize_batch_device_f64(int count, const int* ids, const int* n,
                                          double* const* x, const int* const* nbd,
                                          const double* const* l, const double* const* u,
                                          const lbfgsb_b200_option_f64* option,
                                          lbfgsb_b200_batch_objective_f64 objective, void* user,
                                          void* stream, const lbfgsb_b200_ext* ext,
                                          lbfgsb_b200_summary_f64* summary, int* status);
int lbfgsb_b200_minimize_batch_device_f32(int count, const int* ids, const int* n,
                                          float* const* x, const int* const* nbd,
                                          const float* const* l, const float* const* u,
                                          const lbfgsb_b200_option_f32* option,
                                          lbfgsb_b200_batch_objective_f32 objective, void* user,
                                          void* stream, const lbfgsb_b200_ext* ext,
                                          lbfgsb_b200_summary_f32* summary, int* status);
/* Continuous-batching server for FP32 solves (no counterpart in the reference): one server
 * thread keeps every admitted solve's state on the device and advances all of them together
 * with the batched passes above.  Requests queue in arrival order and are admitted, first
 * come first served, as soon as their workspace segment fits in `hbm_budget_bytes` beside
 * the running solves; requests that arrive while others run join them at the next round,
 * finished solves leave and free their memory for the queue.  `form` is the precision form
 * of every request (LBFGSB_B200_FORM_MIXED: FP32 vectors with FP64 small-matrix steps),
 * `option` their options, `objective` their batched objective (the request's `id` is the
 * entry id it sees); the server runs `rounds_per_loop` rounds (0: 4) between admissions.
 * submit queues a solve on the caller's device arrays (x in / out, nbd, l, u, valid until
 * the request is waited on) and returns a ticket at once; a request larger than the whole
 * budget is refused (LBFGSB_B200_ERR_ARGUMENT).  wait blocks until the ticket's solve has
 * finished and gives its summary, its return code and the seconds from submit to result and
 * from submit to admission; a result equals that of the same solve through
 * lbfgsb_b200_minimize_batch_device_f32 alone.  destroy finishes every queued request
 * first.  submit, wait and peak may be called from any threads. */
typedef struct lbfgsb_b200_batch_server lbfgsb_b200_batch_server;
/* The HBM bytes a request of n elements is admitted against (its workspace segment) in a
 * server of precision form `form` with m = option.hessian_approximate_dimension; host
 * arithmetic only, 0 for a bad argument. */
unsigned long long lbfgsb_b200_batch_request_bytes(int n, int form, int m);
int lbfgsb_b200_batch_server_create_f32(unsigned long long hbm_budget_bytes, int form,
                                        const lbfgsb_b200_option_f32* option,
                                        lbfgsb_b200_batch_objective_f32 objective, void* user,
                                        int rounds_per_loop, lbfgsb_b200_batch_server** server);
int lbfgsb_b200_batch_server_submit_f32(lbfgsb_b200_batch_server* server, int id, int n,
                                        float* x, const int* nbd, const float* l,
                                        const float* u, long long* ticket);
int lbfgsb_b200_batch_server_wait(lbfgsb_b200_batch_server* server, long long ticket,
                                  lbfgsb_b200_summary_f32* summary, int* status,
                                  double* latency_s, double* queue_s);
int lbfgsb_b200_batch_server_peak(lbfgsb_b200_batch_server* server,
                                  unsigned long long* peak_bytes, int* peak_live);
int lbfgsb_b200_batch_server_destroy(lbfgsb_b200_batch_server* server);

/* Override the tuned tiles per CTA of the batched passes for instances in size bucket
 * `bucket` (0: n <= 4096, 1: <= 16384, 2: <= 65536, 3: <= 262144, 4: larger); 0 restores
 * the tuned value.  For the autotuner. */
int lbfgsb_b200_batch_tiles_per_cta(int bucket, int tiles);

/* Statistics of the calling thread's last solve. */
#define LBFGSB_B200_MAX_KERNELS 16
typedef struct {
  int kernels;                       /* number of named kernels below */
  char name[LBFGSB_B200_MAX_KERNELS][32];
  long long launches[LBFGSB_B200_MAX_KERNELS];
  double ms[LBFGSB_B200_MAX_KERNELS];  /* summed CUDA-event time (profile = 1 only) */
  double bytes[LBFGSB_B200_MAX_KERNELS];  /* algorithmic DRAM bytes of one launch */
  long long total_launches;          /* all kernels the solver launched */
  long long host_syncs;              /* stream synchronisations of the solver */
  long long evaluations;             /* funcgrad calls */
  double bytes_per_iteration_model;  /* algorithmic bytes of one steady-state iteration */
  long long rounds;                  /* rounds of a device-driven solve (else 0) */
} lbfgsb_b200_stats;
int lbfgsb_b200_last_stats(lbfgsb_b200_stats* out);

/* Message of the last LBFGSB_B200_ERR_CUDA on the calling thread ("" if none). */
const char* lbfgsb_b200_last_error(void);

/* The solver's workspace comes from a library-owned memory pool per device that keeps its
 * memory between solves (no counterpart in the reference, which allocates and frees with
 * cudaMalloc/cudaFree in every call).  This returns the unused memory of every pool to
 * its device; call it when no solve is running. */
int lbfgsb_b200_trim_memory(void);

/* ---- synthetic objective (test and benchmark glue, no reference counterpart) ---------
 * f(x) = sum_k 0.5*kappa_k*((x_{i+1,j}-x_k)^2 + (x_{i,j+1}-x_k)^2)
 *      + h^2 * sum_k [w_k*softplus(x_k - t_k) - b_k*x_k + 0.05*cos(3*x_k)]
 * on an s x s grid (k = j*s + i, h = 1/(s+1), zero Dirichlet neighbours).  Fields are
 * given as host double arrays of length s*s.  The returned handle is the `user` pointer
 * of the matching funcgrad callback, which computes g on the device and f (deterministic
 * order, accumulated in double) and synchronises the stream to return f on the host. */
void* lbfgsb_b200_synth_create(int s, const double* kappa, const double* w, const double* t,
                               const double* b, int single_precision_fields);
void lbfgsb_b200_synth_destroy(void* handle);
/* Subtract the constant f0 from f (in double, before f is rounded to the solver's
 * precision).  The minimiser and g are unchanged; a float f then resolves decreases near
 * f0 that are below the float spacing of f itself (on a 4096 x 4096 grid f is about 0.45
 * and one iteration lowers it by about 1e-8). */
void lbfgsb_b200_synth_set_offset(void* handle, double f0);
int lbfgsb_b200_synth_funcgrad_f64(void* handle, double* x, double* f, double* g, void* stream,
                                   const lbfgsb_b200_summary_f64* summary);
int lbfgsb_b200_synth_funcgrad_f32(void* handle, float* x, float* f, float* g, void* stream,
                                   const lbfgsb_b200_summary_f32* summary);
/* The same objective for device-driven solves (lbfgsb_b200_device_objective_*): one kernel
 * launch, f written to device memory, nothing synchronised; it does no work when *active
 * is 0. */
int lbfgsb_b200_synth_device_f64(void* handle, const double* const* x, double* const* g,
                                 double* f, const int* active, void* stream);
int lbfgsb_b200_synth_device_f32(void* handle, const float* const* x, float* const* g,
                                 double* f, const int* active, void* stream);

/* A batch of synthetic problems generated on the device (test and benchmark glue): problem
 * p is the grid problem of side sides[p] whose fields, nbd and bounds are those the host
 * generator lbfgsb-gpu_b200/synth.py gives for seed seeds[p] (same counter-based draws,
 * bit-identical).  Fields are stored in float (single_precision_fields) or double; l, u in
 * the solver precision real_size (4 or 8).  _problem gives problem p's device arrays; the
 * _f64 / _f32 functions are its batched objective (lbfgsb_b200_batch_objective_*), the id of
 * an entry being the problem index p. */
void* lbfgsb_b200_synth_batch_create(int count, const int* sides, const unsigned long long* seeds,
                                     int single_precision_fields, int real_size);
void lbfgsb_b200_synth_batch_destroy(void* handle);
int lbfgsb_b200_synth_batch_problem(void* handle, int p, void** l, void** u, int** nbd,
                                    void* fields[4]);
int lbfgsb_b200_synth_batch_f64(void* handle, int count, const int* ids, const int* first,
                                int ctas, const double* const* x, double* const* g, double* f,
                                const int* active, void* stream);
int lbfgsb_b200_synth_batch_f32(void* handle, int count, const int* ids, const int* first,
                                int ctas, const float* const* x, float* const* g, double* f,
                                const int* active, void* stream);

/* ---- dsscfg objective (the reference example's objective, examples/dsscfg/dsscfg_cuda.cu)
 * The MINPACK-2 steady-state combustion problem on an nx x ny grid with parameter lambda,
 * as a device funcgrad callback: the handle is its `user` pointer; g is computed on the
 * device, f in double (deterministic order) and returned after a stream synchronisation.
 * _start writes the example's standard start point into the device vector x. */
void* lbfgsb_b200_dsscfg_create(int nx, int ny, double lambda);
void lbfgsb_b200_dsscfg_destroy(void* handle);
int lbfgsb_b200_dsscfg_funcgrad_f64(void* handle, double* x, double* f, double* g, void* stream,
                                    const lbfgsb_b200_summary_f64* summary);
int lbfgsb_b200_dsscfg_funcgrad_f32(void* handle, float* x, float* f, float* g, void* stream,
                                    const lbfgsb_b200_summary_f32* summary);
int lbfgsb_b200_dsscfg_start_f64(void* handle, double* x, void* stream);
int lbfgsb_b200_dsscfg_start_f32(void* handle, float* x, void* stream);

/* Plain blocking copies for bindings without their own CUDA runtime (kind: 1 host to
 * device, 2 device to host, 3 device to device). */
int lbfgsb_b200_copy(void* dst, const void* src, size_t bytes, int kind);

/* ---- projected-gradient norm that allocates nothing (no counterpart in the reference) --
 * *sbgnrm (device) = max_i |pg_i|, the reference's projgr (culbfgsb/lbfgsbcpu.cpp:1390)
 * and the value the solver reports as summary.residual_g; x, g, nbd, l, u are device
 * arrays of length n.  Enqueued on `stream`, nothing is synchronised.  It calls no
 * allocator: its scratch is a static 64 KB device array, so n is limited to
 * 0..33554432 (8192 per-CTA maxima of 4096 variables); a larger n returns
 * LBFGSB_B200_ERR_ARGUMENT with a message in lbfgsb_b200_last_error().  Meant for callers
 * that must not allocate, such as the solver's callbacks, which run in the middle of its
 * stream work.  Every call on a device shares the scratch: calls that overlap on the GPU
 * (streams not ordered with each other) race, so issue them in order.  The scratch's
 * arrival ticket must be zero when a call starts; it is zero at load and each call leaves
 * it zero.  The first call on a device looks up the scratch address
 * (cudaGetSymbolAddress); make that first call outside any stream capture.  The address is
 * kept for the life of the process: it assumes the device's context is not torn down and
 * created again (cudaDeviceReset) in between.  A call whose grid does not finish (a fault
 * in the caller's arrays) leaves the ticket set; the context is then unusable anyway, and
 * later calls report the sticky error.  Unlike the reference's sequential max, a NaN in g
 * does not propagate into the norm (the reduction keeps the larger of two values, and a NaN
 * compares false); the reference's propagates only a NaN in the last element. */
int lbfgsb_b200_projgr_noalloc_f64(int n, const double* x, const double* g, const int* nbd,
                                   const double* l, const double* u, double* sbgnrm,
                                   void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LBFGSB_B200_H_ */
