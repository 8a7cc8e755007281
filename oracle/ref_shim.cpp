// ref_shim.cpp -- TEST INFRASTRUCTURE.  Binds the reference's own CPU L-BFGS-B
// (culbfgsb/lbfgsbcpu.cpp, entry lbfgsbcuda::cpu::lbfgsbminimize at lbfgsbcpu.cpp:117-465)
// to the plain-C interface of oracle_api.h, so the restatement in lbfgsb_oracle.c can be
// checked call-for-call against the reference built from its own sources (see Makefile).
// Only this adapter is ours; the solver itself is compiled from the reference tree.
#include <cstring>
#include <functional>

#include "culbfgsb/lbfgsbcpu.h"
#include "examples/dsscfg/dsscfg_cpu.h"
#include "oracle_api.h"

namespace {

// lbfgsbcpu.cpp:160 declares `int task;` without an initial value and lbfgsbcpu.cpp:259
// reads it (errclb only writes it on an input error), so the reference can return
// info = -1 for valid input when stale stack bytes happen to hold 2.  Zeroing the stack
// region the solver's frame will occupy makes the reference build deterministic; the
// restatement initialises task to 0 instead.
__attribute__((noinline)) void scrub_stack() {
  volatile unsigned char pad[1 << 16];
  for (unsigned i = 0; i < sizeof(pad); i++) pad[i] = 0;
}

template <typename real, typename csum>
void to_c(const LBFGSB_CUDA_SUMMARY<real>& s, csum* c) {
  c->residual_g = s.residual_g;
  c->residual_f = s.residual_f;
  c->residual_x = s.residual_x;
  c->num_iteration = s.num_iteration;
  c->info = s.info;
}

template <typename real, typename copt, typename csum, typename ccb>
void run(int n, real* x, const int* nbd, const real* l, const real* u, const copt* o,
         ccb funcgrad, ccb after_iter, ccb custom_stop, void* user, csum* summary) {
  LBFGSB_CUDA_OPTION<real> opt;
  opt.machine_epsilon = o->machine_epsilon;
  opt.machine_maximum = o->machine_maximum;
  opt.step_scaling = o->step_scaling;
  opt.eps_g = o->eps_g;
  opt.eps_f = o->eps_f;
  opt.eps_x = o->eps_x;
  opt.hessian_approximate_dimension = o->hessian_approximate_dimension;
  opt.max_iteration = o->max_iteration;
  opt.mode = LCM_NO_ACCELERATION;

  LBFGSB_CUDA_STATE<real> state;
  state.m_cublas_handle = nullptr;
  auto wrap = [user](ccb fn) {
    std::function<int(real*, real&, real*, const cudaStream_t&,
                      const LBFGSB_CUDA_SUMMARY<real>&)> w;
    if (fn)
      w = [fn, user](real* xx, real& f, real* g, const cudaStream_t&,
                     const LBFGSB_CUDA_SUMMARY<real>& s) {
        csum cs;
        to_c(s, &cs);
        return fn(user, xx, &f, g, &cs);
      };
    return w;
  };
  state.m_funcgrad_callback = wrap(funcgrad);
  state.m_after_iteration_callback = wrap(after_iter);
  state.m_customized_stopping_callback = wrap(custom_stop);

  LBFGSB_CUDA_SUMMARY<real> s;
  std::memset(&s, 0, sizeof(s));
  scrub_stack();
  lbfgsbcuda::cpu::lbfgsbminimize<real>(n, state, opt, x, nbd, l, u, s);
  to_c(s, summary);
}

}  // namespace

extern "C" void ref_lbfgsb_minimize_f64(int n, double* x, const int* nbd,
                                        const double* l, const double* u,
                                        const orc_option_f64* opt, orc_cb_f64 funcgrad,
                                        orc_cb_f64 after_iter, orc_cb_f64 custom_stop,
                                        void* user, orc_summary_f64* summary) {
  run<double>(n, x, nbd, l, u, opt, funcgrad, after_iter, custom_stop, user, summary);
}

extern "C" void ref_lbfgsb_minimize_f32(int n, float* x, const int* nbd, const float* l,
                                        const float* u, const orc_option_f32* opt,
                                        orc_cb_f32 funcgrad, orc_cb_f32 after_iter,
                                        orc_cb_f32 custom_stop, void* user,
                                        orc_summary_f32* summary) {
  run<float>(n, x, nbd, l, u, opt, funcgrad, after_iter, custom_stop, user, summary);
}

// The reference's own dsscfg objective (examples/dsscfg/dsscfg_cpu.cpp), compiled from the
// reference tree: task 'XS' writes the standard start point (and allocates work buffers,
// freed here); 'FG' evaluates f and g with four n-vectors of work space.
extern "C" void ref_dsscfg_start_f64(int nx, int ny, double lam, double* x) {
  double* work = nullptr;
  double fdum = 0;
  dsscfg_cpu<double>(nx, ny, x, fdum, nullptr, &work, 'XS', lam);
  delete[] work;
}

extern "C" void ref_dsscfg_start_f32(int nx, int ny, float lam, float* x) {
  float* work = nullptr;
  float fdum = 0;
  dsscfg_cpu<float>(nx, ny, x, fdum, nullptr, &work, 'XS', lam);
  delete[] work;
}

extern "C" void ref_dsscfg_eval_f64(int nx, int ny, double lam, double* x, double* f, double* g) {
  double* work = new double[4 * (size_t)nx * ny];
  dsscfg_cpu<double>(nx, ny, x, *f, g, &work, 'FG', lam);
  delete[] work;
}

extern "C" void ref_dsscfg_eval_f32(int nx, int ny, float lam, float* x, float* f, float* g) {
  float* work = new float[4 * (size_t)nx * ny];
  dsscfg_cpu<float>(nx, ny, x, *f, g, &work, 'FG', lam);
  delete[] work;
}
