/*
 * culbfgsb/culbfgsb.h -- drop-in C++ surface of the reference library (culbfgsb/culbfgsb.h)
 * over the C ABI of lbfgsb_b200.h, at the reference's include path: with this library's
 * include/ directory on the include path, code that writes #include "culbfgsb/culbfgsb.h"
 * compiles unchanged and links against liblbfgsb_b200.so instead of cuLBFGSB:
 *   - enum LBFGSB_CUDA_MODE, LBFGSB_CUDA_OPTION<real>, LBFGSB_CUDA_SUMMARY<real>,
 *     LBFGSB_CUDA_STATE<real> with the same fields in the same order (culbfgsb.h:31-67);
 *   - lbfgsbcuda::lbfgsbminimize<float|double> and lbfgsbcuda::lbfgsbdefaultoption
 *     (culbfgsb.h:157-166, defaults of lbfgsb.cpp:43-66).
 * Differences a caller can observe, all deliberate:
 *   - m_cublas_handle is accepted and ignored (no cuBLAS on the path); it may be null.
 *     <cublas_v2.h> is included, as the reference's header does (culbfgsb.h:26), so that
 *     callers which create and destroy a handle themselves keep compiling; nothing of
 *     cuBLAS is called by the library;
 *   - mode LCM_NO_ACCELERATION is not provided (this library is the GPU path only):
 *     summary.info = -1 and x is left unchanged;
 *   - summary.info reports the real stop reason (the reference's GPU driver overwrites it
 *     with 0, lbfgsbcuda.cpp:393; its CPU driver keeps it, as here);
 *   - a CUDA failure inside the library sets summary.info = LBFGSB_CUDA_INFO_CUDA_FAILURE
 *     (-3) and leaves its message in lbfgsb_b200_last_error(); the reference prints and
 *     exits the process instead (cutil_inline.h:18-25);
 *   - the iteration is the reference's CPU algorithm (full Cauchy breakpoint walk,
 *     2.1-style subspace truncation), not the first-segment approximation of its GPU
 *     kernels (cauchy.cu:596-603).
 */
#ifndef CULBFGSB_CULBFGSB_H_
#define CULBFGSB_CULBFGSB_H_

#include <cublas_v2.h>
#include <cuda_runtime_api.h>

#include <functional>

#include "../lbfgsb_b200.h"

// summary.info after a CUDA failure inside the library (no counterpart in the reference)
#define LBFGSB_CUDA_INFO_CUDA_FAILURE (-3)

enum LBFGSB_CUDA_MODE { LCM_NO_ACCELERATION, LCM_CUDA };

template <typename real>
struct LBFGSB_CUDA_OPTION {
  real machine_epsilon;
  real machine_maximum;
  real step_scaling;
  real eps_g;
  real eps_f;
  real eps_x;
  int hessian_approximate_dimension;
  int max_iteration;
  LBFGSB_CUDA_MODE mode;
};

template <typename real>
struct LBFGSB_CUDA_SUMMARY {
  real residual_g;
  real residual_f;
  real residual_x;
  int num_iteration;
  int info;
};

template <typename real>
struct LBFGSB_CUDA_STATE {
  cublasContext* m_cublas_handle;
  std::function<int(real*, real&, real*, const cudaStream_t&, const LBFGSB_CUDA_SUMMARY<real>&)>
      m_funcgrad_callback;
  std::function<int(real*, real&, real*, const cudaStream_t&, const LBFGSB_CUDA_SUMMARY<real>&)>
      m_after_iteration_callback;
  std::function<int(real*, real&, real*, const cudaStream_t&, const LBFGSB_CUDA_SUMMARY<real>&)>
      m_customized_stopping_callback;
};

namespace lbfgsbcuda {
namespace b200_detail {

template <typename real>
struct CTypes;
template <>
struct CTypes<double> {
  typedef lbfgsb_b200_option_f64 Opt;
  typedef lbfgsb_b200_summary_f64 Sum;
  typedef lbfgsb_b200_callback_f64 Cb;
  static int minimize(int n, double* x, const int* nbd, const double* l, const double* u,
                      const Opt* o, Cb fg, Cb after, Cb stop, void* user, void* stream, Sum* s) {
    return lbfgsb_b200_minimize_f64(n, x, nbd, l, u, o, fg, after, stop, user, stream, s);
  }
  static void defaults(Opt* o) { lbfgsb_b200_default_option_f64(o); }
};
template <>
struct CTypes<float> {
  typedef lbfgsb_b200_option_f32 Opt;
  typedef lbfgsb_b200_summary_f32 Sum;
  typedef lbfgsb_b200_callback_f32 Cb;
  static int minimize(int n, float* x, const int* nbd, const float* l, const float* u,
                      const Opt* o, Cb fg, Cb after, Cb stop, void* user, void* stream, Sum* s) {
    return lbfgsb_b200_minimize_f32(n, x, nbd, l, u, o, fg, after, stop, user, stream, s);
  }
  static void defaults(Opt* o) { lbfgsb_b200_default_option_f32(o); }
};

// The C structs and the templates above have the same layout; the adapter passes the
// caller's summary object itself to the C ABI, so callbacks see it being updated.
template <typename real>
struct LayoutCheck {
  static_assert(sizeof(LBFGSB_CUDA_OPTION<real>) == sizeof(typename CTypes<real>::Opt),
                "option layout");
  static_assert(sizeof(LBFGSB_CUDA_SUMMARY<real>) == sizeof(typename CTypes<real>::Sum),
                "summary layout");
  static_assert(sizeof(LBFGSB_CUDA_MODE) == sizeof(int), "mode size");
};

template <typename real, int Which>
int trampoline(void* user, real* x, real* f, real* g, void* stream,
               const typename CTypes<real>::Sum* s) {
  const LBFGSB_CUDA_STATE<real>* st = static_cast<const LBFGSB_CUDA_STATE<real>*>(user);
  const cudaStream_t cs = static_cast<cudaStream_t>(stream);
  const LBFGSB_CUDA_SUMMARY<real>& sum = *reinterpret_cast<const LBFGSB_CUDA_SUMMARY<real>*>(s);
  if (Which == 0) return st->m_funcgrad_callback(x, *f, g, cs, sum);
  if (Which == 1) return st->m_after_iteration_callback(x, *f, g, cs, sum);
  return st->m_customized_stopping_callback(x, *f, g, cs, sum);
}

}  // namespace b200_detail

template <typename real>
inline void lbfgsbminimize(const int& n, const LBFGSB_CUDA_STATE<real>& state,
                           const LBFGSB_CUDA_OPTION<real>& option, real* x, const int* nbd,
                           const real* l, const real* u, LBFGSB_CUDA_SUMMARY<real>& summary) {
  typedef b200_detail::CTypes<real> T;
  (void)sizeof(b200_detail::LayoutCheck<real>);
  typename T::Cb fg = state.m_funcgrad_callback ? &b200_detail::trampoline<real, 0> : 0;
  typename T::Cb after = state.m_after_iteration_callback ? &b200_detail::trampoline<real, 1> : 0;
  typename T::Cb stop =
      state.m_customized_stopping_callback ? &b200_detail::trampoline<real, 2> : 0;
  const int status =
      T::minimize(n, x, nbd, l, u, reinterpret_cast<const typename T::Opt*>(&option), fg, after,
                  stop, const_cast<LBFGSB_CUDA_STATE<real>*>(&state), 0,
                  reinterpret_cast<typename T::Sum*>(&summary));
  // argument errors already carry info = -1; a CUDA failure gets its own code
  if (status == LBFGSB_B200_ERR_CUDA) summary.info = LBFGSB_CUDA_INFO_CUDA_FAILURE;
}

template <typename real>
inline void lbfgsbdefaultoption(LBFGSB_CUDA_OPTION<real>& option) {
  b200_detail::CTypes<real>::defaults(reinterpret_cast<typename b200_detail::CTypes<real>::Opt*>(&option));
}

}  // namespace lbfgsbcuda

#endif  // CULBFGSB_CULBFGSB_H_
