// objective.cu -- the synthetic grid objective as a device funcgrad callback (benchmark and
// test glue; the reference ships only MINPACK-2 dsscfg as an example objective).
//
//   f(x) = sum_k 0.5*kappa_k*((x_{i+1,j}-x_k)^2 + (x_{i,j+1}-x_k)^2)
//        + h^2 * sum_k [w_k*softplus(x_k - t_k) - b_k*x_k + 0.05*cos(3*x_k)]
//
// One thread per grid point computes g_k and its term of f; f is summed in double through
// per-CTA rows folded in CTA order by the last CTA (bitwise reproducible), then copied to
// pinned host memory.  The callback synchronises the stream: the host needs f.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "../../include/lbfgsb_b200.h"
#include "common.cuh"
#include "reduce.cuh"

namespace lbfgsb_b200 {

struct SynthCtx {
  int s;
  int single;           // fields stored as float
  void* field[4];       // kappa, w, t, b
  double* part;
  double* fdev;
  double* fhost;        // pinned
  unsigned int* ticket;
  int grid[2];          // launch grid of the double / float kernel: one wave of CTAs
  double f0;            // constant subtracted from the double sum before f is rounded
};

// exp, log1p and sincos in the kernel's precision.
__device__ __forceinline__ double rexp(double v) { return exp(v); }
__device__ __forceinline__ float rexp(float v) { return expf(v); }
__device__ __forceinline__ double rlog1p(double v) { return log1p(v); }
__device__ __forceinline__ float rlog1p(float v) { return log1pf(v); }
__device__ __forceinline__ void rsincos(double v, double* s, double* c) { sincos(v, s, c); }
__device__ __forceinline__ void rsincos(float v, float* s, float* c) { sincosf(v, s, c); }

template <typename R, typename F>
__device__ __forceinline__ void synth_body(int s, const R* __restrict__ x, const F* __restrict__ kap,
                                           const F* __restrict__ w, const F* __restrict__ tt,
                                           const F* __restrict__ b, R* __restrict__ g,
                                           double* part, unsigned int* ticket, double f0,
                                           double* fout, CtaPos cp);

template <typename R, typename F>
__global__ void __launch_bounds__(kThreads) k_synth(int s, const R* __restrict__ x,
                                                    const F* __restrict__ kap,
                                                    const F* __restrict__ w,
                                                    const F* __restrict__ tt,
                                                    const F* __restrict__ b, R* __restrict__ g,
                                                    double* part, unsigned int* ticket,
                                                    double f0, double* fout) {
  synth_body<R, F>(s, x, kap, w, tt, b, g, part, ticket, f0, fout, cta_here());
}

// The device-driven form: x and g are read from device memory (the solver's evaluation
// slot), f is left in device memory, and nothing runs when the evaluation is not used.
template <typename R, typename F>
__global__ void __launch_bounds__(kThreads) k_synth_slot(int s, const R* const* xs,
                                                         const F* __restrict__ kap,
                                                         const F* __restrict__ w,
                                                         const F* __restrict__ tt,
                                                         const F* __restrict__ b, R* const* gs,
                                                         const int* active, double* part,
                                                         unsigned int* ticket, double f0,
                                                         double* fout) {
  if (!*active) return;
  synth_body<R, F>(s, *xs, kap, w, tt, b, *gs, part, ticket, f0, fout, cta_here());
}

template <typename R, typename F>
__device__ __forceinline__ void synth_body(int s, const R* __restrict__ x, const F* __restrict__ kap,
                                           const F* __restrict__ w, const F* __restrict__ tt,
                                           const F* __restrict__ b, R* __restrict__ g,
                                           double* part, unsigned int* ticket, double f0,
                                           double* fout, CtaPos cp) {
  const long long n = (long long)s * s;
  const R h = R(1) / (R)(s + 1), h2 = h * h;
  double acc = 0.0;
  for (long long k = (long long)cp.rank * kThreads + threadIdx.x; k < n;
       k += (long long)cp.count * kThreads) {
    const int i = (int)(k % s), j = (int)(k / s);
    const R xk = x[k];
    const R xe = (i + 1 < s) ? x[k + 1] : R(0);
    const R xn = (j + 1 < s) ? x[k + s] : R(0);
    const R de = xe - xk, dn = xn - xk;
    const R kk = (R)kap[k], wk = (R)w[k], bk = (R)b[k];
    const R z = xk - (R)tt[k];
    // softplus(z) = max(z, 0) + log1p(exp(-|z|)) and sigmoid(z) = (z >= 0 ? 1 : e) / (1 + e)
    // share e = exp(-|z|); cos(3x) and sin(3x) share one sincos
    const R e = rexp(-fabs(z));
    const R softplus = (z > R(0) ? z : R(0)) + rlog1p(e);
    const R sigmoid = (z >= R(0) ? R(1) : e) / (R(1) + e);
    R s3, c3;
    rsincos(R(3) * xk, &s3, &c3);
    const R term = R(0.5) * kk * (de * de + dn * dn) + h2 * (wk * softplus - bk * xk + R(0.05) * c3);
    acc += (double)term;
    R gk = -kk * (de + dn);
    if (i > 0) gk += (R)kap[k - 1] * (xk - x[k - 1]);
    if (j > 0) gk += (R)kap[k - s] * (xk - x[k - s]);
    gk += h2 * (wk * sigmoid - bk - R(0.15) * s3);
    g[k] = gk;
  }
  double sarr[1] = {acc}, xd[1] = {0.0}, ld[1] = {0.0};
  MinPair md[1] = {MinPair{0.0, 0}};
  cta_reduce_to_row<kThreads, 1, 0, 0, 0>(sarr, xd, md, ld, part, 1, cp.rank);
  if (!last_cta(ticket, cp.count)) return;
  __shared__ double red[1];
  fold_rows<kThreads>(part, cp.count, 1, 1, 0, 0, red);
  if (threadIdx.x == 0) *fout = red[0] - f0;
}

template <typename R>
static int synth_device(void* handle, const R* const* x, R* const* g, double* f,
                        const int* active, void* stream) {
  SynthCtx* c = static_cast<SynthCtx*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  if (c->single) {
    k_synth_slot<R, float><<<c->grid[sizeof(R) == 8 ? 0 : 1], kThreads, 0, s>>>(
        c->s, x, (const float*)c->field[0], (const float*)c->field[1],
        (const float*)c->field[2], (const float*)c->field[3], g, active, c->part, c->ticket,
        c->f0, f);
  } else {
    k_synth_slot<R, double><<<c->grid[sizeof(R) == 8 ? 0 : 1], kThreads, 0, s>>>(
        c->s, x, (const double*)c->field[0], (const double*)c->field[1],
        (const double*)c->field[2], (const double*)c->field[3], g, active, c->part, c->ticket,
        c->f0, f);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

template <typename R>
static int synth_eval(void* handle, R* x, R* f, R* g, void* stream) {
  SynthCtx* c = static_cast<SynthCtx*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  if (c->single) {
    k_synth<R, float><<<c->grid[sizeof(R) == 8 ? 0 : 1], kThreads, 0, s>>>(
        c->s, x, (const float*)c->field[0], (const float*)c->field[1],
        (const float*)c->field[2], (const float*)c->field[3], g, c->part, c->ticket, c->f0,
        c->fdev);
  } else {
    k_synth<R, double><<<c->grid[sizeof(R) == 8 ? 0 : 1], kThreads, 0, s>>>(
        c->s, x, (const double*)c->field[0], (const double*)c->field[1],
        (const double*)c->field[2], (const double*)c->field[3], g, c->part, c->ticket, c->f0,
        c->fdev);
  }
  cudaMemcpyAsync(c->fhost, c->fdev, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  *f = (R)*c->fhost;
  return 0;
}

}  // namespace lbfgsb_b200

using namespace lbfgsb_b200;

extern "C" {

void* lbfgsb_b200_synth_create(int s, const double* kappa, const double* w, const double* t,
                               const double* b, int single_precision_fields) {
  if (s <= 0 || !kappa || !w || !t || !b) return nullptr;
  SynthCtx* c = new SynthCtx();
  std::memset(c, 0, sizeof(*c));
  c->s = s;
  c->single = single_precision_fields ? 1 : 0;
  const size_t n = (size_t)s * s;
  const double* src[4] = {kappa, w, t, b};
  bool ok = true;
  for (int k = 0; k < 4 && ok; k++) {
    if (c->single) {
      float* tmp = (float*)std::malloc(n * sizeof(float));
      for (size_t i = 0; i < n; i++) tmp[i] = (float)src[k][i];
      ok = cudaMalloc(&c->field[k], n * sizeof(float)) == cudaSuccess &&
           cudaMemcpy(c->field[k], tmp, n * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
      std::free(tmp);
    } else {
      ok = cudaMalloc(&c->field[k], n * sizeof(double)) == cudaSuccess &&
           cudaMemcpy(c->field[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
    }
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = ((long long)n + kThreads - 1) / kThreads;
  for (int r = 0; r < 2; r++) {
    // one wave of resident CTAs; the grid-stride loop covers the rest
    int per_sm = 1;
    if (c->single)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, r == 0 ? (const void*)k_synth<double, float> : (const void*)k_synth<float, float>,
          kThreads, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, r == 0 ? (const void*)k_synth<double, double> : (const void*)k_synth<float, double>,
          kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    c->grid[r] = (int)(want < (long long)sms * per_sm ? want : (long long)sms * per_sm);
  }
  const int rows = c->grid[0] > c->grid[1] ? c->grid[0] : c->grid[1];
  ok = ok && cudaMalloc(&c->part, (size_t)rows * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->fdev, sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->ticket, sizeof(unsigned int)) == cudaSuccess;
  ok = ok && cudaMemset(c->ticket, 0, sizeof(unsigned int)) == cudaSuccess;
  ok = ok && cudaMallocHost(&c->fhost, sizeof(double)) == cudaSuccess;
  if (!ok) {
    lbfgsb_b200_synth_destroy(c);
    return nullptr;
  }
  return c;
}

void lbfgsb_b200_synth_set_offset(void* handle, double f0) {
  if (handle) static_cast<SynthCtx*>(handle)->f0 = f0;
}

void lbfgsb_b200_synth_destroy(void* handle) {
  SynthCtx* c = static_cast<SynthCtx*>(handle);
  if (!c) return;
  for (int k = 0; k < 4; k++)
    if (c->field[k]) cudaFree(c->field[k]);
  if (c->part) cudaFree(c->part);
  if (c->fdev) cudaFree(c->fdev);
  if (c->ticket) cudaFree(c->ticket);
  if (c->fhost) cudaFreeHost(c->fhost);
  delete c;
}

int lbfgsb_b200_synth_funcgrad_f64(void* handle, double* x, double* f, double* g, void* stream,
                                   const lbfgsb_b200_summary_f64*) {
  return synth_eval<double>(handle, x, f, g, stream);
}

int lbfgsb_b200_synth_funcgrad_f32(void* handle, float* x, float* f, float* g, void* stream,
                                   const lbfgsb_b200_summary_f32*) {
  return synth_eval<float>(handle, x, f, g, stream);
}

int lbfgsb_b200_synth_device_f64(void* handle, const double* const* x, double* const* g,
                                 double* f, const int* active, void* stream) {
  return synth_device<double>(handle, x, g, f, active, stream);
}

int lbfgsb_b200_synth_device_f32(void* handle, const float* const* x, float* const* g,
                                 double* f, const int* active, void* stream) {
  return synth_device<float>(handle, x, g, f, active, stream);
}

}  // extern "C"
