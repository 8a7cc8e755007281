// A program written against the reference's public API (culbfgsb.h), as in its dsscfg
// example (examples/dsscfg/dsscfg_main.cpp:115-190): option defaults, a cuBLAS-handle
// field left null, a std::function device callback, lbfgsbcuda::lbfgsbminimize.  It builds
// unchanged against include/culbfgsb.h and runs on liblbfgsb_b200.so.
//   argv[1] = grid side s (objective: separable quadratic sum 0.5*a_k*(x_k - c_k)^2)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "culbfgsb.h"

template <typename real>
__global__ void quad_fg(int n, const real* x, real* g, double* fpart) {
  double acc = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const real a = (real)(1.0 + 0.5 * (k % 3)), c = (real)(k % 2 ? 0.7 : -1.3);
    const real r = x[k] - c;
    g[k] = a * r;
    acc += 0.5 * (double)(a * r * r);
  }
  atomicAdd(fpart, acc);  // order varies; fine for this example
}

template <typename real>
int run(int n) {
  LBFGSB_CUDA_OPTION<real> opt;
  lbfgsbcuda::lbfgsbdefaultoption<real>(opt);
  opt.mode = LCM_CUDA;
  opt.eps_f = opt.eps_g = opt.eps_x = (real)1e-10;
  opt.max_iteration = 200;

  LBFGSB_CUDA_STATE<real> state;
  memset(&state, 0, sizeof(state));
  double* fpart = nullptr;
  cudaMalloc(&fpart, sizeof(double));
  int calls = 0;
  state.m_funcgrad_callback = [&](real* x, real& f, real* g, const cudaStream_t& stream,
                                  const LBFGSB_CUDA_SUMMARY<real>& summary) {
    cudaMemsetAsync(fpart, 0, sizeof(double), stream);
    quad_fg<real><<<64, 256, 0, stream>>>(n, x, g, fpart);
    double h = 0;
    cudaMemcpyAsync(&h, fpart, sizeof(double), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    f = (real)h;
    calls++;
    return 0;
  };

  real *x, *xl, *xu;
  int* nbd;
  cudaMalloc(&x, n * sizeof(real));
  cudaMalloc(&xl, n * sizeof(real));
  cudaMalloc(&xu, n * sizeof(real));
  cudaMalloc(&nbd, n * sizeof(int));
  std::vector<real> hl(n, (real)-1), hu(n, (real)0.5);
  std::vector<int> hb(n, 2);
  cudaMemcpy(xl, hl.data(), n * sizeof(real), cudaMemcpyHostToDevice);
  cudaMemcpy(xu, hu.data(), n * sizeof(real), cudaMemcpyHostToDevice);
  cudaMemcpy(nbd, hb.data(), n * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemset(x, 0, n * sizeof(real));

  LBFGSB_CUDA_SUMMARY<real> summary;
  memset(&summary, 0, sizeof(summary));
  lbfgsbcuda::lbfgsbminimize<real>(n, state, opt, x, nbd, xl, xu, summary);

  std::vector<real> hx(n);
  cudaMemcpy(hx.data(), x, n * sizeof(real), cudaMemcpyDeviceToHost);
  // the minimiser is clamp(c, l, u): -1 for c = -1.3, 0.5 for c = 0.7
  double err = 0;
  for (int k = 0; k < n; k++) {
    const double want = (k % 2) ? 0.5 : -1.0;
    err = std::max(err, std::abs((double)hx[k] - want));
  }
  printf("%s n=%d info=%d iterations=%d evaluations=%d max|x-x*|=%.3e\n",
         sizeof(real) == 8 ? "double" : "float", n, summary.info, summary.num_iteration, calls,
         err);
  cudaFree(x);
  cudaFree(xl);
  cudaFree(xu);
  cudaFree(nbd);
  cudaFree(fpart);
  return (summary.info >= 0 && err < (sizeof(real) == 8 ? 1e-8 : 1e-4)) ? 0 : 1;
}

int main(int argc, char** argv) {
  const int s = argc > 1 ? atoi(argv[1]) : 64;
  const int rc = run<double>(s * s) | run<float>(s * s);
  printf(rc == 0 ? "OK\n" : "FAILED\n");
  return rc;
}
