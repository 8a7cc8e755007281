// dsscfg.cu -- the steady-state combustion objective of the reference's example program
// (examples/dsscfg/dsscfg_cuda.cu; MINPACK-2 dsscfg, Averick, Carter, More and Xue, 1992)
// as a device funcgrad callback, for the example's workload and the parity tests.
//
// nx x ny nodes, k = nx*j + i, hx = 1/(nx+1), hy = 1/(ny+1), zero values outside the
// grid; every node owns a lower triangle (itself, right, top) and an upper triangle
// (itself, left, bottom):
//
//   f = area * (0.5 * sum over triangles of |grad v|^2 - lambda/3 * sum over triangles of
//       the exponentials of their corners),  area = hx*hy/2.
//
// One thread per node gathers its gradient from the six triangles that touch it, in the
// order own lower, own upper, above, right, left, below (each term as the reference forms
// it).  For f, a node's exponential appears once in each triangle that has it as a
// corner (2 + one per existing neighbour), and the zero values outside the grid add
// exp(0) = 1 for 2*(nx + ny) corners; the squared differences are summed per node's two
// triangles.  Both sums run in double through per-CTA rows folded in CTA order by the last
// CTA (bitwise reproducible); the callback synchronises the stream to return f.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "../../include/lbfgsb_b200.h"
#include "common.cuh"
#include "reduce.cuh"

namespace lbfgsb_b200 {

struct DsscfgCtx {
  int nx, ny;
  double lam;
  double* part;
  double* fdev;
  double* fhost;  // pinned
  unsigned int* ticket;
  int grid[2];    // one wave of CTAs of the double / float kernel
};

__device__ __forceinline__ double dexp(double v) { return exp(v); }
__device__ __forceinline__ float dexp(float v) { return expf(v); }

template <typename R>
__global__ void __launch_bounds__(kThreads) k_dsscfg(int nx, int ny, R lam, const R* __restrict__ x,
                                                     R* __restrict__ g, double* part,
                                                     unsigned int* ticket, double* fout) {
  const long long n = (long long)nx * ny;
  const R hx = (R)(1.0 / (double)(nx + 1)), hy = (R)(1.0 / (double)(ny + 1));
  const R area = (R)(0.5 * (double)hx * (double)hy);
  double fquad = 0.0, fexp = 0.0;
  for (long long k = (long long)blockIdx.x * kThreads + threadIdx.x; k < n;
       k += (long long)gridDim.x * kThreads) {
    const int i = (int)(k % nx), j = (int)(k / nx);
    const R v = x[k];
    const R vr = i < nx - 1 ? x[k + 1] : R(0), vt = j < ny - 1 ? x[k + nx] : R(0);
    const R vl = i > 0 ? x[k - 1] : R(0), vb = j > 0 ? x[k - nx] : R(0);
    const R dxl = (vr - v) / hx, dyl = (vt - v) / hy;  // own lower triangle
    const R dxu = (v - vl) / hx, dyu = (v - vb) / hy;  // own upper triangle
    fquad += (double)(dxl * dxl + dyl * dyl) + (double)(dxu * dxu + dyu * dyu);
    const R ev = dexp(v);
    const int corners = 2 + (i > 0) + (j > 0) + (i < nx - 1) + (j < ny - 1);
    fexp += (double)corners * (double)ev;
    const R e3 = lam * ev / R(3);
    R gk = (-dxl / hx - dyl / hy - e3) + (dxu / hx + dyu / hy - e3);
    gk = gk + (j < ny - 1 ? -dyl / hy - e3 : R(0));
    gk = gk + (i < nx - 1 ? -dxl / hx - e3 : R(0));
    gk = gk + (i > 0 ? dxu / hx - e3 : R(0));
    gk = gk + (j > 0 ? dyu / hy - e3 : R(0));
    g[k] = gk * area;
  }
  double sarr[2] = {fquad, fexp}, xd[1] = {0.0}, ld[1] = {0.0};
  MinPair md[1] = {MinPair{0.0, 0}};
  cta_reduce_to_row<kThreads, 2, 0, 0, 0>(sarr, xd, md, ld, part, 2, (int)blockIdx.x,
                                          (int)gridDim.x);
  if (!last_cta(ticket, (int)gridDim.x)) return;
  __shared__ double red[2];
  fold_rows<kThreads>(part, gridDim.x, 2, 2, 0, 0, red);
  if (threadIdx.x == 0) {
    const double boundary = 2.0 * ((double)nx + (double)ny);
    *fout = (double)area * (0.5 * red[0] - (double)lam / 3.0 * (red[1] + boundary));
  }
}

// The example's standard start point: lambda/(lambda+1) * sqrt(min(dist_x, dist_y)),
// with dist the smaller node distance to the two edges of each axis.
template <typename R>
__global__ void k_dsscfg_start(int nx, int ny, R lam, R* __restrict__ x) {
  const long long n = (long long)nx * ny;
  const R hx = (R)(1.0 / (double)(nx + 1)), hy = (R)(1.0 / (double)(ny + 1));
  const R c = (R)((double)lam / ((double)lam + 1.0));
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % nx), j = (int)(k / nx);
    const R ty = (R)(j < ny - j ? j : ny - j) * hy;
    const R tx = (R)(i < nx - i ? i : nx - i) * hx;
    x[k] = c * sqrt(ty < tx ? ty : tx);
  }
}

template <typename R>
static int dsscfg_eval(void* handle, R* x, R* f, R* g, void* stream) {
  DsscfgCtx* c = static_cast<DsscfgCtx*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  k_dsscfg<R><<<c->grid[sizeof(R) == 8 ? 0 : 1], kThreads, 0, s>>>(c->nx, c->ny, (R)c->lam, x, g,
                                                                   c->part, c->ticket, c->fdev);
  cudaMemcpyAsync(c->fhost, c->fdev, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
  *f = (R)*c->fhost;
  return 0;
}

template <typename R>
static int dsscfg_start(void* handle, R* x, void* stream) {
  DsscfgCtx* c = static_cast<DsscfgCtx*>(handle);
  if (!c || !x) return LBFGSB_B200_ERR_ARGUMENT;
  const long long n = (long long)c->nx * c->ny;
  const int grid = (int)((n + kThreads - 1) / kThreads < 4096 ? (n + kThreads - 1) / kThreads : 4096);
  k_dsscfg_start<R><<<grid, kThreads, 0, (cudaStream_t)stream>>>(c->nx, c->ny, (R)c->lam, x);
  return cudaGetLastError() == cudaSuccess ? LBFGSB_B200_OK : LBFGSB_B200_ERR_CUDA;
}

}  // namespace lbfgsb_b200

using namespace lbfgsb_b200;

extern "C" {

void* lbfgsb_b200_dsscfg_create(int nx, int ny, double lambda) {
  if (nx <= 0 || ny <= 0 || (long long)nx * ny > 0x7fffffffLL) return nullptr;
  DsscfgCtx* c = new DsscfgCtx();
  std::memset(c, 0, sizeof(*c));
  c->nx = nx;
  c->ny = ny;
  c->lam = lambda;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = ((long long)nx * ny + kThreads - 1) / kThreads;
  for (int r = 0; r < 2; r++) {
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, r == 0 ? (const void*)k_dsscfg<double> : (const void*)k_dsscfg<float>, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    c->grid[r] = (int)(want < (long long)sms * per_sm ? want : (long long)sms * per_sm);
  }
  const int rows = c->grid[0] > c->grid[1] ? c->grid[0] : c->grid[1];
  bool ok = cudaMalloc(&c->part, (size_t)rows * 2 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->fdev, sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->ticket, sizeof(unsigned int)) == cudaSuccess;
  ok = ok && cudaMemset(c->ticket, 0, sizeof(unsigned int)) == cudaSuccess;
  ok = ok && cudaMallocHost(&c->fhost, sizeof(double)) == cudaSuccess;
  if (!ok) {
    lbfgsb_b200_dsscfg_destroy(c);
    return nullptr;
  }
  return c;
}

void lbfgsb_b200_dsscfg_destroy(void* handle) {
  DsscfgCtx* c = static_cast<DsscfgCtx*>(handle);
  if (!c) return;
  if (c->part) cudaFree(c->part);
  if (c->fdev) cudaFree(c->fdev);
  if (c->ticket) cudaFree(c->ticket);
  if (c->fhost) cudaFreeHost(c->fhost);
  delete c;
}

int lbfgsb_b200_dsscfg_funcgrad_f64(void* handle, double* x, double* f, double* g, void* stream,
                                    const lbfgsb_b200_summary_f64*) {
  return dsscfg_eval<double>(handle, x, f, g, stream);
}

int lbfgsb_b200_dsscfg_funcgrad_f32(void* handle, float* x, float* f, float* g, void* stream,
                                    const lbfgsb_b200_summary_f32*) {
  return dsscfg_eval<float>(handle, x, f, g, stream);
}

int lbfgsb_b200_dsscfg_start_f64(void* handle, double* x, void* stream) {
  return dsscfg_start<double>(handle, x, stream);
}

int lbfgsb_b200_dsscfg_start_f32(void* handle, float* x, void* stream) {
  return dsscfg_start<float>(handle, x, stream);
}

}  // extern "C"
