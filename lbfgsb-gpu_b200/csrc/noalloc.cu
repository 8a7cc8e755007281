// noalloc.cu -- projected-gradient norm with no allocation at all.
//
// lbfgsb_b200_projgr_noalloc_f64 computes the reference's projgr
// (culbfgsb/lbfgsbcpu.cpp:1390-1415): sbgnrm = max_i |pg_i| with pg_i = g_i, clipped to
// x_i - u_i (g_i < 0, nbd_i >= 2) or x_i - l_i (g_i >= 0, nbd_i <= 2).  It is the same
// computation as the solver's k_projgr (which reports it as summary.residual_g), except
// that its scratch lives in the static device array below instead of the solver's
// workspace, so a call allocates nothing: no cudaMalloc/cudaFree, no pool, no pinned
// host memory.  Callers that cannot allocate are the solver's own callbacks
// (after_iteration, customized_stopping, funcgrad): they run in the middle of the
// solver's stream work, where cudaMalloc/cudaFree would synchronise the device.
//
// Scratch (shared by every call on a device):
//   word 0                  arrival ticket; must be 0 when a call starts.  It is 0 at
//                           module load and the last CTA of every call resets it to 0.
//   words 32 .. 32+rows-1   per-CTA maxima (bits of doubles); each CTA writes its own
//                           word before it takes a ticket, so they need no initial value.
// Calls that overlap on the GPU (on streams not ordered with each other) race on this
// scratch; issue them on one stream or order them with events.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/lbfgsb_b200.h"
#include "common.cuh"

namespace lbfgsb_b200 {

extern thread_local std::string g_last_error;

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerCta = 4096;   // elements per CTA (16 per thread)
constexpr int kNoAllocRows = 8192;     // per-CTA maxima: at most 8192 CTAs
constexpr long long kNoAllocMaxN = (long long)kNoAllocRows * kNoAllocPerCta;  // 2^25
constexpr int kNoAllocMaxDevices = 64;

// 64 KB of per-CTA maxima plus a 256-byte header holding the ticket.
static __device__ __align__(256) unsigned long long g_projgr_scratch[32 + kNoAllocRows];

__global__ void __launch_bounds__(kNoAllocThreads)
    k_projgr_noalloc(int n, const double* __restrict__ x, const double* __restrict__ g,
                     const int* __restrict__ nbd, const double* __restrict__ l,
                     const double* __restrict__ u, unsigned long long* scratch, double* out) {
  unsigned long long* ticket = scratch;
  unsigned long long* rows = scratch + 32;
  const long long base = (long long)blockIdx.x * kNoAllocPerCta;
  double m = 0.0;
  for (int k = threadIdx.x; k < kNoAllocPerCta; k += kNoAllocThreads) {
    const long long i = base + k;
    if (i >= n) break;
    const double xi = x[i], gi = g[i];
    const int nb = nbd[i];
    double pg = gi;
    if (nb != 0) {  // the reference's maxreal / minreal: (a > b) ? a : b, (a < b) ? a : b
      if (gi < 0.0) {
        if (nb >= 2) {
          const double d = __dsub_rn(xi, u[i]);
          pg = d > gi ? d : gi;
        }
      } else {
        if (nb <= 2) {
          const double d = __dsub_rn(xi, l[i]);
          pg = d < gi ? d : gi;
        }
      }
    }
    const double a = fabs(pg);
    m = a > m ? a : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, m, o);
    m = w > m ? w : m;
  }
  __shared__ double wm[kNoAllocThreads / 32];
  __shared__ bool last;
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = wm[0];
    for (int w = 1; w < kNoAllocThreads / 32; w++) c = wm[w] > c ? wm[w] : c;
    rows[blockIdx.x] = (unsigned long long)__double_as_longlong(c);
    __threadfence();
    last = atomicAdd(ticket, 1ull) == (unsigned long long)(gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double r = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kNoAllocThreads) {
    const double v = __longlong_as_double((long long)*(volatile unsigned long long*)&rows[b]);
    r = v > r ? v : r;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, r, o);
    r = w > r ? w : r;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = wm[0];
    for (int w = 1; w < kNoAllocThreads / 32; w++) c = wm[w] > c ? wm[w] : c;
    *out = c;
    *ticket = 0ull;  // ready for the next call
  }
}

// Address of the scratch on the current device, looked up once per device.
static int scratch_on_device(unsigned long long** ptr) {
  static std::mutex mu;
  static unsigned long long* cache[kNoAllocMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_last_error = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return LBFGSB_B200_ERR_CUDA;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    g_last_error = "lbfgsb_b200_projgr_noalloc_f64: device ordinal beyond 63";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!cache[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_projgr_scratch);
    if (e != cudaSuccess) {
      g_last_error = std::string("cudaGetSymbolAddress(g_projgr_scratch): ") + cudaGetErrorString(e);
      return LBFGSB_B200_ERR_CUDA;
    }
    cache[dev] = static_cast<unsigned long long*>(p);
  }
  *ptr = cache[dev];
  return LBFGSB_B200_OK;
}

}  // namespace lbfgsb_b200

using namespace lbfgsb_b200;

extern "C" int lbfgsb_b200_projgr_noalloc_f64(int n, const double* x, const double* g,
                                              const int* nbd, const double* l,
                                              const double* u, double* sbgnrm, void* stream) {
  g_last_error.clear();
  if (n < 0 || (long long)n > kNoAllocMaxN) {
    g_last_error = "lbfgsb_b200_projgr_noalloc_f64: n = " + std::to_string(n) +
                   " is outside 0..33554432 (the static scratch holds 8192 per-CTA maxima "
                   "of 4096 variables each)";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  if (!sbgnrm || (n > 0 && (!x || !g || !nbd || !l || !u))) {
    g_last_error = "lbfgsb_b200_projgr_noalloc_f64: null pointer argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  unsigned long long* scratch = nullptr;
  const int st = scratch_on_device(&scratch);
  if (st != LBFGSB_B200_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (n == 0) {
    e = cudaMemsetAsync(sbgnrm, 0, sizeof(double), s);  // the reference's sbgnrm = 0
  } else {
    const int rows = (int)(((long long)n + kNoAllocPerCta - 1) / kNoAllocPerCta);
    k_projgr_noalloc<<<rows, kNoAllocThreads, 0, s>>>(n, x, g, nbd, l, u, scratch, sbgnrm);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    g_last_error = std::string("lbfgsb_b200_projgr_noalloc_f64: ") + cudaGetErrorString(e);
    return LBFGSB_B200_ERR_CUDA;
  }
  return LBFGSB_B200_OK;
}
