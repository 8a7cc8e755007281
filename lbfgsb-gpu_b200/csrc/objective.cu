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
#include <vector>

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
  const R h = R(1) / (R)(s + 1), h2 = h * h;
  double acc = 0.0;
  // work units: segments of kThreads columns of one row (segs per row), unit u = CTA rank
  // + m * count for m = 0, 1, ...; the unit's row and segment are stepped along, so no
  // element needs a division to find its row and column
  const int segs = (s + kThreads - 1) / kThreads;
  const long long units = (long long)s * segs;
  const int dj = cp.count / segs, dseg = cp.count % segs;
  int j = cp.rank / segs, seg = cp.rank % segs;
  for (long long u = cp.rank; u < units; u += cp.count) {
    const int row = j, i = seg * kThreads + (int)threadIdx.x;
    seg += dseg;
    j += dj;
    if (seg >= segs) {
      seg -= segs;
      j++;
    }
    if (i >= s) continue;
    const long long k = (long long)row * s + i;
    const R xk = x[k];
    const R xe = (i + 1 < s) ? x[k + 1] : R(0);
    const R xn = (row + 1 < s) ? x[k + s] : R(0);
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
    if (row > 0) gk += (R)kap[k - s] * (xk - x[k - s]);
    gk += h2 * (wk * sigmoid - bk - R(0.15) * s3);
    g[k] = gk;
  }
  double sarr[1] = {acc}, xd[1] = {0.0}, ld[1] = {0.0};
  MinPair md[1] = {MinPair{0.0, 0}};
  cta_reduce_to_row<kThreads, 1, 0, 0, 0>(sarr, xd, md, ld, part, 1, cp.rank, cp.count);
  if (!last_cta(ticket, cp.count)) return;
  __shared__ double red[1];
  fold_rows<kThreads>(part, cp.count, 1, 1, 0, 0, red);
  if (threadIdx.x == 0) *fout = red[0] - f0;
}

// ---- a batch of synthetic problems, generated on the device ------------------------------
// The fields of problem p (grid side s_p, seed_p) are those of lbfgsb-gpu_b200/synth.py
// (synth_problem(s_p, seed_p)): the same counter-based generator in the same IEEE operations
// (splitmix64 draws, the Marsaglia polar method with the series logarithm), so they are
// bit-identical to the host generator's.
__device__ __forceinline__ unsigned long long synth_stream_base(unsigned long long seed, int field) {
  return mix64(seed ^ ((unsigned long long)field * 0xD1B54A32D192ED03ULL));
}
__device__ __forceinline__ double synth_uniform(unsigned long long base, long long k, int draw) {
  const unsigned long long z = mix64(base + ((unsigned long long)k << 6) + (unsigned long long)draw);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ double synth_log(double x) {
  int e;
  double m = frexp(x, &e);
  if (m < 0.7071067811865476) {
    m = m * 2.0;
    e = e - 1;
  }
  const double z = (m - 1.0) / (m + 1.0), z2 = z * z;
  double acc = 0.0;
  for (int odd = 27; odd > 1; odd -= 2) acc = acc * z2 + 1.0 / (double)odd;
  acc = acc * z2 + 1.0;
  return (double)e * 0.6931471805599453 + 2.0 * z * acc;
}
__device__ __forceinline__ double synth_normal(unsigned long long base, long long k) {
  for (int attempt = 0; attempt < 32; attempt++) {
    const double u = 2.0 * synth_uniform(base, k, 2 * attempt) - 1.0;
    const double v = 2.0 * synth_uniform(base, k, 2 * attempt + 1) - 1.0;
    const double sq = u * u + v * v;
    if (sq > 0.0 && sq < 1.0) return u * __dsqrt_rn(-2.0 * synth_log(sq) / sq);
  }
  return 0.0;
}

struct SynthDesc {
  int s;
  int pad;
  long long off;  // first element of the problem in the packed arrays
  unsigned long long seed;
};

// the problem holding packed element e (the largest p with off[p] <= e)
__device__ __forceinline__ int synth_problem_of(const SynthDesc* d, int count, long long e) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d[mid].off <= e)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <typename F, typename RB>
__global__ void k_synth_generate(const SynthDesc* d, int count, long long total, F* kap, F* w,
                                 F* tt, F* b, RB* l, RB* u, int* nbd) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int p = synth_problem_of(d, count, e);
    const long long k = e - d[p].off;
    if (k >= (long long)d[p].s * d[p].s) continue;  // alignment padding between problems
    const unsigned long long seed = d[p].seed;
    kap[e] = (F)(0.5 + 1.5 * synth_uniform(synth_stream_base(seed, 1), k, 0));
    w[e] = (F)synth_uniform(synth_stream_base(seed, 2), k, 0);
    tt[e] = (F)synth_normal(synth_stream_base(seed, 3), k);
    b[e] = (F)(2.0 * synth_normal(synth_stream_base(seed, 4), k));
    const double r = synth_uniform(synth_stream_base(seed, 5), k, 0);
    nbd[e] = r < 0.8 ? 2 : (r < 0.9 ? 1 : 0);
    l[e] = (RB)-1.0;
    u[e] = (RB)1.0;
  }
}

// The batched objective: entry j (problem ids[j]) owns CTAs first[j] .. first[j+1]-1 and
// reduces f over that problem's rows and ticket.
template <typename R, typename F>
__global__ void __launch_bounds__(kThreads) k_synth_batch(const SynthDesc* d, const F* kap,
                                                          const F* w, const F* tt, const F* b,
                                                          int count, const int* ids,
                                                          const int* first, const R* const* xs,
                                                          R* const* gs, double* f,
                                                          const int* active, double* part,
                                                          unsigned int* tickets, int rows) {
  __shared__ int s_j;
  if (threadIdx.x == 0) {
    int lo = 0, hi = count - 1;
    const int bi = (int)blockIdx.x;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (first[mid] <= bi)
        lo = mid;
      else
        hi = mid - 1;
    }
    s_j = lo;
  }
  __syncthreads();
  const int j = s_j;
  if (!active[j]) return;
  const int p = ids[j];
  const long long off = d[p].off;
  const CtaPos cp{(int)blockIdx.x - first[j], first[j + 1] - first[j]};
  synth_body<R, F>(d[p].s, xs[j], kap + off, w + off, tt + off, b + off, gs[j],
                   part + (size_t)p * rows, tickets + p, 0.0, f + j, cp);
}

struct SynthBatch {
  int count = 0, single = 0, real_size = 8;
  long long total = 0;
  std::vector<SynthDesc> desc;
  SynthDesc* desc_dev = nullptr;
  void* field[4] = {nullptr, nullptr, nullptr, nullptr};
  void* l = nullptr;
  void* u = nullptr;
  int* nbd = nullptr;
  double* part = nullptr;
  unsigned int* tickets = nullptr;
  static constexpr int kRows = 64;  // reduction rows per problem (the most a batched launch gives)
};

template <typename R>
static int synth_batch_eval(void* handle, int count, const int* ids, const int* first, int ctas,
                            const R* const* x, R* const* g, double* f, const int* active,
                            void* stream) {
  SynthBatch* h = static_cast<SynthBatch*>(handle);
  cudaStream_t s = (cudaStream_t)stream;
  if (count <= 0 || ctas <= 0) return 0;
  if (h->single)
    k_synth_batch<R, float><<<ctas, kThreads, 0, s>>>(
        h->desc_dev, (const float*)h->field[0], (const float*)h->field[1],
        (const float*)h->field[2], (const float*)h->field[3], count, ids, first, x, g, f, active,
        h->part, h->tickets, SynthBatch::kRows);
  else
    k_synth_batch<R, double><<<ctas, kThreads, 0, s>>>(
        h->desc_dev, (const double*)h->field[0], (const double*)h->field[1],
        (const double*)h->field[2], (const double*)h->field[3], count, ids, first, x, g, f, active,
        h->part, h->tickets, SynthBatch::kRows);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
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

void* lbfgsb_b200_synth_batch_create(int count, const int* sides, const unsigned long long* seeds,
                                     int single_precision_fields, int real_size) {
  if (count <= 0 || !sides || !seeds || (real_size != 4 && real_size != 8)) return nullptr;
  SynthBatch* h = new SynthBatch();
  h->count = count;
  h->single = single_precision_fields ? 1 : 0;
  h->real_size = real_size;
  h->desc.resize(count);
  long long off = 0;
  for (int p = 0; p < count; p++) {
    if (sides[p] <= 0) {
      delete h;
      return nullptr;
    }
    h->desc[p].s = sides[p];
    h->desc[p].pad = 0;
    h->desc[p].off = off;
    h->desc[p].seed = seeds[p];
    off += (long long)sides[p] * sides[p];
    off = (off + 63) / 64 * 64;  // every problem's arrays start 256-byte aligned
  }
  h->total = off;
  const size_t fb = h->single ? 4 : 8;
  bool ok = cudaMalloc(&h->desc_dev, count * sizeof(SynthDesc)) == cudaSuccess &&
            cudaMemcpy(h->desc_dev, h->desc.data(), count * sizeof(SynthDesc),
                       cudaMemcpyHostToDevice) == cudaSuccess;
  for (int k = 0; k < 4 && ok; k++) {
    ok = cudaMalloc(&h->field[k], (size_t)off * fb) == cudaSuccess &&
         cudaMemset(h->field[k], 0, (size_t)off * fb) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&h->l, (size_t)off * real_size) == cudaSuccess;
  ok = ok && cudaMalloc(&h->u, (size_t)off * real_size) == cudaSuccess;
  ok = ok && cudaMalloc(&h->nbd, (size_t)off * 4) == cudaSuccess;
  ok = ok && cudaMalloc(&h->part, (size_t)count * SynthBatch::kRows * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&h->tickets, (size_t)count * sizeof(unsigned int)) == cudaSuccess;
  ok = ok && cudaMemset(h->tickets, 0, (size_t)count * sizeof(unsigned int)) == cudaSuccess;
  ok = ok && cudaMemset(h->nbd, 0, (size_t)off * 4) == cudaSuccess;
  if (ok) {
    const int grid = 148 * 8;
    if (h->single && real_size == 4)
      k_synth_generate<float, float><<<grid, 256>>>(h->desc_dev, count, off, (float*)h->field[0],
          (float*)h->field[1], (float*)h->field[2], (float*)h->field[3], (float*)h->l,
          (float*)h->u, h->nbd);
    else if (h->single)
      k_synth_generate<float, double><<<grid, 256>>>(h->desc_dev, count, off, (float*)h->field[0],
          (float*)h->field[1], (float*)h->field[2], (float*)h->field[3], (double*)h->l,
          (double*)h->u, h->nbd);
    else if (real_size == 4)
      k_synth_generate<double, float><<<grid, 256>>>(h->desc_dev, count, off, (double*)h->field[0],
          (double*)h->field[1], (double*)h->field[2], (double*)h->field[3], (float*)h->l,
          (float*)h->u, h->nbd);
    else
      k_synth_generate<double, double><<<grid, 256>>>(h->desc_dev, count, off, (double*)h->field[0],
          (double*)h->field[1], (double*)h->field[2], (double*)h->field[3], (double*)h->l,
          (double*)h->u, h->nbd);
    ok = cudaDeviceSynchronize() == cudaSuccess;
  }
  if (!ok) {
    lbfgsb_b200_synth_batch_destroy(h);
    return nullptr;
  }
  return h;
}

void lbfgsb_b200_synth_batch_destroy(void* handle) {
  SynthBatch* h = static_cast<SynthBatch*>(handle);
  if (!h) return;
  if (h->desc_dev) cudaFree(h->desc_dev);
  for (int k = 0; k < 4; k++)
    if (h->field[k]) cudaFree(h->field[k]);
  if (h->l) cudaFree(h->l);
  if (h->u) cudaFree(h->u);
  if (h->nbd) cudaFree(h->nbd);
  if (h->part) cudaFree(h->part);
  if (h->tickets) cudaFree(h->tickets);
  delete h;
}

int lbfgsb_b200_synth_batch_problem(void* handle, int p, void** l, void** u, int** nbd,
                                    void* fields[4]) {
  SynthBatch* h = static_cast<SynthBatch*>(handle);
  if (!h || p < 0 || p >= h->count) return 1;
  const long long off = h->desc[p].off;
  const size_t fb = h->single ? 4 : 8;
  if (l) *l = (unsigned char*)h->l + (size_t)off * h->real_size;
  if (u) *u = (unsigned char*)h->u + (size_t)off * h->real_size;
  if (nbd) *nbd = h->nbd + off;
  if (fields)
    for (int k = 0; k < 4; k++) fields[k] = (unsigned char*)h->field[k] + (size_t)off * fb;
  return 0;
}

int lbfgsb_b200_synth_batch_f64(void* handle, int count, const int* ids, const int* first,
                                int ctas, const double* const* x, double* const* g, double* f,
                                const int* active, void* stream) {
  return synth_batch_eval<double>(handle, count, ids, first, ctas, x, g, f, active, stream);
}

int lbfgsb_b200_synth_batch_f32(void* handle, int count, const int* ids, const int* first,
                                int ctas, const float* const* x, float* const* g, double* f,
                                const int* active, void* stream) {
  return synth_batch_eval<float>(handle, count, ids, first, ctas, x, g, f, active, stream);
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
