// walk.cuh -- the breakpoint walk of the generalized Cauchy point (the part of
// culbfgsb/lbfgsbcpu.cpp:725-816 after the first breakpoint test).
//
// The reference keeps the breakpoints in a heap (hpsolb, 1175-1233) and pops them one at
// a time.  Here, only when the scan found that the first breakpoint is passed:
//   k_walk_gather  lists every breakpoint (t_i, i) (one grid-wide pass; same arithmetic
//                  as the scan, so the same t_i);
//   k_walk         one CTA repeatedly selects the next chunk of the smallest remaining
//                  breakpoints (radix select on the 96-bit key (bits of t, i) over the
//                  list), sorts the chunk in shared memory, computes each candidate's
//                  row of W, M*wbp and wbp'M wbp in parallel, and walks the chunk in key
//                  order on one thread with the reference's recurrence for f', f'', c, p.
// Breakpoints with equal t are passed in increasing variable index (the heap's order
// among exact ties is an artefact of its layout).
#pragma once

#include "common.cuh"
#include "passes.cuh"
#include "small.cuh"
#include "state.cuh"

namespace lbfgsb_b200 {

template <typename R, typename H, typename S>
__device__ __forceinline__ void walk_gather_pass(const Ctx<R, H, S>& c, CtaPos cp,
                                                 const R* __restrict__ x, const R* __restrict__ g) {
  if (c.rounds) {
    const DevState<S>* st = c.st;
    if (!st->rp_sub || st->gcp_state != GCP_WALK || st->internal_fail != 0) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
  }
  const int n = c.n;
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)cp.rank * kThreads; base < n;
       base += (long long)cp.count * kThreads) {
    const long long i = base + threadIdx.x;
    bool has_bp = false;
    R t = 0;
    if (i < n) classify(x[i], g[i], c.l[i], c.u[i], c.nbd[i], has_bp, t);
    const uint32_t mask = __ballot_sync(0xffffffffu, has_bp);
    if (mask == 0) continue;
    unsigned int start = 0;
    if (lane == 0) start = atomicAdd(c.wl_n, (unsigned int)__popc(mask));
    start = __shfl_sync(0xffffffffu, start, 0);
    if (has_bp) {
      const unsigned int pos = start + __popc(mask & ((1u << lane) - 1u));
      c.wl_t[pos] = (double)t;
      c.wl_i[pos] = (int)i;
    }
  }
}
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kThreads) k_walk_gather(Ctx<R, H, S> c, const R* __restrict__ x,
                                                          const R* __restrict__ g) {
  walk_gather_pass<R, H, S>(c, cta_here(), x, g);
}

constexpr int kWalkThreads = 512;
constexpr int kChunk = 1024;  // breakpoints selected and sorted per round
constexpr int kBatch = 64;    // candidates prepared in parallel per walking step

struct Key96 {
  unsigned long long hi;  // bits of t (t >= 0, so the bits order like the values)
  unsigned int lo;        // variable index
};
__device__ __forceinline__ bool key_less(const Key96& a, const Key96& b) {
  return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}
__device__ __forceinline__ Key96 make_key(double t, int i) {
  return Key96{(unsigned long long)__double_as_longlong(t), (unsigned int)i};
}
__device__ __forceinline__ int key_digit(const Key96& k, int level) {
  return level < 8 ? (int)((k.hi >> (56 - 8 * level)) & 255ull) : (int)((k.lo >> (24 - 8 * (level - 8))) & 255u);
}
// true when the first `level` digits of k equal those of p
__device__ __forceinline__ bool key_prefix_eq(const Key96& k, const Key96& p, int level) {
  if (level == 0) return true;
  if (level <= 8) {
    const int sh = 64 - 8 * level;
    return (sh == 0) ? k.hi == p.hi : (k.hi >> sh) == (p.hi >> sh);
  }
  if (k.hi != p.hi) return false;
  const int sh = 32 - 8 * (level - 8);
  return (sh == 0) ? k.lo == p.lo : (k.lo >> sh) == (p.lo >> sh);
}
__device__ __forceinline__ void key_set_digit(Key96& k, int level, int d) {
  if (level < 8) {
    const int sh = 56 - 8 * level;
    k.hi = (k.hi & ~(255ull << sh)) | ((unsigned long long)d << sh);
  } else {
    const int sh = 24 - 8 * (level - 8);
    k.lo = (k.lo & ~(255u << sh)) | ((unsigned int)d << sh);
  }
}

template <typename R, typename H, typename S>
__device__ __forceinline__ void walk_pass(const Ctx<R, H, S>& c, const R* __restrict__ x,
                                          const R* __restrict__ g) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!st->rp_sub || st->internal_fail != 0) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
  }
  if (st->gcp_state != GCP_WALK) return;
  const int n = c.n, col = st->col, col2 = 2 * col;
  const long long L = *c.wl_n;
  const S theta = st->theta;
  const H *Y[kMaxM], *Sl[kMaxM];
  ring_ptrs(st, c.wy, c.ld, Y);
  ring_ptrs(st, c.ws, c.ld, Sl);

  __shared__ unsigned long long k_hi[kChunk];
  __shared__ unsigned int k_lo[kChunk];
  __shared__ unsigned int hist[256];
  __shared__ int sh_count, sh_done;
  __shared__ Key96 sh_prefix, sh_last;
  __shared__ long long sh_kk;
  __shared__ S b_wbp[kBatch][2 * kMaxM + 1];
  __shared__ S b_v[kBatch][2 * kMaxM + 1];
  __shared__ S b_wmw[kBatch], b_dibp[kBatch], b_zibp[kBatch];
  __shared__ S b_work[kBatch][kMaxM + 1];
  __shared__ int b_info;

  // walk state (thread 0 only)
  S f1 = st->f1, f2 = st->f2, f2org = st->f2org, dtm = st->dtm, tsum = st->tsum, tj = st->tj;
  int nleft = st->nleft, nint = st->nint;
  const int nbreak = st->nbreak, bnded = st->bnded;
  bool all_fixed = false;

  if (threadIdx.x == 0) {
    sh_done = 0;
    sh_last = Key96{0ull, 0u};
    b_info = 0;
  }
  __syncthreads();
  bool first_round = true;
  long long consumed = 0;
  while (true) {
    // ---- select the next chunk: the kChunk smallest keys greater than sh_last ----
    const long long remaining = L - consumed;
    Key96 thr;
    thr.hi = ~0ull;
    thr.lo = ~0u;
    if (remaining > kChunk) {
      if (threadIdx.x == 0) {
        sh_prefix = Key96{0ull, 0u};
        sh_kk = kChunk;
      }
      __syncthreads();
      for (int level = 0; level < 12; level++) {
        for (int b = threadIdx.x; b < 256; b += kWalkThreads) hist[b] = 0;
        __syncthreads();
        const Key96 pre = sh_prefix, last = sh_last;
        for (long long e = threadIdx.x; e < L; e += kWalkThreads) {
          const Key96 k = make_key(c.wl_t[e], c.wl_i[e]);
          if (!first_round && !key_less(last, k)) continue;
          if (!key_prefix_eq(k, pre, level)) continue;
          atomicAdd(&hist[key_digit(k, level)], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          long long cum = 0, kk = sh_kk;
          int d = 255;
          for (int b = 0; b < 256; b++) {
            if (cum + hist[b] >= kk) {
              d = b;
              break;
            }
            cum += hist[b];
          }
          sh_kk = kk - cum;
          Key96 p = sh_prefix;
          key_set_digit(p, level, d);
          sh_prefix = p;
        }
        __syncthreads();
      }
      thr = sh_prefix;
    }
    // ---- extract keys in (sh_last, thr] into shared memory ----
    if (threadIdx.x == 0) sh_count = 0;
    __syncthreads();
    {
      const Key96 last = sh_last;
      for (long long e = threadIdx.x; e < L; e += kWalkThreads) {
        const Key96 k = make_key(c.wl_t[e], c.wl_i[e]);
        if (!first_round && !key_less(last, k)) continue;
        if (key_less(thr, k)) continue;
        const int pos = atomicAdd(&sh_count, 1);
        if (pos < kChunk) {
          k_hi[pos] = k.hi;
          k_lo[pos] = k.lo;
        }
      }
    }
    __syncthreads();
    const int cnt = sh_count < kChunk ? sh_count : kChunk;
    // ---- bitonic sort of the chunk by (hi, lo), padded with maximal keys ----
    for (int e = cnt + threadIdx.x; e < kChunk; e += kWalkThreads) {
      k_hi[e] = ~0ull;
      k_lo[e] = ~0u;
    }
    __syncthreads();
    for (int size = 2; size <= kChunk; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int e = threadIdx.x; e < kChunk; e += kWalkThreads) {
          const int p = e ^ stride;
          if (p > e) {
            const bool up = (e & size) == 0;
            const Key96 a{k_hi[e], k_lo[e]}, b{k_hi[p], k_lo[p]};
            if (key_less(b, a) == up) {
              k_hi[e] = b.hi;
              k_lo[e] = b.lo;
              k_hi[p] = a.hi;
              k_lo[p] = a.lo;
            }
          }
        }
        __syncthreads();
      }
    }
    // ---- walk the chunk in batches ----
    for (int b0 = 0; b0 < cnt; b0 += kBatch) {
      const int nb = (cnt - b0) < kBatch ? (cnt - b0) : kBatch;
      if (threadIdx.x < nb) {
        const int k = b0 + threadIdx.x;
        const int i = (int)k_lo[k];
        const R xi = x[i], gi = g[i];
        const R dibp = -gi;
        const R zibp = (dibp > R(0)) ? rsub(c.u[i], xi) : rsub(c.l[i], xi);
        b_dibp[threadIdx.x] = (S)dibp;
        b_zibp[threadIdx.x] = (S)zibp;
        S* wbp = b_wbp[threadIdx.x];
        for (int j = 0; j < col; j++) {
          wbp[1 + j] = (S)HistTraits<H>::load(Y[j] + i);
          wbp[1 + col + j] = theta * (S)HistTraits<H>::load(Sl[j] + i);
        }
        if (col > 0) {
          int info = 0;
          sbmv(st->sy, st->wt, col, wbp, b_v[threadIdx.x], &info, b_work[threadIdx.x]);
          if (info != 0) atomicExch(&b_info, info);
          b_wmw[threadIdx.x] = sdot(&wbp[1], 1, &b_v[threadIdx.x][1], 1, col2);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        if (b_info != 0) {
          st->internal_fail = b_info;
          sh_done = 2;
        }
        for (int q = 0; q < nb && sh_done == 0; q++) {
          const int k = b0 + q;
          const S tk = (S)__longlong_as_double((long long)k_hi[k]);
          const int ibp = (int)k_lo[k];
          const S tj0 = tj;
          tj = tk;
          const S dt = tj - tj0;
          if (dtm < dt) {
            sh_done = 1;
            break;
          }
          tsum = tsum + dt;
          nleft = nleft - 1;
          const S dibp = b_dibp[q];
          c.code[ibp] = (int8_t)(dibp > S(0) ? IW_WALK_UPP : IW_WALK_LOW);
          if (nleft == 0 && nbreak == n) {
            dtm = dt;
            for (int j = 1; j <= col2; j++) st->c[j] += dtm * st->p[j];
            all_fixed = true;
            sh_done = 1;
            break;
          }
          nint = nint + 1;
          const S dibp2 = dibp * dibp;
          f1 = f1 + dt * f2 + dibp2 - theta * dibp * b_zibp[q];
          f2 = f2 - theta * dibp2;
          if (col > 0) {
            for (int j = 1; j <= col2; j++) st->c[j] += dt * st->p[j];
            const S wmc = sdot(&st->c[1], 1, &b_v[q][1], 1, col2);
            const S wmp = sdot(&st->p[1], 1, &b_v[q][1], 1, col2);
            const S wmw = b_wmw[q];
            for (int j = 1; j <= col2; j++) st->p[j] += (-dibp) * b_wbp[q][j];
            f1 = f1 + dibp * wmc;
            f2 = f2 + (S)2.0 * dibp * wmp - dibp2 * wmw;
          }
          f2 = smax((S)(5e-16 * (double)f2org), f2);
          if (nleft > 0) {
            dtm = -f1 / f2;
            continue;
          }
          if (bnded) {
            f1 = 0;
            f2 = 0;
            dtm = 0;
          } else {
            dtm = -f1 / f2;
          }
          sh_done = 1;
          break;
        }
      }
      __syncthreads();
      if (sh_done) break;
    }
    consumed += cnt;
    if (sh_done || consumed >= L || cnt == 0) break;
    if (threadIdx.x == 0) sh_last = Key96{k_hi[cnt - 1], k_lo[cnt - 1]};
    first_round = false;
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (sh_done == 2) return;  // a failed M*wbp: the driver resets the memory
  if (!all_fixed) {
    if (dtm <= S(0)) dtm = 0;
    tsum = tsum + dtm;
    for (int j = 1; j <= col2; j++) st->c[j] += dtm * st->p[j];
  }
  st->f1 = f1;
  st->f2 = f2;
  st->dtm = dtm;
  st->tsum = tsum;
  st->tj = tj;
  st->nleft = nleft;
  st->nint = nint;
  if (col > 0) {
    int info = 0;
    sbmv(st->sy, st->wt, col, st->c, st->mc, &info, b_work[0]);
    if (info != 0) {
      st->internal_fail = -8;
      return;
    }
  }
  st->gcp_state = GCP_DONE;
}
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kWalkThreads) k_walk(Ctx<R, H, S> c, const R* __restrict__ x,
                                                       const R* __restrict__ g) {
  walk_pass<R, H, S>(c, x, g);
}

}  // namespace lbfgsb_b200
