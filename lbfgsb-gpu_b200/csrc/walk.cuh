// walk.cuh -- the breakpoint walk of the generalized Cauchy point (the part of
// culbfgsb/lbfgsbcpu.cpp:725-816 after the first breakpoint test).
//
// The reference keeps the breakpoints in a heap (hpsolb, 1175-1233) and pops them one at
// a time.  Here, only when the scan found that the first breakpoint is passed, the
// breakpoints (t_i, i) are listed (same arithmetic as the scan, so the same t_i) and walked
// in chunks of the smallest remaining keys (96-bit key: the bits of t, then i):
//   select   a radix select over the list, 8 bits a level, that stops as soon as the
//            buckets below the boundary hold a large enough chunk (usually after one or
//            two levels), and the extraction of that chunk;
//   walk     the chunk is sorted in shared memory (bitonic), each candidate's row of W,
//            M*wbp and wbp'M wbp are formed in parallel, and one thread walks the chunk in
//            key order with the reference's recurrence for f', f'', c and p.
// Two forms: k_walk_coop (single-instance solves) lists and selects with the whole grid, a
// cooperative launch with a bounded grid barrier, and walks in CTA 0; k_walk (one CTA per
// instance, used by batched solves, with k_walk_gather before it) does everything in one
// CTA.  Breakpoints with equal t are passed in increasing variable index (the heap's order
// among exact ties is an artefact of its layout).
#pragma once

#include "common.cuh"
#include "passes.cuh"
#include "small.cuh"
#include "state.cuh"

namespace lbfgsb_b200 {

// Appends the breakpoints of the CTA's share of the variables to (wl_t, wl_i).
template <typename R, typename H, typename S>
__device__ __forceinline__ void gather_breakpoints(const Ctx<R, H, S>& c, CtaPos cp, int nthreads,
                                                   const R* __restrict__ x, const R* __restrict__ g) {
  const int n = c.n;
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)cp.rank * nthreads; base < n;
       base += (long long)cp.count * nthreads) {
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
__device__ __forceinline__ void walk_gather_pass(const Ctx<R, H, S>& c, CtaPos cp,
                                                 const R* __restrict__ x, const R* __restrict__ g) {
  if (c.rounds) {
    const DevState<S>* st = c.st;
    if (!st->rp_sub || st->gcp_state != GCP_WALK || st->internal_fail != 0) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
  }
  gather_breakpoints<R, H, S>(c, cp, kThreads, x, g);
}
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kThreads) k_walk_gather(Ctx<R, H, S> c, const R* __restrict__ x,
                                                          const R* __restrict__ g) {
  walk_gather_pass<R, H, S>(c, cta_here(), x, g);
}

constexpr int kWalkThreads = 512;
constexpr int kChunk = kWalkChunk;
constexpr int kChunkMin = kChunk / 4;  // the smallest chunk the select may stop at
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
// the key just below k (k > 0)
__device__ __forceinline__ Key96 key_prev(Key96 k) {
  if (k.lo > 0) return Key96{k.hi, k.lo - 1};
  return Key96{k.hi - 1, ~0u};
}

// One level of the radix select, from the level's histogram (the same in every thread that
// runs it): the boundary digit d, the keys below it, and whether the select may stop here
// with the chunk "every candidate below bucket d" (at least chunk_min keys in all).  taken:
// keys already below the prefix from earlier levels; kk: keys still wanted.
__device__ __forceinline__ void select_level(const unsigned int* hist, long long taken,
                                             long long kk, long long chunk_min, int& d,
                                             long long& cum, bool& stop) {
  cum = 0;
  d = 255;
  for (int b = 0; b < 256; b++) {
    if (cum + hist[b] >= kk) {
      d = b;
      break;
    }
    cum += hist[b];
  }
  stop = taken + cum >= chunk_min;
}

// Thread 0's running walk (lbfgsbcpu.cpp:725-809) across chunks.
template <typename S>
struct WalkCarry {
  S f1, f2, f2org, dtm, tsum, tj;
  int nleft, nint;
  bool all_fixed;
};

template <typename S>
struct WalkSmem {
  unsigned long long k_hi[kChunk];
  unsigned int k_lo[kChunk];
  unsigned int hist[256];
  int count, done, info;
  Key96 prefix, last;
  long long kk, taken;
  S wbp[kBatch][2 * kMaxM + 1];
  S v[kBatch][2 * kMaxM + 1];
  S wmw[kBatch], dibp[kBatch], zibp[kBatch];
  S work[kBatch][kMaxM + 1];
};

// Bitonic sort of the cnt keys in sm.k_hi / k_lo by (hi, lo), padded with maximal keys
// (all threads of the CTA).
template <typename S>
__device__ void sort_chunk(WalkSmem<S>& sm, int cnt) {
  for (int e = cnt + threadIdx.x; e < kChunk; e += blockDim.x) {
    sm.k_hi[e] = ~0ull;
    sm.k_lo[e] = ~0u;
  }
  __syncthreads();
  for (int size = 2; size <= kChunk; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int e = threadIdx.x; e < kChunk; e += blockDim.x) {
        const int p = e ^ stride;
        if (p > e) {
          const bool up = (e & size) == 0;
          const Key96 a{sm.k_hi[e], sm.k_lo[e]}, b{sm.k_hi[p], sm.k_lo[p]};
          if (key_less(b, a) == up) {
            sm.k_hi[e] = b.hi;
            sm.k_lo[e] = b.lo;
            sm.k_hi[p] = a.hi;
            sm.k_lo[p] = a.lo;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Walk the cnt sorted keys of sm (all threads of the CTA) with the reference's recurrence
// (lbfgsbcpu.cpp:725-809).  prep(q, k) fills sm.dibp[q], sm.zibp[q] and sm.wbp[q][1..2col]
// for key k of the chunk (run by thread q of a batch); pass(k, dibp) records that the walk
// passed key k (thread 0).  Sets sm.done: 1 the walk ended, 2 a step of M*wbp failed (the
// driver resets the memory).
template <typename S, typename Prep, typename Pass>
__device__ void walk_sorted(DevState<S>* st, WalkSmem<S>& sm, int cnt, WalkCarry<S>& w,
                            Prep&& prep, Pass&& pass) {
  const int n = st->n, col = st->col, col2 = 2 * col, nbreak = st->nbreak, bnded = st->bnded;
  const S theta = st->theta;
  for (int b0 = 0; b0 < cnt; b0 += kBatch) {
    const int nb = (cnt - b0) < kBatch ? (cnt - b0) : kBatch;
    if (threadIdx.x < nb) {
      prep((int)threadIdx.x, b0 + (int)threadIdx.x);
      const S* wbp = sm.wbp[threadIdx.x];
      if (col > 0) {
        int info = 0;
        sbmv(st->sy, st->wt, col, wbp, sm.v[threadIdx.x], &info, sm.work[threadIdx.x]);
        if (info != 0) atomicExch(&sm.info, info);
        sm.wmw[threadIdx.x] = sdot(&wbp[1], 1, &sm.v[threadIdx.x][1], 1, col2);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (sm.info != 0) {
        st->internal_fail = sm.info;
        sm.done = 2;
      }
      #pragma unroll 1
      for (int q = 0; q < nb && sm.done == 0; q++) {
        const int k = b0 + q;
        const S tk = (S)__longlong_as_double((long long)sm.k_hi[k]);
        const S tj0 = w.tj;
        w.tj = tk;
        const S dt = w.tj - tj0;
        if (w.dtm < dt) {
          sm.done = 1;
          break;
        }
        w.tsum = w.tsum + dt;
        w.nleft = w.nleft - 1;
        const S dibp = sm.dibp[q];
        pass(k, dibp);
        if (w.nleft == 0 && nbreak == n) {
          w.dtm = dt;
          #pragma unroll 1
          for (int j = 1; j <= col2; j++) st->c[j] += w.dtm * st->p[j];
          w.all_fixed = true;
          sm.done = 1;
          break;
        }
        w.nint = w.nint + 1;
        const S dibp2 = dibp * dibp;
        w.f1 = w.f1 + dt * w.f2 + dibp2 - theta * dibp * sm.zibp[q];
        w.f2 = w.f2 - theta * dibp2;
        if (col > 0) {
          #pragma unroll 1
          for (int j = 1; j <= col2; j++) st->c[j] += dt * st->p[j];
          const S wmc = sdot(&st->c[1], 1, &sm.v[q][1], 1, col2);
          const S wmp = sdot(&st->p[1], 1, &sm.v[q][1], 1, col2);
          const S wmw = sm.wmw[q];
          #pragma unroll 1
          for (int j = 1; j <= col2; j++) st->p[j] += (-dibp) * sm.wbp[q][j];
          w.f1 = w.f1 + dibp * wmc;
          w.f2 = w.f2 + (S)2.0 * dibp * wmp - dibp2 * wmw;
        }
        w.f2 = smax((S)(5e-16 * (double)w.f2org), w.f2);
        if (w.nleft > 0) {
          w.dtm = -w.f1 / w.f2;
          continue;
        }
        if (bnded) {
          w.f1 = 0;
          w.f2 = 0;
          w.dtm = 0;
        } else {
          w.dtm = -w.f1 / w.f2;
        }
        sm.done = 1;
        break;
      }
    }
    __syncthreads();
    if (sm.done) break;
  }
}

// Sort the cnt keys in sm.k_hi / k_lo and walk them, reading each candidate's x, g, bounds
// and history row from the solve's arrays (all threads of the CTA).
template <typename R, typename H, typename S>
__device__ void walk_chunk(const Ctx<R, H, S>& c, const R* __restrict__ x, const R* __restrict__ g,
                           const H* const (&Y)[kMaxM], const H* const (&Sl)[kMaxM], WalkSmem<S>& sm,
                           int cnt, WalkCarry<S>& w) {
  DevState<S>* st = c.st;
  const int col = st->col;
  const S theta = st->theta;
  sort_chunk(sm, cnt);
  walk_sorted(st, sm, cnt, w,
      [&](int q, int k) {
        const int i = (int)sm.k_lo[k];
        const R xi = x[i], gi = g[i];
        const R dibp = -gi;
        const R zibp = (dibp > R(0)) ? rsub(c.u[i], xi) : rsub(c.l[i], xi);
        sm.dibp[q] = (S)dibp;
        sm.zibp[q] = (S)zibp;
        S* wbp = sm.wbp[q];
        #pragma unroll 1
        for (int j = 0; j < col; j++) {
          wbp[1 + j] = (S)HistTraits<H>::load(Y[j] + i);
          wbp[1 + col + j] = theta * (S)HistTraits<H>::load(Sl[j] + i);
        }
      },
      [&](int k, S dibp) {
        c.code[(int)sm.k_lo[k]] = (int8_t)(dibp > S(0) ? IW_WALK_UPP : IW_WALK_LOW);
      });
}

// The walk's start from the state and its end into it (thread 0).
template <typename S>
__device__ __forceinline__ WalkCarry<S> walk_start(const DevState<S>* st) {
  WalkCarry<S> w;
  w.f1 = st->f1;
  w.f2 = st->f2;
  w.f2org = st->f2org;
  w.dtm = st->dtm;
  w.tsum = st->tsum;
  w.tj = st->tj;
  w.nleft = st->nleft;
  w.nint = st->nint;
  w.all_fixed = false;
  return w;
}
template <typename S>
__device__ __forceinline__ void walk_end(DevState<S>* st, WalkCarry<S>& w, S* work) {
  const int col = st->col, col2 = 2 * col;
  if (!w.all_fixed) {
    if (w.dtm <= S(0)) w.dtm = 0;
    w.tsum = w.tsum + w.dtm;
    #pragma unroll 1
    for (int j = 1; j <= col2; j++) st->c[j] += w.dtm * st->p[j];
  }
  st->f1 = w.f1;
  st->f2 = w.f2;
  st->dtm = w.dtm;
  st->tsum = w.tsum;
  st->tj = w.tj;
  st->nleft = w.nleft;
  st->nint = w.nint;
  if (col > 0) {
    int info = 0;
    sbmv(st->sy, st->wt, col, st->c, st->mc, &info, work);
    if (info != 0) {
      st->internal_fail = -8;
      return;
    }
  }
  st->gcp_state = GCP_DONE;
}

// The whole walk in one CTA (batched solves: one CTA per instance, after k_walk_gather).
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
  const long long L = *c.wl_n;
  const H *Y[kMaxM], *Sl[kMaxM];
  ring_ptrs(st, c.wy, c.ld, Y);
  ring_ptrs(st, c.ws, c.ld, Sl);
  __shared__ WalkSmem<S> sm;
  WalkCarry<S> w{};
  if (threadIdx.x == 0) {
    w = walk_start(st);
    sm.done = 0;
    sm.last = Key96{0ull, 0u};
    sm.info = 0;
  }
  __syncthreads();
  bool first_round = true;
  long long consumed = 0;
  while (true) {
    // ---- select the next chunk: the smallest keys greater than sm.last ----
    const long long remaining = L - consumed;
    Key96 thr;
    thr.hi = ~0ull;
    thr.lo = ~0u;
    if (remaining > kChunk) {
      if (threadIdx.x == 0) {
        sm.prefix = Key96{0ull, 0u};
        sm.kk = kChunk;
        sm.taken = 0;
        sm.done = 0;
      }
      __syncthreads();
      for (int level = 0; level < 12; level++) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) sm.hist[b] = 0;
        __syncthreads();
        const Key96 pre = sm.prefix, last = sm.last;
        for (long long e = threadIdx.x; e < L; e += blockDim.x) {
          const Key96 k = make_key(c.wl_t[e], c.wl_i[e]);
          if (!first_round && !key_less(last, k)) continue;
          if (!key_prefix_eq(k, pre, level)) continue;
          atomicAdd(&sm.hist[key_digit(k, level)], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          int d;
          long long cum;
          bool stop;
          select_level(sm.hist, sm.taken, sm.kk, kChunkMin, d, cum, stop);
          Key96 p = sm.prefix;
          key_set_digit(p, level, d);
          if (stop) {
            // every candidate below bucket d: the prefix with digit d and zeros after it
            sm.prefix = key_prev(p);
            sm.done = 1;  // used here as "select finished early"
          } else {
            sm.prefix = p;
            sm.kk = sm.kk - cum;
            sm.taken = sm.taken + cum;
          }
        }
        __syncthreads();
        if (sm.done) break;
      }
      thr = sm.prefix;
      __syncthreads();
      if (threadIdx.x == 0) sm.done = 0;
    }
    // ---- extract keys in (sm.last, thr] into shared memory ----
    if (threadIdx.x == 0) sm.count = 0;
    __syncthreads();
    {
      const Key96 last = sm.last;
      for (long long e = threadIdx.x; e < L; e += blockDim.x) {
        const Key96 k = make_key(c.wl_t[e], c.wl_i[e]);
        if (!first_round && !key_less(last, k)) continue;
        if (key_less(thr, k)) continue;
        const int pos = atomicAdd(&sm.count, 1);
        if (pos < kChunk) {
          sm.k_hi[pos] = k.hi;
          sm.k_lo[pos] = k.lo;
        }
      }
    }
    __syncthreads();
    const int cnt = sm.count < kChunk ? sm.count : kChunk;
    walk_chunk<R, H, S>(c, x, g, Y, Sl, sm, cnt, w);
    consumed += cnt;
    if (sm.done || consumed >= L || cnt == 0) break;
    if (threadIdx.x == 0) sm.last = Key96{sm.k_hi[cnt - 1], sm.k_lo[cnt - 1]};
    first_round = false;
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (sm.done == 2) return;  // a failed M*wbp: the driver resets the memory
  walk_end(st, w, sm.work[0]);
}
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kWalkThreads) k_walk(Ctx<R, H, S> c, const R* __restrict__ x,
                                                       const R* __restrict__ g) {
  walk_pass<R, H, S>(c, x, g);
}

// ---- the cooperative walk of single-instance solves ------------------------------------

// Bounded grid barrier of a cooperative launch: every CTA adds one arrival to *bar and
// waits until all of this barrier's arrivals are in (target counts up by gridDim.x per
// barrier; *bar is zero at launch).  Returns false in every CTA whose wait gave up.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int& target) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    target += gridDim.x;
    __threadfence();
    atomicAdd(bar, 1u);
    long long k = 0;
    while (*(volatile unsigned int*)bar < target && k < 4 * kWaitPolls) k++;
    s_ok = k < 4 * kWaitPolls ? 1 : 0;
    __threadfence();
  }
  __syncthreads();
  return s_ok != 0;
}

// Lists the breakpoints with the whole grid, selects each chunk with the whole grid
// (histograms in global memory, the same digit decided redundantly by every CTA) and walks
// it in CTA 0.  wsc->bar and *wl_n are zero at launch.
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kWalkThreads) k_walk_coop(Ctx<R, H, S> c, const R* __restrict__ x,
                                                            const R* __restrict__ g) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!st->rp_sub || st->internal_fail != 0) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
  }
  if (st->gcp_state != GCP_WALK) return;
  WalkScratch* ws = c.wsc;
  unsigned int target = 0;
  auto fail = [&]() {
    if (threadIdx.x == 0) atomicExch(&st->device_error, 1);
  };
  __shared__ WalkSmem<S> sm;
  const bool lead = blockIdx.x == 0;
  if (lead) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) ws->hist[0][b] = 0;
    if (threadIdx.x == 0) ws->chunk_n = 0;
  }
  gather_breakpoints<R, H, S>(c, cta_here(), blockDim.x, x, g);
  if (!grid_barrier(&ws->bar, target)) return fail();
  const long long L = (long long)*(volatile unsigned int*)c.wl_n;
  const H *Y[kMaxM], *Sl[kMaxM];
  WalkCarry<S> w{};
  if (lead) {
    ring_ptrs(st, c.wy, c.ld, Y);
    ring_ptrs(st, c.ws, c.ld, Sl);
    if (threadIdx.x == 0) {
      w = walk_start(st);
      sm.done = 0;
      sm.info = 0;
    }
  }
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long e0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool first_round = true;
  Key96 last{0ull, 0u};
  long long consumed = 0;
  int hb = 0;  // the histogram buffer of the next level (rotating over three)
  __shared__ unsigned int s_hist[256];
  while (true) {
    const long long remaining = L - consumed;
    Key96 thr{~0ull, ~0u};
    if (remaining > kChunk) {
      Key96 prefix{0ull, 0u};
      long long kk = kChunk, taken = 0;
      for (int level = 0; level < 12; level++) {
        unsigned int* h = ws->hist[hb];
        // the buffer after this one was last read two levels ago, before the previous
        // barrier: clear it for the next level
        if (lead)
          for (int b = threadIdx.x; b < 256; b += blockDim.x) ws->hist[(hb + 1) % 3][b] = 0;
        for (int b = threadIdx.x; b < 256; b += blockDim.x) s_hist[b] = 0;
        __syncthreads();
        for (long long e = e0; e < L; e += stride) {
          const Key96 k = make_key(c.wl_t[e], c.wl_i[e]);
          if (!first_round && !key_less(last, k)) continue;
          if (!key_prefix_eq(k, prefix, level)) continue;
          atomicAdd(&s_hist[key_digit(k, level)], 1u);
        }
        __syncthreads();
        for (int b = threadIdx.x; b < 256; b += blockDim.x)
          if (s_hist[b]) atomicAdd(&h[b], s_hist[b]);
        if (!grid_barrier(&ws->bar, target)) return fail();
        for (int b = threadIdx.x; b < 256; b += blockDim.x) s_hist[b] = __ldcg(&h[b]);
        __syncthreads();
        hb = (hb + 1) % 3;
        int d;
        long long cum;
        bool stop;
        select_level(s_hist, taken, kk, kChunkMin, d, cum, stop);
        __syncthreads();  // every thread has read s_hist before the next level clears it
        key_set_digit(prefix, level, d);
        if (stop) {
          prefix = key_prev(prefix);
          break;
        }
        kk -= cum;
        taken += cum;
      }
      thr = prefix;
    }
    // extract the chunk: keys in (last, thr]
    for (long long e = e0; e < L; e += stride) {
      const Key96 k = make_key(c.wl_t[e], c.wl_i[e]);
      if (!first_round && !key_less(last, k)) continue;
      if (key_less(thr, k)) continue;
      const unsigned int pos = atomicAdd(&ws->chunk_n, 1u);
      if (pos < (unsigned int)kChunk) {
        ws->chunk_hi[pos] = k.hi;
        ws->chunk_lo[pos] = k.lo;
      }
    }
    if (!grid_barrier(&ws->bar, target)) return fail();
    if (lead) {
      const unsigned int n_sel = __ldcg(&ws->chunk_n);
      const int cnt = n_sel < (unsigned int)kChunk ? (int)n_sel : kChunk;
      for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        sm.k_hi[e] = __ldcg(&ws->chunk_hi[e]);
        sm.k_lo[e] = __ldcg(&ws->chunk_lo[e]);
      }
      __syncthreads();
      walk_chunk<R, H, S>(c, x, g, Y, Sl, sm, cnt, w);
      if (threadIdx.x == 0) {
        ws->chunk_n = 0;
        ws->cnt = cnt;
        ws->done = sm.done;
        if (cnt > 0) {
          ws->last_hi = sm.k_hi[cnt - 1];
          ws->last_lo = sm.k_lo[cnt - 1];
        }
      }
    }
    if (!grid_barrier(&ws->bar, target)) return fail();
    const int cnt = *(volatile int*)&ws->cnt;
    const int done = *(volatile int*)&ws->done;
    consumed += cnt;
    if (done || consumed >= L || cnt == 0) break;
    last = Key96{*(volatile unsigned long long*)&ws->last_hi, *(volatile unsigned int*)&ws->last_lo};
    first_round = false;
  }
  if (!lead || threadIdx.x != 0) return;
  if (sm.done == 2) return;  // a failed M*wbp: the driver resets the memory
  walk_end(st, w, sm.work[0]);
}

}  // namespace lbfgsb_b200
