// shard.cuh -- device side of sharded solves: one problem held by several ranks, rank r
// owning the variables ioff .. ioff + n of the problem's n_global (one process per GPU).
//
// The reference solves one problem on one GPU (culbfgsb/lbfgsbcuda.cpp:39-441); its only
// concurrency is a stream pool (lbfgsbcuda.cpp:144-148).  Every pass of an iteration here
// is an elementwise sweep plus a small reduction, so a problem splits by index range: the
// sweeps stay local and only the reductions cross ranks.  The passes do that through
// pass_fold (reduce.cuh): each rank folds its own CTA rows, the host gathers the rank rows
// with the caller's all-gather, and one CTA per rank folds them in rank order and runs the
// epilogue, so every rank keeps the same scalar state.  This file has the remaining pieces:
//   * the start point's flags (input errors, constrained, boxed), combined over the ranks;
//   * the function value, whose parts (one per rank) are summed in rank order;
//   * the breakpoint walk (walk.cuh) over all ranks' breakpoints in global key order: each
//     rank selects its smallest remaining keys with their walk records (the variable's
//     -g, distance to the bound and row of W), the records are gathered, and every rank
//     sorts the union and walks the keys up to the frontier (the smallest boundary of a
//     rank that still has keys beyond its selection), then marks the breakpoints it owns
//     that the walk passed.
#pragma once

#include "passes.cuh"
#include "walk.cuh"

namespace lbfgsb_b200 {

// Start-point flags: rank row [input_error, cnstnd, boxed].
template <typename S>
__global__ void k_shard_flags_put(const DevState<S>* st, double* send) {
  if (threadIdx.x == 0) {
    send[0] = (double)st->input_error;
    send[1] = (double)st->cnstnd;
    send[2] = (double)st->boxed;
  }
}
template <typename S>
__global__ void k_shard_flags_get(DevState<S>* st, const double* recv, int world) {
  if (threadIdx.x != 0) return;
  int err = 0, cn = 0, boxed = 1;
  for (int r = 0; r < world; r++) {
    const double* row = recv + (size_t)r * kShardRow;
    err |= (int)row[0];
    cn |= (int)row[1];
    boxed &= (int)row[2];
  }
  st->input_error = err;
  st->cnstnd = cn;
  st->boxed = boxed;
}

// ---- the sharded breakpoint walk ----------------------------------------------------

// Doubles per walk record: the key (bits of t, global index), -g, the distance to the
// bound passed, and the variable's row of W (2 col values, y then theta * s).
constexpr int kWalkRec = 4 + 2 * kMaxM;
constexpr int kWalkHead = 4;  // a rank block: [count, more, boundary hi, boundary lo]

// Doubles of one rank's block of gathered walk records, for `chunk` records.
__host__ __device__ inline int shard_walk_block(int chunk) { return kWalkHead + chunk * kWalkRec; }

// The walk's progress kept between launches (one per rank, the same on every rank).
template <typename S>
struct ShardWalk {
  WalkCarry<S> w;
  unsigned long long front_hi;  // every key <= the frontier has been walked
  unsigned int front_lo;
  int rounds;                   // selection rounds so far
  unsigned long long pass_hi;   // the largest key the walk passed
  unsigned int pass_lo;
  int npassed;
  int done;                     // 1 the walk ended, 2 a step of M*wbp failed
};

__device__ __forceinline__ double key_word(unsigned long long v) {
  return __longlong_as_double((long long)v);
}
__device__ __forceinline__ unsigned long long word_key(double d) {
  return (unsigned long long)__double_as_longlong(d);
}

// Selects this rank's smallest keys above the frontier (at most `chunk`, at least a
// quarter of it unless fewer remain) and writes them with their records to send (one CTA
// of kWalkThreads).  x, g: the iterate and its gradient; the keys come from the list that
// k_walk_gather made (local indices, keyed by global index).
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kWalkThreads) k_shard_walk_select(Ctx<R, H, S> c, const R* __restrict__ x,
                                                                    const R* __restrict__ g,
                                                                    const ShardWalk<S>* sw,
                                                                    int chunk, double* send) {
  const DevState<S>* st = c.st;
  const long long L = *c.wl_n;
  const bool first = sw->rounds == 0;
  const Key96 last{sw->front_hi, sw->front_lo};
  __shared__ WalkSmem<S> sm;
  __shared__ unsigned long long s_remaining;
  if (threadIdx.x == 0) {
    s_remaining = 0;
    sm.count = 0;
  }
  __syncthreads();
  // keys above the frontier
  {
    unsigned long long mine = 0;
    for (long long e = threadIdx.x; e < L; e += blockDim.x) {
      const Key96 k = make_key(c.wl_t[e], c.wl_i[e] + c.ioff);
      if (first || key_less(last, k)) mine++;
    }
    atomicAdd(&s_remaining, mine);
  }
  __syncthreads();
  const long long remaining = (long long)s_remaining;
  Key96 thr{~0ull, ~0u};
  if (remaining > chunk) {
    if (threadIdx.x == 0) {
      sm.prefix = Key96{0ull, 0u};
      sm.kk = chunk;
      sm.taken = 0;
      sm.done = 0;
    }
    __syncthreads();
    for (int level = 0; level < 12; level++) {
      for (int b = threadIdx.x; b < 256; b += blockDim.x) sm.hist[b] = 0;
      __syncthreads();
      const Key96 pre = sm.prefix;
      for (long long e = threadIdx.x; e < L; e += blockDim.x) {
        const Key96 k = make_key(c.wl_t[e], c.wl_i[e] + c.ioff);
        if (!first && !key_less(last, k)) continue;
        if (!key_prefix_eq(k, pre, level)) continue;
        atomicAdd(&sm.hist[key_digit(k, level)], 1u);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int d;
        long long cum;
        bool stop;
        select_level(sm.hist, sm.taken, sm.kk, chunk / 4, d, cum, stop);
        Key96 p = sm.prefix;
        key_set_digit(p, level, d);
        if (stop) {
          sm.prefix = key_prev(p);
          sm.done = 1;
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
  }
  // the records of the keys in (frontier, thr]
  const int col = st->col;
  const S theta = st->theta;
  const H *Y[kMaxM], *Sl[kMaxM];
  ring_ptrs(st, c.wy, c.ld, Y);
  ring_ptrs(st, c.ws, c.ld, Sl);
  double* rec0 = send + kWalkHead;
  for (long long e = threadIdx.x; e < L; e += blockDim.x) {
    const int i = c.wl_i[e];
    const Key96 k = make_key(c.wl_t[e], i + c.ioff);
    if (!first && !key_less(last, k)) continue;
    if (key_less(thr, k)) continue;
    const int pos = atomicAdd(&sm.count, 1);
    if (pos >= chunk) continue;
    double* rec = rec0 + (size_t)pos * kWalkRec;
    const R xi = x[i], gi = g[i];
    const R dibp = -gi;
    const R zibp = (dibp > R(0)) ? rsub(c.u[i], xi) : rsub(c.l[i], xi);
    rec[0] = key_word(k.hi);
    rec[1] = (double)k.lo;
    rec[2] = (double)(S)dibp;
    rec[3] = (double)(S)zibp;
    for (int j = 0; j < col; j++) {
      rec[4 + j] = (double)(S)HistTraits<H>::load(Y[j] + i);
      rec[4 + col + j] = (double)(theta * (S)HistTraits<H>::load(Sl[j] + i));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int cnt = sm.count < chunk ? sm.count : chunk;
    send[0] = (double)cnt;
    send[1] = remaining > cnt ? 1.0 : 0.0;
    send[2] = key_word(thr.hi);
    send[3] = (double)thr.lo;
  }
}

// Every rank: sorts the gathered records of all ranks, walks the keys up to the frontier
// and updates the progress (one CTA of kWalkThreads).  recv: world blocks of
// shard_walk_block(chunk) doubles.
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kWalkThreads) k_shard_walk_merge(Ctx<R, H, S> c, const double* recv,
                                                                   int world, int chunk,
                                                                   ShardWalk<S>* swk) {
  DevState<S>* st = c.st;
  const int block = shard_walk_block(chunk);
  __shared__ WalkSmem<S> sm;
  __shared__ unsigned short k_id[kChunk];  // the record of each sorted key
  __shared__ Key96 s_front;
  __shared__ WalkCarry<S> s_w;
  if (threadIdx.x == 0) {
    // the frontier: the smallest boundary of a rank with keys beyond its selection
    Key96 f{~0ull, ~0u};
    for (int r = 0; r < world; r++) {
      const double* head = recv + (size_t)r * block;
      if (head[1] != 0.0) {
        const Key96 b{word_key(head[2]), (unsigned int)head[3]};
        if (key_less(b, f)) f = b;
      }
    }
    s_front = f;
    sm.count = 0;
    sm.done = 0;
    sm.info = 0;
    s_w = swk->rounds == 0 ? walk_start(st) : swk->w;
  }
  __syncthreads();
  const Key96 front = s_front;
  // the keys up to the frontier (world * chunk <= kChunk records in all)
  for (int id = threadIdx.x; id < world * chunk; id += blockDim.x) {
    const int r = id / chunk, slot = id % chunk;
    const double* head = recv + (size_t)r * block;
    if (slot >= (int)head[0]) continue;
    const double* rec = head + kWalkHead + (size_t)slot * kWalkRec;
    const Key96 k{word_key(rec[0]), (unsigned int)rec[1]};
    if (key_less(front, k)) continue;
    const int pos = atomicAdd(&sm.count, 1);
    sm.k_hi[pos] = k.hi;
    sm.k_lo[pos] = k.lo;
  }
  __syncthreads();
  const int cnt = sm.count;
  sort_chunk(sm, cnt);
  // each record finds its key's place in the sorted chunk (keys are distinct)
  for (int id = threadIdx.x; id < world * chunk; id += blockDim.x) {
    const int r = id / chunk, slot = id % chunk;
    const double* head = recv + (size_t)r * block;
    if (slot >= (int)head[0]) continue;
    const double* rec = head + kWalkHead + (size_t)slot * kWalkRec;
    const Key96 k{word_key(rec[0]), (unsigned int)rec[1]};
    if (key_less(front, k)) continue;
    int lo = 0, hi = cnt;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (key_less(Key96{sm.k_hi[mid], sm.k_lo[mid]}, k)) lo = mid + 1;
      else hi = mid;
    }
    k_id[lo] = (unsigned short)id;
  }
  __syncthreads();
  const int col = st->col;
  WalkCarry<S> w = s_w;  // thread 0's copy is the one that walks
  __shared__ int s_np;
  __shared__ Key96 s_pass;
  if (threadIdx.x == 0) s_np = 0;
  __syncthreads();
  walk_sorted(st, sm, cnt, w,
      [&](int q, int k) {
        const int id = k_id[k];
        const double* rec = recv + (size_t)(id / chunk) * block + kWalkHead +
                            (size_t)(id % chunk) * kWalkRec;
        sm.dibp[q] = (S)rec[2];
        sm.zibp[q] = (S)rec[3];
        S* wbp = sm.wbp[q];
        for (int j = 0; j < 2 * col; j++) wbp[1 + j] = (S)rec[4 + j];
      },
      [&](int k, S) {
        s_pass = Key96{sm.k_hi[k], sm.k_lo[k]};
        s_np++;
      });
  if (threadIdx.x != 0) return;
  swk->w = w;
  if (s_np > 0) {
    swk->pass_hi = s_pass.hi;
    swk->pass_lo = s_pass.lo;
    swk->npassed += s_np;
  }
  swk->front_hi = front.hi;
  swk->front_lo = front.lo;
  swk->rounds++;
  const bool all_walked = front.hi == ~0ull && front.lo == ~0u;
  swk->done = sm.done ? sm.done : (all_walked || cnt == 0) ? 1 : 0;
}

// The walk's end into the state (thread 0), unless a step failed.
template <typename S>
__global__ void k_shard_walk_end(DevState<S>* st, ShardWalk<S>* swk) {
  if (threadIdx.x != 0 || swk->done == 2) return;
  __shared__ S work[kMaxM + 1];
  walk_end(st, swk->w, work);
}

// Marks this rank's breakpoints that the walk passed (keys up to the last one passed).
template <typename R, typename H, typename S>
__global__ void k_shard_walk_mark(Ctx<R, H, S> c, const R* __restrict__ g, const ShardWalk<S>* swk) {
  if (swk->npassed == 0 || swk->done == 2) return;
  const Key96 last{swk->pass_hi, swk->pass_lo};
  const long long L = *c.wl_n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < L;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = c.wl_i[e];
    const Key96 k = make_key(c.wl_t[e], i + c.ioff);
    if (key_less(last, k)) continue;
    const S dibp = (S)(-g[i]);
    c.code[i] = (int8_t)(dibp > S(0) ? IW_WALK_UPP : IW_WALK_LOW);
  }
}

}  // namespace lbfgsb_b200
