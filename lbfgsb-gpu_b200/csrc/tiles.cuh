// tiles.cuh -- TMA-staged tile pipeline for the streaming passes.
//
// Each pass reads up to ~22 element streams (x, g, l, u, nbd, iwhere codes, and the 2*col
// history columns).  Instead of relying on warps in flight to hide HBM latency (the pass
// kernels carry many accumulators and run one CTA per SM), the lanes of one warp issue one
// bulk asynchronous copy (cp.async.bulk, completion counted on an mbarrier) per stream per
// kTile-element tile into a multi-stage shared-memory ring; the CTA's threads compute on
// stage s while stages s+1.. are in flight.  No multicast is used.
//
// Every wait on an mbarrier is bounded: after kWaitNs nanoseconds without completion the
// CTA records the failure in *err and stops issuing; the host turns the flag into an error
// status.
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace lbfgsb_b200 {

constexpr int kTile = 512;          // elements per tile
constexpr int kMaxStreams = 24;
constexpr int kWaitPolls = 1 << 24;

// Bulk copies need 16-byte aligned addresses and sizes; the host pads the history slot
// stride to a multiple of kTile elements and checks the user's arrays.
struct StreamSet {
  const unsigned char* src[kMaxStreams];  // base of element 0 of the stream
  int tile_bytes[kMaxStreams];            // bytes of one tile of the stream
  int off[kMaxStreams];                   // byte offset of the stream in a stage buffer
  int count;
  int stage_bytes;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint: a thread whose phase is not complete sleeps until it
// completes or `ns` nanoseconds pass, instead of returning after the system's shorter limit
// (fewer polls, so fewer issue slots taken from the warps that compute).
__device__ __forceinline__ bool mbar_try_wait_for(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr uint32_t kSuspendNs = 1000000;            // 1 ms per try_wait at most
constexpr unsigned long long kWaitNs = 2000000000;  // give up after 2 s

// Bounded wait; false after kWaitNs nanoseconds (device global timer) without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try_wait_for(bar, parity, kSuspendNs)) return true;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}

// L2 policy of the streamed tiles: evict first.  An n-vector is read once or twice per
// pass and is larger than L2 at the sizes where it matters, so the tiles gain nothing from
// staying; marked evict-first they leave L2 to what is re-read (the state, the reduction
// rows, the code of the pass epilogues).  Measured 1.7-1.9% faster per iteration at
// n = 4096² and 2048² (FP64), with identical results.
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
      : "memory");
}

// Issue the copies of tile t into stage buffer `buf`, called by all lanes of warp 0:
// lane 0 posts the byte count, then each lane issues the copies of its streams.
__device__ __forceinline__ void issue_tile(const StreamSet& ss, long long t, unsigned char* buf,
                                           uint64_t* bar) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)ss.stage_bytes);
  __syncwarp();
  const uint64_t pol = l2_evict_first();
  for (int j = lane; j < ss.count; j += 32)
    bulk_g2s(buf + ss.off[j], ss.src[j] + (size_t)t * ss.tile_bytes[j], (uint32_t)ss.tile_bytes[j],
             bar, pol);
}

// Fill the partial last tile (elements [t*kTile, n)) with plain loads by the `nthr`
// threads rank = 0..nthr-1; the rest of the stage is left as is (callers mask by index).
__device__ __forceinline__ void fill_tail(const StreamSet& ss, long long t, long long n,
                                          unsigned char* buf, int rank, int nthr) {
  const long long first = t * kTile;
  const long long valid = n - first;  // 0 < valid < kTile
  for (int j = 0; j < ss.count; j++) {
    const int tb = ss.tile_bytes[j];
    // bytes of the valid prefix (bit streams round up to whole 32-bit words)
    long long vb = (long long)tb * valid / kTile;
    if ((long long)tb * valid % kTile) vb++;
    if (tb < kTile) vb = ((vb + 3) / 4) * 4;
    const unsigned char* src = ss.src[j] + (size_t)t * tb;
    for (long long b = rank; b < vb; b += nthr) buf[ss.off[j] + b] = src[b];
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Stage buffer of tile t: full tiles by bulk copies (lanes of the calling warp issue the
// copies of their streams), the partial last tile by plain loads of the warp's lanes and a
// plain arrive.  Called by a whole warp.
__device__ __forceinline__ void load_tile(const StreamSet& ss, long long t, long long n,
                                          unsigned char* buf, uint64_t* full) {
  const int lane = threadIdx.x & 31;
  if ((t + 1) * kTile <= n) {
    issue_tile(ss, t, buf, full);
  } else {
    fill_tail(ss, t, n, buf, lane, 32);
    __syncwarp();
    if (lane == 0) mbar_arrive(full);
  }
}

constexpr int kMaxStages = 8;

// Warp-specialised tile pipeline.  The CTA has CONSUMERS + 32 threads: the last warp is
// the producer, which issues the copies of the CTA's tiles (tiles rank, rank + count, ...
// of the instance's n elements) into a ring of `stages` stage buffers; the consumer threads run
// body(buf, t, valid) once per tile.  full[s] completes when the bytes of the tile in
// stage s have landed; empty[s] completes when every consumer warp has finished with it.
// There is no CTA-wide barrier per tile, and the producer issues a freed stage's next
// tile while the consumers work on the other stages.  body(buf, t, valid, release) must
// call release() exactly once, with the whole warp, after its last read of the stage
// buffer; a body that reads its data into registers first can release the stage before it
// computes, so that the producer refills it sooner.  body must not contain block-level
// barriers nor write the stage buffer.  Every wait is bounded; on a timeout the CTA sets
// *err and leaves the loop (returns false).
template <int CONSUMERS, typename Body>
__device__ __forceinline__ bool run_stages(const StreamSet& ss, long long n, int stages,
                                           unsigned char* ring, uint64_t* bars, int* err,
                                           CtaPos cp, Body&& body) {
  constexpr int kConsumerWarps = CONSUMERS / 32;
  uint64_t* full = bars;
  uint64_t* empty = bars + stages;
  const long long ntiles = (n + kTile - 1) / kTile;
  __shared__ int timed_out;
  if (threadIdx.x == 0) {
    timed_out = 0;
    for (int s = 0; s < stages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    mbar_init_fence();
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // The k-th tile of the CTA goes to stage s = k mod stages in round k / stages; both are
  // stepped along (no division per tile), with ph the parity of the round.
  if (warp == kConsumerWarps) {
    // producer
    int s = 0;
    uint32_t ph = 0;
    bool wrapped = false;
    for (long long t = cp.rank; t < ntiles; t += cp.count) {
      if (wrapped) {
        // the stage's previous tile (one round earlier) must have been released
        bool ok = true;
        if (lane == 0) ok = mbar_wait(&empty[s], ph ^ 1u);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok || *(volatile int*)&timed_out) {
          if (lane == 0) timed_out = 1;
          break;
        }
      }
      load_tile(ss, t, n, ring + (size_t)s * ss.stage_bytes, &full[s]);
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
        wrapped = true;
      }
    }
  } else {
    // consumers
    int s = 0;
    uint32_t ph = 0;
    for (long long t = cp.rank; t < ntiles; t += cp.count) {
      const unsigned char* buf = ring + (size_t)s * ss.stage_bytes;
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&full[s], ph));
      if (!ok) {
        if (lane == 0) timed_out = 1;
        break;
      }
      const int valid = t * kTile + kTile <= n ? kTile : (int)(n - t * kTile);
      body(buf, t, valid, [&] {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
      });
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
      }
    }
  }
  __syncthreads();
  if (timed_out) {
    // let the copies still in flight land (bounded) before the CTA's shared memory goes
    // away: wait on every stage's barrier at each of its two parities
    if (threadIdx.x == 0) {
      for (int s = 0; s < stages; s++) {
        mbar_wait(&full[s], 0);
        mbar_wait(&full[s], 1);
      }
      atomicExch(err, 1);
    }
    __syncthreads();
    return false;
  }
  return true;
}

// run_stages with consumer thread e handling elements e, e + CONSUMERS, ... of each
// tile: body(buf, t, valid, e).
template <int CONSUMERS, typename Body>
__device__ __forceinline__ bool run_tiles(const StreamSet& ss, long long n, int stages,
                                          unsigned char* ring, uint64_t* bars, int* err,
                                          CtaPos cp, Body&& body) {
  return run_stages<CONSUMERS>(ss, n, stages, ring, bars, err, cp,
                               [&](const unsigned char* buf, long long t, int valid, auto release) {
#pragma unroll
    for (int h = 0; h < kTile / CONSUMERS; h++)
      body(buf, t, valid, (int)threadIdx.x + h * CONSUMERS);
    release();
  });
}

// run_tiles in two phases: load(buf, t, valid, e) reads element e of the tile into a value
// (registers), the stage is released, then compute(value, t, valid, e) runs.
template <int CONSUMERS, typename Load, typename Compute>
__device__ __forceinline__ bool run_tiles_split(const StreamSet& ss, long long n, int stages,
                                                unsigned char* ring, uint64_t* bars, int* err,
                                                CtaPos cp, Load&& load, Compute&& compute) {
  static_assert(kTile == CONSUMERS, "one element per consumer thread and tile");
  return run_stages<CONSUMERS>(ss, n, stages, ring, bars, err, cp,
                               [&](const unsigned char* buf, long long t, int valid, auto release) {
    const int e = (int)threadIdx.x;
    const auto v = load(buf, t, valid, e);
    release();
    compute(v, t, valid, e);
  });
}

}  // namespace lbfgsb_b200
