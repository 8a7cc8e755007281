// reduce.cuh -- deterministic grid reductions for the streaming passes.
//
// Each CTA reduces its threads' accumulators (warp butterflies, then a fixed-order sum
// over warps) into one row of `part` (one row per CTA of the instance, by rank).  `part` is
// stored column by column (entry k of row r at part[k * rows + r]), so that the last CTA
// reads each column with coalesced loads when it folds the rows.  The CTA that finishes last (an
// atomic ticket after a fence) folds the rows in CTA order and runs the pass epilogue.
// The order of every addition is fixed by the launch shape, so results are bitwise
// reproducible from run to run.
#pragma once

#include "common.cuh"
#include "state.cuh"

namespace lbfgsb_b200 {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v) ? w : v;
  }
  return v;
}
__device__ __forceinline__ MinPair warp_min(MinPair a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    MinPair b;
    b.v = __shfl_xor_sync(0xffffffffu, a.v, o);
    b.i = __shfl_xor_sync(0xffffffffu, a.i, o);
    a = minpair(a, b);
  }
  return a;
}

// Row layout of `part`: [ sums (NS) | maxima (NX) | min pairs (2*NM: value, index) ].
template <int NS, int NX, int NM>
struct RowLayout {
  static constexpr int kSums = NS, kMax = NX, kMin = NM;
  static constexpr int kWidth = NS + NX + 2 * NM;
};

// CTA-level reduction of per-thread values into row `rank` of the `count` rows of part.  `lane_owned`
// values (one distinct output per lane, NL per lane) are summed across warps only.
template <int NT, int NS, int NX, int NM, int NL = 0>
__device__ __forceinline__ void cta_reduce_to_row(const double (&s)[NS > 0 ? NS : 1],
                                                  const double (&x)[NX > 0 ? NX : 1],
                                                  const MinPair (&mn)[NM > 0 ? NM : 1],
                                                  const double (&lo)[NL > 0 ? NL : 1],
                                                  double* part, int width, int rank,
                                                  int count) {
  constexpr int kWarps = NT / 32;
  constexpr int kVals = NS + NX + 2 * NM + 32 * NL;
  __shared__ double sm[kWarps][kVals > 0 ? kVals : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double v = warp_sum(s[k]);
    if (lane == 0) sm[warp][k] = v;
  }
#pragma unroll
  for (int k = 0; k < NX; k++) {
    double v = warp_max(x[k]);
    if (lane == 0) sm[warp][NS + k] = v;
  }
#pragma unroll
  for (int k = 0; k < NM; k++) {
    MinPair v = warp_min(mn[k]);
    if (lane == 0) {
      sm[warp][NS + NX + 2 * k] = v.v;
      sm[warp][NS + NX + 2 * k + 1] = (double)v.i;
    }
  }
#pragma unroll
  for (int k = 0; k < NL; k++) sm[warp][NS + NX + 2 * NM + 32 * k + lane] = lo[k];
  __syncthreads();
  (void)width;
  double* row = part + rank;  // entry k at row[k * count]
  for (int k = threadIdx.x; k < kVals; k += NT) {
    if (k >= NS && k < NS + NX) {
      double a = sm[0][k];
      for (int w = 1; w < kWarps; w++) a = (sm[w][k] > a) ? sm[w][k] : a;
      row[(size_t)k * count] = a;
    } else if (k >= NS + NX && k < NS + NX + 2 * NM) {
      if (((k - NS - NX) & 1) != 0) continue;
      MinPair a = {sm[0][k], (long long)sm[0][k + 1]};
      for (int w = 1; w < kWarps; w++) a = minpair(a, MinPair{sm[w][k], (long long)sm[w][k + 1]});
      row[(size_t)k * count] = a.v;
      row[(size_t)(k + 1) * count] = (double)a.i;
    } else {
      double a = 0;
      for (int w = 0; w < kWarps; w++) a += sm[w][k];
      row[(size_t)k * count] = a;
    }
  }
}

// Ticket: returns true in exactly one of the instance's `count` CTAs (the last to
// arrive), after all rows are visible.  Resets the ticket for the next launch.
__device__ __forceinline__ bool last_cta(unsigned int* ticket, int count) {
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == (unsigned int)count - 1u);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    if (threadIdx.x == 0) *ticket = 0u;
  }
  return am_last;
}

// Final fold in the last CTA: out[k] for the `width` columns of part[0..rows).  Sums
// for k < ns and k >= ns + nx + 2*nm (lane-owned block), max for the next nx columns,
// min pairs for the next 2*nm columns.  Warps take columns round robin; lanes stride over
// rows; a fixed butterfly finishes each column.  A warp works on kFoldCols of its columns
// at once, and a lane issues the loads of all its rows of those columns (kFoldRows of
// them, 32 * kFoldRows rows a round) before it adds them, so that the fold waits about one
// memory round trip per kFoldCols columns (one CTA reading the rows is latency-bound);
// each column's operations and their order (a lane's rows in increasing order, then the
// butterfly) do not depend on that grouping.
constexpr int kFoldCols = 4;
constexpr int kFoldRows = 5;
template <int NT>
__device__ __forceinline__ void fold_rows(const double* part, int rows, int width, int ns,
                                          int nx, int nm, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = NT / 32;
  // column kinds: 0 sum, 1 max, 2 min pair (value column; the index is the next one),
  // 3 nothing (past the end, or the index column of a min pair)
  auto kind_of = [&](int k) {
    if (k >= width) return 3;
    if (k >= ns && k < ns + nx) return 1;
    if (k >= ns + nx && k < ns + nx + 2 * nm) return ((k - ns - nx) & 1) ? 3 : 2;
    return 0;
  };
  for (int k0 = warp; k0 < width; k0 += kWarps * kFoldCols) {
    int kind[kFoldCols];
    double acc[kFoldCols];
    MinPair mp[kFoldCols];
#pragma unroll
    for (int u = 0; u < kFoldCols; u++) {
      kind[u] = kind_of(k0 + u * kWarps);
      acc[u] = kind[u] == 1 ? -INFINITY : 0.0;
      mp[u] = MinPair{INFINITY, kNoIndex};
    }
    for (int r0 = lane; r0 < rows; r0 += 32 * kFoldRows) {
      double v[kFoldCols][kFoldRows];
#pragma unroll
      for (int u = 0; u < kFoldCols; u++) {
        const double* col = part + (size_t)(k0 + u * kWarps) * rows;  // entry k at [k * rows + r]
#pragma unroll
        for (int q = 0; q < kFoldRows; q++) {
          const int r = r0 + 32 * q;
          v[u][q] = (kind[u] != 3 && r < rows) ? col[r] : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < kFoldCols; u++) {
        const int k = k0 + u * kWarps;
#pragma unroll
        for (int q = 0; q < kFoldRows; q++) {
          const int r = r0 + 32 * q;
          if (r >= rows) break;
          if (kind[u] == 0) {
            acc[u] += v[u][q];
          } else if (kind[u] == 1) {
            acc[u] = (v[u][q] > acc[u]) ? v[u][q] : acc[u];
          } else if (kind[u] == 2) {
            mp[u] = minpair(mp[u], MinPair{v[u][q], (long long)part[(size_t)(k + 1) * rows + r]});
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kFoldCols; u++) {
      const int k = k0 + u * kWarps;
      if (kind[u] == 0) {
        const double a = warp_sum(acc[u]);
        if (lane == 0) out[k] = a;
      } else if (kind[u] == 1) {
        const double a = warp_max(acc[u]);
        if (lane == 0) out[k] = a;
      } else if (kind[u] == 2) {
        const MinPair a = warp_min(mp[u]);
        if (lane == 0) {
          out[k] = a.v;
          out[k + 1] = (double)a.i;
        }
      }
    }
  }
  __syncthreads();
}

// ---- sharded solves: one problem over several ranks, each holding an index range ----
//
// A pass's reduction then spans the ranks.  Each rank's last CTA folds its own rows
// (fold_rows) and, instead of running the epilogue, writes the folded row to c.shard_send
// (kShardRow doubles: the row, then one extra slot) and returns.  The host gathers every
// rank's row into c.shard_recv (rank r at r * kShardRow, the caller's all-gather) and
// launches the pass again in one CTA with c.epi_only set: that CTA folds the rank rows in
// rank order and runs the epilogue, so every rank runs it on the same values.
constexpr int kShardRow = 256;

// out[k] from the world rank rows of recv, column kinds as in fold_rows, each column
// folded in rank order.
template <int NT>
__device__ __forceinline__ void fold_rank_rows(const double* recv, int world, int width, int ns,
                                               int nx, int nm, double* out) {
  for (int k = threadIdx.x; k < width; k += NT) {
    if (k >= ns && k < ns + nx) {
      double a = -INFINITY;
      for (int r = 0; r < world; r++) {
        const double v = recv[(size_t)r * kShardRow + k];
        a = (v > a) ? v : a;
      }
      out[k] = a;
    } else if (k >= ns + nx && k < ns + nx + 2 * nm) {
      if (((k - ns - nx) & 1) != 0) continue;  // the index column of a min pair
      MinPair a{INFINITY, kNoIndex};
      for (int r = 0; r < world; r++) {
        const double* row = recv + (size_t)r * kShardRow;
        a = minpair(a, MinPair{row[k], (long long)row[k + 1]});
      }
      out[k] = a.v;
      out[k + 1] = (double)a.i;
    } else {
      double a = 0.0;
      for (int r = 0; r < world; r++) a += recv[(size_t)r * kShardRow + k];
      out[k] = a;
    }
  }
  __syncthreads();
}

// The fold of a pass's rows before its epilogue.  Returns true in the one CTA that runs
// the epilogue, with the folded row in red.  hash: a 64-bit sum the pass's CTAs added up
// in device memory (the free-set hash), carried in the extra slot of a rank row and summed
// (mod 2^64) over the ranks.
template <int NT, typename C>
__device__ __forceinline__ bool pass_fold(const C& c, CtaPos cp, int width, int ns, int nx,
                                          int nm, double* red,
                                          unsigned long long* hash = nullptr) {
  if (c.epi_only) {
    fold_rank_rows<NT>(c.shard_recv, c.shard_world, width, ns, nx, nm, red);
    if (hash && threadIdx.x == 0) {
      unsigned long long h = 0;
      for (int r = 0; r < c.shard_world; r++)
        h += (unsigned long long)__double_as_longlong(c.shard_recv[(size_t)r * kShardRow + width]);
      *hash = h;
    }
    __syncthreads();
    return true;
  }
  if (!last_cta(c.ticket, cp.count)) return false;
  fold_rows<NT>(c.part, cp.count, width, ns, nx, nm, red);
  if (c.shard_send) {
    for (int k = threadIdx.x; k < width; k += NT) c.shard_send[k] = red[k];
    if (threadIdx.x == 0)
      c.shard_send[width] = hash ? __longlong_as_double((long long)*(volatile unsigned long long*)hash) : 0.0;
    return false;
  }
  return true;
}

}  // namespace lbfgsb_b200
