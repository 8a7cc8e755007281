// reduce.cuh -- deterministic grid reductions for the streaming passes.
//
// Each CTA reduces its threads' accumulators (warp butterflies, then a fixed-order sum
// over warps) into one row of `part` (gridDim.x rows).  The CTA that finishes last (an
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

// CTA-level reduction of per-thread values into part[blockIdx.x * W + ...].  `lane_owned`
// values (one distinct output per lane, NL per lane) are summed across warps only.
template <int NT, int NS, int NX, int NM, int NL = 0>
__device__ __forceinline__ void cta_reduce_to_row(const double (&s)[NS > 0 ? NS : 1],
                                                  const double (&x)[NX > 0 ? NX : 1],
                                                  const MinPair (&mn)[NM > 0 ? NM : 1],
                                                  const double (&lo)[NL > 0 ? NL : 1],
                                                  double* part, int width) {
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
  double* row = part + (size_t)blockIdx.x * width;
  for (int k = threadIdx.x; k < kVals; k += NT) {
    if (k >= NS && k < NS + NX) {
      double a = sm[0][k];
      for (int w = 1; w < kWarps; w++) a = (sm[w][k] > a) ? sm[w][k] : a;
      row[k] = a;
    } else if (k >= NS + NX && k < NS + NX + 2 * NM) {
      if (((k - NS - NX) & 1) != 0) continue;
      MinPair a = {sm[0][k], (long long)sm[0][k + 1]};
      for (int w = 1; w < kWarps; w++) a = minpair(a, MinPair{sm[w][k], (long long)sm[w][k + 1]});
      row[k] = a.v;
      row[k + 1] = (double)a.i;
    } else {
      double a = 0;
      for (int w = 0; w < kWarps; w++) a += sm[w][k];
      row[k] = a;
    }
  }
}

// Ticket: returns true in exactly one CTA (the last to arrive), after all rows are
// visible.  Resets the ticket for the next launch.
__device__ __forceinline__ bool last_cta(unsigned int* ticket) {
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == gridDim.x - 1);
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
// rows; a fixed butterfly finishes each column.
template <int NT>
__device__ __forceinline__ void fold_rows(const double* part, int rows, int width, int ns,
                                          int nx, int nm, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = NT / 32;
  for (int k = warp; k < width; k += kWarps) {
    const bool is_max = (k >= ns && k < ns + nx);
    const bool is_min = (k >= ns + nx && k < ns + nx + 2 * nm);
    if (is_min) {
      if (((k - ns - nx) & 1) != 0) continue;  // handled with its value column
      MinPair a = {INFINITY, kNoIndex};
      for (int r = lane; r < rows; r += 32)
        a = minpair(a, MinPair{part[(size_t)r * width + k], (long long)part[(size_t)r * width + k + 1]});
      a = warp_min(a);
      if (lane == 0) {
        out[k] = a.v;
        out[k + 1] = (double)a.i;
      }
    } else if (is_max) {
      double a = -INFINITY;
      for (int r = lane; r < rows; r += 32) {
        double v = part[(size_t)r * width + k];
        a = (v > a) ? v : a;
      }
      a = warp_max(a);
      if (lane == 0) out[k] = a;
    } else {
      double a = 0;
      for (int r = lane; r < rows; r += 32) a += part[(size_t)r * width + k];
      a = warp_sum(a);
      if (lane == 0) out[k] = a;
    }
  }
  __syncthreads();
}

}  // namespace lbfgsb_b200
