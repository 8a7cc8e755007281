// state.cuh -- the solver's device-resident state and reduction scratch.
//
// Every scalar the reference keeps in local variables of lbfgsbminimize
// (culbfgsb/lbfgsbcpu.cpp:132-245: col, head, itail, iupdat, theta, the line-search
// scalars, the dcsrch save arrays, the m x m and 2m x 2m matrices) lives here, in device
// memory, and is advanced by the epilogues of the streaming passes.  The host reads the
// control header (everything before `big`) after each synchronisation point.
#pragma once

#include "common.cuh"
#include "small.cuh"

namespace lbfgsb_b200 {

// gcp_state
enum : int { GCP_DONE = 0, GCP_WALK = 1, GCP_EARLY = 2, GCP_SKIPPED = 3 };
// phase of a device-driven solve, what its next round does: start an iteration, evaluate
// the line search's next trial point, accept the 20th backtrack without evaluating it (the
// reference's exit from the search, lbfgsbcpu.cpp:352-358), or nothing (finished)
enum : int { PH_ITER = 0, PH_LS = 1, PH_QUIRK = 2, PH_DONE = 3 };
// ls_task: 1 = evaluate f, g at the trial point, 5 = the line search has converged
// fail codes (internal_fail): nonzero requests the memory reset of the reference driver.

template <typename S>
struct DevState {
  // ---------------- control header (copied to the host) ----------------
  int n, m, cnstnd, boxed;
  int col, head, itail, iupdat, updatd;
  int iter, ifun, iback, nfgv, ls_info, ls_task, csave;
  int gcp_state, nint, bnded, iword, subsm_active, wrk, uncon_branch;
  int internal_fail;   // 0, or the info code of a failed small-matrix step
  int input_error;     // errclb: bit 0 nbd out of range, bit 1 l > u on a boxed variable
  int device_error;    // 1 if a bounded wait of a staged-tile pipeline gave up
  int ibkmin, ibd;
  int nbreak, nleft, nfree_mov, nfree, nenter, nleave;
  int spec_gcp;       // 1: the post-evaluation pass also ran the next Cauchy scan
  int spec_apply;     // 1: the direction pass also applied the (untruncated) step
  int dir_no_spec;    // 1 after a truncated step: the next direction pass does not try
  int subsm_proj;     // 1: the L-BFGS-B 3.0 subspace step (projection), 0: the 2.1 step
  // device-driven solves (rounds.cuh): the round plan and the outer loop's decisions
  int phase;          // PH_*
  int reset_pending;  // the next iteration starts with the memory reset
  int rp_scan, rp_sub;  // this round runs cauchy's scan / the walk and the subspace passes
  int ev_active, ev_force, ev_is_z, ev_trial;  // this round's evaluation (see k_pre_eval)
  int xr[3];          // roles of the x buffers: [0] the iterate, [1] z, [2] the trial point
  int gr[2];          // roles of the g buffers: [0] at the iterate, [1] at the trial point
  int info_final;     // summary.info once phase == PH_DONE
  int max_iteration;  // option.max_iteration
  int rounds;         // rounds run so far
  int pad_rounds;
  unsigned long long free_hash, free_hash_acc, at_lower, at_upper;
  S theta, f, fold, gd, gdold, stp, dnrm, dtd, xstep, stpmx;
  S sbgnrm, tf, rr, dr, ddum_dr;
  S f1, f2, f2org, dtm, tsum, tj, bkmin, alpha, f1_0, f2_0;
  S eps_g, eps_x, eps_f;        // the stopping tolerances (device-driven solves)
  S res_g, res_x, res_f;        // summary.residual_* as the host loop would leave them
  // ---------------- large part ----------------
  S big;  // marks the end of the header
  int phys[kMaxM + 1];  // physical history slot of ring index r = 1..m
  int spare;            // physical slot receiving the speculative (s, y) pair
  S sy[kMaxM * kMaxM], ss[kMaxM * kMaxM], wt[kMaxM * kMaxM];
  S wn[4 * kMaxM * kMaxM], wn1[4 * kMaxM * kMaxM];
  S p[2 * kMaxM + 1], c[2 * kMaxM + 1], mc[2 * kMaxM + 1], wv[2 * kMaxM + 1];  // 1-based
  S prod_sy[kMaxM], prod_ss[kMaxM];  // s'y_j and s_j's of the pending pair, old positions
  LineSearchSave<S> ls;
};

// The pass epilogues read and write the small matrices of the state many times over; from
// global memory every such access would wait hundreds of cycles.  The last CTA therefore
// copies the whole state into shared memory (all threads, 4-byte words, loads that bypass
// L1 so that the other CTAs' writes are seen), runs the epilogue f on that copy, and all
// threads store the copy back.  epilogue_on_shared runs f(st) on thread 0;
// epilogue_on_shared_warp runs f(st, lane) on the 32 lanes of warp 0, for epilogues whose
// matrix algebra is shared out over a warp (warp_small.cuh).
template <bool kWarp, typename S, typename F>
__device__ __forceinline__ void epilogue_in_shared(DevState<S>* st, F&& f) {
  static_assert(sizeof(DevState<S>) % 4 == 0, "the state is copied in 4-byte words");
  constexpr int kWords = (int)(sizeof(DevState<S>) / 4);
  __shared__ __align__(16) unsigned int words[kWords];
  const unsigned int* src = reinterpret_cast<const unsigned int*>(st);
  for (int k = threadIdx.x; k < kWords; k += blockDim.x) words[k] = __ldcg(src + k);
  __syncthreads();
  if constexpr (kWarp) {
    if (threadIdx.x < 32) f(reinterpret_cast<DevState<S>*>(words), (int)threadIdx.x);
  } else {
    if (threadIdx.x == 0) f(reinterpret_cast<DevState<S>*>(words));
  }
  __syncthreads();
  unsigned int* dst = reinterpret_cast<unsigned int*>(st);
  for (int k = threadIdx.x; k < kWords; k += blockDim.x) dst[k] = words[k];
}
template <typename S, typename F>
__device__ __forceinline__ void epilogue_on_shared(DevState<S>* st, F&& f) {
  epilogue_in_shared<false>(st, f);
}
template <typename S, typename F>
__device__ __forceinline__ void epilogue_on_shared_warp(DevState<S>* st, F&& f) {
  epilogue_in_shared<true>(st, f);
}

// A (value, index) pair reduced by minimum value, ties to the lower index.  kNoIndex
// marks "no candidate" (exactly representable in the double rows of the reduction).
constexpr long long kNoIndex = 1LL << 62;
struct MinPair {
  double v;
  long long i;
};
__host__ __device__ __forceinline__ MinPair minpair(MinPair a, MinPair b) {
  if (b.v < a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}

// One thread's running arg-min of candidate values in their own type T (breakpoints,
// steps to a bound), with the filter bound thr = the least T above the minimum
// (quotient_exceeds).  A thread meets its elements in increasing index order, so a
// candidate replaces the minimum only when it is strictly smaller; across threads the
// reductions break ties by the lower index (minpair).  A thread without a candidate
// reports (+inf, kNoIndex).
template <typename T>
struct ArgMin {
  T v;
  int i;
  T thr;
  __device__ __forceinline__ ArgMin() : v(T(INFINITY)), i(-1), thr(T(INFINITY)) {}
  __device__ __forceinline__ void offer(T c, int k) {
    if (c < v) {
      v = c;
      i = k;
      thr = next_up(c);
    }
  }
  // the candidate num/den, formed (correctly rounded) only when it may be the minimum
  __device__ __forceinline__ void offer_quotient(T num, T den, int k) {
    if (!quotient_exceeds(num, den, thr)) offer(rdiv(num, den), k);
  }
  __device__ __forceinline__ MinPair pair() const {
    return MinPair{(double)v, i < 0 ? kNoIndex : (long long)i};
  }
};

}  // namespace lbfgsb_b200
