// rounds.cuh -- the outer loop of the reference driver (culbfgsb/lbfgsbcpu.cpp:279-462) as
// device decisions, for solves whose objective keeps f on the device.
//
// A device-driven solve repeats one fixed sequence of launches, a round:
//
//   k_round_begin   the loop top (279-284): the memory reset when one is pending, the
//                   branch flags, and the round plan (scan? subspace passes?)
//   k_gcp_scan, k_walk_coop, k_freev_formk, k_subsm_dir, k_subsm_apply
//                   each returns at once unless the plan (and the state) asks for it
//   k_pre_eval      the checks between the subspace step and the line search (the memory
//                   reset after a failed step, 297-341; the g'd >= 0 exit, 359-387), and
//                   where the objective reads x and writes g this round
//   k_trial_round   the trial point stp*d + t when stp != 1 (1332-1334)
//   objective       the caller's, enqueued once per round; it reads x and writes g and f
//                   through the evaluation slot (Ctx::ev_*)
//   k_post_eval / k_post_gcp, k_post_round
//                   dcsrch, and on acceptance the role rotation of the x and g buffers
//                   and the stopping tests in the reference's order (394-429)
//
// so that the host enqueues rounds without reading anything back: the sequence is captured
// once into a CUDA graph and relaunched, and the host reads the state only every few rounds
// to see whether the solve has finished.  Rounds after the finish do nothing (every kernel
// returns at once and the objective is told, through *ev_act, that its result is not
// used).  Each decision is the one the host loop of driver.cu makes from the same state,
// so a device-driven solve gives the host-driven solve's results bit for bit.
#pragma once

#include "passes.cuh"

namespace lbfgsb_b200 {

// The round kernels are run by one thread per instance (round_begin, pre_eval, post_round
// below); k_round_* run them for a single instance.
template <typename R, typename H, typename S>
__device__ __forceinline__ void round_begin(const Ctx<R, H, S>& c) {
  DevState<S>* st = c.st;
  st->rounds = st->rounds + 1;
  st->rp_scan = 0;
  st->rp_sub = 0;
  if (c.wl_n) *c.wl_n = 0;  // the breakpoint list of this round's walk, if any
  if (c.wsc) c.wsc->bar = 0;  // and the cooperative walk's grid barrier
  if (st->phase != PH_ITER) return;
  // the post-evaluation pass may already have started this iteration and run its Cauchy
  // scan (spec_gcp); otherwise, and after a reset, the loop top runs here
  const bool spec = st->cnstnd && st->spec_gcp;
  const bool start_here = st->reset_pending || !spec;
  if (start_here) begin_state(st, st->reset_pending);
  st->rp_scan = (start_here && !st->uncon_branch) ? 1 : 0;
  st->rp_sub = 1;
  st->reset_pending = 0;
  st->spec_gcp = 0;
}

template <typename R, typename H, typename S>
__device__ __forceinline__ void pre_eval(const Ctx<R, H, S>& c) {
  DevState<S>* st = c.st;
  st->ev_active = 0;
  st->ev_force = 0;
  if (st->phase == PH_ITER) {
    if (st->internal_fail != 0) {
      st->reset_pending = 1;  // cauchy / formk / cmprlb / subsm failed (297-341)
    } else if (st->ls_info != 0) {
      // g'd >= 0 at the start of the line search (359-387)
      if (st->col == 0) {
        st->phase = PH_DONE;
        st->info_final = -2;
      } else {
        st->reset_pending = 1;
      }
    } else {
      st->ev_active = 1;
    }
  } else if (st->phase == PH_LS) {
    st->ev_active = 1;
  } else if (st->phase == PH_QUIRK) {
    st->ev_force = 1;
  }
  const bool ev = st->ev_active || st->ev_force;
  const bool unit = st->stp == S(1);
  st->ev_is_z = (ev && unit) ? 1 : 0;
  st->ev_trial = (ev && !unit) ? 1 : 0;
  *c.ev_x = ev ? (unit ? c.X[st->xr[1]] : c.X[st->xr[2]]) : c.X[st->xr[0]];
  *c.ev_g = st->ev_active ? c.G[st->gr[1]] : c.gdummy;
  *c.ev_act = st->ev_active;
}

template <typename S>
__device__ __forceinline__ void finish_solve(DevState<S>* st, int info) {
  st->phase = PH_DONE;
  st->info_final = info;
}

template <typename R, typename H, typename S>
__device__ __forceinline__ void post_round(const Ctx<R, H, S>& c) {
  DevState<S>* st = c.st;
  if (!(st->ev_active || st->ev_force)) return;
  if (!st->ev_force && st->ls_task == 1) {
    // the line search goes on; after 20 backtracks the reference leaves it at the next,
    // unevaluated trial point (352-358)
    st->phase = st->iback >= 20 ? PH_QUIRK : PH_LS;
    return;
  }
  // accepted: the evaluated point and its gradient become the iterate
  if (st->ev_is_z) {
    const int t = st->xr[0];
    st->xr[0] = st->xr[1];
    st->xr[1] = t;
  } else {
    const int t = st->xr[0];
    st->xr[0] = st->xr[2];
    st->xr[2] = t;
  }
  const int tg = st->gr[0];
  st->gr[0] = st->gr[1];
  st->gr[1] = tg;
  st->phase = PH_ITER;
  // stopping tests in the reference's order (394-429), leaving the summary's residuals as
  // the host loop does (each is updated only when its test is reached)
  st->res_g = st->sbgnrm;
  if (st->sbgnrm <= st->eps_g) {
    finish_solve(st, 4);
    return;
  }
  st->res_x = st->tf;
  if (st->tf <= st->eps_x) {
    finish_solve(st, 2);
    return;
  }
  const S fold = st->fold, fc = st->f;
  const S ddum = smax<S>(sabs(fold), smax<S>(sabs(fc), S(1)));
  st->res_f = (fold - fc) / ddum;
  if (fold - fc <= st->eps_f * ddum) {
    finish_solve(st, 1);
    return;
  }
  if (st->iter > st->max_iteration && st->max_iteration > 0) {
    finish_solve(st, 5);
    return;
  }
  if (st->internal_fail != 0) st->reset_pending = 1;  // formt failed (451-459)
}

template <typename R, typename H, typename S>
__global__ void k_round_begin(Ctx<R, H, S> c) {
  if (threadIdx.x == 0 && blockIdx.x == 0) round_begin<R, H, S>(c);
}
template <typename R, typename H, typename S>
__global__ void k_pre_eval(Ctx<R, H, S> c) {
  if (threadIdx.x == 0 && blockIdx.x == 0) pre_eval<R, H, S>(c);
}
template <typename R, typename H, typename S>
__global__ void k_post_round(Ctx<R, H, S> c) {
  if (threadIdx.x == 0 && blockIdx.x == 0) post_round<R, H, S>(c);
}

}  // namespace lbfgsb_b200
