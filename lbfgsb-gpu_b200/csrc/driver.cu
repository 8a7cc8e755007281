// driver.cu -- host driver and C ABI of the sm_100a L-BFGS-B library.
//
// The outer loop restates the reference's CPU driver (culbfgsb/lbfgsbcpu.cpp:117-465)
// over the device passes of passes.cuh / walk.cuh.  All solver state stays on the
// device; the host reads a small control header twice per iteration: once after the
// subspace step (to call the user's funcgrad at the trial point) and once after each
// function evaluation (the line-search decision and the stopping-test quantities).  The
// reference's GPU driver synchronises about 15 times and launches 30-60 kernels and
// cuBLAS/Thrust calls per iteration (lbfgsbcuda.cpp:212-390); this one launches 5.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lbfgsb_b200.h"
#include "host.cuh"
#include "shard.cuh"

namespace lbfgsb_b200 {

thread_local std::string g_last_error;
thread_local lbfgsb_b200_stats g_last_stats;

// A sharded solve's all-gather returned an error code.
struct ShardFailure {
  int rc;
};

// Page-locked host doubles for a sharded solve's small exchanges.
struct PinnedDoubles {
  double* p = nullptr;
  explicit PinnedDoubles(size_t n) { CK(cudaMallocHost(&p, n * sizeof(double))); }
  ~PinnedDoubles() {
    if (p) cudaFreeHost(p);
  }
  PinnedDoubles(const PinnedDoubles&) = delete;
  PinnedDoubles& operator=(const PinnedDoubles&) = delete;
};

constexpr int kMaxDevices = 64;
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[kMaxDevices] = {};

cudaMemPool_t workspace_pool() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw CudaFailure{cudaErrorInvalidDevice, "device ordinal", __LINE__};
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    CK(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~0ull;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}

template <typename R, typename H, typename S>
static int solve(int n, R* x_user, const int* nbd, const R* l, const R* u,
                 const typename Api<R>::Opt* opt, typename Api<R>::Cb funcgrad,
                 typename Api<R>::Cb after_iter, typename Api<R>::Cb custom_stop, void* user,
                 cudaStream_t stream, const lbfgsb_b200_ext* ext,
                 typename Api<R>::Sum* summary, const lbfgsb_b200_shard* sh = nullptr) {
  using Sum = typename Api<R>::Sum;
  g_last_error.clear();
  std::memset(&g_last_stats, 0, sizeof(g_last_stats));
  if (!opt || !summary || !x_user || !nbd || !l || !u) return LBFGSB_B200_ERR_ARGUMENT;
  if (opt->mode != LBFGSB_B200_MODE_CUDA) {
    summary->info = -1;
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  const int m = std::min(opt->hessian_approximate_dimension, kMaxM);
  // a sharded solve: this rank's n variables start at global index sh->offset
  if (sh && (sh->world < 1 || sh->rank < 0 || sh->rank >= sh->world || !sh->allgather ||
             sh->offset < 0 || n <= 0 || (long long)sh->offset + n > (long long)sh->n_global ||
             sh->world * kShardRow > (1 << 30)))
    return LBFGSB_B200_ERR_ARGUMENT;
  const int n_all = sh ? sh->n_global : n;
  // errclb's scalar checks and the driver's option checks (lbfgsbcpu.cpp:258-264, 879-890)
  if (n <= 0 || m <= 0 || m > n_all || opt->eps_f < 0 || opt->max_iteration < 0 ||
      opt->eps_g < 0 || opt->eps_x < 0) {
    summary->info = -1;
    return LBFGSB_B200_OK;
  }
  if (!funcgrad) {  // the reference's GPU driver rejects a missing callback (lbfgsbcuda.cpp:28-33)
    summary->info = -1;
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  const bool profile = ext && ext->profile;
  lbfgsb_b200_trace_callback trace = ext ? ext->trace : nullptr;
  void* trace_user = ext ? ext->trace_user : nullptr;

  Workspace<R, H, S> w;
  w.s = stream;
  Launcher L(stream, profile);
  bool fused = false;  // the post-evaluation pass runs the next Cauchy scan (k_post_gcp)
  long long syncs = 0, evals = 0;
  // direction passes that wrote the speculative z: for the per-launch byte counts of the
  // stats
  long long dir_spec = 0;
  int prev_no_spec = 0;
  try {
    const size_t N = (size_t)n;
    Ctx<R, H, S> c;
    Plan p;
    prepare<R, H, S>(w, c, p, n, m, nbd, l, u, stream, ext, false);
    const PassCfg &p_gcp = p.gcp, &p_freev = p.freev, &p_dir = p.dir, &p_apply = p.apply,
                  &p_post = p.post, &p_pgcp = p.pgcp;
    const int g_proj = p.g_proj, g_elem = p.g_elem;
    const int g_walk = walk_coop_grid<R, H, S>();
    DevState<S>& hs = *w.hs;
    // sharded: the buffers of the rank rows (shard.cuh, reduce.cuh) and of the walk records
    const int world = sh ? sh->world : 1;
    const int walk_chunk = kWalkChunk / world;
    std::unique_ptr<PinnedDoubles> pin;
    double *f_send = nullptr, *f_recv = nullptr, *rows_recv = nullptr;
    double *walk_send = nullptr, *walk_recv = nullptr;
    ShardWalk<S>* swk = nullptr;
    if (sh) {
      hs.n = sh->n_global;
      c.shard_world = world;
      c.ioff = sh->offset;
      c.shard_send = w.template alloc<double>(kShardRow);
      rows_recv = w.template alloc<double>((size_t)world * kShardRow);
      c.shard_recv = rows_recv;
      f_send = w.template alloc<double>(2);
      f_recv = w.template alloc<double>((size_t)world * 2);
      pin.reset(new PinnedDoubles((size_t)world * 2 + 4));
    }
    CK(cudaMemcpyAsync(w.st, &hs, sizeof(hs), cudaMemcpyHostToDevice, stream));
    const size_t header = offsetof(DevState<S>, big);
    auto pull = [&]() {
      CK(cudaMemcpyAsync(w.hs, w.st, header, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      syncs++;
      if (w.hs->device_error) throw CudaFailure{cudaErrorLaunchTimeout, "staged-tile wait", __LINE__};
    };
    auto exchange = [&](const double* send, double* recv, int count) {
      const int rc = sh->allgather(sh->allgather_user, send, recv, count, (void*)stream);
      if (rc != 0) throw ShardFailure{rc};
    };
    // two values of every rank (host side, in rank order) into pin->p[2 + 2r .. 3 + 2r]
    auto gather2 = [&](double a, double b) {
      pin->p[0] = a;
      pin->p[1] = b;
      CK(cudaMemcpyAsync(f_send, pin->p, 2 * sizeof(double), cudaMemcpyHostToDevice, stream));
      exchange(f_send, f_recv, 2);
      CK(cudaMemcpyAsync(pin->p + 2, f_recv, (size_t)world * 2 * sizeof(double),
                         cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      syncs++;
    };
    // the function value of a sharded solve: the ranks' shares added in rank order
    auto total_f = [&](R part) -> R {
      if (!sh) return part;
      gather2((double)part, 0.0);
      double a = 0.0;
      for (int r = 0; r < world; r++) a += pin->p[2 + 2 * r];
      return (R)a;
    };
    // a pass: the streaming launch, and for a sharded solve the exchange of the rank rows
    // and the one-CTA launch that folds them and runs the epilogue
    auto run_pass = [&](int kid, int grid, auto launch) {
      L.run(kid, [&] {
        launch(c, grid);
        if (sh) {
          exchange(c.shard_send, rows_recv, kShardRow);
          Ctx<R, H, S> e = c;
          e.epi_only = 1;
          launch(e, 1);
        }
      });
    };
    if (sh) {
      // the ranks' index ranges must tile 0 .. n_global in rank order
      gather2((double)n, (double)sh->offset);
      long long next = 0;
      bool tiled = true;
      for (int r = 0; r < world; r++) {
        const long long nr = (long long)pin->p[2 + 2 * r], orr = (long long)pin->p[3 + 2 * r];
        if (nr < 1 || orr != next) tiled = false;
        next += nr;
      }
      if (!tiled || next != sh->n_global) {
        summary->info = -1;
        CK(cudaStreamSynchronize(stream));
        return LBFGSB_B200_ERR_ARGUMENT;
      }
    }

    R* xcur = w.X[0];
    R* zb = w.X[1];
    R* tb = w.X[2];
    R* gcur = w.G[0];
    R* gnew = w.G[1];
    int info = 0;
    bool finished = false;
    auto finish = [&](int code) {
      summary->info = code;
      finished = true;
    };

    // errclb's per-variable checks and lbfgsbactive, into the solver's x buffer
    L.run(KID_INIT, [&] {
      k_init<R, S><<<g_elem, 256, 0, stream>>>(n, x_user, xcur, nbd, l, u, w.st);
    });
    if (sh) {
      k_shard_flags_put<S><<<1, 32, 0, stream>>>(w.st, c.shard_send);
      exchange(c.shard_send, rows_recv, kShardRow);
      k_shard_flags_get<S><<<1, 32, 0, stream>>>(w.st, rows_recv, world);
    }
    pull();
    if (hs.input_error) {
      summary->info = -1;  // x is left as given (lbfgsbcpu.cpp:259-264)
      CK(cudaStreamSynchronize(stream));
      goto done;
    }
    {
      const bool cnstnd = hs.cnstnd != 0;
      R f = 0;
      funcgrad(user, xcur, &f, gcur, (void*)stream, summary);
      evals++;
      f = total_f(f);
      run_pass(KID_PROJGR, g_proj, [&](const Ctx<R, H, S>& cc, int grid) {
        k_projgr<R, H, S><<<grid, kThreads, 0, stream>>>(cc, xcur, gcur, (S)f);
      });
      pull();
      summary->residual_g = (R)hs.sbgnrm;
      if (hs.sbgnrm <= (S)opt->eps_g) finish(4);

      int reset = 0;
      // with bounds, the post-evaluation pass also runs the next iteration's Cauchy scan
      // (k_post_gcp); spec: the last accepted step left that scan's result in the state
      fused = cnstnd;
      bool spec = false;
      DevState<S> snap;
      while (!finished) {
        const bool start_here = reset || !spec;
        if (start_here)
          L.run(KID_BEGIN, [&] { k_begin_iteration<S><<<1, 1, 0, stream>>>(w.st, reset); });
        spec = false;
        const int reset_before = reset;
        reset = 0;
        const int col_now = reset_before ? 0 : hs.col;
        const bool uncon = !cnstnd && col_now > 0;
        auto subspace = [&]() {
          c.stages = p_freev.stages;
          run_pass(KID_FREEV, p_freev.grid, [&](const Ctx<R, H, S>& cc, int grid) {
            k_freev_formk<R, H, S, kConsWide><<<grid, p_freev.threads, p_freev.smem, stream>>>(cc, xcur, gcur);
          });
          c.stages = p_dir.stages;
          run_pass(KID_SUBDIR, p_dir.grid, [&](const Ctx<R, H, S>& cc, int grid) {
            k_subsm_dir<R, H, S, kConsWide><<<grid, p_dir.threads, p_dir.smem, stream>>>(cc, xcur, gcur, zb);
          });
          // the direction pass applies an untruncated step itself (spec_apply); the apply
          // pass runs only when it has work, which the host learns from the state
          pull();
          if (!(hs.gcp_state == GCP_WALK || hs.internal_fail != 0 || hs.spec_apply)) {
            c.stages = p_apply.stages;
            run_pass(KID_SUBAPPLY, p_apply.grid, [&](const Ctx<R, H, S>& cc, int grid) {
              k_subsm_apply<R, H, S, kConsWide><<<grid, p_apply.threads, p_apply.smem, stream>>>(cc, xcur, gcur, zb);
            });
            pull();
          }
        };
        if (!uncon && start_here) {
          c.stages = p_gcp.stages;
          run_pass(KID_GCP, p_gcp.grid, [&](const Ctx<R, H, S>& cc, int grid) {
            k_gcp_scan<R, H, S, kConsWide><<<grid, p_gcp.threads, p_gcp.smem, stream>>>(cc, xcur, gcur);
          });
        }
        auto count_dir = [&]() {
          if (hs.subsm_active && hs.gcp_state != GCP_WALK && hs.internal_fail == 0) {
            if (!prev_no_spec) dir_spec++;
            prev_no_spec = hs.dir_no_spec;
          }
        };
        subspace();
        count_dir();
        if (hs.gcp_state == GCP_WALK && hs.internal_fail == 0) {
          if (!c.wl_t) walk_buffers(w, c, N);
          CK(cudaMemsetAsync(w.wl_n, 0, sizeof(unsigned int), stream));
          CK(cudaMemsetAsync(&c.wsc->bar, 0, sizeof(unsigned int), stream));
          if (!sh) {
            L.run(KID_WALK, [&] { launch_walk_coop<R, H, S>(c, xcur, gcur, g_walk, stream); });
          } else {
            // the walk over every rank's breakpoints (shard.cuh): select, gather, walk up to
            // the frontier, until the walk ends; then each rank marks what it owns
            if (!swk) {
              swk = w.template alloc<ShardWalk<S>>(1);
              walk_send = w.template alloc<double>(shard_walk_block(walk_chunk));
              walk_recv = w.template alloc<double>((size_t)world * shard_walk_block(walk_chunk));
            }
            L.run(KID_WALK, [&] {
              k_walk_gather<R, H, S><<<g_elem, kThreads, 0, stream>>>(c, xcur, gcur);
              CK(cudaMemsetAsync(swk, 0, sizeof(ShardWalk<S>), stream));
              int* h_done = reinterpret_cast<int*>(pin->p);
              while (true) {
                k_shard_walk_select<R, H, S><<<1, kWalkThreads, 0, stream>>>(c, xcur, gcur, swk,
                                                                             walk_chunk, walk_send);
                exchange(walk_send, walk_recv, shard_walk_block(walk_chunk));
                k_shard_walk_merge<R, H, S><<<1, kWalkThreads, 0, stream>>>(c, walk_recv, world,
                                                                            walk_chunk, swk);
                CK(cudaMemcpyAsync(h_done, reinterpret_cast<char*>(swk) + offsetof(ShardWalk<S>, done),
                                   sizeof(int), cudaMemcpyDeviceToHost, stream));
                CK(cudaStreamSynchronize(stream));
                syncs++;
                if (*h_done) break;
              }
              k_shard_walk_end<S><<<1, 32, 0, stream>>>(w.st, swk);
              k_shard_walk_mark<R, H, S><<<g_elem, 256, 0, stream>>>(c, gcur, swk);
            });
          }
          subspace();
          count_dir();
        }
        if (hs.internal_fail != 0) {  // cauchy/formk/cmprlb/subsm failed: reset (297-341)
          reset = 1;
          continue;
        }
        snap = hs;
        if (trace) {  // the trace also reports a few entries of the small matrices
          CK(cudaMemcpyAsync(&snap, w.st, sizeof(snap), cudaMemcpyDeviceToHost, stream));
          CK(cudaStreamSynchronize(stream));
        }
        if (hs.ls_info != 0) {
          // g'd >= 0 at the start of the line search: x, g, f stay (359-387)
          if (hs.col == 0) {
            finish(-2);
            break;
          }
          reset = 1;
          continue;
        }
        auto post = [&](R* xt_, R fval, int force) {
          if (fused) {
            c.stages = p_pgcp.stages;
            run_pass(KID_POSTGCP, p_pgcp.grid, [&](const Ctx<R, H, S>& cc, int grid) {
              k_post_gcp<R, H, S, kConsWide><<<grid, p_pgcp.threads, p_pgcp.smem, stream>>>(
                  cc, xcur, zb, xt_, gnew, gcur, (S)fval, force);
            });
          } else {
            c.stages = p_post.stages;
            run_pass(KID_POST, p_post.grid, [&](const Ctx<R, H, S>& cc, int grid) {
              k_post_eval<R, H, S, kConsWide><<<grid, p_post.threads, p_post.smem, stream>>>(
                  cc, xcur, zb, xt_, gnew, gcur, (S)fval, force);
            });
          }
        };
        // line search (347-358)
        R* xt = zb;
        bool quirk = false;
        while (true) {
          if (hs.stp == S(1)) {
            xt = zb;
          } else {
            L.run(KID_TRIAL, [&] {
              k_trial<R, S><<<g_elem, 256, 0, stream>>>(n, xcur, zb, tb, w.st);
            });
            xt = tb;
          }
          funcgrad(user, xt, &f, gnew, (void*)stream, summary);
          evals++;
          f = total_f(f);
          post(xt, f, 0);
          pull();
          if (hs.ls_task != 1) break;
          if (hs.iback >= 20) {
            quirk = true;
            break;
          }
        }
        if (quirk) {
          // the reference leaves the search after 20 backtracks with x at the new,
          // unevaluated trial point and f, g of the previous one (352-358)
          if (hs.stp == S(1)) {
            xt = zb;
          } else {
            L.run(KID_TRIAL, [&] {
              k_trial<R, S><<<g_elem, 256, 0, stream>>>(n, xcur, zb, tb, w.st);
            });
            xt = tb;
          }
          post(xt, f, 1);
          pull();
        }
        if (xt == zb)
          std::swap(xcur, zb);
        else
          std::swap(xcur, tb);
        std::swap(gcur, gnew);
        spec = fused && hs.spec_gcp != 0;
        summary->num_iteration = hs.iter;
        if (trace) {
          lbfgsb_b200_trace_record rec;
          rec.iter = hs.iter;
          rec.nint = snap.nint;
          rec.nbreak = snap.gcp_state == GCP_SKIPPED ? 0 : snap.nbreak;
          rec.nfree = snap.nfree;
          rec.nenter = snap.nenter;
          rec.nleave = snap.nleave;
          rec.col = snap.col;
          rec.head = snap.head;
          rec.nfgv = hs.nfgv + 1;  // the oracle counts the first evaluation too
          rec.ifun = hs.ifun;
          rec.iword = snap.subsm_active ? snap.iword : -1;
          rec.reset = reset_before;
          rec.free_hash = snap.free_hash;
          rec.at_lower = snap.at_lower;
          rec.at_upper = snap.at_upper;
          rec.f = (double)hs.f;
          rec.theta = (double)snap.theta;
          rec.stp = (double)hs.stp;
          rec.dtm = (double)snap.dtm;
          rec.tsum = (double)snap.tsum;
          rec.gd = (double)hs.gd;
          rec.gdold = (double)hs.gdold;
          rec.dtd = (double)hs.dtd;
          rec.stpmx = (double)hs.stpmx;
          rec.f1_0 = (double)snap.f1_0;
          rec.f2_0 = (double)snap.f2_0;
          const int cc = snap.col;
          rec.dbg[0] = cc > 0 ? (double)snap.p[1] : 0;
          rec.dbg[1] = cc > 0 ? (double)snap.p[cc + 1] : 0;
          rec.dbg[2] = cc > 0 ? (double)snap.c[1] : 0;
          rec.dbg[3] = cc > 0 ? (double)snap.c[cc + 1] : 0;
          rec.dbg[4] = cc > 0 ? (double)snap.mc[1] : 0;
          rec.dbg[5] = cc > 0 ? (double)snap.mc[cc + 1] : 0;
          rec.dbg[6] = cc > 0 ? (double)snap.sy[0] : 0;
          rec.dbg[7] = cc > 0 ? (double)snap.wt[0] : 0;
          trace(trace_user, &rec);
        }
        if (after_iter) after_iter(user, xcur, &f, gcur, (void*)stream, summary);
        // stopping tests in the reference's order (394-429)
        summary->residual_g = (R)hs.sbgnrm;
        if (hs.sbgnrm <= (S)opt->eps_g) {
          finish(4);
          break;
        }
        summary->residual_x = (R)hs.tf;
        if (hs.tf <= (S)opt->eps_x) {
          finish(2);
          break;
        }
        {
          const S fold = hs.fold, fc = hs.f;
          const S ddum = smax<S>(sabs(fold), smax<S>(sabs(fc), S(1)));
          summary->residual_f = (R)((fold - fc) / ddum);
          if (fold - fc <= (S)opt->eps_f * ddum) {
            finish(1);
            break;
          }
        }
        if (hs.iter > opt->max_iteration && opt->max_iteration > 0) {
          finish(5);
          break;
        }
        if (custom_stop && custom_stop(user, xcur, &f, gcur, (void*)stream, summary)) {
          finish(0);
          break;
        }
        if (hs.internal_fail != 0) {  // formt failed (451-459)
          reset = 1;
          continue;
        }
      }
      (void)info;
    }
    CK(cudaMemcpyAsync(x_user, xcur, N * sizeof(R), cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  done:
    lbfgsb_b200_stats& st = g_last_stats;
    st.kernels = KID_COUNT;
    for (int k = 0; k < KID_COUNT; k++) {
      std::snprintf(st.name[k], sizeof(st.name[k]), "%s", kKernelNames[k]);
    }
    L.collect(&st);
    st.host_syncs = syncs;
    st.evaluations = evals;
    // algorithmic bytes of one launch (steady state, all variables free, col = m)
    const double Rb = sizeof(R), Hb = sizeof(H), hist = 2.0 * m * Hb, nn = (double)n;
    st.bytes[KID_GCP] = nn * (4 * Rb + 4 + hist + 1);
    st.bytes[KID_FREEV] = nn * (2 * Rb + hist + 1 + 0.25);
    // per launch, averaged over the launches made: the direction pass writes z when it
    // speculates; k_subsm_apply is launched only for the steps it applies
    const double ndir = std::max<double>(1.0, (double)g_last_stats.launches[KID_SUBDIR]);
    st.bytes[KID_SUBDIR] = nn * (5 * Rb + hist + 5 + Rb * (double)dir_spec / ndir);
    st.bytes[KID_SUBAPPLY] = nn * (6 * Rb + 5);
    st.bytes[KID_POST] = nn * (6 * Rb + 4 + hist + 2 * Hb);
    st.bytes[KID_POSTGCP] = nn * (6 * Rb + 4 + hist + 2 * Hb + 1);
    st.bytes[KID_TRIAL] = nn * 3 * Rb;
    st.bytes[KID_WALK] = nn * (4 * Rb + 4);  // the listing pass of the cooperative walk
    st.bytes[KID_PROJGR] = nn * (4 * Rb + 4);
    st.bytes[KID_INIT] = nn * (4 * Rb + 4);
    st.bytes_per_iteration_model =
        (fused ? st.bytes[KID_POSTGCP] : st.bytes[KID_POST] + st.bytes[KID_GCP]) +
        st.bytes[KID_FREEV] + st.bytes[KID_SUBDIR] +
        st.bytes[KID_SUBAPPLY] * (double)g_last_stats.launches[KID_SUBAPPLY] / ndir;  // averaged
  } catch (const CudaFailure& e) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s failed at driver.cu:%d: %s", e.call, e.line,
                  cudaGetErrorString(e.err));
    g_last_error = buf;
    return LBFGSB_B200_ERR_CUDA;
  } catch (const ShardFailure& e) {
    g_last_error = "the sharded solve's allgather returned " + std::to_string(e.rc);
    return LBFGSB_B200_ERR_CALLBACK;
  }
  return LBFGSB_B200_OK;
}

// A solve whose objective keeps f on the device (no counterpart in the reference, whose
// callback returns f on the host): the outer loop's decisions run on the device
// (rounds.cuh), one round is captured into a CUDA graph and relaunched, and the host reads
// the state once before the first iteration and then every few rounds.  The results equal
// those of solve() with the same objective, bit for bit.
template <typename R, typename H, typename S>
static int solve_device(int n, R* x_user, const int* nbd, const R* l, const R* u,
                        const typename Api<R>::Opt* opt, typename DevObjective<R>::Fn objective,
                        void* user, cudaStream_t ustream, const lbfgsb_b200_ext* ext,
                        typename Api<R>::Sum* summary) {
  g_last_error.clear();
  std::memset(&g_last_stats, 0, sizeof(g_last_stats));
  if (!opt || !summary || !x_user || !nbd || !l || !u) return LBFGSB_B200_ERR_ARGUMENT;
  if (opt->mode != LBFGSB_B200_MODE_CUDA) {
    summary->info = -1;
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  const int m = std::min(opt->hessian_approximate_dimension, kMaxM);
  if (n <= 0 || m <= 0 || m > n || opt->eps_f < 0 || opt->max_iteration < 0 ||
      opt->eps_g < 0 || opt->eps_x < 0) {
    summary->info = -1;
    return LBFGSB_B200_OK;
  }
  if (!objective) {
    summary->info = -1;
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  long long syncs = 0, rounds_launched = 0, launches = 0;
  try {
    RoundStream& rs = round_stream();
    const cudaStream_t stream = rs.s;
    CK(cudaEventRecord(rs.in, ustream));
    CK(cudaStreamWaitEvent(stream, rs.in, 0));
    Workspace<R, H, S> w;
    w.s = stream;
    const size_t N = (size_t)n;
    Ctx<R, H, S> c;
    Plan p;
    prepare<R, H, S>(w, c, p, n, m, nbd, l, u, stream, ext, true);
    EvalSlots* slot = w.template alloc<EvalSlots>(1);
    c.ev_x = reinterpret_cast<R**>(&slot->x);
    c.ev_g = reinterpret_cast<R**>(&slot->g);
    c.ev_f = &slot->f;
    c.ev_act = &slot->active;
    c.gdummy = w.template alloc<R>(N);
    DevState<S>& hs = *w.hs;
    hs.phase = PH_ITER;
    hs.eps_g = (S)opt->eps_g;
    hs.eps_x = (S)opt->eps_x;
    hs.eps_f = (S)opt->eps_f;
    hs.max_iteration = opt->max_iteration;
    hs.res_x = (S)summary->residual_x;  // left as given unless a test reaches them
    hs.res_f = (S)summary->residual_f;
    CK(cudaMemcpyAsync(w.st, &hs, sizeof(hs), cudaMemcpyHostToDevice, stream));
    const size_t header = offsetof(DevState<S>, big);
    auto pull = [&]() {
      CK(cudaMemcpyAsync(w.hs, w.st, header, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      syncs++;
      if (w.hs->device_error) throw CudaFailure{cudaErrorLaunchTimeout, "staged-tile wait", __LINE__};
    };
    k_init<R, S><<<p.g_elem, 256, 0, stream>>>(n, x_user, w.X[0], nbd, l, u, w.st);
    CK(cudaGetLastError());
    launches++;
    pull();
    bool done = false;
    if (hs.input_error) {
      summary->info = -1;  // x is left as given (lbfgsbcpu.cpp:259-264)
      done = true;
    }
    if (!done) {
      // the first evaluation, at x0, and projgr there (lbfgsbcpu.cpp:266-276)
      c.rounds = 1;
      EvalSlots* hslot = static_cast<EvalSlots*>(pinned_mirror_slot(sizeof(EvalSlots)));
      hslot->x = w.X[0];
      hslot->g = w.G[0];
      hslot->f = 0;
      hslot->active = 1;
      CK(cudaMemcpyAsync(slot, hslot, sizeof(EvalSlots), cudaMemcpyHostToDevice, stream));
      objective(user, (const R* const*)c.ev_x, c.ev_g, c.ev_f, c.ev_act, (void*)stream);
      CK(cudaGetLastError());
      k_projgr<R, H, S><<<p.g_proj, kThreads, 0, stream>>>(c, nullptr, nullptr, S(0));
      CK(cudaGetLastError());
      launches++;
      pull();
      summary->residual_g = (R)hs.sbgnrm;
      if (hs.sbgnrm <= (S)opt->eps_g) {
        summary->info = 4;
        done = true;
      }
    }
    if (!done) {
      const bool fused = hs.cnstnd != 0;
      const int g_walk = walk_coop_grid<R, H, S>();
      auto round = [&]() {
        k_round_begin<R, H, S><<<1, 32, 0, stream>>>(c);
        c.stages = p.gcp.stages;
        k_gcp_scan<R, H, S, kConsWide><<<p.gcp.grid, p.gcp.threads, p.gcp.smem, stream>>>(c, nullptr, nullptr);
        launch_walk_coop<R, H, S>(c, (const R*)nullptr, (const R*)nullptr, g_walk, stream);
        c.stages = p.freev.stages;
        k_freev_formk<R, H, S, kConsWide><<<p.freev.grid, p.freev.threads, p.freev.smem, stream>>>(c, nullptr, nullptr);
        c.stages = p.dir.stages;
        k_subsm_dir<R, H, S, kConsWide><<<p.dir.grid, p.dir.threads, p.dir.smem, stream>>>(c, nullptr, nullptr, nullptr);
        c.stages = p.apply.stages;
        k_subsm_apply<R, H, S, kConsWide><<<p.apply.grid, p.apply.threads, p.apply.smem, stream>>>(c, nullptr, nullptr, nullptr);
        k_pre_eval<R, H, S><<<1, 32, 0, stream>>>(c);
        k_trial_round<R, H, S><<<p.g_elem, 256, 0, stream>>>(c);
        objective(user, (const R* const*)c.ev_x, c.ev_g, c.ev_f, c.ev_act, (void*)stream);
        if (fused) {
          c.stages = p.pgcp.stages;
          k_post_gcp<R, H, S, kConsWide><<<p.pgcp.grid, p.pgcp.threads, p.pgcp.smem, stream>>>(
              c, nullptr, nullptr, nullptr, nullptr, nullptr, S(0), 0);
        } else {
          c.stages = p.post.stages;
          k_post_eval<R, H, S, kConsWide><<<p.post.grid, p.post.threads, p.post.smem, stream>>>(
              c, nullptr, nullptr, nullptr, nullptr, nullptr, S(0), 0);
        }
        k_post_round<R, H, S><<<1, 32, 0, stream>>>(c);
      };
      constexpr int kRoundKernels = 11;
      RoundGraph rg;
      CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      round();
      const cudaError_t launch_err = cudaGetLastError();
      const cudaError_t cap_err = cudaStreamEndCapture(stream, &rg.g);
      CK(launch_err);
      CK(cap_err);
      CK(cudaGraphInstantiate(&rg.e, rg.g, 0));
      // rounds between two reads of the state: few at first, then about a quarter of the
      // rounds so far (a finished solve idles through at most that many rounds)
      int batch = 4;
      while (true) {
        for (int r = 0; r < batch; r++) CK(cudaGraphLaunch(rg.e, stream));
        rounds_launched += batch;
        pull();
        if (hs.phase == PH_DONE) break;
        batch = (int)std::min<long long>(64, std::max<long long>(4, rounds_launched / 4));
      }
      launches += rounds_launched * kRoundKernels;
      summary->info = hs.info_final;
      summary->num_iteration = hs.iter;
      summary->residual_g = (R)hs.res_g;
      summary->residual_x = (R)hs.res_x;
      summary->residual_f = (R)hs.res_f;
    }
    if (!hs.input_error) {
      CK(cudaMemcpyAsync(x_user, w.X[hs.xr[0]], N * sizeof(R), cudaMemcpyDeviceToDevice, stream));
    }
    CK(cudaEventRecord(rs.out, stream));
    CK(cudaStreamWaitEvent(ustream, rs.out, 0));
    w.release();  // the workspace returns to the pool on the solve's stream
    CK(cudaStreamSynchronize(stream));
    lbfgsb_b200_stats& st = g_last_stats;
    st.kernels = 0;
    st.total_launches = launches;
    st.host_syncs = syncs;
    st.evaluations = hs.nfgv + 1;
    st.rounds = rounds_launched;
  } catch (const CudaFailure& e) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s failed at driver.cu:%d: %s", e.call, e.line,
                  cudaGetErrorString(e.err));
    g_last_error = buf;
    return LBFGSB_B200_ERR_CUDA;
  }
  return LBFGSB_B200_OK;
}

template <typename R, typename Opt>
static void default_option(Opt* o, R meps, R mmax) {
  o->eps_f = o->eps_g = o->eps_x = (R)1e-15;
  o->hessian_approximate_dimension = 8;
  o->machine_epsilon = meps;
  o->machine_maximum = mmax;
  o->max_iteration = 1000;
  o->mode = LBFGSB_B200_MODE_CUDA;
  o->step_scaling = (R)1.0;
}

// Independent solves side by side: `concurrency` host workers, each with its own
// non-blocking stream on the caller's device, take instances in order and run the plain
// solve on them; instance k's result is the one its solo solve gives (the solve is
// deterministic and its workspace private).  status[k] gets the instance's return code
// and seconds[k] (optional) its wall time; the return value is the first failing code.
template <typename R>
static int minimize_batch(int count, const int* n, R* const* x, const int* const* nbd,
                          const R* const* l, const R* const* u,
                          const typename Api<R>::Opt* option, typename Api<R>::Cb funcgrad,
                          void* const* user, int concurrency, typename Api<R>::Sum* summary,
                          int* status, double* seconds) {
  g_last_error.clear();
  if (count < 0 || (count > 0 && (!n || !x || !nbd || !l || !u || !option || !funcgrad ||
                                  !summary || !status))) {
    g_last_error = "minimize_batch: null argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  if (count == 0) return LBFGSB_B200_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_last_error = cudaGetErrorString(e);
    return LBFGSB_B200_ERR_CUDA;
  }
  const int workers = std::max(1, std::min(concurrency > 0 ? concurrency : 16, count));
  std::atomic<int> next{0};
  std::mutex mu;
  std::string first_error;
  int first_status = LBFGSB_B200_OK;
  auto work = [&]() {
    cudaStream_t s = nullptr;
    if (cudaSetDevice(dev) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      std::lock_guard<std::mutex> lock(mu);
      if (first_status == LBFGSB_B200_OK) {
        first_status = LBFGSB_B200_ERR_CUDA;
        first_error = "minimize_batch: worker stream set-up failed";
      }
      return;
    }
    for (int k = next++; k < count; k = next++) {
      const auto t0 = std::chrono::steady_clock::now();
      const int st = solve<R, R, R>(n[k], x[k], nbd[k], l[k], u[k], option, funcgrad, nullptr,
                                    nullptr, user ? user[k] : nullptr, s, nullptr, &summary[k]);
      status[k] = st;
      if (seconds)
        seconds[k] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (st != LBFGSB_B200_OK) {
        std::lock_guard<std::mutex> lock(mu);
        if (first_status == LBFGSB_B200_OK) {
          first_status = st;
          first_error = g_last_error;
        }
      }
    }
    cudaStreamDestroy(s);
  };
  for (int k = 0; k < count; k++) status[k] = -1;
  std::vector<std::thread> pool;
  for (int w = 0; w < workers; w++) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  if (first_status != LBFGSB_B200_OK) g_last_error = first_error;
  return first_status;
}

// Bytes that one solve of n elements may take from the workspace pool: an upper bound
// (the 16-byte aligned copies of l, u and nbd, the breakpoint-walk buffers, and reduction
// rows for up to 4096 CTAs included).  It calls nothing on the device.
static size_t workspace_bound(long long n, size_t real, size_t hist) {
  const size_t N = (size_t)std::max<long long>(n, 1);
  const size_t ld = ((N + kTile - 1) / kTile) * kTile;
  constexpr size_t kRowsBound = 4096;
  return N * (8 * real + 4 + 1 + 12) + 2 * ld * kSlots * hist + (N / 32 + 2) * 4 +
         sizeof(DevState<double>) + kRowsBound * 256 * 8 + ((size_t)1 << 20);
}

// Serving front end.  Requests (whole FP32 solves on the caller's device arrays) arrive
// one by one, wait in arrival order until their workspace fits in the HBM budget beside
// the solves already running, and run on a pool of host workers, each with its own
// stream.  Admission is first come, first served: a request that does not fit holds back
// the ones behind it until running solves release enough memory.
struct ServeRequest {
  int n = 0;
  float* x = nullptr;
  const int* nbd = nullptr;
  const float* l = nullptr;
  const float* u = nullptr;
  lbfgsb_b200_option_f32 option{};
  lbfgsb_b200_callback_f32 funcgrad = nullptr;
  void* user = nullptr;
  size_t bytes = 0;
  std::chrono::steady_clock::time_point arrive, start, finish;
  lbfgsb_b200_summary_f32 summary{};
  int status = -1;
  bool done = false;
  std::string error;
};

struct Server {
  int dev = 0, form = LBFGSB_B200_FORM_MIXED;
  size_t budget = 0, in_use = 0, peak_bytes = 0;
  int running = 0, peak_running = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServeRequest> reqs;  // by id (push_back keeps references to the others valid)
  std::deque<long long> queue;    // ids waiting for admission, in arrival order
  bool stop = false;
  std::vector<std::thread> workers;
};

static void serve_worker(Server* sv) {
  cudaStream_t s = nullptr;
  const bool ok = cudaSetDevice(sv->dev) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
  std::unique_lock<std::mutex> lock(sv->mu);
  for (;;) {
    sv->cv_work.wait(lock, [&] {
      return (sv->stop && sv->queue.empty()) ||
             (!sv->queue.empty() && sv->in_use + sv->reqs[(size_t)sv->queue.front()].bytes <= sv->budget);
    });
    if (sv->queue.empty()) break;
    const long long id = sv->queue.front();
    sv->queue.pop_front();
    ServeRequest& r = sv->reqs[(size_t)id];
    sv->in_use += r.bytes;
    sv->peak_bytes = std::max(sv->peak_bytes, sv->in_use);
    sv->peak_running = std::max(sv->peak_running, ++sv->running);
    r.start = std::chrono::steady_clock::now();
    lock.unlock();
    int st = LBFGSB_B200_ERR_CUDA;
    std::string err = "server: worker stream set-up failed";
    if (ok) {
      lbfgsb_b200_ext ext{};
      ext.form = sv->form;
      if (sv->form == LBFGSB_B200_FORM_MIXED)
        st = solve<float, float, double>(r.n, r.x, r.nbd, r.l, r.u, &r.option, r.funcgrad, nullptr,
                                         nullptr, r.user, s, &ext, &r.summary);
      else if (sv->form == LBFGSB_B200_FORM_MIXED_BF16)
        st = solve<float, __nv_bfloat16, double>(r.n, r.x, r.nbd, r.l, r.u, &r.option, r.funcgrad,
                                                 nullptr, nullptr, r.user, s, &ext, &r.summary);
      else
        st = solve<float, float, float>(r.n, r.x, r.nbd, r.l, r.u, &r.option, r.funcgrad, nullptr,
                                        nullptr, r.user, s, &ext, &r.summary);
      err = st == LBFGSB_B200_OK ? std::string() : g_last_error;
    }
    lock.lock();
    sv->in_use -= r.bytes;
    sv->running--;
    r.finish = std::chrono::steady_clock::now();
    r.status = st;
    r.error = err;
    r.done = true;
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
  }
  lock.unlock();
  if (s) cudaStreamDestroy(s);
}

}  // namespace lbfgsb_b200

using namespace lbfgsb_b200;

extern "C" {

void lbfgsb_b200_default_option_f64(lbfgsb_b200_option_f64* o) {
  if (o) default_option<double>(o, 1e-15, 1.7976931348623157e308);
}
void lbfgsb_b200_default_option_f32(lbfgsb_b200_option_f32* o) {
  if (o) default_option<float>(o, 1e-8f, 3.40282347e38f);
}

int lbfgsb_b200_minimize_ext_f64(int n, double* x, const int* nbd, const double* l,
                                 const double* u, const lbfgsb_b200_option_f64* option,
                                 lbfgsb_b200_callback_f64 funcgrad,
                                 lbfgsb_b200_callback_f64 after_iteration,
                                 lbfgsb_b200_callback_f64 customized_stopping, void* user,
                                 void* stream, const lbfgsb_b200_ext* ext,
                                 lbfgsb_b200_summary_f64* summary) {
  return solve<double, double, double>(n, x, nbd, l, u, option, funcgrad, after_iteration,
                                       customized_stopping, user, (cudaStream_t)stream, ext,
                                       summary);
}

int lbfgsb_b200_minimize_ext_f32(int n, float* x, const int* nbd, const float* l,
                                 const float* u, const lbfgsb_b200_option_f32* option,
                                 lbfgsb_b200_callback_f32 funcgrad,
                                 lbfgsb_b200_callback_f32 after_iteration,
                                 lbfgsb_b200_callback_f32 customized_stopping, void* user,
                                 void* stream, const lbfgsb_b200_ext* ext,
                                 lbfgsb_b200_summary_f32* summary) {
  const int form = ext ? ext->form : LBFGSB_B200_FORM_PLAIN;
  cudaStream_t s = (cudaStream_t)stream;
  if (form == LBFGSB_B200_FORM_MIXED)
    return solve<float, float, double>(n, x, nbd, l, u, option, funcgrad, after_iteration,
                                       customized_stopping, user, s, ext, summary);
  if (form == LBFGSB_B200_FORM_MIXED_BF16)
    return solve<float, __nv_bfloat16, double>(n, x, nbd, l, u, option, funcgrad,
                                               after_iteration, customized_stopping, user, s,
                                               ext, summary);
  return solve<float, float, float>(n, x, nbd, l, u, option, funcgrad, after_iteration,
                                    customized_stopping, user, s, ext, summary);
}

int lbfgsb_b200_minimize_sharded_f64(const lbfgsb_b200_shard* shard, int n_local, double* x,
                                     const int* nbd, const double* l, const double* u,
                                     const lbfgsb_b200_option_f64* option,
                                     lbfgsb_b200_callback_f64 funcgrad,
                                     lbfgsb_b200_callback_f64 after_iteration,
                                     lbfgsb_b200_callback_f64 customized_stopping, void* user,
                                     void* stream, const lbfgsb_b200_ext* ext,
                                     lbfgsb_b200_summary_f64* summary) {
  if (!shard) return LBFGSB_B200_ERR_ARGUMENT;
  return solve<double, double, double>(n_local, x, nbd, l, u, option, funcgrad, after_iteration,
                                       customized_stopping, user, (cudaStream_t)stream, ext,
                                       summary, shard);
}

int lbfgsb_b200_minimize_sharded_f32(const lbfgsb_b200_shard* shard, int n_local, float* x,
                                     const int* nbd, const float* l, const float* u,
                                     const lbfgsb_b200_option_f32* option,
                                     lbfgsb_b200_callback_f32 funcgrad,
                                     lbfgsb_b200_callback_f32 after_iteration,
                                     lbfgsb_b200_callback_f32 customized_stopping, void* user,
                                     void* stream, const lbfgsb_b200_ext* ext,
                                     lbfgsb_b200_summary_f32* summary) {
  if (!shard) return LBFGSB_B200_ERR_ARGUMENT;
  const int form = ext ? ext->form : LBFGSB_B200_FORM_PLAIN;
  cudaStream_t s = (cudaStream_t)stream;
  if (form == LBFGSB_B200_FORM_MIXED)
    return solve<float, float, double>(n_local, x, nbd, l, u, option, funcgrad, after_iteration,
                                       customized_stopping, user, s, ext, summary, shard);
  if (form == LBFGSB_B200_FORM_MIXED_BF16)
    return solve<float, __nv_bfloat16, double>(n_local, x, nbd, l, u, option, funcgrad,
                                               after_iteration, customized_stopping, user, s,
                                               ext, summary, shard);
  return solve<float, float, float>(n_local, x, nbd, l, u, option, funcgrad, after_iteration,
                                    customized_stopping, user, s, ext, summary, shard);
}

int lbfgsb_b200_minimize_device_f64(int n, double* x, const int* nbd, const double* l,
                                    const double* u, const lbfgsb_b200_option_f64* option,
                                    lbfgsb_b200_device_objective_f64 objective, void* user,
                                    void* stream, const lbfgsb_b200_ext* ext,
                                    lbfgsb_b200_summary_f64* summary) {
  return solve_device<double, double, double>(n, x, nbd, l, u, option, objective, user,
                                              (cudaStream_t)stream, ext, summary);
}

int lbfgsb_b200_minimize_device_f32(int n, float* x, const int* nbd, const float* l,
                                    const float* u, const lbfgsb_b200_option_f32* option,
                                    lbfgsb_b200_device_objective_f32 objective, void* user,
                                    void* stream, const lbfgsb_b200_ext* ext,
                                    lbfgsb_b200_summary_f32* summary) {
  const int form = ext ? ext->form : LBFGSB_B200_FORM_PLAIN;
  cudaStream_t s = (cudaStream_t)stream;
  if (form == LBFGSB_B200_FORM_MIXED)
    return solve_device<float, float, double>(n, x, nbd, l, u, option, objective, user, s, ext,
                                              summary);
  if (form == LBFGSB_B200_FORM_MIXED_BF16)
    return solve_device<float, __nv_bfloat16, double>(n, x, nbd, l, u, option, objective, user,
                                                      s, ext, summary);
  return solve_device<float, float, float>(n, x, nbd, l, u, option, objective, user, s, ext,
                                           summary);
}

int lbfgsb_b200_minimize_f64(int n, double* x, const int* nbd, const double* l,
                             const double* u, const lbfgsb_b200_option_f64* option,
                             lbfgsb_b200_callback_f64 funcgrad,
                             lbfgsb_b200_callback_f64 after_iteration,
                             lbfgsb_b200_callback_f64 customized_stopping, void* user,
                             void* stream, lbfgsb_b200_summary_f64* summary) {
  return lbfgsb_b200_minimize_ext_f64(n, x, nbd, l, u, option, funcgrad, after_iteration,
                                      customized_stopping, user, stream, nullptr, summary);
}

int lbfgsb_b200_minimize_f32(int n, float* x, const int* nbd, const float* l, const float* u,
                             const lbfgsb_b200_option_f32* option,
                             lbfgsb_b200_callback_f32 funcgrad,
                             lbfgsb_b200_callback_f32 after_iteration,
                             lbfgsb_b200_callback_f32 customized_stopping, void* user,
                             void* stream, lbfgsb_b200_summary_f32* summary) {
  return lbfgsb_b200_minimize_ext_f32(n, x, nbd, l, u, option, funcgrad, after_iteration,
                                      customized_stopping, user, stream, nullptr, summary);
}

int lbfgsb_b200_minimize_batch_f64(int count, const int* n, double* const* x,
                                   const int* const* nbd, const double* const* l,
                                   const double* const* u, const lbfgsb_b200_option_f64* option,
                                   lbfgsb_b200_callback_f64 funcgrad, void* const* user,
                                   int concurrency, lbfgsb_b200_summary_f64* summary,
                                   int* status, double* seconds) {
  return lbfgsb_b200::minimize_batch<double>(count, n, x, nbd, l, u, option, funcgrad, user,
                                             concurrency, summary, status, seconds);
}

int lbfgsb_b200_minimize_batch_f32(int count, const int* n, float* const* x,
                                   const int* const* nbd, const float* const* l,
                                   const float* const* u, const lbfgsb_b200_option_f32* option,
                                   lbfgsb_b200_callback_f32 funcgrad, void* const* user,
                                   int concurrency, lbfgsb_b200_summary_f32* summary,
                                   int* status, double* seconds) {
  return lbfgsb_b200::minimize_batch<float>(count, n, x, nbd, l, u, option, funcgrad, user,
                                            concurrency, summary, status, seconds);
}

unsigned long long lbfgsb_b200_workspace_bytes(int n, int real_size, int form) {
  if (n <= 0 || (real_size != 4 && real_size != 8)) return 0;
  const size_t hist = (real_size == 4 && form == LBFGSB_B200_FORM_MIXED_BF16) ? 2 : (size_t)real_size;
  return (unsigned long long)workspace_bound(n, (size_t)real_size, hist);
}

int lbfgsb_b200_server_create(int workers, unsigned long long hbm_budget_bytes, int form,
                              lbfgsb_b200_server** out) {
  g_last_error.clear();
  if (!out || workers < 0 || form < LBFGSB_B200_FORM_PLAIN || form > LBFGSB_B200_FORM_MIXED_BF16) {
    g_last_error = "server_create: bad argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_last_error = cudaGetErrorString(e);
    return LBFGSB_B200_ERR_CUDA;
  }
  auto* sv = new Server;
  sv->dev = dev;
  sv->form = form;
  sv->budget = (size_t)hbm_budget_bytes;
  const int nw = workers > 0 ? workers : 16;
  for (int w = 0; w < nw; w++) sv->workers.emplace_back(serve_worker, sv);
  *out = reinterpret_cast<lbfgsb_b200_server*>(sv);
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_server_submit_f32(lbfgsb_b200_server* server, int n, float* x, const int* nbd,
                                  const float* l, const float* u,
                                  const lbfgsb_b200_option_f32* option,
                                  lbfgsb_b200_callback_f32 funcgrad, void* user, long long* id) {
  g_last_error.clear();
  auto* sv = reinterpret_cast<Server*>(server);
  if (!sv || n <= 0 || !x || !nbd || !l || !u || !option || !funcgrad || !id) {
    g_last_error = "server_submit: null argument or n <= 0";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  const size_t bytes = workspace_bound(n, 4, sv->form == LBFGSB_B200_FORM_MIXED_BF16 ? 2 : 4);
  if (bytes > sv->budget) {
    g_last_error = "server_submit: the solve's workspace (" + std::to_string(bytes) +
                   " bytes) exceeds the server's HBM budget (" + std::to_string(sv->budget) + ")";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->stop) {
    g_last_error = "server_submit: the server is shutting down";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  sv->reqs.emplace_back();
  ServeRequest& r = sv->reqs.back();
  r.n = n;
  r.x = x;
  r.nbd = nbd;
  r.l = l;
  r.u = u;
  r.option = *option;
  r.funcgrad = funcgrad;
  r.user = user;
  r.bytes = bytes;
  r.arrive = std::chrono::steady_clock::now();
  *id = (long long)sv->reqs.size() - 1;
  sv->queue.push_back(*id);
  sv->cv_work.notify_all();
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_server_wait(lbfgsb_b200_server* server, long long id,
                            lbfgsb_b200_summary_f32* summary, int* status, double* latency_s,
                            double* queue_s) {
  g_last_error.clear();
  auto* sv = reinterpret_cast<Server*>(server);
  if (!sv || id < 0) {
    g_last_error = "server_wait: bad argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  std::unique_lock<std::mutex> lock(sv->mu);
  if ((size_t)id >= sv->reqs.size()) {
    g_last_error = "server_wait: unknown request id";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  sv->cv_done.wait(lock, [&] { return sv->reqs[(size_t)id].done; });
  const ServeRequest& r = sv->reqs[(size_t)id];
  if (summary) *summary = r.summary;
  if (status) *status = r.status;
  if (latency_s) *latency_s = std::chrono::duration<double>(r.finish - r.arrive).count();
  if (queue_s) *queue_s = std::chrono::duration<double>(r.start - r.arrive).count();
  if (r.status != LBFGSB_B200_OK) g_last_error = r.error;
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_server_peak(lbfgsb_b200_server* server, unsigned long long* peak_bytes,
                            int* peak_running) {
  auto* sv = reinterpret_cast<Server*>(server);
  if (!sv) return LBFGSB_B200_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(sv->mu);
  if (peak_bytes) *peak_bytes = (unsigned long long)sv->peak_bytes;
  if (peak_running) *peak_running = sv->peak_running;
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_server_destroy(lbfgsb_b200_server* server) {
  auto* sv = reinterpret_cast<Server*>(server);
  if (!sv) return LBFGSB_B200_ERR_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto& t : sv->workers) t.join();
  delete sv;
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_last_stats(lbfgsb_b200_stats* out) {
  if (!out) return LBFGSB_B200_ERR_ARGUMENT;
  *out = g_last_stats;
  return LBFGSB_B200_OK;
}

const char* lbfgsb_b200_last_error(void) { return g_last_error.c_str(); }

int lbfgsb_b200_trim_memory(void) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  for (int d = 0; d < kMaxDevices; d++) {
    if (!g_pools[d]) continue;
    cudaError_t e = cudaMemPoolTrimTo(g_pools[d], 0);
    if (e != cudaSuccess) {
      g_last_error = cudaGetErrorString(e);
      return LBFGSB_B200_ERR_CUDA;
    }
  }
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_copy(void* dst, const void* src, size_t bytes, int kind) {
  cudaMemcpyKind k = kind == 1   ? cudaMemcpyHostToDevice
                     : kind == 2 ? cudaMemcpyDeviceToHost
                                 : cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaMemcpy(dst, src, bytes, k);
  if (e != cudaSuccess) {
    g_last_error = cudaGetErrorString(e);
    return LBFGSB_B200_ERR_CUDA;
  }
  return LBFGSB_B200_OK;
}

}  // extern "C"
