// batch.cu -- many independent solves advanced together: one launch per pass for every live
// instance, device-driven rounds (rounds.cuh) captured into a CUDA graph, and the
// continuous-batching server built on it.  The reference solves one problem per call
// (culbfgsb/culbfgsb.h:157-163); everything here is an extension.
//
// Layout: each instance owns one segment of the workspace pool, cut into its vectors (x, z,
// trial point, two gradients, the subspace direction), its slot-major S/Y history, its
// iwhere codes and free-set bits, its state, its reduction rows and ticket, and its
// breakpoint-walk buffers.  A batched launch lists the live instances in a table of their
// pass contexts; instance k owns CTAs first[k] .. first[k+1]-1 of the launch and runs the
// same pass body as a single-instance launch on its own rows and ticket, so its results do
// not depend on the other instances in the launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

#include "batch_tune.h"
#include "host.cuh"

namespace lbfgsb_b200 {

template <typename R, typename H, typename S>
struct BatchLaunch {
  const Ctx<R, H, S>* table;
  const int* first;
  int count;
  int stages;
};

// The instance of this CTA (the largest k with first[k] <= blockIdx.x) and its place among
// that instance's CTAs.
__device__ __forceinline__ int batch_instance(const int* first, int count, CtaPos& cp) {
  __shared__ int s_k;
  if (threadIdx.x == 0) {
    int lo = 0, hi = count - 1;
    const int b = (int)blockIdx.x;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (first[mid] <= b)
        lo = mid;
      else
        hi = mid - 1;
    }
    s_k = lo;
  }
  __syncthreads();
  const int k = s_k;
  cp.rank = (int)blockIdx.x - first[k];
  cp.count = first[k + 1] - first[k];
  return k;
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) kb_gcp_scan(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  gcp_scan_pass<R, H, S, CONS>(b.table[k], cp, b.stages, nullptr, nullptr);
}
template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) kb_freev_formk(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  freev_formk_pass<R, H, S, CONS>(b.table[k], cp, b.stages, nullptr, nullptr);
}
template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) kb_subsm_dir(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  subsm_dir_pass<R, H, S, CONS>(b.table[k], cp, b.stages, nullptr, nullptr, nullptr);
}
template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) kb_subsm_apply(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  subsm_apply_pass<R, H, S, CONS>(b.table[k], cp, b.stages, nullptr, nullptr, nullptr);
}
// the post-evaluation pass with the next Cauchy scan for instances with bounds, the plain
// one for the others (as the single-instance driver chooses)
template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) kb_post_gcp(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  const Ctx<R, H, S>& c = b.table[k];
  if (!c.st->cnstnd) return;
  post_gcp_pass<R, H, S, CONS>(c, cp, b.stages, nullptr, nullptr, nullptr, nullptr, nullptr, S(0), 0);
}
template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) kb_post_eval(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  const Ctx<R, H, S>& c = b.table[k];
  if (c.st->cnstnd) return;
  post_eval_pass<R, H, S, CONS>(c, cp, b.stages, nullptr, nullptr, nullptr, nullptr, nullptr, S(0), 0);
}
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kThreads) kb_walk_gather(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  walk_gather_pass<R, H, S>(b.table[k], cp, nullptr, nullptr);
}
// one CTA per instance
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kWalkThreads) kb_walk(const Ctx<R, H, S>* table) {
  walk_pass<R, H, S>(table[blockIdx.x], nullptr, nullptr);
}
template <typename R, typename H, typename S>
__global__ void kb_trial_round(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  trial_round_pass<R, H, S>(b.table[k], cp);
}
// projgr at the start point, skipped by instances whose input was rejected
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kThreads) kb_projgr(BatchLaunch<R, H, S> b) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  const Ctx<R, H, S>& c = b.table[k];
  if (c.st->input_error) return;
  projgr_pass<R, H, S>(c, cp, nullptr, nullptr, S(0));
}
// errclb and lbfgsbactive: x_in[k] is instance k's start point
template <typename R, typename H, typename S>
__global__ void kb_init(BatchLaunch<R, H, S> b, const R* const* x_in) {
  CtaPos cp;
  const int k = batch_instance(b.first, b.count, cp);
  const Ctx<R, H, S>& c = b.table[k];
  init_pass<R, S>(c.n, x_in[k], c.X[0], c.nbd, c.l, c.u, c.st, cp);
}
// the first evaluation's slot: x0 into the gradient at the iterate; instances whose input
// was rejected are not evaluated
template <typename R, typename H, typename S>
__global__ void kb_first_slot(const Ctx<R, H, S>* table, int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const Ctx<R, H, S>& c = table[k];
  *c.ev_x = c.X[0];
  *c.ev_g = c.G[0];
  *c.ev_act = c.st->input_error ? 0 : 1;
}

enum { RK_BEGIN = 0, RK_PRE = 1, RK_POST = 2 };
template <typename R, typename H, typename S, int WHICH>
__global__ void kb_round(const Ctx<R, H, S>* table, int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  if (WHICH == RK_BEGIN) round_begin<R, H, S>(table[k]);
  if (WHICH == RK_PRE) pre_eval<R, H, S>(table[k]);
  if (WHICH == RK_POST) post_round<R, H, S>(table[k]);
}

// What the host needs of each instance after a batch of rounds.
struct BatchRow {
  int phase, info, iter, xr0, device_error, input_error, cnstnd, pad;
  double res_g, res_x, res_f, sbgnrm;
};
template <typename R, typename H, typename S>
__global__ void kb_collect(const Ctx<R, H, S>* table, int count, BatchRow* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const DevState<S>* st = table[k].st;
  BatchRow r;
  r.phase = st->phase;
  r.info = st->info_final;
  r.iter = st->iter;
  r.xr0 = st->xr[0];
  r.device_error = st->device_error;
  r.input_error = st->input_error;
  r.cnstnd = st->cnstnd;
  r.pad = 0;
  r.res_g = (double)st->res_g;
  r.res_x = (double)st->res_x;
  r.res_f = (double)st->res_f;
  r.sbgnrm = (double)st->sbgnrm;
  out[k] = r;
}

// ---- host side -------------------------------------------------------------------------

template <typename R>
struct BatchObjective;
template <>
struct BatchObjective<double> {
  using Fn = lbfgsb_b200_batch_objective_f64;
};
template <>
struct BatchObjective<float> {
  using Fn = lbfgsb_b200_batch_objective_f32;
};

// Tiles per CTA of the batched passes, by instance size: the table the autotuner writes
// (batch_tune.h), overridable at run time (lbfgsb_b200_batch_tiles_per_cta).
static int g_tiles_override[kTuneBuckets] = {};
static int tune_bucket(long long n) {
  int b = 0;
  for (long long lim = 1LL << 12; b < kTuneBuckets - 1 && n > lim; lim <<= 2) b++;
  return b;
}
static int tiles_per_cta(long long n) {
  const int b = tune_bucket(n);
  return g_tiles_override[b] > 0 ? g_tiles_override[b] : kTunedTilesPerCta[b];
}

// Pinned host buffer that grows (owned by one runner).
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void* get(size_t want) {
    if (want > bytes) {
      if (p) CK(cudaFreeHost(p));
      p = nullptr;
      bytes = 0;
      CK(cudaMallocHost(&p, want));
      bytes = want;
    }
    return p;
  }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

// Device buffer of the workspace pool that grows (owned by one runner).
struct PoolBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void* get(size_t want, cudaStream_t stream) {
    if (want > bytes) {
      if (p) CK(cudaFreeAsync(p, stream));
      p = nullptr;
      bytes = 0;
      CK(cudaMallocFromPoolAsync(&p, want, workspace_pool(), stream));
      bytes = want;
    }
    return p;
  }
  void release(cudaStream_t stream) {
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
    bytes = 0;
  }
};

// Runs a changing set of instances.  admit() sets new instances up and evaluates them at
// their start points; run() launches rounds of every live instance; poll() finishes the
// instances that are done (x copied back, summary written, segment released).  All work is
// enqueued on one stream; the calls are not thread-safe.
template <typename R, typename H, typename S>
class BatchRunner {
 public:
  using Opt = typename Api<R>::Opt;
  using Sum = typename Api<R>::Sum;
  using Fn = typename BatchObjective<R>::Fn;

  struct Inst {
    int id = 0;  // the id the objective sees
    int n = 0;
    R* x_user = nullptr;
    const int* nbd = nullptr;
    const R* l = nullptr;
    const R* u = nullptr;
    Sum* summary = nullptr;
    int* status = nullptr;
    void* tag = nullptr;  // the caller's (the server's request)
    // set up by admit()
    Ctx<R, H, S> c{};
    void* seg = nullptr;
    size_t seg_bytes = 0;
    int gp = 1, ge = 1;  // CTAs of a pass launch / of an elementwise launch
    int cnstnd = 1;
  };

  BatchRunner(cudaStream_t s, const Opt& opt, const lbfgsb_b200_ext* ext, Fn objective, void* user)
      : s_(s), opt_(opt), objective_(objective), user_(user) {
    subsm_proj_ = (ext && ext->subsm_projection) ? 1 : 0;
    m_ = std::min(opt.hessian_approximate_dimension, kMaxM);
    int dev = 0, optin = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    sms_ = device_sms();
    const int hsz = (int)sizeof(H);
    cap_gcp_ = stage_capacity(StageBytes<R>::gcp, 0, m_, hsz);
    cap_freev_ = stage_capacity(StageBytes<R>::freev, kTile / 8, m_, hsz);
    cap_dir_ = stage_capacity(StageBytes<R>::dir, 0, m_, hsz);
    cap_apply_ = stage_capacity(StageBytes<R>::apply, 0, 0, hsz);
    cap_post_ = stage_capacity(StageBytes<R>::post, 0, m_, hsz);
    set_smem(kb_gcp_scan<R, H, S, kConsWide>, optin);
    set_smem(kb_freev_formk<R, H, S, kConsWide>, optin);
    set_smem(kb_subsm_dir<R, H, S, kConsWide>, optin);
    set_smem(kb_subsm_apply<R, H, S, kConsWide>, optin);
    set_smem(kb_post_gcp<R, H, S, kConsWide>, optin);
    set_smem(kb_post_eval<R, H, S, kConsWide>, optin);
  }
  ~BatchRunner() {
    drop_graph();
    for (auto& in : live_)
      if (in.seg) cudaFreeAsync(in.seg, s_);
    tables_.release(s_);
    cudaStreamSynchronize(s_);
  }

  size_t live() const { return live_.size(); }
  long long rounds() const { return rounds_; }
  long long launches() const { return launches_; }
  long long syncs() const { return syncs_; }
  size_t live_bytes() const { return live_bytes_; }

  // The pool bytes one instance of n elements takes (its segment), host arithmetic only.
  static size_t segment_bytes(long long n, int m, int sms) {
    Layout L = layout(n, m, sms, true);
    return L.total;
  }

  // Validate, set up and evaluate new instances at their start points.  Instances that end
  // before their first iteration (rejected input, ||proj g|| <= eps_g at x0) are finished
  // here and appended to `finished`; the others join the live set.
  void admit(std::vector<Inst>& fresh, std::vector<Inst>* finished) {
    std::vector<Inst> ok;
    for (auto& in : fresh) {
      if (!in.x_user || !in.nbd || !in.l || !in.u || in.n <= 0) {
        in.summary->info = -1;
        *in.status = LBFGSB_B200_ERR_ARGUMENT;
        finished->push_back(in);
        continue;
      }
      // errclb's scalar checks (lbfgsbcpu.cpp:258-264, 879-890)
      if (m_ <= 0 || m_ > in.n || opt_.eps_f < 0 || opt_.max_iteration < 0 || opt_.eps_g < 0 ||
          opt_.eps_x < 0) {
        in.summary->info = -1;
        *in.status = LBFGSB_B200_OK;
        finished->push_back(in);
        continue;
      }
      ok.push_back(in);
    }
    if (ok.empty()) return;
    CK(cudaStreamSynchronize(s_));  // the pinned state buffer may still be read
    DevState<S>* hs = static_cast<DevState<S>*>(state_buf_.get(ok.size() * sizeof(DevState<S>)));
    for (size_t j = 0; j < ok.size(); j++) setup(ok[j], hs + j);
    // errclb / lbfgsbactive, the first evaluation and projgr over the new instances
    upload_tables(ok);
    const int cnt = (int)ok.size();
    const BatchLaunch<R, H, S> be{table_, first_elem_, cnt, 2};
    kb_init<R, H, S><<<ctas_elem_, 256, 0, s_>>>(be, xin_);
    kb_first_slot<R, H, S><<<(cnt + 127) / 128, 128, 0, s_>>>(table_, cnt);
    objective_(user_, cnt, ids_, first_elem_, ctas_elem_, (const R* const*)ev_x_, ev_g_, ev_f_,
               ev_act_, (void*)s_);
    kb_projgr<R, H, S><<<ctas_elem_, kThreads, 0, s_>>>(be);
    CK(cudaGetLastError());
    launches_ += 4;
    std::vector<BatchRow> rows = collect(cnt);
    for (int j = 0; j < cnt; j++) {
      Inst& in = ok[j];
      const BatchRow& r = rows[j];
      in.cnstnd = r.cnstnd;
      if (r.input_error) {
        in.summary->info = -1;  // x is left as given (lbfgsbcpu.cpp:259-264)
        *in.status = LBFGSB_B200_OK;
        release(in);
        finished->push_back(in);
        continue;
      }
      in.summary->residual_g = (R)r.sbgnrm;
      if ((S)r.sbgnrm <= (S)opt_.eps_g) {
        in.summary->info = 4;
        *in.status = LBFGSB_B200_OK;
        CK(cudaMemcpyAsync(in.x_user, in.c.X[0], (size_t)in.n * sizeof(R), cudaMemcpyDeviceToDevice, s_));
        release(in);
        finished->push_back(in);
        continue;
      }
      live_.push_back(in);
    }
    dirty_ = true;
  }

  // `count` rounds of every live instance.
  void run(int count) {
    if (live_.empty()) return;
    if (dirty_) rebuild();
    for (int r = 0; r < count; r++) CK(cudaGraphLaunch(exec_, s_));
    rounds_ += count;
    launches_ += (long long)count * kernels_per_round_;
  }

  // Finish the instances that are done; returns how many are still live.
  size_t poll(std::vector<Inst>* finished) {
    if (live_.empty()) return 0;
    if (dirty_) rebuild();
    std::vector<BatchRow> rows = collect((int)live_.size());
    std::vector<Inst> keep;
    for (size_t j = 0; j < live_.size(); j++) {
      Inst& in = live_[j];
      const BatchRow& r = rows[j];
      if (r.device_error) throw CudaFailure{cudaErrorLaunchTimeout, "staged-tile wait", __LINE__};
      if (r.phase != PH_DONE) {
        keep.push_back(in);
        continue;
      }
      in.summary->info = r.info;
      in.summary->num_iteration = r.iter;
      in.summary->residual_g = (R)r.res_g;
      in.summary->residual_x = (R)r.res_x;
      in.summary->residual_f = (R)r.res_f;
      *in.status = LBFGSB_B200_OK;
      CK(cudaMemcpyAsync(in.x_user, in.c.X[r.xr0], (size_t)in.n * sizeof(R), cudaMemcpyDeviceToDevice, s_));
      release(in);
      finished->push_back(in);
    }
    if (keep.size() != live_.size()) {
      live_.swap(keep);
      dirty_ = true;
    }
    return live_.size();
  }

 private:
  template <typename K>
  void set_smem(K kernel, int optin) {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            optin - (int)fa.sharedSizeBytes));
  }

  static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

  // Offsets of one instance's buffers in its segment.
  struct Layout {
    size_t X[3], G[2], dsub, gdummy, ws, wy, code, fbits, st, ticket, part, wlt, wli, wln, l, u, nbd;
    size_t total, ld;
    int gp, ge;
  };
  static Layout layout(long long n, int m, int sms, bool copy_bounds) {
    (void)m;
    Layout L{};
    const size_t N = (size_t)n;
    L.ld = align_up(N, kTile);
    const long long tiles = (long long)L.ld / kTile;
    const int tpc = tiles_per_cta(n);
    L.gp = (int)std::max<long long>(1, std::min<long long>(sms, (tiles + tpc - 1) / tpc));
    L.ge = (int)std::max<long long>(1, std::min<long long>(64, (n + 4095) / 4096));
    const int rows = std::max(L.gp, L.ge);
    size_t off = 0;
    auto take = [&](size_t bytes) {
      off = align_up(off, 256);
      const size_t o = off;
      off += std::max<size_t>(bytes, 1);
      return o;
    };
    for (int k = 0; k < 3; k++) L.X[k] = take(L.ld * sizeof(R));
    for (int k = 0; k < 2; k++) L.G[k] = take(L.ld * sizeof(R));
    L.dsub = take(L.ld * sizeof(R));
    L.gdummy = take(L.ld * sizeof(R));
    L.ws = take(L.ld * kSlots * sizeof(H));
    L.wy = take(L.ld * kSlots * sizeof(H));
    L.code = take(L.ld);
    L.fbits = take((L.ld / 32 + 4) * 4);
    L.st = take(sizeof(DevState<S>));
    L.ticket = take(16);
    L.part = take((size_t)rows * 256 * 8);
    L.wlt = take(N * 8);
    L.wli = take(N * 4);
    L.wln = take(16);
    L.l = L.u = L.nbd = 0;
    if (copy_bounds) {
      L.l = take(N * sizeof(R));
      L.u = take(N * sizeof(R));
      L.nbd = take(N * 4);
    }
    L.total = align_up(off, 256);
    return L;
  }

  // One segment of the pool per instance, cut into its buffers; its initial state in hs.
  void setup(Inst& in, DevState<S>* hs) {
    const size_t N = (size_t)in.n;
    auto misaligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) != 0; };
    const bool copy_bounds = misaligned(in.l) || misaligned(in.u) || misaligned(in.nbd);
    const Layout L = layout(in.n, m_, sms_, copy_bounds);
    in.gp = L.gp;
    in.ge = L.ge;
    in.seg_bytes = L.total;
    CK(cudaMallocFromPoolAsync(&in.seg, L.total, workspace_pool(), s_));
    live_bytes_ += L.total;
    unsigned char* b = static_cast<unsigned char*>(in.seg);
    Ctx<R, H, S>& c = in.c;
    c = Ctx<R, H, S>{};
    c.n = in.n;
    c.l = in.l;
    c.u = in.u;
    c.nbd = in.nbd;
    if (copy_bounds) {
      CK(cudaMemcpyAsync(b + L.l, in.l, N * sizeof(R), cudaMemcpyDeviceToDevice, s_));
      CK(cudaMemcpyAsync(b + L.u, in.u, N * sizeof(R), cudaMemcpyDeviceToDevice, s_));
      CK(cudaMemcpyAsync(b + L.nbd, in.nbd, N * 4, cudaMemcpyDeviceToDevice, s_));
      c.l = reinterpret_cast<const R*>(b + L.l);
      c.u = reinterpret_cast<const R*>(b + L.u);
      c.nbd = reinterpret_cast<const int*>(b + L.nbd);
    }
    c.ws = reinterpret_cast<H*>(b + L.ws);
    c.wy = reinterpret_cast<H*>(b + L.wy);
    c.ld = (long long)L.ld;
    c.stages = 2;
    c.code = reinterpret_cast<int8_t*>(b + L.code);
    c.fbits = reinterpret_cast<uint32_t*>(b + L.fbits);
    c.dsub = reinterpret_cast<R*>(b + L.dsub);
    c.st = reinterpret_cast<DevState<S>*>(b + L.st);
    c.part = reinterpret_cast<double*>(b + L.part);
    c.ticket = reinterpret_cast<unsigned int*>(b + L.ticket);
    c.wl_t = reinterpret_cast<double*>(b + L.wlt);
    c.wl_i = reinterpret_cast<int*>(b + L.wli);
    c.wl_n = reinterpret_cast<unsigned int*>(b + L.wln);
    c.rounds = 1;
    for (int k = 0; k < 3; k++) c.X[k] = reinterpret_cast<R*>(b + L.X[k]);
    for (int k = 0; k < 2; k++) c.G[k] = reinterpret_cast<R*>(b + L.G[k]);
    c.gdummy = reinterpret_cast<R*>(b + L.gdummy);
    CK(cudaMemsetAsync(b + L.ws, 0, L.ld * kSlots * sizeof(H), s_));
    CK(cudaMemsetAsync(b + L.wy, 0, L.ld * kSlots * sizeof(H), s_));
    CK(cudaMemsetAsync(b + L.fbits, 0, (L.ld / 32 + 4) * 4, s_));
    CK(cudaMemsetAsync(b + L.ticket, 0, 16, s_));
    // the state: the start of the reference driver (as prepare() writes it) and the round
    // bookkeeping of a device-driven solve
    std::memset(hs, 0, sizeof(*hs));
    hs->n = in.n;
    hs->m = m_;
    hs->subsm_proj = subsm_proj_;
    hs->boxed = 1;
    hs->head = 1;
    hs->theta = 1;
    hs->iword = -1;
    hs->big = (S)1.0e10;
    for (int r = 1; r <= m_; r++) hs->phys[r] = r - 1;
    hs->spare = m_;
    hs->xr[0] = 0;
    hs->xr[1] = 1;
    hs->xr[2] = 2;
    hs->gr[0] = 0;
    hs->gr[1] = 1;
    hs->phase = PH_ITER;
    hs->eps_g = (S)opt_.eps_g;
    hs->eps_x = (S)opt_.eps_x;
    hs->eps_f = (S)opt_.eps_f;
    hs->max_iteration = opt_.max_iteration;
    hs->res_x = (S)in.summary->residual_x;
    hs->res_f = (S)in.summary->residual_f;
    CK(cudaMemcpyAsync(c.st, hs, sizeof(*hs), cudaMemcpyHostToDevice, s_));
  }

  void release(Inst& in) {
    if (in.seg) CK(cudaFreeAsync(in.seg, s_));
    in.seg = nullptr;
    live_bytes_ -= in.seg_bytes;
    in.seg_bytes = 0;
  }

  // The launch tables of a set of instances: contexts (with their evaluation slots), the
  // CTA prefixes of pass and elementwise launches, the ids and start points.
  void upload_tables(std::vector<Inst>& set) {
    const int cnt = (int)set.size();
    const size_t a = 256;
    const size_t o_tab = 0;
    const size_t o_fp = align_up(o_tab + cnt * sizeof(Ctx<R, H, S>), a);
    const size_t o_fe = align_up(o_fp + (cnt + 1) * sizeof(int), a);
    const size_t o_ids = align_up(o_fe + (cnt + 1) * sizeof(int), a);
    const size_t o_xin = align_up(o_ids + cnt * sizeof(int), a);
    const size_t o_evx = align_up(o_xin + cnt * sizeof(void*), a);
    const size_t o_evg = align_up(o_evx + cnt * sizeof(void*), a);
    const size_t o_evf = align_up(o_evg + cnt * sizeof(void*), a);
    const size_t o_eva = align_up(o_evf + cnt * sizeof(double), a);
    const size_t o_rows = align_up(o_eva + cnt * sizeof(int), a);
    const size_t total = align_up(o_rows + cnt * sizeof(BatchRow), a);
    CK(cudaStreamSynchronize(s_));  // the previous tables may still be read
    unsigned char* h = static_cast<unsigned char*>(host_tables_.get(total));
    unsigned char* d = static_cast<unsigned char*>(tables_.get(total, s_));
    table_ = reinterpret_cast<Ctx<R, H, S>*>(d + o_tab);
    first_pass_ = reinterpret_cast<int*>(d + o_fp);
    first_elem_ = reinterpret_cast<int*>(d + o_fe);
    ids_ = reinterpret_cast<int*>(d + o_ids);
    xin_ = reinterpret_cast<const R**>(d + o_xin);
    ev_x_ = reinterpret_cast<R**>(d + o_evx);
    ev_g_ = reinterpret_cast<R**>(d + o_evg);
    ev_f_ = reinterpret_cast<double*>(d + o_evf);
    ev_act_ = reinterpret_cast<int*>(d + o_eva);
    rows_ = reinterpret_cast<BatchRow*>(d + o_rows);
    Ctx<R, H, S>* ht = reinterpret_cast<Ctx<R, H, S>*>(h + o_tab);
    int* hfp = reinterpret_cast<int*>(h + o_fp);
    int* hfe = reinterpret_cast<int*>(h + o_fe);
    int* hid = reinterpret_cast<int*>(h + o_ids);
    const R** hxin = reinterpret_cast<const R**>(h + o_xin);
    int fp = 0, fe = 0;
    any_uncon_ = false;
    for (int j = 0; j < cnt; j++) {
      Inst& in = set[j];
      in.c.ev_x = ev_x_ + j;
      in.c.ev_g = ev_g_ + j;
      in.c.ev_f = ev_f_ + j;
      in.c.ev_act = ev_act_ + j;
      ht[j] = in.c;
      hfp[j] = fp;
      hfe[j] = fe;
      fp += in.gp;
      fe += in.ge;
      hid[j] = in.id;
      hxin[j] = in.x_user;
      if (!in.cnstnd) any_uncon_ = true;
    }
    hfp[cnt] = fp;
    hfe[cnt] = fe;
    ctas_pass_ = fp;
    ctas_elem_ = fe;
    count_ = cnt;
    CK(cudaMemcpyAsync(d, h, o_rows, cudaMemcpyHostToDevice, s_));
  }

  std::vector<BatchRow> collect(int cnt) {
    kb_collect<R, H, S><<<(cnt + 127) / 128, 128, 0, s_>>>(table_, cnt, rows_);
    CK(cudaGetLastError());
    BatchRow* h = static_cast<BatchRow*>(row_buf_.get(cnt * sizeof(BatchRow)));
    CK(cudaMemcpyAsync(h, rows_, cnt * sizeof(BatchRow), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    syncs_++;
    return std::vector<BatchRow>(h, h + cnt);
  }

  void drop_graph() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
  }

  // Tables and the captured round for the live set.
  void rebuild() {
    drop_graph();
    upload_tables(live_);
    const int cnt = count_;
    const int rb = (cnt + 127) / 128;
    const BatchLaunch<R, H, S> bp{table_, first_pass_, cnt, 2};
    const BatchLaunch<R, H, S> be{table_, first_elem_, cnt, 2};
    const int thr = kConsWide + 32;
    CK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
    kb_round<R, H, S, RK_BEGIN><<<rb, 128, 0, s_>>>(table_, cnt);
    kb_gcp_scan<R, H, S, kConsWide><<<ctas_pass_, thr, ring_bytes(2, cap_gcp_), s_>>>(bp);
    kb_walk_gather<R, H, S><<<ctas_elem_, kThreads, 0, s_>>>(be);
    kb_walk<R, H, S><<<cnt, kWalkThreads, 0, s_>>>(table_);
    kb_freev_formk<R, H, S, kConsWide><<<ctas_pass_, thr, ring_bytes(2, cap_freev_) + freev_extra_smem<S>(), s_>>>(bp);
    kb_subsm_dir<R, H, S, kConsWide><<<ctas_pass_, thr, ring_bytes(2, cap_dir_), s_>>>(bp);
    kb_subsm_apply<R, H, S, kConsWide><<<ctas_pass_, thr, ring_bytes(2, cap_apply_), s_>>>(bp);
    kb_round<R, H, S, RK_PRE><<<rb, 128, 0, s_>>>(table_, cnt);
    kb_trial_round<R, H, S><<<ctas_elem_, 256, 0, s_>>>(be);
    objective_(user_, cnt, ids_, first_elem_, ctas_elem_, (const R* const*)ev_x_, ev_g_, ev_f_,
               ev_act_, (void*)s_);
    kb_post_gcp<R, H, S, kConsWide><<<ctas_pass_, thr, ring_bytes(2, cap_post_), s_>>>(bp);
    if (any_uncon_)
      kb_post_eval<R, H, S, kConsWide><<<ctas_pass_, thr, ring_bytes(2, cap_post_), s_>>>(bp);
    kb_round<R, H, S, RK_POST><<<rb, 128, 0, s_>>>(table_, cnt);
    const cudaError_t launch_err = cudaGetLastError();
    const cudaError_t cap_err = cudaStreamEndCapture(s_, &graph_);
    CK(launch_err);
    CK(cap_err);
    CK(cudaGraphInstantiate(&exec_, graph_, 0));
    kernels_per_round_ = any_uncon_ ? 13 : 12;
    dirty_ = false;
  }

  cudaStream_t s_;
  Opt opt_;
  Fn objective_;
  void* user_;
  int m_ = 8, sms_ = 148, subsm_proj_ = 0;
  int cap_gcp_ = 0, cap_freev_ = 0, cap_dir_ = 0, cap_apply_ = 0, cap_post_ = 0;
  std::vector<Inst> live_;
  bool dirty_ = true, any_uncon_ = false;
  PoolBuf tables_;
  PinnedBuf host_tables_, row_buf_, state_buf_;
  Ctx<R, H, S>* table_ = nullptr;
  int *first_pass_ = nullptr, *first_elem_ = nullptr, *ids_ = nullptr;
  const R** xin_ = nullptr;
  R** ev_x_ = nullptr;
  R** ev_g_ = nullptr;
  double* ev_f_ = nullptr;
  int* ev_act_ = nullptr;
  BatchRow* rows_ = nullptr;
  int count_ = 0, ctas_pass_ = 0, ctas_elem_ = 0, kernels_per_round_ = 12;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  long long rounds_ = 0, launches_ = 0, syncs_ = 0;
  size_t live_bytes_ = 0;
};

// Batched device-driven solves of `count` instances, all given at once.
template <typename R, typename H, typename S>
static int solve_batch_device(int count, const int* ids, const int* n, R* const* x,
                              const int* const* nbd, const R* const* l, const R* const* u,
                              const typename Api<R>::Opt* opt,
                              typename BatchObjective<R>::Fn objective, void* user,
                              cudaStream_t ustream, const lbfgsb_b200_ext* ext,
                              typename Api<R>::Sum* summary, int* status) {
  g_last_error.clear();
  std::memset(&g_last_stats, 0, sizeof(g_last_stats));
  if (count < 0 || (count > 0 && (!n || !x || !nbd || !l || !u || !opt || !objective || !summary ||
                                  !status))) {
    g_last_error = "minimize_batch_device: null argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  if (count == 0) return LBFGSB_B200_OK;
  if (opt->mode != LBFGSB_B200_MODE_CUDA) {
    for (int k = 0; k < count; k++) {
      summary[k].info = -1;
      status[k] = LBFGSB_B200_ERR_ARGUMENT;
    }
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  using Runner = BatchRunner<R, H, S>;
  try {
    RoundStream& rs = round_stream();
    const cudaStream_t stream = rs.s;
    CK(cudaEventRecord(rs.in, ustream));
    CK(cudaStreamWaitEvent(stream, rs.in, 0));
    long long rounds = 0, launches = 0, syncs = 0;
    {
      Runner run(stream, *opt, ext, objective, user);
      std::vector<typename Runner::Inst> fresh(count), done;
      for (int k = 0; k < count; k++) {
        auto& in = fresh[k];
        in.id = ids ? ids[k] : k;
        in.n = n[k];
        in.x_user = x[k];
        in.nbd = nbd[k];
        in.l = l[k];
        in.u = u[k];
        in.summary = &summary[k];
        in.status = &status[k];
        status[k] = -1;
      }
      run.admit(fresh, &done);
      // rounds between two polls: a few at first, then about an eighth of the rounds so far
      int batch = 4;
      while (run.live() > 0) {
        run.run(batch);
        run.poll(&done);
        batch = (int)std::min<long long>(32, std::max<long long>(4, run.rounds() / 8));
      }
      rounds = run.rounds();
      launches = run.launches();
      syncs = run.syncs();
    }
    CK(cudaEventRecord(rs.out, stream));
    CK(cudaStreamWaitEvent(ustream, rs.out, 0));
    CK(cudaStreamSynchronize(stream));
    g_last_stats.rounds = rounds;
    g_last_stats.total_launches = launches;
    g_last_stats.host_syncs = syncs;
  } catch (const CudaFailure& e) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s failed at batch.cu:%d: %s", e.call, e.line,
                  cudaGetErrorString(e.err));
    g_last_error = buf;
    return LBFGSB_B200_ERR_CUDA;
  }
  int first_bad = LBFGSB_B200_OK;
  for (int k = 0; k < count; k++)
    if (status[k] != LBFGSB_B200_OK && first_bad == LBFGSB_B200_OK) first_bad = status[k];
  return first_bad;
}

// ---- continuous batching ----------------------------------------------------------------
// A server thread owns a BatchRunner on its own stream.  Requests queue in arrival order and
// are admitted, first come first served, as soon as their segment fits in the HBM budget
// beside the live solves; every loop admits what fits, runs a few rounds of every live
// solve (old and new together, one launch per pass) and retires the finished ones, whose
// memory then admits the next requests.
struct BatchServeRequest {
  int id = 0, n = 0;
  float* x = nullptr;
  const int* nbd = nullptr;
  const float* l = nullptr;
  const float* u = nullptr;
  size_t bytes = 0;
  std::chrono::steady_clock::time_point arrive, start, finish;
  lbfgsb_b200_summary_f32 summary{};
  int status = -1;
  bool done = false;
};

struct BatchServer {
  int dev = 0, form = LBFGSB_B200_FORM_MIXED, rounds_per_loop = 4;
  lbfgsb_b200_option_f32 opt{};
  lbfgsb_b200_batch_objective_f32 objective = nullptr;
  void* user = nullptr;
  size_t budget = 0, in_use = 0, peak_bytes = 0;
  int live = 0, peak_live = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<BatchServeRequest> reqs;  // by ticket
  std::deque<long long> queue;         // tickets waiting for admission, in arrival order
  bool stop = false;
  std::string error;
  long long rounds = 0, launches = 0;
  std::thread thread;
};

template <typename H, typename S>
static void batch_serve_loop(BatchServer* sv) {
  using Runner = BatchRunner<float, H, S>;
  cudaStream_t s = nullptr;
  try {
    CK(cudaSetDevice(sv->dev));
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    lbfgsb_b200_ext ext{};
    ext.form = sv->form;
    Runner run(s, sv->opt, &ext, sv->objective, sv->user);
    std::vector<typename Runner::Inst> fresh, finished;
    auto complete = [&](std::vector<typename Runner::Inst>& fin) {
      if (fin.empty()) return;
      CK(cudaStreamSynchronize(s));  // x is copied back
      const auto now = std::chrono::steady_clock::now();
      std::lock_guard<std::mutex> lock(sv->mu);
      for (auto& in : fin) {
        BatchServeRequest& r = *static_cast<BatchServeRequest*>(in.tag);
        r.finish = now;
        r.done = true;
        sv->in_use -= r.bytes;
        sv->live--;
      }
      fin.clear();
      sv->cv_done.notify_all();
    };
    for (;;) {
      fresh.clear();
      {
        std::unique_lock<std::mutex> lock(sv->mu);
        if (run.live() == 0)
          sv->cv_work.wait(lock, [&] { return sv->stop || !sv->queue.empty(); });
        if (sv->stop && sv->queue.empty() && run.live() == 0) break;
        const auto now = std::chrono::steady_clock::now();
        while (!sv->queue.empty()) {
          BatchServeRequest& r = sv->reqs[(size_t)sv->queue.front()];
          if (sv->in_use + r.bytes > sv->budget) break;  // first come, first served
          sv->queue.pop_front();
          sv->in_use += r.bytes;
          sv->peak_bytes = std::max(sv->peak_bytes, sv->in_use);
          sv->peak_live = std::max(sv->peak_live, ++sv->live);
          r.start = now;
          typename Runner::Inst in;
          in.id = r.id;
          in.n = r.n;
          in.x_user = r.x;
          in.nbd = r.nbd;
          in.l = r.l;
          in.u = r.u;
          in.summary = &r.summary;
          in.status = &r.status;
          in.tag = &r;
          fresh.push_back(in);
        }
      }
      if (!fresh.empty()) {
        run.admit(fresh, &finished);
        complete(finished);
      }
      if (run.live() > 0) {
        run.run(sv->rounds_per_loop);
        run.poll(&finished);
        complete(finished);
      }
    }
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->rounds = run.rounds();
    sv->launches = run.launches();
  } catch (const CudaFailure& e) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s failed at batch.cu:%d: %s", e.call, e.line,
                  cudaGetErrorString(e.err));
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->error = buf;
    // every request not finished fails
    for (auto& r : sv->reqs)
      if (!r.done) {
        r.status = LBFGSB_B200_ERR_CUDA;
        r.done = true;
        r.finish = std::chrono::steady_clock::now();
      }
    sv->queue.clear();
    sv->cv_done.notify_all();
  }
  if (s) cudaStreamDestroy(s);
}

}  // namespace lbfgsb_b200

using namespace lbfgsb_b200;

extern "C" {

unsigned long long lbfgsb_b200_batch_request_bytes(int n, int form, int m);

int lbfgsb_b200_minimize_batch_device_f64(int count, const int* ids, const int* n,
                                          double* const* x, const int* const* nbd,
                                          const double* const* l, const double* const* u,
                                          const lbfgsb_b200_option_f64* option,
                                          lbfgsb_b200_batch_objective_f64 objective, void* user,
                                          void* stream, const lbfgsb_b200_ext* ext,
                                          lbfgsb_b200_summary_f64* summary, int* status) {
  return solve_batch_device<double, double, double>(count, ids, n, x, nbd, l, u, option,
                                                    objective, user, (cudaStream_t)stream, ext,
                                                    summary, status);
}

int lbfgsb_b200_minimize_batch_device_f32(int count, const int* ids, const int* n,
                                          float* const* x, const int* const* nbd,
                                          const float* const* l, const float* const* u,
                                          const lbfgsb_b200_option_f32* option,
                                          lbfgsb_b200_batch_objective_f32 objective, void* user,
                                          void* stream, const lbfgsb_b200_ext* ext,
                                          lbfgsb_b200_summary_f32* summary, int* status) {
  const int form = ext ? ext->form : LBFGSB_B200_FORM_PLAIN;
  cudaStream_t s = (cudaStream_t)stream;
  if (form == LBFGSB_B200_FORM_MIXED)
    return solve_batch_device<float, float, double>(count, ids, n, x, nbd, l, u, option,
                                                    objective, user, s, ext, summary, status);
  if (form == LBFGSB_B200_FORM_MIXED_BF16)
    return solve_batch_device<float, __nv_bfloat16, double>(count, ids, n, x, nbd, l, u, option,
                                                            objective, user, s, ext, summary,
                                                            status);
  return solve_batch_device<float, float, float>(count, ids, n, x, nbd, l, u, option, objective,
                                                 user, s, ext, summary, status);
}

int lbfgsb_b200_batch_server_create_f32(unsigned long long hbm_budget_bytes, int form,
                                        const lbfgsb_b200_option_f32* option,
                                        lbfgsb_b200_batch_objective_f32 objective, void* user,
                                        int rounds_per_loop, lbfgsb_b200_batch_server** out) {
  g_last_error.clear();
  if (!out || !option || !objective || form < LBFGSB_B200_FORM_PLAIN ||
      form > LBFGSB_B200_FORM_MIXED_BF16 || option->mode != LBFGSB_B200_MODE_CUDA) {
    g_last_error = "batch_server_create: bad argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_last_error = cudaGetErrorString(e);
    return LBFGSB_B200_ERR_CUDA;
  }
  auto* sv = new BatchServer;
  sv->dev = dev;
  sv->form = form;
  sv->opt = *option;
  sv->objective = objective;
  sv->user = user;
  sv->budget = (size_t)hbm_budget_bytes;
  sv->rounds_per_loop = rounds_per_loop > 0 ? rounds_per_loop : 4;
  if (form == LBFGSB_B200_FORM_MIXED)
    sv->thread = std::thread(batch_serve_loop<float, double>, sv);
  else if (form == LBFGSB_B200_FORM_MIXED_BF16)
    sv->thread = std::thread(batch_serve_loop<__nv_bfloat16, double>, sv);
  else
    sv->thread = std::thread(batch_serve_loop<float, float>, sv);
  *out = reinterpret_cast<lbfgsb_b200_batch_server*>(sv);
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_batch_server_submit_f32(lbfgsb_b200_batch_server* server, int id, int n, float* x,
                                        const int* nbd, const float* l, const float* u,
                                        long long* ticket) {
  g_last_error.clear();
  auto* sv = reinterpret_cast<BatchServer*>(server);
  if (!sv || n <= 0 || !x || !nbd || !l || !u || !ticket) {
    g_last_error = "batch_server_submit: null argument or n <= 0";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  const size_t bytes =
      (size_t)lbfgsb_b200_batch_request_bytes(n, sv->form, sv->opt.hessian_approximate_dimension);
  if (bytes > sv->budget) {
    g_last_error = "batch_server_submit: the solve's workspace (" + std::to_string(bytes) +
                   " bytes) exceeds the server's HBM budget (" + std::to_string(sv->budget) + ")";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->stop || !sv->error.empty()) {
    g_last_error = sv->error.empty() ? "batch_server_submit: the server is shutting down" : sv->error;
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  sv->reqs.emplace_back();
  BatchServeRequest& r = sv->reqs.back();
  r.id = id;
  r.n = n;
  r.x = x;
  r.nbd = nbd;
  r.l = l;
  r.u = u;
  r.bytes = bytes;
  r.arrive = std::chrono::steady_clock::now();
  *ticket = (long long)sv->reqs.size() - 1;
  sv->queue.push_back(*ticket);
  sv->cv_work.notify_all();
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_batch_server_wait(lbfgsb_b200_batch_server* server, long long ticket,
                                  lbfgsb_b200_summary_f32* summary, int* status,
                                  double* latency_s, double* queue_s) {
  g_last_error.clear();
  auto* sv = reinterpret_cast<BatchServer*>(server);
  if (!sv || ticket < 0) {
    g_last_error = "batch_server_wait: bad argument";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  std::unique_lock<std::mutex> lock(sv->mu);
  if ((size_t)ticket >= sv->reqs.size()) {
    g_last_error = "batch_server_wait: unknown ticket";
    return LBFGSB_B200_ERR_ARGUMENT;
  }
  sv->cv_done.wait(lock, [&] { return sv->reqs[(size_t)ticket].done; });
  const BatchServeRequest& r = sv->reqs[(size_t)ticket];
  if (summary) *summary = r.summary;
  if (status) *status = r.status;
  if (latency_s) *latency_s = std::chrono::duration<double>(r.finish - r.arrive).count();
  if (queue_s) *queue_s = std::chrono::duration<double>(r.start - r.arrive).count();
  if (r.status != LBFGSB_B200_OK) g_last_error = sv->error;
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_batch_server_peak(lbfgsb_b200_batch_server* server, unsigned long long* peak_bytes,
                                  int* peak_live) {
  auto* sv = reinterpret_cast<BatchServer*>(server);
  if (!sv) return LBFGSB_B200_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(sv->mu);
  if (peak_bytes) *peak_bytes = (unsigned long long)sv->peak_bytes;
  if (peak_live) *peak_live = sv->peak_live;
  return LBFGSB_B200_OK;
}

int lbfgsb_b200_batch_server_destroy(lbfgsb_b200_batch_server* server) {
  auto* sv = reinterpret_cast<BatchServer*>(server);
  if (!sv) return LBFGSB_B200_ERR_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  if (sv->thread.joinable()) sv->thread.join();
  delete sv;
  return LBFGSB_B200_OK;
}

unsigned long long lbfgsb_b200_batch_request_bytes(int n, int form, int m) {
  if (n <= 0 || m <= 0) return 0;
  m = std::min(m, kMaxM);
  return form == LBFGSB_B200_FORM_MIXED_BF16
             ? BatchRunner<float, __nv_bfloat16, double>::segment_bytes(n, m, 148)
             : BatchRunner<float, float, double>::segment_bytes(n, m, 148);
}

int lbfgsb_b200_batch_tiles_per_cta(int bucket, int tiles) {
  if (bucket < 0 || bucket >= kTuneBuckets || tiles < 0) return LBFGSB_B200_ERR_ARGUMENT;
  g_tiles_override[bucket] = tiles;
  return LBFGSB_B200_OK;
}

}  // extern "C"
