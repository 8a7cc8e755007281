// host.cuh -- host-side pieces shared by the library's translation units (driver.cu, the
// single-instance solves; batch.cu, the batched solves and the server): error handling,
// the workspace pool, launch bookkeeping, pass launch shapes and one solve's workspace.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lbfgsb_b200.h"
#include "passes.cuh"
#include "rounds.cuh"
#include "walk.cuh"

namespace lbfgsb_b200 {

// the message of the calling thread's last LBFGSB_B200_ERR_CUDA and its last solve's
// statistics (defined in driver.cu)
extern thread_local std::string g_last_error;
extern thread_local lbfgsb_b200_stats g_last_stats;

struct CudaFailure {
  cudaError_t err;
  const char* call;
  int line;
};
#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) throw CudaFailure{e_, #call, __LINE__}; \
  } while (0)

enum KernelId {
  KID_INIT,
  KID_PROJGR,
  KID_BEGIN,
  KID_GCP,
  KID_WALK_GATHER,
  KID_WALK,
  KID_FREEV,
  KID_SUBDIR,
  KID_SUBAPPLY,
  KID_TRIAL,
  KID_POST,
  KID_POSTGCP,
  KID_COUNT
};
static const char* kKernelNames[KID_COUNT] = {
    "k_init",      "k_projgr",    "k_begin_iteration", "k_gcp_scan",
    "k_walk_gather", "k_walk_coop", "k_freev_formk",   "k_subsm_dir",
    "k_subsm_apply", "k_trial",   "k_post_eval",       "k_post_gcp"};

template <typename R>
struct Api;
template <>
struct Api<double> {
  using Opt = lbfgsb_b200_option_f64;
  using Sum = lbfgsb_b200_summary_f64;
  using Cb = lbfgsb_b200_callback_f64;
};
template <>
struct Api<float> {
  using Opt = lbfgsb_b200_option_f32;
  using Sum = lbfgsb_b200_summary_f32;
  using Cb = lbfgsb_b200_callback_f32;
};

// Launch bookkeeping: counts every launch, and with profiling brackets it with events.
class Launcher {
 public:
  Launcher(cudaStream_t s, bool profile) : s_(s), profile_(profile) {
    std::fill(count_, count_ + KID_COUNT, 0LL);
  }
  ~Launcher() {
    for (auto& e : pool_) cudaEventDestroy(e);
  }
  template <typename F>
  void run(int kid, F&& launch) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (profile_) {
      a = event();
      b = event();
      CK(cudaEventRecord(a, s_));
    }
    launch();
    CK(cudaGetLastError());
    if (profile_) {
      CK(cudaEventRecord(b, s_));
      timed_.push_back({kid, a, b});
    }
    count_[kid]++;
  }
  void collect(lbfgsb_b200_stats* st) {
    for (int k = 0; k < KID_COUNT; k++) {
      st->launches[k] = count_[k];
      st->total_launches += count_[k];
      st->ms[k] = 0;
    }
    for (auto& t : timed_) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) st->ms[t.kid] += ms;
    }
  }

 private:
  struct Timed {
    int kid;
    cudaEvent_t a, b;
  };
  cudaEvent_t event() {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    pool_.push_back(e);
    return e;
  }
  cudaStream_t s_;
  bool profile_;
  long long count_[KID_COUNT];
  std::vector<Timed> timed_;
  std::vector<cudaEvent_t> pool_;
};

// Owns the device workspace of one solve.
// Workspace memory comes from a library-owned stream-ordered pool per device that keeps
// its memory between solves (release threshold: unlimited), so repeated solves do not map
// and unmap gigabytes each time; lbfgsb_b200_trim_memory() returns it to the device.
// The library-owned stream-ordered memory pool of the current device (driver.cu); its
// release threshold is unlimited, so memory stays mapped between solves.
cudaMemPool_t workspace_pool();

template <typename R, typename H, typename S>
struct Workspace {
  cudaStream_t s = nullptr;
  std::vector<void*> blocks;
  R* X[3] = {nullptr, nullptr, nullptr};
  R* G[2] = {nullptr, nullptr};
  R* dsub = nullptr;
  H* ws = nullptr;
  H* wy = nullptr;
  int8_t* code = nullptr;
  uint32_t* fbits = nullptr;
  DevState<S>* st = nullptr;
  DevState<S>* hs = nullptr;  // pinned mirror
  double* part = nullptr;
  unsigned int* ticket = nullptr;
  double* wl_t = nullptr;
  int* wl_i = nullptr;
  unsigned int* wl_n = nullptr;

  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    CK(cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), workspace_pool(), s));
    blocks.push_back(p);
    return static_cast<T*>(p);
  }
  void release() {
    for (void* p : blocks) cudaFreeAsync(p, s);
    blocks.clear();
  }
  ~Workspace() { release(); }
};

// Pinned host scratch of the calling thread, `which` = 0 the state header's mirror, 1 the
// device-driven solve's evaluation slot (each allocated once, grown when needed).
static void* pinned_scratch(int which, size_t bytes) {
  struct Mirror {
    void* p = nullptr;
    size_t bytes = 0;
    ~Mirror() {
      if (p) cudaFreeHost(p);
    }
  };
  thread_local Mirror m[2];
  Mirror& mm = m[which];
  if (mm.bytes < bytes) {
    if (mm.p) CK(cudaFreeHost(mm.p));
    mm.p = nullptr;
    mm.bytes = 0;
    CK(cudaMallocHost(&mm.p, bytes));
    mm.bytes = bytes;
  }
  return mm.p;
}
static void* pinned_mirror(size_t bytes) { return pinned_scratch(0, bytes); }
static void* pinned_mirror_slot(size_t bytes) { return pinned_scratch(1, bytes); }

static int device_sms() {
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return sms;
}

// Launch shape of a staged-tile pass: as many ring stages as fit a shared-memory budget
// (2..8), the dynamic shared memory that needs, and a grid of resident CTAs.
struct PassCfg {
  int grid = 1, stages = 2, smem = 0, threads = 0;
};
constexpr int kConsWide = 512;    // consumer threads of the staged passes
constexpr int kRingBudget = 176 * 1024;

// extra: dynamic shared memory the pass uses after its ring (freev_extra_smem).
template <typename K>
static PassCfg pass_cfg(K kernel, int cap, long long n, int threads, int extra = 0) {
  PassCfg p;
  p.threads = threads;
  // a CTA never has more tiles in flight than it processes: small problems take fewer
  // stages, which leaves room for other streams' CTAs on the same SM
  const long long tiles = (n + kTile - 1) / kTile;
  const long long per_cta = (tiles + device_sms() - 1) / device_sms();
  p.stages = std::max(2, std::min<int>(std::min(kMaxStages, kRingBudget / cap), (int)per_cta + 1));
  // the attribute is per kernel and process-wide, while solves of different sizes may run
  // concurrently on other threads: it is always set to the full opt-in allowance (the same
  // value from every thread), and each launch asks only for its own ring
  int dev = 0, optin = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, kernel));
  const int allowance = optin - (int)fa.sharedSizeBytes;
  while (p.stages > 2 && ring_bytes(p.stages, cap) + extra > allowance) p.stages--;
  p.smem = ring_bytes(p.stages, cap) + extra;
  if (p.smem > allowance) throw CudaFailure{cudaErrorInvalidValue, "stage ring exceeds shared memory", __LINE__};
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, allowance));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, p.smem));
  per_sm = std::max(per_sm, 1);
  p.grid = (int)std::max<long long>(1, std::min<long long>(tiles, (long long)device_sms() * per_sm));
  return p;
}

template <typename K>
static int grid_for(K kernel, int n, int threads) {
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
  per_sm = std::max(per_sm, 1);
  long long want = ((long long)n + threads - 1) / threads;
  long long cap = (long long)device_sms() * per_sm;
  return (int)std::max<long long>(1, std::min(want, cap));
}

// The breakpoint-walk buffers of one solve: the list of (t, i) and the cooperative walk's
// scratch.
template <typename R, typename H, typename S>
static void walk_buffers(Workspace<R, H, S>& w, Ctx<R, H, S>& c, size_t N) {
  w.wl_t = w.template alloc<double>(N);
  w.wl_i = w.template alloc<int>(N);
  w.wl_n = w.template alloc<unsigned int>(1);
  c.wl_t = w.wl_t;
  c.wl_i = w.wl_i;
  c.wl_n = w.wl_n;
  c.wsc = w.template alloc<WalkScratch>(1);
}

// Grid of the cooperative walk: CTAs that are all resident at once (one per SM at most).
template <typename R, typename H, typename S>
static int walk_coop_grid() {
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_coop<R, H, S>, kWalkThreads, 0));
  if (per_sm < 1) throw CudaFailure{cudaErrorCooperativeLaunchTooLarge, "k_walk_coop occupancy", __LINE__};
  return device_sms();
}

// The cooperative walk: listing, selection and walk in one launch whose CTAs are
// guaranteed to be resident together (its grid barrier relies on that).  *wl_n and the
// barrier must be zero (the host clears them, or a device-driven round's k_round_begin).
template <typename R, typename H, typename S>
static void launch_walk_coop(const Ctx<R, H, S>& c, const R* x, const R* g, int grid,
                             cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kWalkThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, k_walk_coop<R, H, S>, c, x, g));
}

// Launch shapes of one solve's passes.
struct Plan {
  PassCfg gcp, freev, dir, apply, post, pgcp;
  int g_proj = 1, g_elem = 1;
};

// Takes one solve's workspace from the pool, checks its alignment, fills the pass context
// and the launch shapes, zeroes the history, and fills the host copy of the state (w.hs)
// with the start of the reference driver (head = 1, theta = 1, col = 0).  walk: allocate
// the breakpoint-walk buffers now (device-driven solves cannot allocate them on demand).
template <typename R, typename H, typename S>
static void prepare(Workspace<R, H, S>& w, Ctx<R, H, S>& c, Plan& p, int n, int m, const int* nbd,
                    const R* l, const R* u, cudaStream_t stream, const lbfgsb_b200_ext* ext,
                    bool walk) {
  const size_t N = (size_t)n;
  for (int k = 0; k < 3; k++) w.X[k] = w.template alloc<R>(N);
  for (int k = 0; k < 2; k++) w.G[k] = w.template alloc<R>(N);
  w.dsub = w.template alloc<R>(N);
  const size_t ld = ((N + kTile - 1) / kTile) * kTile;  // 16-byte aligned slots
  w.ws = w.template alloc<H>(ld * kSlots);
  w.wy = w.template alloc<H>(ld * kSlots);
  w.code = w.template alloc<int8_t>(N);
  const size_t words = (N + 31) / 32 + 1;
  w.fbits = w.template alloc<uint32_t>(words);
  w.st = w.template alloc<DevState<S>>(1);
  w.ticket = w.template alloc<unsigned int>(1);
  w.hs = static_cast<DevState<S>*>(pinned_mirror(sizeof(DevState<S>)));

  // the staged passes copy l, u and nbd in 16-byte aligned tiles
  const R* la = l;
  const R* ua = u;
  const int* nbda = nbd;
  auto misaligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) != 0; };
  if (misaligned(l) || misaligned(u) || misaligned(nbd)) {
    R* lc = w.template alloc<R>(N);
    R* uc = w.template alloc<R>(N);
    int* nc = w.template alloc<int>(N);
    CK(cudaMemcpyAsync(lc, l, N * sizeof(R), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(uc, u, N * sizeof(R), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(nc, nbd, N * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    la = lc;
    ua = uc;
    nbda = nc;
  }

  // every stream the staged passes copy with cp.async.bulk starts on a 16-byte boundary
  for (const void* q : {(const void*)la, (const void*)ua, (const void*)nbda, (const void*)w.X[0],
                        (const void*)w.X[1], (const void*)w.X[2], (const void*)w.G[0],
                        (const void*)w.G[1], (const void*)w.dsub, (const void*)w.code,
                        (const void*)w.fbits, (const void*)w.ws, (const void*)w.wy}) {
    if (misaligned(q)) throw CudaFailure{cudaErrorMisalignedAddress, "workspace alignment", __LINE__};
  }

  c = Ctx<R, H, S>{};
  c.n = n;
  c.l = la;
  c.u = ua;
  c.nbd = nbda;
  c.ws = w.ws;
  c.wy = w.wy;
  c.ld = (long long)ld;
  c.stages = 2;
  c.code = w.code;
  c.fbits = w.fbits;
  c.dsub = w.dsub;
  c.st = w.st;
  c.ticket = w.ticket;
  c.wl_t = nullptr;
  c.wl_i = nullptr;
  c.wl_n = nullptr;
  c.rounds = 0;
  c.hash_free = (ext && ext->trace) ? 1 : 0;
  for (int k = 0; k < 3; k++) c.X[k] = w.X[k];
  for (int k = 0; k < 2; k++) c.G[k] = w.G[k];
  c.gdummy = nullptr;
  c.ev_x = nullptr;
  c.ev_g = nullptr;
  c.ev_f = nullptr;
  c.ev_act = nullptr;
  c.wsc = nullptr;
  if (walk) walk_buffers(w, c, N);

  const int hsz = (int)sizeof(H);
  p.gcp = pass_cfg(k_gcp_scan<R, H, S, kConsWide>,
                   stage_capacity(StageBytes<R>::gcp, 0, m, hsz), n, kConsWide + 32);
  p.freev = pass_cfg(k_freev_formk<R, H, S, kConsWide>,
                     stage_capacity(StageBytes<R>::freev, kTile / 8, m, hsz), n, kConsWide + 32,
                     freev_extra_smem<S>());
  p.dir = pass_cfg(k_subsm_dir<R, H, S, kConsWide>,
                   stage_capacity(StageBytes<R>::dir, 0, m, hsz), n, kConsWide + 32);
  p.apply = pass_cfg(k_subsm_apply<R, H, S, kConsWide>,
                     stage_capacity(StageBytes<R>::apply, 0, 0, hsz), n, kConsWide + 32);
  p.post = pass_cfg(k_post_eval<R, H, S, kConsWide>,
                    stage_capacity(StageBytes<R>::post, 0, m, hsz), n, kConsWide + 32);
  p.pgcp = pass_cfg(k_post_gcp<R, H, S, kConsWide>,
                    stage_capacity(StageBytes<R>::post, 0, m, hsz), n, kConsWide + 32);
  p.g_proj = grid_for(k_projgr<R, H, S>, n, kThreads);
  const int g_max = std::max({p.gcp.grid, p.freev.grid, p.dir.grid, p.apply.grid, p.post.grid,
                              p.pgcp.grid, p.g_proj});
  w.part = w.template alloc<double>((size_t)g_max * 256);
  c.part = w.part;
  p.g_elem = (int)std::min<long long>(((long long)n + 255) / 256, (long long)device_sms() * 8);

  // history slots start at zero so that unused positions read as finite values
  CK(cudaMemsetAsync(w.ws, 0, N * kSlots * sizeof(H), stream));
  CK(cudaMemsetAsync(w.wy, 0, N * kSlots * sizeof(H), stream));
  CK(cudaMemsetAsync(w.fbits, 0, words * sizeof(uint32_t), stream));
  CK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned int), stream));

  DevState<S>& hs = *w.hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.n = n;
  hs.m = m;
  hs.subsm_proj = (ext && ext->subsm_projection) ? 1 : 0;
  hs.boxed = 1;
  hs.head = 1;
  hs.theta = 1;
  hs.iword = -1;
  hs.big = (S)1.0e10;
  for (int r = 1; r <= m; r++) hs.phys[r] = r - 1;
  hs.spare = m;
  hs.xr[0] = 0;
  hs.xr[1] = 1;
  hs.xr[2] = 2;
  hs.gr[0] = 0;
  hs.gr[1] = 1;
}

template <typename R>
struct DevObjective;
template <>
struct DevObjective<double> {
  using Fn = lbfgsb_b200_device_objective_f64;
};
template <>
struct DevObjective<float> {
  using Fn = lbfgsb_b200_device_objective_f32;
};

// The calling thread's stream for device-driven solves (capture needs a stream other than
// the legacy default stream) and the two events that order it after / before the caller's.
struct RoundStream {
  cudaStream_t s = nullptr;
  cudaEvent_t in = nullptr, out = nullptr;
  int dev = -1;
  ~RoundStream() {
    if (in) cudaEventDestroy(in);
    if (out) cudaEventDestroy(out);
    if (s) cudaStreamDestroy(s);
  }
};
static RoundStream& round_stream() {
  thread_local RoundStream rs;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (rs.dev != dev) {
    if (rs.s) {
      cudaEventDestroy(rs.in);
      cudaEventDestroy(rs.out);
      cudaStreamDestroy(rs.s);
    }
    rs.s = nullptr;
    CK(cudaStreamCreateWithFlags(&rs.s, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&rs.in, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&rs.out, cudaEventDisableTiming));
    rs.dev = dev;
  }
  return rs;
}

// The evaluation slot of one device-driven solve (device memory): the objective reads x at
// *x, writes g to *g and f to f; active = 0 marks an evaluation whose result is not used.
struct EvalSlots {
  void* x;
  void* g;
  double f;
  int active;
  int pad;
};

// Owns a captured round graph.
struct RoundGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t e = nullptr;
  ~RoundGraph() {
    if (e) cudaGraphExecDestroy(e);
    if (g) cudaGraphDestroy(g);
  }
};

}  // namespace lbfgsb_b200
