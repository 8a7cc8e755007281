// passes.cuh -- the streaming passes of one L-BFGS-B iteration on sm_100a.
//
// One iteration of the reference's outer loop (culbfgsb/lbfgsbcpu.cpp:279-462) is cut into
// five grid-wide passes over the n-vectors and the slot-major S/Y history, each ending
// in a deterministic reduction whose last CTA runs the scalar / small-matrix epilogue:
//
//   A  k_gcp_scan        cauchy's scan (lbfgsbcpu.cpp:634-701): iwhere, d = -g, p = W'd,
//                        f', breakpoints; epilogue: f'', dtm, first-breakpoint test
//                        (the full breakpoint walk, when needed, is walk.cuh)
//   B  k_freev_formk     freev (1135-1173) as a bitmask, the formk products (972-1054:
//                        new row over F/A, entering/leaving corrections), cmprlb's reduced
//                        gradient r (819-869) and subsm's W'r (1446-1458); epilogue:
//                        formk assembly + factorisation, the two K solves
//   C  k_subsm_dir       subsm's direction (1472-1483) and the step to the first bound
//                        (1484-1516) as an arg-min reduction
//   D  k_subsm_apply     the truncated step (1517-1533), d = z - x, and lnsrlb's start
//                        (1263-1320): dtd, stpmx, g'd; epilogue: dcsrch start
//   E  k_post_eval       after each function evaluation: g'd and dcsrch (1312-1338); on
//                        acceptance the stopping-test quantities (projgr, |dx|, rr) and
//                        matupd/formt (1341-1387, 1105-1133), with (s, y) written to a
//                        spare history slot that the epilogue commits to the ring
//
// Elementwise arithmetic that feeds a comparison or a stored vector repeats the
// reference's operations in its order (the build uses -fmad=false, so no FMA is
// contracted); reductions accumulate in double with explicit fma().
#pragma once

#include <type_traits>

#include "common.cuh"
#include "reduce.cuh"
#include "small.cuh"
#include "state.cuh"
#include "tiles.cuh"
#include "warp_small.cuh"

namespace lbfgsb_b200 {

// Scratch of the cooperative breakpoint walk (walk.cuh, k_walk_coop): its grid barrier,
// the radix-select histograms (three, used in rotation), and the selected chunk.
constexpr int kWalkChunk = 1024;  // breakpoints selected and sorted at a time
struct WalkScratch {
  unsigned int bar;      // grid-barrier arrivals; zero before each launch
  unsigned int chunk_n;  // keys of the selected chunk
  int done;              // the walk has ended
  int cnt;               // keys in the chunk just walked
  unsigned long long last_hi;  // largest key walked so far
  unsigned int last_lo;
  unsigned int pad;
  unsigned int hist[3][256];
  unsigned long long chunk_hi[kWalkChunk];
  unsigned int chunk_lo[kWalkChunk];
};

template <typename R, typename H, typename S>
struct Ctx {
  int n;
  const R* __restrict__ l;
  const R* __restrict__ u;
  const int* __restrict__ nbd;
  H* ws;             // kSlots slot-major arrays, slot stride ld elements
  H* wy;
  long long ld;      // history slot stride (n rounded up to a multiple of kTile)
  int stages;        // depth of the staged-tile ring of the passes
  int8_t* code;      // iwhere codes
  uint32_t* fbits;   // free set of the last freev, one bit per variable
  R* dsub;           // subspace direction on the free set
  DevState<S>* st;
  double* part;      // reduction rows
  unsigned int* ticket;
  double* wl_t;      // breakpoint list (walk)
  int* wl_i;
  unsigned int* wl_n;
  WalkScratch* wsc;  // the cooperative walk's scratch (single-instance solves)
  // device-driven solves: rounds = 1 makes every pass gate itself on the round plan in the
  // state and take its vectors from the buffers below by the roles st->xr / st->gr
  int rounds;
  int hash_free;     // 1: form the free-set hash (reported only by the per-iteration trace)
  R* X[3];
  R* G[2];
  R* gdummy;         // g of evaluations whose result is not used
  // where the objective of a device-driven solve reads x (*ev_x) and writes g (*ev_g) and
  // f (*ev_f); *ev_act = 0 marks an evaluation whose result is not used (device memory;
  // a batch keeps each of them as one array over its instances)
  R** ev_x;
  R** ev_g;
  double* ev_f;
  int* ev_act;
  // sharded solves (reduce.cuh): this rank's variables are global indices ioff .. ioff + n;
  // shard_send / shard_recv hold the rank rows of a pass's reduction (null and 0 otherwise),
  // epi_only = 1 in the one-CTA launch that folds the gathered rows and runs the epilogue
  int shard_world = 0;
  int ioff = 0;
  int epi_only = 0;
  double* shard_send = nullptr;
  const double* shard_recv = nullptr;
};

// Physical slot pointers of ring positions 1..kMaxM counted from head.
template <typename H, typename S>
__device__ __forceinline__ void ring_ptrs(const DevState<S>* st, const H* base, long long ld,
                                          const H* (&out)[kMaxM]) {
  const int m = st->m, head = st->head;
#pragma unroll
  for (int j = 0; j < kMaxM; j++) {
    int r = (head - 1 + j) % m + 1;
    out[j] = base + (size_t)st->phys[r] * (size_t)ld;
  }
}

// Bytes per element of the scalar streams each pass stages (the history columns add
// 2*col*sizeof(H) per element, the free-set bits 32 bytes per tile).
template <typename R>
struct StageBytes {
  static constexpr int gcp = 4 * (int)sizeof(R) + 4;        // x g l u nbd
  static constexpr int freev = 1 + 2 * (int)sizeof(R);      // code x g
  static constexpr int dir = 1 + 4 * (int)sizeof(R) + 4;    // code x g l u nbd
  static constexpr int apply = 1 + 5 * (int)sizeof(R) + 4;  // code x g l u dsub nbd
  static constexpr int post = 7 * (int)sizeof(R) + 4;       // t z g go l u nbd (+ xt)
};
// Shared-memory ring capacity of one stage for a pass with `scalar` bytes per element.
__host__ __device__ inline int stage_capacity(int scalar, int extra_tile, int m, int hsize) {
  return kTile * scalar + extra_tile + 2 * m * kTile * hsize;
}
__host__ __device__ inline int ring_bytes(int stages, int cap) { return stages * cap + 16 * stages; }
// Dynamic shared memory the free-set pass needs after its stage ring: the per-thread
// active-set sums of its one-role form (float sums), 16 floats for each of kTile threads.
template <typename S>
__host__ __device__ constexpr int freev_extra_smem() {
  return sizeof(typename AccOf<S>::type) == 4 ? 16 * kTile * (int)sizeof(float) : 0;
}

__device__ __forceinline__ int add_stream(StreamSet& ss, const void* base, int tile_bytes) {
  const int j = ss.count++;
  ss.src[j] = static_cast<const unsigned char*>(base);
  ss.tile_bytes[j] = tile_bytes;
  ss.off[j] = ss.stage_bytes;
  ss.stage_bytes += tile_bytes;
  return j;
}

// Appends the col y-columns, then the col s-columns, of the ring (positions 1..col from
// head); returns the stage offsets of the first y and s column.
template <typename R, typename H, typename S>
__device__ __forceinline__ void add_history(StreamSet& ss, const Ctx<R, H, S>& c,
                                            const DevState<S>* st, int& hy, int& hs) {
  const int col = st->col, m = st->m, head = st->head;
  const int hb = kTile * (int)sizeof(H);
  hy = ss.stage_bytes;
  for (int j = 0; j < col; j++) {
    const int r = (head - 1 + j) % m + 1;
    add_stream(ss, c.wy + (size_t)st->phys[r] * (size_t)c.ld, hb);
  }
  hs = ss.stage_bytes;
  for (int j = 0; j < col; j++) {
    const int r = (head - 1 + j) % m + 1;
    add_stream(ss, c.ws + (size_t)st->phys[r] * (size_t)c.ld, hb);
  }
}

template <typename T>
__device__ __forceinline__ T stage_at(const unsigned char* buf, int off, int e) {
  return reinterpret_cast<const T*>(buf + off)[e];
}
// A history element of the stage as the accumulator type A.
template <typename H, typename A = double>
__device__ __forceinline__ A hist_at(const unsigned char* buf, int off, int e) {
  const H v = reinterpret_cast<const H*>(buf + off)[e];
  if constexpr (sizeof(H) == 2) {
    return (A)__bfloat162float(v);
  } else {
    return (A)v;
  }
}

// The per-thread sums as doubles, for the CTA and grid levels of a reduction.
template <typename A, int N>
__device__ __forceinline__ void sums_to_double(const A (&a)[N], double (&d)[N]) {
#pragma unroll
  for (int k = 0; k < N; k++) d[k] = (double)a[k];
}

// The history loops run over the col live columns.  In the steady state col == kMaxM and
// the pass body is compiled with that as a constant (the unrolled loops carry no
// per-column tests); otherwise with the runtime col.  f(tag): decltype(tag)::value is
// kMaxM or -1.
template <int V>
struct Cols {
  static constexpr int value = V;
};
template <typename F>
__device__ __forceinline__ void dispatch_cols(int col, F&& f) {
  if (col == kMaxM)
    f(Cols<kMaxM>{});
  else
    f(Cols<-1>{});
}

// cauchy's per-variable classification (lbfgsbcpu.cpp:635-663) and breakpoint
// (675-699).  Returns the iwhere code; for a movable variable with a breakpoint sets
// has_bp and the breakpoint as the quotient num/den (the reference's tl/(-g) or tu/g).
// The static codes -1 (nbd 0) and 3 (l == u) come from nbd, l, u, which is what
// lbfgsbactive stored (467-515).
template <typename R>
__device__ __forceinline__ int classify_q(R x, R g, R l, R u, int nb, bool& has_bp, R& num,
                                          R& den) {
  // written with selects rather than branches (the lanes of a warp take different ones):
  // every value is the reference's, formed from the same operands; bounds that nb does
  // not declare are read but never selected
  const R neggi = -g;
  const bool hl = nb <= 2, hu = nb >= 2;
  const R tl = rsub(x, l), tu = rsub(u, x);
  const bool xlower = hl && tl <= R(0);
  const bool xupper = hu && tu <= R(0);
  int code = xlower   ? (neggi <= R(0) ? IW_LOW : IW_FREE)
             : xupper ? (neggi >= R(0) ? IW_UPP : IW_FREE)
                      : (fabs(neggi) <= R(0) ? IW_ZERO : IW_FREE);
  const bool fixed = nb == 2 && rsub(u, l) <= R(0);
  code = nb == 0 ? IW_UNB : fixed ? IW_FIX : code;
  const bool isfree = code == IW_FREE;
  const bool bl = isfree && hl && neggi < R(0);
  const bool bu = isfree && !bl && hu && neggi > R(0);
  has_bp = bl || bu;
  num = bl ? tl : bu ? tu : R(0);
  den = bl ? -neggi : bu ? neggi : R(1);
  return code;
}
// classify_q with the breakpoint t = num/den correctly rounded.
template <typename R>
__device__ __forceinline__ int classify(R x, R g, R l, R u, int nb, bool& has_bp, R& t) {
  R num, den;
  const int code = classify_q(x, g, l, u, nb, has_bp, num, den);
  t = has_bp ? rdiv(num, den) : R(0);
  return code;
}

// The generalized Cauchy point of one variable, rebuilt from its code: xcp = x + tsum*d
// for a variable that moves along d = -g (lbfgsbcpu.cpp:813), its bound when the walk
// fixed it (755-761), x otherwise.
template <typename R, typename S>
__device__ __forceinline__ R gcp_point(int code, R x, R g, R l, R u, S tsum) {
  const S d = (S)(-g);
  const R moved = (R)((S)x + tsum * d);
  return (code == IW_FREE || code == IW_UNB) ? moved
         : code == IW_WALK_LOW             ? l
         : code == IW_WALK_UPP             ? u
                                           : x;
}

// cmprlb's reduced gradient of one free variable (lbfgsbcpu.cpp:842-867), in the
// reference's operation order.  uncon: the !cnstnd && col > 0 branch (r = -g).
template <typename R, typename S>
__device__ __forceinline__ S reduced_grad(bool uncon, R x, R z, R g, int col,
                                          const S (&yv)[kMaxM], const S (&sv)[kMaxM],
                                          const S* a1, const S* a2) {
  if (uncon) return -(S)g;
  S r = -a1[kMaxM] * ((S)z - (S)x) - (S)g;  // a1[kMaxM] holds theta
#pragma unroll
  for (int j = 0; j < kMaxM; j++)
    if (j < col) r = r + yv[j] * a1[j] + sv[j] * a2[j];
  return r;
}

// cauchy's epilogue (lbfgsbcpu.cpp:702-733) and the first breakpoint test of the walk
// (745-747), from the sums of the scan over the movable variables: red[0] sum g^2,
// red[1..8] / red[9..16] the y / s parts of p = W'd by ring position, red[17] nbreak,
// red[18] movable variables without a breakpoint, red[19] > 0 if one of them has g != 0,
// red[20] / red[21] the smallest breakpoint and its index.
template <typename S>
__device__ void gcp_epilogue(DevState<S>* st, const double* red, int col, SmallWork<S>& sw,
                             int lane) {
  // run by the 32 lanes of one warp: lane 0 writes the scalars, the products with the
  // middle matrix are shared out (wbmv); every branch below depends only on red, st->theta
  // and values that all lanes compute alike, so the warp never splits
  const S theta = st->theta;
  const S f1 = -(S)red[0];
  const int col2 = 2 * col;
  const int nbreak = (int)red[17], nfree_mov = (int)red[18];
  if (lane == 0) {
    #pragma unroll 1
    for (int j = 1; j <= col; j++) {
      st->p[j] = (S)red[j];
      st->p[col + j] = (S)red[8 + j];
    }
    if (theta != S(1))
      #pragma unroll 1
      for (int j = col + 1; j <= col2; j++) st->p[j] *= theta;
    st->nbreak = nbreak;
    st->nfree_mov = nfree_mov;
    st->bnded = red[19] > 0.0 ? 0 : 1;
    st->internal_fail = 0;
  }
  __syncwarp();
  if (nbreak == 0 && nfree_mov == 0) {
    // xcp = x; c is left as it was (lbfgsbcpu.cpp:706-708), and cmprlb still applies the
    // current middle matrix to it
    if (lane == 0) {
      st->gcp_state = GCP_EARLY;
      st->tsum = 0;
    }
    if (col > 0) {
      const int info = wbmv(st->sy, st->wt, col, st->c, st->mc, sw.work, lane);
      if (lane == 0 && info != 0) st->internal_fail = -8;
    }
    return;
  }
  if (lane == 0)
    #pragma unroll 1
    for (int j = 1; j <= col2; j++) st->c[j] = 0;
  S f2 = -theta * f1;
  const S f2org = f2;
  if (col > 0) {
    S* v = sw.v;
    const int info = wbmv(st->sy, st->wt, col, st->p, v, sw.work, lane);
    if (info != 0) {
      if (lane == 0) st->internal_fail = info;
      return;
    }
    f2 = f2 - sdot(&v[1], 1, &st->p[1], 1, col2);
  }
  S dtm = -f1 / f2;
  if (lane == 0) {
    st->f1 = f1;
    st->f2 = f2;
    st->f1_0 = f1;
    st->f2_0 = f2;
    st->f2org = f2org;
    st->tsum = 0;
    st->tj = 0;
    st->nint = 1;
    st->nleft = nbreak;
  }
  if (nbreak != 0) {
    const S bkmin = (S)red[20];
    if (lane == 0) {
      st->bkmin = bkmin;
      st->ibkmin = (int)red[21];
    }
    if (!(dtm < bkmin - S(0))) {
      if (lane == 0) {
        st->dtm = dtm;
        st->gcp_state = GCP_WALK;  // at least one breakpoint is passed
      }
      return;
    }
  }
  if (dtm <= S(0)) dtm = 0;
  if (lane == 0) {
    st->dtm = dtm;
    st->tsum = st->tsum + dtm;
    #pragma unroll 1
    for (int j = 1; j <= col2; j++) st->c[j] += dtm * st->p[j];
  }
  __syncwarp();
  if (col > 0) {
    const int info = wbmv(st->sy, st->wt, col, st->c, st->mc, sw.work, lane);  // cmprlb's M c (852)
    if (lane == 0 && info != 0) st->internal_fail = -8;
  }
  if (lane == 0) st->gcp_state = GCP_DONE;
}

// ------------------------------------------------------------------------------------
// A: the Cauchy-point scan.
template <typename R, typename H, typename S, int CONS>
__device__ __forceinline__ void gcp_scan_pass(const Ctx<R, H, S>& c, CtaPos cp, int stages,
    const R* __restrict__ x,
                                                       const R* __restrict__ g) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!st->rp_scan) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
  }
  const int n = c.epi_only ? 0 : c.n, col = st->col;
  // sums: [0] sum neggi^2, [1..16] p (y part 1..8, s part 9..16), [17] nbreak,
  // [18] movable variables without breakpoint; max: [0] any such with g != 0;
  // min pair: smallest breakpoint
  constexpr int NS = 19, NX = 1, NM = 1;
  using A = typename AccOf<S>::type;
  A s[NS];
  double xm[NX];
  ArgMin<R> bp;  // the smallest breakpoint
#pragma unroll
  for (int k = 0; k < NS; k++) s[k] = A(0);
  xm[0] = 0.0;

  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ StreamSet ss;
  __shared__ int s_hy, s_hs;
  if (threadIdx.x == 0) {
    ss.count = 0;
    ss.stage_bytes = 0;
    add_stream(ss, x, kTile * (int)sizeof(R));
    add_stream(ss, g, kTile * (int)sizeof(R));
    add_stream(ss, c.l, kTile * (int)sizeof(R));
    add_stream(ss, c.u, kTile * (int)sizeof(R));
    add_stream(ss, c.nbd, kTile * 4);
    add_history(ss, c, st, s_hy, s_hs);
  }
  __syncthreads();
  const int o_x = ss.off[0], o_g = ss.off[1], o_l = ss.off[2], o_u = ss.off[3], o_nb = ss.off[4];
  const int hy = s_hy, hs = s_hs, hb = kTile * (int)sizeof(H);
  const int cap = stage_capacity(StageBytes<R>::gcp, 0, st->m, (int)sizeof(H));
  dispatch_cols(col, [&](auto cols_tag) {
    constexpr bool kFull = decltype(cols_tag)::value == kMaxM;
    run_tiles<CONS>(ss, n, stages, dyn, reinterpret_cast<uint64_t*>(dyn + (size_t)stages * cap),
              &st->device_error, cp, [&](const unsigned char* buf, long long t, int valid, int e) {
      if (e >= valid) return;
      const int i = (int)(t * kTile) + e;
      const R xi = stage_at<R>(buf, o_x, e), gi = stage_at<R>(buf, o_g, e);
      const R li = stage_at<R>(buf, o_l, e), ui = stage_at<R>(buf, o_u, e);
      const int nb = stage_at<int>(buf, o_nb, e);
      bool has_bp;
      R tnum, tden;
      const int code = classify_q(xi, gi, li, ui, nb, has_bp, tnum, tden);
      c.code[i] = (int8_t)code;
      if (code == IW_FREE || code == IW_UNB) {
        const A neggi = -(A)gi;
        s[0] = fma(neggi, neggi, s[0]);
  #pragma unroll
        for (int j = 0; j < kMaxM; j++) {
          if (kFull || j < col) {
            s[1 + j] = fma(hist_at<H, A>(buf, hy + j * hb, e), neggi, s[1 + j]);
            s[9 + j] = fma(hist_at<H, A>(buf, hs + j * hb, e), neggi, s[9 + j]);
          }
        }
        if (has_bp) {
          s[17] += A(1);
          // the smallest breakpoint: only candidates that can reach it are divided exactly
          bp.offer_quotient(tnum, tden, i + c.ioff);
        } else {
          s[18] += A(1);
          if (neggi != A(0)) xm[0] = 1.0;
        }
      }
    });
  });
  constexpr int W = NS + NX + 2 * NM;
  double lo[1] = {0.0}, sd[NS];
  MinPair mn[NM] = {bp.pair()};
  sums_to_double(s, sd);
  if (!c.epi_only) cta_reduce_to_row<CONS + 32, NS, NX, NM, 0>(sd, xm, mn, lo, c.part, W, cp.rank, cp.count);
  __shared__ double red[W];
  if (!pass_fold<CONS + 32>(c, cp, W, NS, NX, NM, red)) return;
  __shared__ SmallWork<S> sw;
  epilogue_on_shared_warp<S>(st, [&](DevState<S>* st, int lane) {
    gcp_epilogue<S>(st, red, col, sw, lane);
  });
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) k_gcp_scan(Ctx<R, H, S> c,
    const R* __restrict__ x, const R* __restrict__ g) {
  gcp_scan_pass<R, H, S, CONS>(c, cta_here(), c.stages, x, g);
}

// ------------------------------------------------------------------------------------
// B: freev + formk products + reduced gradient + W'r.  One warp handles 32 consecutive
// variables per step so that the free-set bitmask is read and written a word at a time.
constexpr int kLaneOwned = 5;  // 136 correction products over 32 lanes

// Output q of the 136 entering/leaving products: kind 0 y_a y_b (a >= b, q < 36),
// kind 1 s_a s_b (a >= b, q < 72), kind 2 s_a y_b (q < 136), kind 3 unused.
__host__ __device__ inline void corr_map(int q, int& kind, int& a, int& b) {
  if (q < 72) {
    kind = q < 36 ? 0 : 1;
    int t = q < 36 ? q : q - 36;
    a = 0;
    while ((a + 1) * (a + 2) / 2 <= t) a++;
    b = t - a * (a + 1) / 2;
  } else if (q < 136) {
    kind = 2;
    a = (q - 72) / kMaxM;
    b = (q - 72) % kMaxM;
  } else {
    kind = 3;
    a = b = 0;
  }
}

template <typename R, typename H, typename S, int CONS>
__device__ __forceinline__ void freev_formk_pass(const Ctx<R, H, S>& c, CtaPos cp, int stages,
    const R* __restrict__ x,
                                                          const R* __restrict__ g) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!st->rp_sub) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
  }
  if (st->gcp_state == GCP_WALK || st->internal_fail != 0) return;
  const int n = c.epi_only ? 0 : c.n, col = st->col, iter = st->iter;
  const bool uncon = st->uncon_branch != 0;
  const bool track = !uncon && iter > 0 && st->cnstnd;
  const bool updatd = st->updatd != 0;
  const S theta = st->theta, tsum = st->tsum;
  __shared__ __align__(16) S a1[kMaxM + 1], a2[kMaxM];  // cmprlb's coefficients (uniform)
  if (threadIdx.x < kMaxM) {
    const int j = threadIdx.x;
    a1[j] = (j < col) ? st->mc[1 + j] : S(0);
    a2[j] = (j < col) ? theta * st->mc[col + 1 + j] : S(0);
    if (j == 0) a1[kMaxM] = theta;
  }
  // Three warp roles over every tile (each role covers all kTile elements, so that the
  // accumulator sets never live in the same thread):
  //   role 0 (consumer warps 0..7, 2 elements per thread): acc[0..7] sum_F y_j r,
  //     acc[8..15] sum_F s_j r, the counts (nfree, nenter, nleave, at lower, at upper),
  //     the free-set bitmask and hash, and the entering / leaving corrections (lane-owned,
  //     accumulated in shared memory: corr_sm[warp][q] belongs to lane q mod 32);
  //   role 1 (warps 8..11, 4 elements per thread), when a pair was just added:
  //     acc[0..7] sum_F y_col y_j, acc[8..15] sum_F s_j y_col;
  //   role 2 (warps 12..15): acc[0..7] sum_A s_col s_j, acc[8..15] sum_A s_col y_j.
  //
  // With float sums (the FP32 plain form) the accumulators are small enough for one role:
  // every consumer thread does all of one element's work per tile (kOneRole), so that the
  // work stays balanced over the 16 warps whatever the share of free variables (with the
  // role split, the warps of the role that has no variables in a tile wait for the others).
  static_assert(CONS == 512, "the role split assumes 16 consumer warps");
  using A = typename AccOf<S>::type;
  constexpr bool kOneRole = sizeof(A) == 4;
  static_assert(!kOneRole || CONS == kTile, "one element per consumer thread and tile");
  constexpr int kRole0Warps = kOneRole ? CONS / 32 : 8, kRole12Warps = 4;
  constexpr int NA = 2 * kMaxM + 5, NB = 2 * kMaxM, NC = 2 * kMaxM;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int role = warp < kRole0Warps ? 0
                 : kOneRole ? 3
                 : warp < kRole0Warps + kRole12Warps ? 1
                 : warp < kRole0Warps + 2 * kRole12Warps ? 2 : 3;  // 3: the producer
  const int rt = role == 0 ? (int)threadIdx.x
               : (int)threadIdx.x - 32 * (kRole0Warps + (role - 1) * kRole12Warps);
  A acc[2 * kMaxM];
#pragma unroll
  for (int k = 0; k < 2 * kMaxM; k++) acc[k] = A(0);
  // kOneRole: the new row's products (roles 1 and 2 of the split): [0..7] sum_F y_col y_j,
  // [8..15] sum_F s_j y_col in registers; sum_A s_col s_j and sum_A s_col y_j per thread in
  // shared memory after the stage ring (entry q of thread e at nra[(q / 4) * CONS + e],
  // component q % 4), which keeps the thread within the register file's share of a
  // 17-warp CTA
  A nrow[kOneRole ? 2 * kMaxM : 1];
#pragma unroll
  for (int k = 0; k < (kOneRole ? 2 * kMaxM : 1); k++) nrow[k] = A(0);

  int cnt[5] = {0, 0, 0, 0, 0};
  unsigned long long hash = 0;
  __shared__ double corr_sm[kRole0Warps][32 * kLaneOwned];
  __shared__ double bc[kRole0Warps][2 * kMaxM];
  if (role == 0) {
#pragma unroll
    for (int k = 0; k < kLaneOwned; k++) corr_sm[warp][32 * k + lane] = 0.0;
  }
  const int newest = col - 1;
  const bool need_row = updatd && col > 0;

  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ StreamSet ss;
  __shared__ int s_hy, s_hs;
  if (threadIdx.x == 0) {
    ss.count = 0;
    ss.stage_bytes = 0;
    add_stream(ss, c.code, kTile);
    add_stream(ss, c.fbits, kTile / 8);
    add_stream(ss, x, kTile * (int)sizeof(R));
    add_stream(ss, g, kTile * (int)sizeof(R));
    add_history(ss, c, st, s_hy, s_hs);
  }
  __syncthreads();
  const int o_code = ss.off[0], o_bits = ss.off[1], o_x = ss.off[2], o_g = ss.off[3];
  const int hy = s_hy, hs = s_hs, hb = kTile * (int)sizeof(H);
  const int cap = stage_capacity(StageBytes<R>::freev, kTile / 8, st->m, (int)sizeof(H));
  float4* nra = reinterpret_cast<float4*>(dyn + ring_bytes(stages, cap));
  if (kOneRole && threadIdx.x < CONS) {
#pragma unroll
    for (int q = 0; q < 4; q++) nra[q * CONS + threadIdx.x] = make_float4(0.f, 0.f, 0.f, 0.f);
  }

  dispatch_cols(col, [&](auto cols_tag) {
    constexpr bool kFull = decltype(cols_tag)::value == kMaxM;
    auto role0 = [&](const unsigned char* buf, long long t, int valid, int e) {
      // the whole warp runs every call (ballots); word e/32 of the tile's free-set bits
      const int i = (int)(t * kTile) + e;
      const bool ok = e < valid;
      int code = IW_LOW;
      if (ok) code = stage_at<int8_t>(buf, o_code, e);
      const bool fnow = ok && (uncon || iw_free(code));
      const int wi = e >> 5;
      const uint32_t word = stage_at<uint32_t>(buf, o_bits, wi);
      const bool fprev = (word >> lane) & 1u;
      const bool enter = track && ok && !fprev && fnow;
      const bool leave = track && ok && fprev && !fnow;
      const uint32_t newword = __ballot_sync(0xffffffffu, fnow);
      if (!uncon && lane == 0 && wi * 32 < valid) c.fbits[t * (kTile / 32) + wi] = newword;
      if (ok) {
        if (fnow) {
          cnt[0]++;
          if (c.hash_free) hash += mix64((unsigned long long)(i + c.ioff));
          const R xi = stage_at<R>(buf, o_x, e), gi = stage_at<R>(buf, o_g, e);
          const R zi = uncon ? xi : gcp_point<R, S>(code, xi, gi, R(0), R(0), tsum);
          // cmprlb's r (842-867).  Here it only feeds the W'r reductions (the subspace
          // pass recomputes r in the reference's operation order for the stored
          // direction), so it is accumulated with fma in two independent chains.  The
          // history rows stay in the stage buffer (re-read, not held in registers).
          S r = -(S)gi;
          if (!uncon) {
            S ry = -a1[kMaxM] * ((S)zi - (S)xi) - (S)gi, rs = S(0);
  #pragma unroll
            for (int j = 0; j < kMaxM; j++)
              if (kFull || j < col) {
                ry = fma(hist_at<H, S>(buf, hy + j * hb, e), a1[j], ry);
                rs = fma(hist_at<H, S>(buf, hs + j * hb, e), a2[j], rs);
              }
            r = ry + rs;
          }
  #pragma unroll
          for (int j = 0; j < kMaxM; j++) {
            if (kFull || j < col) {
              acc[j] = fma(hist_at<H, A>(buf, hy + j * hb, e), (A)r, acc[j]);
              acc[8 + j] = fma(hist_at<H, A>(buf, hs + j * hb, e), (A)r, acc[8 + j]);
            }
          }
        } else {
          if (code == IW_LOW || code == IW_WALK_LOW) cnt[3]++;
          if (code == IW_UPP || code == IW_WALK_UPP) cnt[4]++;
        }
        if (enter) cnt[1]++;
        if (leave) cnt[2]++;
      }
      // entering (+) / leaving (-) variables: the whole warp adds the products of the
      // variable's rows, each lane its kLaneOwned outputs
      uint32_t pick = __ballot_sync(0xffffffffu, enter || leave);
      while (pick) {
        const int src = __ffs(pick) - 1;
        pick &= pick - 1;
        const double sign = __shfl_sync(0xffffffffu, enter ? 1.0 : -1.0, src);
        // the source variable's y and s rows, read from the stage buffer by lanes 0..15
        const int es = e - lane + src;
        if (lane < kMaxM)
          bc[warp][lane] = lane < col ? hist_at<H>(buf, hy + lane * hb, es) : 0.0;
        else if (lane < 2 * kMaxM)
          bc[warp][lane] = lane - kMaxM < col ? hist_at<H>(buf, hs + (lane - kMaxM) * hb, es) : 0.0;
        __syncwarp();
  #pragma unroll
        for (int k = 0; k < kLaneOwned; k++) {
          int kind, a, b;
          corr_map(lane + 32 * k, kind, a, b);
          if (kind < 3) {
            const int oa = kind == 0 ? a : kMaxM + a;
            const int ob = kind == 1 ? kMaxM + b : b;
            double& cq = corr_sm[warp][32 * k + lane];
            cq = fma(sign * bc[warp][oa], bc[warp][ob], cq);
          }
        }
        __syncwarp();
      }
    };
    // kOneRole: all of element e's work.  Its 2*col history values are read from the stage
    // once, into registers; the sums are those of roles 0, 1 and 2 below, with the same
    // operands in each fma.
    // fast: the steady state of a bounded problem (every column live, the free set tracked,
    // a new pair to multiply, no hash), compiled with those flags as constants
    // Every input of the element is read into registers first and the stage released, so
    // that the producer refills it while the sums are formed.
    auto one_role = [&](const unsigned char* buf, long long t, int valid, int e, auto fast,
                        auto release) {
      constexpr bool F = decltype(fast)::value;
      const bool uncon_ = F ? false : uncon;
      const bool track_ = F ? true : track;
      const bool need_row_ = F ? true : need_row;
      const bool hash_ = F ? false : c.hash_free != 0;
      const int i = (int)(t * kTile) + e;
      const bool ok = e < valid;
      int code = IW_LOW;
      if (ok) code = stage_at<int8_t>(buf, o_code, e);
      const int wi = e >> 5;
      const uint32_t word = stage_at<uint32_t>(buf, o_bits, wi);
      // past the tile's end the values are stale stage bytes, never used
      const R xi = stage_at<R>(buf, o_x, e), gi = stage_at<R>(buf, o_g, e);
      A yv[kMaxM], sv[kMaxM];
  #pragma unroll
      for (int j = 0; j < kMaxM; j++) {
        const bool live = kFull || j < col;
        yv[j] = live ? hist_at<H, A>(buf, hy + j * hb, e) : A(0);
        sv[j] = live ? hist_at<H, A>(buf, hs + j * hb, e) : A(0);
      }
      release();
      const bool fnow = ok && (uncon_ || iw_free(code));
      const bool fprev = (word >> lane) & 1u;
      const bool enter = track_ && ok && !fprev && fnow;
      const bool leave = track_ && ok && fprev && !fnow;
      const uint32_t newword = __ballot_sync(0xffffffffu, fnow);
      if (!uncon_ && lane == 0 && wi * 32 < valid) c.fbits[t * (kTile / 32) + wi] = newword;
      // the newest column, selected without a runtime register index
      const int nw = kFull ? kMaxM - 1 : newest;
      A ynew = A(0), snew = A(0);
#pragma unroll
      for (int j = 0; j < kMaxM; j++)
        if (j == nw) {
          ynew = yv[j];
          snew = sv[j];
        }
      // a free variable's sums (cmprlb's r with the W'r sums, the new row over the free set)
      auto free_elem = [&]() {
        cnt[0]++;
        if (hash_) hash += mix64((unsigned long long)(i + c.ioff));
        const R zi = uncon_ ? xi : gcp_point<R, S>(code, xi, gi, R(0), R(0), tsum);
        S r = -(S)gi;
        if (!uncon_) {
          S ry = -a1[kMaxM] * ((S)zi - (S)xi) - (S)gi, rs = S(0);
#pragma unroll
          for (int j = 0; j < kMaxM; j++)
            if (kFull || j < col) {
              ry = fma((S)yv[j], a1[j], ry);
              rs = fma((S)sv[j], a2[j], rs);
            }
          r = ry + rs;
        }
#pragma unroll
        for (int j = 0; j < kMaxM; j++) {
          if (kFull || j < col) {
            acc[j] = fma(yv[j], (A)r, acc[j]);
            acc[8 + j] = fma(sv[j], (A)r, acc[8 + j]);
          }
        }
        if (need_row_) {
#pragma unroll
          for (int j = 0; j < kMaxM; j++) {
            if (kFull || j < col) {
              nrow[j] = fma(ynew, yv[j], nrow[j]);
              nrow[8 + j] = fma(sv[j], ynew, nrow[8 + j]);
            }
          }
        }
      };
      if (F && __all_sync(0xffffffffu, fnow)) {
        free_elem();  // the steady state: every lane's variable free, no active-set code
      } else if (ok) {
        if (fnow) {
          free_elem();
        } else {
          if (code == IW_LOW || code == IW_WALK_LOW) cnt[3]++;
          if (code == IW_UPP || code == IW_WALK_UPP) cnt[4]++;
          if (need_row_) {
            // columns past col hold zeros and add nothing
#pragma unroll
            for (int q = 0; q < 4; q++) {
              float4 v = nra[q * CONS + e];
              const A* src = q < 2 ? sv : yv;
              const int j0 = (q & 1) * 4;
              v.x = fmaf((float)snew, (float)src[j0 + 0], v.x);
              v.y = fmaf((float)snew, (float)src[j0 + 1], v.y);
              v.z = fmaf((float)snew, (float)src[j0 + 2], v.z);
              v.w = fmaf((float)snew, (float)src[j0 + 3], v.w);
              nra[q * CONS + e] = v;
            }
          }
        }
      }
      if (enter) cnt[1]++;
      if (leave) cnt[2]++;
      // entering (+) / leaving (-) variables, as in role 0
      uint32_t pick = __ballot_sync(0xffffffffu, enter || leave);
      while (pick) {
        const int src = __ffs(pick) - 1;
        pick &= pick - 1;
        const double sign = __shfl_sync(0xffffffffu, enter ? 1.0 : -1.0, src);
        // the source variable's rows, from its lane's registers (columns past col are 0)
  #pragma unroll
        for (int j = 0; j < kMaxM; j++) {
          const A vy = __shfl_sync(0xffffffffu, yv[j], src);
          const A vs = __shfl_sync(0xffffffffu, sv[j], src);
          if (lane == 0) {
            bc[warp][j] = (double)vy;
            bc[warp][kMaxM + j] = (double)vs;
          }
        }
        __syncwarp();
  #pragma unroll
        for (int k = 0; k < kLaneOwned; k++) {
          int kind, a, b;
          corr_map(lane + 32 * k, kind, a, b);
          if (kind < 3) {
            const int oa = kind == 0 ? a : kMaxM + a;
            const int ob = kind == 1 ? kMaxM + b : b;
            double& cq = corr_sm[warp][32 * k + lane];
            cq = fma(sign * bc[warp][oa], bc[warp][ob], cq);
          }
        }
        __syncwarp();
      }
    };
    // roles 1 and 2: the new row's products over the free (role 1) or active (role 2) set
    auto rowprod = [&](const unsigned char* buf, int valid, int e) {
      if (e >= valid) return;
      const int code = stage_at<int8_t>(buf, o_code, e);
      const bool fnow = uncon || iw_free(code);
      if (fnow != (role == 1)) return;
      const A a = hist_at<H, A>(buf, (role == 1 ? hy : hs) + newest * hb, e);
      const int o1 = role == 1 ? hy : hs;
  #pragma unroll
      for (int j = 0; j < kMaxM; j++) {
        if (kFull || j < col) {
          acc[j] = fma(a, hist_at<H, A>(buf, o1 + j * hb, e), acc[j]);
          acc[8 + j] = role == 1 ? fma(hist_at<H, A>(buf, hs + j * hb, e), a, acc[8 + j])
                                 : fma(a, hist_at<H, A>(buf, hy + j * hb, e), acc[8 + j]);
        }
      }
    };
    auto stream_tiles = [&](auto fast) {
    run_stages<CONS>(ss, n, stages, dyn, reinterpret_cast<uint64_t*>(dyn + (size_t)stages * cap),
                     &st->device_error, cp, [&](const unsigned char* buf, long long t, int valid,
                                            auto release) {
      if constexpr (kOneRole) {
        one_role(buf, t, valid, (int)threadIdx.x, fast, release);
        return;
      } else if (role == 0) {
  #pragma unroll
        for (int h = 0; h < kTile / (32 * kRole0Warps); h++)
          role0(buf, t, valid, rt + h * 32 * kRole0Warps);
      } else if (need_row) {
  #pragma unroll
        for (int h = 0; h < kTile / (32 * kRole12Warps); h++)
          rowprod(buf, valid, rt + h * 32 * kRole12Warps);
      }
      release();
    });
    };
    if constexpr (kOneRole) {
      if (kFull && !uncon && track && need_row && !c.hash_free)
        stream_tiles(std::true_type{});
      else
        stream_tiles(std::false_type{});
    } else {
      stream_tiles(std::false_type{});
    }
  });
  // the free-set hash sums mod 2^64 (order free), one atomic per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) hash += __shfl_xor_sync(0xffffffffu, hash, o);
  if (lane == 0 && hash != 0) atomicAdd(&st->free_hash_acc, hash);

  // CTA row: [ role 0: 16 sums + 5 counts | role 1: 16 | role 2: 16 | corrections ];
  // every column is summed over the warps in warp order (fixed)
  constexpr int NS = NA + NB + NC;
  constexpr int W = NS + 32 * kLaneOwned;
  constexpr int kAllWarps = CONS / 32 + 1;
  if (!c.epi_only) {
    __shared__ double wsum[kAllWarps][NS];
    for (int k = lane; k < NS; k += 32) wsum[warp][k] = 0.0;
    __syncwarp();
    const int off = role == 0 ? 0 : role == 1 ? NA : NA + NB;
#pragma unroll
    for (int k = 0; k < 2 * kMaxM; k++) {
      const double v = warp_sum((double)acc[k]);
      if (lane == 0 && role < 3) wsum[warp][off + k] = v;
    }
    if constexpr (kOneRole) {
#pragma unroll
      for (int k = 0; k < 2 * kMaxM; k++) {
        const double v = warp_sum((double)nrow[k]);
        if (lane == 0 && role == 0) wsum[warp][NA + k] = v;
      }
      const int me = role == 0 ? (int)threadIdx.x : 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 a = nra[q * CONS + me];
        const float comp[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const double v = warp_sum(role == 0 ? (double)comp[k] : 0.0);
          if (lane == 0 && role == 0) wsum[warp][NA + NB + 4 * q + k] = v;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const double v = warp_sum((double)cnt[k]);
      if (lane == 0 && role == 0) wsum[warp][2 * kMaxM + k] = v;
    }
    __syncthreads();
    double* row = c.part + cp.rank;  // entry k at row[k * cp.count] (reduce.cuh)
    for (int k = threadIdx.x; k < W; k += CONS + 32) {
      double a = 0.0;
      if (k < NS) {
        for (int w = 0; w < kAllWarps; w++) a += wsum[w][k];
      } else {
        for (int w = 0; w < kRole0Warps; w++) a += corr_sm[w][k - NS];
      }
      row[(size_t)k * cp.count] = a;
    }
  }
  __shared__ double red[W];
  if (!pass_fold<CONS + 32>(c, cp, W, W, 0, 0, red, &st->free_hash_acc)) return;
  __shared__ SmallWork<S> sw;
  __shared__ S wn1_snap[4 * kMaxM * kMaxM];
  epilogue_on_shared_warp<S>(st, [&](DevState<S>* st, int lane) {
    // epilogue: freev's counts and wrk (1143-1161), formk (907-1103), subsm's K solves
    // (1459-1471); lane 0 writes the scalars, the matrix work is shared out over the warp
    if (lane == 0) {
      const int nfree = (int)red[16];
      if (!uncon) {
        st->nfree = nfree;
        st->nenter = (int)red[17];
        st->nleave = (int)red[18];
        st->wrk = (st->nleave > 0 || st->nenter > 0 || updatd) ? 1 : 0;
      } else {
        st->wrk = updatd ? 1 : 0;
        st->nenter = 0;
        st->nleave = 0;
      }
      st->free_hash = st->free_hash_acc;
      st->free_hash_acc = 0;
      st->spec_apply = 0;  // set by the direction pass when it applies an untruncated step
      st->at_lower = (unsigned long long)red[19];
      st->at_upper = (unsigned long long)red[20];
      st->subsm_active = (st->nfree != 0 && col != 0) ? 1 : 0;
    }
    __syncwarp();
    if (!st->subsm_active) return;
    if (st->wrk) {
      FormkSums<S>& fs = sw.fs;
      if (lane < kMaxM) {
        const int j = lane;
        fs.yy_new[j] = (S)red[NA + j];
        fs.sy_col[j] = (S)red[NA + kMaxM + j];
        fs.ss_new[j] = (S)red[NA + NB + j];
        fs.sy_row[j] = (S)red[NA + NB + kMaxM + j];
      }
      for (int q = lane; q < 32 * kLaneOwned; q += 32) {
        int kind, a, b;
        corr_map(q, kind, a, b);
        if (kind >= 3) continue;
        const S v = (S)red[NS + q];
        if (kind == 0) fs.dyy[a][b] = v;
        if (kind == 1) fs.dss[a][b] = v;
        if (kind == 2) fs.dsy[a][b] = v;
      }
      __syncwarp();
      const int info = wformk<S>(st->m, col, st->updatd, st->iupdat, theta, st->sy, st->wn,
                                 st->wn1, fs, sw.wm, wn1_snap, lane);
      if (info != 0) {
        if (lane == 0) st->internal_fail = info;
        return;
      }
    }
    S* wv = sw.wv;
    if (lane < col) {
      const int j = lane + 1;
      wv[j] = (S)red[j - 1];
      wv[col + j] = theta * (S)red[8 + j - 1];
    }
    __syncwarp();
    const int info = wdiag_zero(st->wn, 2 * kMaxM, 2 * col, lane);
    if (info != 0) {
      if (lane == 0) st->internal_fail = info;
      return;
    }
    wdtrsl11(st->wn, 2 * kMaxM, 2 * col, wv, lane);
    if (lane < col) wv[lane + 1] = -wv[lane + 1];
    __syncwarp();
    wdtrsl1(st->wn, 2 * kMaxM, 2 * col, wv, lane);  // the same diagonal: no zero
    if (lane < 2 * col) st->wv[lane + 1] = wv[lane + 1];
  });
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) k_freev_formk(Ctx<R, H, S> c,
    const R* __restrict__ x, const R* __restrict__ g) {
  freev_formk_pass<R, H, S, CONS>(c, cta_here(), c.stages, x, g);
}

// lnsrlb's per-variable start at the subspace point z (lbfgsbcpu.cpp:1263-1299): d = z - x,
// d'd, g'd, and the step along d to the first bound (stpmx), filtered as for stpmx = 1e10;
// candidates that cannot reach the running minimum skip the exact division.
template <typename R, typename A>
__device__ __forceinline__ void lnsrlb_elem(R zi, R xi, R gi, R li, R ui, int nb, bool want_stpmx,
                                            int i, A& dtd, A& gd, ArgMin<R>& mn) {
  const R big = (R)1.0e10;
  const R d = rsub(zi, xi);
  dtd = fma((A)d, (A)d, dtd);
  gd = fma((A)gi, (A)d, gd);
  if (!want_stpmx) return;
  // the two cases as selects (the lanes of a warp take different ones); a variable with
  // neither has no candidate
  const bool lo = nb != 0 && d < R(0) && nb <= 2;
  const bool hi = nb != 0 && !lo && d > R(0) && nb >= 2;
  const R a2 = rsub(lo ? li : ui, xi);
  const R db = rmul(d, big);
  const bool at = lo ? a2 >= R(0) : a2 <= R(0);
  const bool reach = lo ? db < a2 : db > a2;
  if (lo || hi) {
    if (at)
      mn.offer(R(0), i);
    else if (reach)
      mn.offer_quotient(a2, d, i);
  }
}

// lnsrlb with task != 1 (1263-1311), then its first dcsrch call (1312-1338), from
// red[0] d'd, red[1] g'd and red[2] the smallest step to a bound.
template <typename S>
__device__ void lnsrlb_start(DevState<S>* st, const double* red) {
  const S sbig = (S)1.0e10;
  st->dtd = (S)red[0];
  st->dnrm = ssqrt(st->dtd);
  st->stpmx = sbig;
  if (st->cnstnd) {
    if (st->iter == 0)
      st->stpmx = 1;
    else if ((S)red[2] < st->stpmx)
      st->stpmx = (S)red[2];
  }
  if (st->iter == 0 && !st->boxed)
    st->stp = smin((S)1 / st->dnrm, st->stpmx);
  else
    st->stp = 1;
  st->fold = st->f;
  st->ifun = 0;
  st->iback = 0;
  st->csave = 0;
  st->gd = (S)red[1];
  st->gdold = st->gd;
  st->ls_info = 0;
  if (st->gd >= S(0)) {
    st->ls_info = -4;
    return;
  }
  sdcsrch<S>(st->f, st->gd, st->stp, (S)1.0e-3, (S)0.9, (S)0.1, (S)0, st->stpmx, st->csave,
             st->ls);
  st->xstep = st->stp * st->dnrm;
  if (st->csave != 4 && st->csave != 3) {
    st->ls_task = 1;
    st->ifun = st->ifun + 1;
    st->nfgv = st->nfgv + 1;
    st->iback = st->ifun - 1;
  } else {
    st->ls_task = 5;
  }
}

// One variable's inputs to the direction pass, read from the stage into registers.
template <typename R, typename S>
struct DirElem {
  int code, nb;
  R x, g, l, u;
  S yv[kMaxM], sv[kMaxM];
};

// ------------------------------------------------------------------------------------
// C: subspace direction on the free set and the step to the first bound it meets.
template <typename R, typename H, typename S, int CONS>
__device__ __forceinline__ void subsm_dir_pass(const Ctx<R, H, S>& c, CtaPos cp, int stages,
    const R* __restrict__ x,
                                                        const R* __restrict__ g, R* __restrict__ z) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!st->rp_sub) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
    z = c.X[st->xr[1]];
  }
  if (st->gcp_state == GCP_WALK || st->internal_fail != 0 || !st->subsm_active) return;
  const int n = c.epi_only ? 0 : c.n, col = st->col;
  const bool uncon = st->uncon_branch != 0;
  const S theta = st->theta, tsum = st->tsum;
  __shared__ __align__(16) S a1[kMaxM + 1], a2[kMaxM], w1[kMaxM], w2[kMaxM];  // uniform
  if (threadIdx.x < kMaxM) {
    const int j = threadIdx.x;
    a1[j] = (j < col) ? st->mc[1 + j] : S(0);
    a2[j] = (j < col) ? theta * st->mc[col + 1 + j] : S(0);
    w1[j] = (j < col) ? st->wv[1 + j] : S(0);
    w2[j] = (j < col) ? st->wv[col + 1 + j] : S(0);
    if (j == 0) a1[kMaxM] = theta;
  }
  // mb: the step to the first bound (alpha); the speculative lnsrlb start at the
  // untruncated step (alpha = 1): sums d'd, g'd and ms the smallest step to a bound
  ArgMin<S> mb;
  ArgMin<R> ms;
  using A = typename AccOf<S>::type;
  A sl[2] = {A(0), A(0)};
  const bool want_stpmx = st->cnstnd && st->iter > 0;
  // speculate unless the last step was truncated (then this one likely is too); the 3.0
  // step always needs the projected point
  const bool proj = st->subsm_proj != 0;
  const bool spec = proj || st->dir_no_spec == 0;
  __shared__ int s_projected;  // 1 once the 3.0 projection has put a variable on a bound
  const FixedDiv<S> divt(theta);

  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ StreamSet ss;
  __shared__ int s_hy, s_hs;
  if (threadIdx.x == 0) {
    s_projected = 0;
    ss.count = 0;
    ss.stage_bytes = 0;
    add_stream(ss, c.code, kTile);
    add_stream(ss, x, kTile * (int)sizeof(R));
    add_stream(ss, g, kTile * (int)sizeof(R));
    add_stream(ss, c.l, kTile * (int)sizeof(R));
    add_stream(ss, c.u, kTile * (int)sizeof(R));
    add_stream(ss, c.nbd, kTile * 4);
    add_history(ss, c, st, s_hy, s_hs);
  }
  __syncthreads();
  const int o_code = ss.off[0], o_x = ss.off[1], o_g = ss.off[2], o_l = ss.off[3];
  const int o_u = ss.off[4], o_nb = ss.off[5];
  const int hy = s_hy, hs = s_hs, hb = kTile * (int)sizeof(H);
  const int cap = stage_capacity(StageBytes<R>::dir, 0, st->m, (int)sizeof(H));
  dispatch_cols(col, [&](auto cols_tag) {
    constexpr bool kFull = decltype(cols_tag)::value == kMaxM;
    // each thread reads its variable's inputs and history row into registers and the stage
    // is released before the arithmetic, so that the producer refills it sooner
    run_tiles_split<CONS>(ss, n, stages, dyn, reinterpret_cast<uint64_t*>(dyn + (size_t)stages * cap),
              &st->device_error, cp, [&](const unsigned char* buf, long long t, int valid, int e) {
      DirElem<R, S> v{};
      if (e < valid) {
        v.code = stage_at<int8_t>(buf, o_code, e);
        v.x = stage_at<R>(buf, o_x, e);
        v.g = stage_at<R>(buf, o_g, e);
        v.l = stage_at<R>(buf, o_l, e);
        v.u = stage_at<R>(buf, o_u, e);
        v.nb = stage_at<int>(buf, o_nb, e);
        if (uncon || iw_free(v.code)) {
  #pragma unroll
          for (int j = 0; j < kMaxM; j++) {
            v.yv[j] = (kFull || j < col) ? hist_at<H, S>(buf, hy + j * hb, e) : S(0);
            v.sv[j] = (kFull || j < col) ? hist_at<H, S>(buf, hs + j * hb, e) : S(0);
          }
        }
      }
      return v;
    }, [&](const DirElem<R, S>& v, long long t, int valid, int e) {
      if (e >= valid) return;
      const int i = (int)(t * kTile) + e;
      const int code = v.code;
      if (!(uncon || iw_free(code))) {
        if (!spec) return;
        // an active variable: z is its Cauchy point
        const R zi = gcp_point<R, S>(code, v.x, v.g, v.l, v.u, tsum);
        z[i] = zi;
        lnsrlb_elem<R, A>(zi, v.x, v.g, v.l, v.u, v.nb, want_stpmx, i + c.ioff, sl[0], sl[1], ms);
        return;
      }
      const S(&yv)[kMaxM] = v.yv;
      const S(&sv)[kMaxM] = v.sv;
      const R xi = v.x, gi = v.g, li = v.l, ui = v.u;
      const R zi = uncon ? xi : gcp_point<R, S>(code, xi, gi, li, ui, tsum);
      S d;
      if constexpr (sizeof(S) == 4) {
        // The FP32 form: r, then d = (r + sum_j wy_j wv_j / theta + ws_j wv_j) / theta
        // (1472-1483) with fused multiply-adds and the reciprocal of theta, one rounding
        // more per quotient than the division (the form is held to the FP32 tolerance)
        const S rth = divt.y;
        d = uncon ? -(S)gi : -a1[kMaxM] * ((S)zi - (S)xi) - (S)gi;
        if (!uncon) {
  #pragma unroll
          for (int j = 0; j < kMaxM; j++)
            if (kFull || j < col) d = fmaf(sv[j], a2[j], fmaf(yv[j], a1[j], d));
        }
  #pragma unroll
        for (int j = 0; j < kMaxM; j++)
          if (kFull || j < col) d = fmaf(sv[j], w2[j], fmaf(yv[j] * w1[j], rth, d));
        d = d * rth;
      } else {
        d = reduced_grad<R, S>(uncon, xi, zi, gi, kFull ? kMaxM : col, yv, sv, a1, a2);
        // ... + wy*wv(jy)/theta + ws*wv(js), then d/theta (1472-1483): the divisions by
        // the pass-constant theta use its reciprocal with Markstein's correction (FixedDiv),
        // which rounds exactly like the division; the quotients do not depend on d: they are
        // formed side by side without branches, the rare out-of-range ones redone with the
        // full division, then summed in order
        S q[kMaxM];
        bool ok = true;
  #pragma unroll
        for (int j = 0; j < kMaxM; j++) {
          if (kFull || j < col) {
            const S a = yv[j] * w1[j];
            q[j] = divt.markstein(a);
            ok = ok && divt.in_range(a);
          }
        }
        if (!ok) {
  #pragma unroll
          for (int j = 0; j < kMaxM; j++) {
            if (kFull || j < col) {
              const S a = yv[j] * w1[j];
              if (!divt.in_range(a)) q[j] = divt.full(a);
            }
          }
        }
  #pragma unroll
        for (int j = 0; j < kMaxM; j++)
          if (kFull || j < col) d = d + q[j] + sv[j] * w2[j];
        d = divt(d);
      }
      const R dr = (R)d;
      c.dsub[i] = dr;
      // candidate step to the bound (1486-1516), filtered as for alpha = 1; the two cases
      // as selects
      const int nb = v.nb;
      const S dk = (S)dr;
      {
        const bool lo = nb != 0 && dk < S(0) && nb <= 2;
        const bool hi = nb != 0 && !lo && dk > S(0) && nb >= 2;
        const S temp2 = (S)(lo ? li : ui) - (S)zi;
        const S dk1 = dk * S(1);
        const bool at = lo ? temp2 >= S(0) : temp2 <= S(0);
        const bool reach = lo ? dk1 < temp2 : dk1 > temp2;
        if (lo || hi) {
          if (at)
            mb.offer(S(0), i + c.ioff);
          else if (reach && !quotient_exceeds(temp2, dk, mb.thr))
            mb.offer(temp2 / dk, i + c.ioff);
        }
      }
      // the subspace step with alpha = 1 (1517-1533): z = xcp + d; with the 3.0 step,
      // projected onto the box (the lower bound, then the upper one)
      if (spec) {
        R zs = (R)((S)zi + dk);
        if (proj) {
          const bool lo = nb == 1 || nb == 2, hi = nb == 2 || nb == 3;
          if (lo) zs = li > zs ? li : zs;
          if (hi) zs = ui > zs ? zs : ui;
          if ((lo && zs == li) || (hi && zs == ui)) s_projected = 1;
        }
        z[i] = zs;
        lnsrlb_elem<R, A>(zs, xi, gi, li, ui, nb, want_stpmx, i + c.ioff, sl[0], sl[1], ms);
      }
    });
  });
  // row: [ d'd, g'd | projected | alpha candidate (value, index) | stpmx candidate
  // (value, index) ]
  constexpr int W = 7;
  // (the pipeline ends with a block barrier, so every thread's flag store is visible)
  double xm[1] = {s_projected ? 1.0 : 0.0}, ldum[1] = {0.0}, sld[2];
  MinPair mn[2] = {mb.pair(), ms.pair()};
  sums_to_double(sl, sld);
  if (!c.epi_only) cta_reduce_to_row<CONS + 32, 2, 1, 2, 0>(sld, xm, mn, ldum, c.part, W, cp.rank, cp.count);
  __shared__ double red[W];
  __shared__ double rl[3];
  if (!pass_fold<CONS + 32>(c, cp, W, 2, 1, 2, red)) return;
  epilogue_on_shared<S>(st, [&](DevState<S>* st) {
    // the 3.0 step keeps the projected point when it gives a descent direction from x
    // (g'd <= 0 over the written z); otherwise, and always with the 2.1 step, the step is
    // truncated at the first bound when one is met before alpha = 1
    const bool keep_projection = proj && red[2] > 0.0 && red[1] <= 0.0;
    const S cand = (S)red[3];
    if (!keep_projection && cand < S(1)) {
      st->alpha = cand;
      st->ibd = (int)red[4];
      st->iword = 1;
      st->dir_no_spec = proj ? 0 : 1;
      return;  // truncated: k_subsm_apply applies the step
    }
    st->alpha = 1;
    st->ibd = -1;
    st->iword = keep_projection ? 1 : 0;
    st->dir_no_spec = 0;
    if (!spec) return;  // k_subsm_apply applies the step
    // the step written above is the subspace point; start the line search
    rl[0] = red[0];
    rl[1] = red[1];
    rl[2] = red[5];
    lnsrlb_start<S>(st, rl);
    st->spec_apply = 1;
  });
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) k_subsm_dir(Ctx<R, H, S> c,
    const R* __restrict__ x, const R* __restrict__ g, R* __restrict__ z) {
  subsm_dir_pass<R, H, S, CONS>(c, cta_here(), c.stages, x, g, z);
}

// ------------------------------------------------------------------------------------
// D: apply the subspace step, form z and d = z - x, and start the line search.
template <typename R, typename H, typename S, int CONS>
__device__ __forceinline__ void subsm_apply_pass(const Ctx<R, H, S>& c, CtaPos cp, int stages,
    const R* __restrict__ x,
                                                          const R* __restrict__ g, R* __restrict__ z) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!st->rp_sub) return;
    x = c.X[st->xr[0]];
    g = c.G[st->gr[0]];
    z = c.X[st->xr[1]];
  }
  if (st->gcp_state == GCP_WALK || st->internal_fail != 0 || st->spec_apply) return;
  const int n = c.epi_only ? 0 : c.n;
  const bool uncon = st->uncon_branch != 0;
  const bool sub = st->subsm_active != 0;
  const S alpha = sub ? st->alpha : S(1), tsum = st->tsum;
  const long long ibd = sub ? st->ibd : -1;
  const bool want_stpmx = st->cnstnd && st->iter > 0;
  using A = typename AccOf<S>::type;
  A s[2] = {A(0), A(0)};
  ArgMin<R> ms;

  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ StreamSet ss;
  if (threadIdx.x == 0) {
    ss.count = 0;
    ss.stage_bytes = 0;
    add_stream(ss, c.code, kTile);
    add_stream(ss, x, kTile * (int)sizeof(R));
    add_stream(ss, g, kTile * (int)sizeof(R));
    add_stream(ss, c.l, kTile * (int)sizeof(R));
    add_stream(ss, c.u, kTile * (int)sizeof(R));
    add_stream(ss, c.dsub, kTile * (int)sizeof(R));
    add_stream(ss, c.nbd, kTile * 4);
  }
  __syncthreads();
  const int o_code = ss.off[0], o_x = ss.off[1], o_g = ss.off[2], o_l = ss.off[3];
  const int o_u = ss.off[4], o_ds = ss.off[5], o_nb = ss.off[6];
  const int cap = stage_capacity(StageBytes<R>::apply, 0, 0, (int)sizeof(H));
  run_tiles<CONS>(ss, n, stages, dyn, reinterpret_cast<uint64_t*>(dyn + (size_t)stages * cap),
            &st->device_error, cp, [&](const unsigned char* buf, long long t, int valid, int e) {
    if (e >= valid) return;
    const int i = (int)(t * kTile) + e;
    const R xi = stage_at<R>(buf, o_x, e), gi = stage_at<R>(buf, o_g, e);
    const R li = stage_at<R>(buf, o_l, e), ui = stage_at<R>(buf, o_u, e);
    const int code = stage_at<int8_t>(buf, o_code, e);
    R zi = uncon ? xi : gcp_point<R, S>(code, xi, gi, li, ui, tsum);
    if (sub && (uncon || iw_free(code))) {
      S dk = (S)stage_at<R>(buf, o_ds, e);
      if (i + c.ioff == ibd) {
        if (dk > S(0)) {
          zi = ui;
          dk = 0;
        } else if (dk < S(0)) {
          zi = li;
          dk = 0;
        }
      }
      zi = (R)((S)zi + alpha * dk);
    }
    z[i] = zi;
    lnsrlb_elem<R, A>(zi, xi, gi, li, ui, want_stpmx ? stage_at<int>(buf, o_nb, e) : 0, want_stpmx,
                      i + c.ioff, s[0], s[1], ms);
  });
  constexpr int W = 4;
  double xdum[1] = {0.0}, ldum[1] = {0.0}, sd[2];
  MinPair mn[1] = {ms.pair()};
  sums_to_double(s, sd);
  if (!c.epi_only) cta_reduce_to_row<CONS + 32, 2, 0, 1, 0>(sd, xdum, mn, ldum, c.part, W, cp.rank, cp.count);
  __shared__ double red[W];
  if (!pass_fold<CONS + 32>(c, cp, W, 2, 0, 1, red)) return;
  epilogue_on_shared<S>(st, [&](DevState<S>* st) {

    lnsrlb_start<S>(st, red);
  });
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) k_subsm_apply(Ctx<R, H, S> c,
    const R* __restrict__ x, const R* __restrict__ g, R* __restrict__ z) {
  subsm_apply_pass<R, H, S, CONS>(c, cta_here(), c.stages, x, g, z);
}

// Trial point x = stp*d + t with d = z - t (lbfgsbcpu.cpp:1332-1334).
template <typename R, typename S>
__device__ __forceinline__ void trial_point(int n, const R* __restrict__ t, const R* __restrict__ z,
                                            R* __restrict__ xt, const DevState<S>* st, CtaPos cp) {
  const R stp = (R)st->stp;
  for (long long i = (long long)cp.rank * blockDim.x + threadIdx.x; i < n;
       i += (long long)cp.count * blockDim.x) {
    const R ti = t[i];
    const R d = rsub(z[i], ti);
    xt[i] = radd(rmul(stp, d), ti);
  }
}
template <typename R, typename S>
__global__ void k_trial(int n, const R* __restrict__ t, const R* __restrict__ z, R* __restrict__ xt,
                        const DevState<S>* st) {
  trial_point<R, S>(n, t, z, xt, st, cta_here());
}
// The trial point of a device-driven round, when the round evaluates at stp != 1.
template <typename R, typename H, typename S>
__device__ __forceinline__ void trial_round_pass(const Ctx<R, H, S>& c, CtaPos cp) {
  const DevState<S>* st = c.st;
  if (!st->ev_trial) return;
  trial_point<R, S>(c.n, c.X[st->xr[0]], c.X[st->xr[1]], c.X[st->xr[2]], st, cp);
}
template <typename R, typename H, typename S>
__global__ void k_trial_round(Ctx<R, H, S> c) {
  trial_round_pass<R, H, S>(c, cta_here());
}

// The epilogue after a function evaluation: g'd and dcsrch (lbfgsbcpu.cpp:1312-1338); on
// acceptance the stopping-test quantities (394-417) and matupd/formt (431-461, 1105-1133),
// committing the spare slot that holds (s, y) to the ring.  red[0] g'd, red[1] |xold-x|^2,
// red[2] y'y, red[3..10] s'y_j and red[11..18] s_j's by old ring position, red[19] the
// projected-gradient norm.  post_scalar runs on one lane and returns 0 while the line
// search goes on, 1 when the step is accepted without an update, 2 when formt is due;
// post_epilogue is run by the 32 lanes of a warp and returns false while the line search
// goes on.
template <typename S>
__device__ int post_scalar(DevState<S>* st, const double* red, S f, int force_accept) {
  st->f = f;
  st->gd = (S)red[0];
  if (!force_accept) {
    // lnsrlb with task == 1 (1312-1338)
    sdcsrch<S>(f, st->gd, st->stp, (S)1.0e-3, (S)0.9, (S)0.1, (S)0, st->stpmx, st->csave,
               st->ls);
    st->xstep = st->stp * st->dnrm;
    if (st->csave != 4 && st->csave != 3) {
      st->ls_task = 1;
      st->ifun = st->ifun + 1;
      st->nfgv = st->nfgv + 1;
      st->iback = st->ifun - 1;
      return 0;
    }
    st->ls_task = 5;
  }
  // accepted: quantities of the stopping tests (394-417)
  st->iter = st->iter + 1;
  st->sbgnrm = (S)red[19];
  st->tf = ssqrt((S)red[1]);
  st->rr = (S)red[2];
  // the update (431-461), carried out ahead of the host-side tests; if a test stops the
  // solve the updated memory is simply discarded
  S dr, ddum;
  const S sstp = st->stp;
  if (sstp == S(1)) {
    dr = st->gd - st->gdold;
    ddum = -st->gdold;
  } else {
    dr = (st->gd - st->gdold) * sstp;
    ddum = -st->gdold * sstp;
  }
  st->dr = dr;
  st->ddum_dr = ddum;
  st->internal_fail = 0;
  if ((double)dr <= 5e-16 * (double)ddum) {
    st->updatd = 0;
    return 1;
  }
  st->updatd = 1;
  st->iupdat = st->iupdat + 1;
  const int m = st->m;
  int shifted = 0;
  if (st->iupdat <= m) {
    st->col = st->iupdat;
    st->itail = (st->head + st->iupdat - 2) % m + 1;
  } else {
    st->itail = st->itail % m + 1;
    st->head = st->head % m + 1;
    shifted = 1;
  }
  const int old = st->phys[st->itail];
  st->phys[st->itail] = st->spare;
  st->spare = old;
  st->theta = st->rr / dr;
  const int ncol = st->col;
  constexpr int ld = kMaxM;
  if (st->iupdat > m) {
    #pragma unroll 1
    for (int j = 1; j <= ncol - 1; j++) {
      #pragma unroll 1
      for (int i = 1; i <= j; i++) LB_AT(st->ss, ld, i, j) = LB_AT(st->ss, ld, i + 1, j + 1);
      #pragma unroll 1
      for (int i = j; i <= ncol - 1; i++) LB_AT(st->sy, ld, i, j) = LB_AT(st->sy, ld, i + 1, j + 1);
    }
  }
  #pragma unroll 1
  for (int j = 1; j <= ncol - 1; j++) {
    LB_AT(st->sy, ld, ncol, j) = (S)red[3 + j - 1 + shifted];
    LB_AT(st->ss, ld, j, ncol) = (S)red[11 + j - 1 + shifted];
  }
  LB_AT(st->ss, ld, ncol, ncol) = (sstp == S(1)) ? st->dtd : sstp * sstp * st->dtd;
  LB_AT(st->sy, ld, ncol, ncol) = dr;
  return 2;
}
template <typename S>
__device__ bool post_epilogue(DevState<S>* st, const double* red, S f, int force_accept,
                              int lane) {
  int r = 0;
  if (lane == 0) r = post_scalar<S>(st, red, f, force_accept);
  r = __shfl_sync(kFullMask, r, 0);
  __syncwarp();
  if (r == 2) {
    const int info = wformt<S>(st->wt, st->sy, st->ss, st->col, st->theta, lane);
    if (lane == 0 && info != 0) st->internal_fail = info;
    __syncwarp();
  }
  return r != 0;
}

// ------------------------------------------------------------------------------------
// E: after a function evaluation at xt (gradient gt; t and go are the point and the
// gradient where the line search started).
template <typename R, typename H, typename S, int CONS>
__device__ __forceinline__ void post_eval_pass(const Ctx<R, H, S>& c, CtaPos cp, int stages,
    const R* __restrict__ t,
                                                        const R* __restrict__ z,
                                                        const R* __restrict__ xt,
                                                        const R* __restrict__ gt,
                                                        const R* __restrict__ go, S f,
                                                        int force_accept) {
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!(st->ev_active || st->ev_force)) return;
    t = c.X[st->xr[0]];
    z = c.X[st->xr[1]];
    xt = st->ev_is_z ? z : c.X[st->xr[2]];
    gt = c.G[st->gr[1]];
    go = c.G[st->gr[0]];
    force_accept = st->ev_force;
    f = st->ev_force ? st->f : (S)(R)*c.ev_f;
  }
  const int n = c.epi_only ? 0 : c.n, col = st->col;
  const R stp = (R)st->stp;
  const bool unit = st->stp == S(1);
  H* ysp = c.wy + (size_t)st->spare * (size_t)c.ld;
  H* ssp = c.ws + (size_t)st->spare * (size_t)c.ld;
  // sums: [0] g'd, [1] |xold - x|^2, [2] y'y, [3..10] s'y_j, [11..18] s_j's; max: |proj g|
  constexpr int NS = 19, NX = 1;
  using A = typename AccOf<S>::type;
  A s[NS], xa = A(0);
#pragma unroll
  for (int k = 0; k < NS; k++) s[k] = A(0);

  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ StreamSet ss;
  __shared__ int s_hy, s_hs;
  const bool xt_is_z = xt == z;
  if (threadIdx.x == 0) {
    ss.count = 0;
    ss.stage_bytes = 0;
    add_stream(ss, t, kTile * (int)sizeof(R));
    add_stream(ss, z, kTile * (int)sizeof(R));
    add_stream(ss, gt, kTile * (int)sizeof(R));
    add_stream(ss, go, kTile * (int)sizeof(R));
    add_stream(ss, c.l, kTile * (int)sizeof(R));
    add_stream(ss, c.u, kTile * (int)sizeof(R));
    add_stream(ss, c.nbd, kTile * 4);
    if (!xt_is_z) add_stream(ss, xt, kTile * (int)sizeof(R));
    add_history(ss, c, st, s_hy, s_hs);
  }
  __syncthreads();
  const int o_t = ss.off[0], o_z = ss.off[1], o_g = ss.off[2], o_go = ss.off[3];
  const int o_l = ss.off[4], o_u = ss.off[5], o_nb = ss.off[6];
  const int o_xt = xt_is_z ? o_z : ss.off[7];
  const int hy = s_hy, hs = s_hs, hb = kTile * (int)sizeof(H);
  const int cap = stage_capacity(StageBytes<R>::post, 0, st->m, (int)sizeof(H));
  dispatch_cols(col, [&](auto cols_tag) {
    constexpr bool kFull = decltype(cols_tag)::value == kMaxM;
    run_tiles<CONS>(ss, n, stages, dyn, reinterpret_cast<uint64_t*>(dyn + (size_t)stages * cap),
              &st->device_error, cp, [&](const unsigned char* buf, long long tt, int valid, int e) {
      if (e >= valid) return;
      const int i = (int)(tt * kTile) + e;
      const R ti = stage_at<R>(buf, o_t, e), zi = stage_at<R>(buf, o_z, e);
      const R xi = stage_at<R>(buf, o_xt, e), gi = stage_at<R>(buf, o_g, e);
      const R gold = stage_at<R>(buf, o_go, e);
      const R d = rsub(zi, ti);
      s[0] = fma((A)gi, (A)d, s[0]);
      // projgr (1389-1414), its cases as selects
      const int nb = stage_at<int>(buf, o_nb, e);
      const bool neg = gi < R(0);
      const R tb = rsub(xi, stage_at<R>(buf, neg ? o_u : o_l, e));
      const bool clip = nb != 0 && (neg ? nb >= 2 : nb <= 2);
      const R pg = clip ? (neg ? smax<R>(tb, gi) : smin<R>(tb, gi)) : gi;
      const A apg = fabs((A)pg);
      xa = (apg > xa) ? apg : xa;
      const R xd = rsub(ti, xi);
      s[1] = fma((A)xd, (A)xd, s[1]);
      const R y = rsub(gi, gold);
      s[2] = fma((A)y, (A)y, s[2]);
      const R sv = unit ? d : rmul(d, stp);
  #pragma unroll
      for (int j = 0; j < kMaxM; j++) {
        if (kFull || j < col) {
          s[3 + j] = fma((A)sv, hist_at<H, A>(buf, hy + j * hb, e), s[3 + j]);
          s[11 + j] = fma(hist_at<H, A>(buf, hs + j * hb, e), (A)sv, s[11 + j]);
        }
      }
      ssp[i] = HistTraits<H>::from(sv);
      ysp[i] = HistTraits<H>::from(y);
    });
  });
  constexpr int W = NS + NX;
  MinPair mdum[1] = {MinPair{0.0, 0}};
  double ldum[1] = {0.0}, sd[NS], xm[NX] = {(double)xa};
  sums_to_double(s, sd);
  if (!c.epi_only) cta_reduce_to_row<CONS + 32, NS, NX, 0, 0>(sd, xm, mdum, ldum, c.part, W, cp.rank, cp.count);
  __shared__ double red[W];
  if (!pass_fold<CONS + 32>(c, cp, W, NS, NX, 0, red)) return;
  epilogue_on_shared_warp<S>(st, [&](DevState<S>* st, int lane) {
    post_epilogue<S>(st, red, f, force_accept, lane);
  });
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) k_post_eval(Ctx<R, H, S> c,
    const R* __restrict__ t, const R* __restrict__ z, const R* __restrict__ xt,
    const R* __restrict__ gt, const R* __restrict__ go, S f, int force_accept) {
  post_eval_pass<R, H, S, CONS>(c, cta_here(), c.stages, t, z, xt, gt, go, f, force_accept);
}

// ------------------------------------------------------------------------------------
// Set-up: errclb (871-905), lbfgsbactive (467-515) into the solver's x buffer.
template <typename R, typename S>
__device__ __forceinline__ void init_pass(int n, const R* __restrict__ x_in, R* __restrict__ x,
                                          const int* __restrict__ nbd, const R* __restrict__ l,
                                          const R* __restrict__ u, DevState<S>* st, CtaPos cp) {
  int err = 0, any_c = 0, not_boxed = 0;
  for (long long i = (long long)cp.rank * blockDim.x + threadIdx.x; i < n;
       i += (long long)cp.count * blockDim.x) {
    const int nb = nbd[i];
    const R li = l[i], ui = u[i];
    R xi = x_in[i];
    if (nb < 0 || nb > 3) err |= 1;
    if (nb == 2 && li > ui) err |= 2;
    if (nb > 0) {
      if (nb <= 2 && xi <= li) {
        if (xi < li) xi = li;
      } else if (nb >= 2 && xi >= ui) {
        if (xi > ui) xi = ui;
      }
    }
    x[i] = xi;
    if (nb != 2) not_boxed = 1;
    if (nb != 0) any_c = 1;
  }
  err = __reduce_or_sync(0xffffffffu, err);
  any_c = __reduce_or_sync(0xffffffffu, any_c);
  not_boxed = __reduce_or_sync(0xffffffffu, not_boxed);
  if ((threadIdx.x & 31) == 0) {
    if (err) atomicOr(&st->input_error, err);
    if (any_c) atomicOr(&st->cnstnd, 1);
    if (not_boxed) atomicAnd(&st->boxed, 0);
  }
}
template <typename R, typename S>
__global__ void k_init(int n, const R* __restrict__ x_in, R* __restrict__ x, const int* __restrict__ nbd,
                       const R* __restrict__ l, const R* __restrict__ u, DevState<S>* st) {
  init_pass<R, S>(n, x_in, x, nbd, l, u, st, cta_here());
}

// projgr at the start point (lbfgsbcpu.cpp:272-273); also records f.
template <typename R, typename H, typename S>
__device__ __forceinline__ void projgr_pass(const Ctx<R, H, S>& c, CtaPos cp, const R* __restrict__ x,
                                            const R* __restrict__ g, S f) {
  if (c.rounds) {
    x = c.X[c.st->xr[0]];
    g = c.G[c.st->gr[0]];
    f = (S)(R)*c.ev_f;
  }
  double xm[1] = {0.0};
  const int n = c.epi_only ? 0 : c.n;
  for (long long i = (long long)cp.rank * kThreads + threadIdx.x; i < n;
       i += (long long)cp.count * kThreads) {
    const R xi = x[i], gi = g[i];
    const int nb = c.nbd[i];
    R pg = gi;
    if (nb != 0) {
      if (gi < R(0)) {
        if (nb >= 2) pg = smax<R>(rsub(xi, c.u[i]), gi);
      } else {
        if (nb <= 2) pg = smin<R>(rsub(xi, c.l[i]), gi);
      }
    }
    const double a = fabs((double)pg);
    xm[0] = (a > xm[0]) ? a : xm[0];
  }
  double sdum[1] = {0.0}, ldum[1] = {0.0};
  MinPair mdum[1] = {MinPair{0.0, 0}};
  if (!c.epi_only) cta_reduce_to_row<kThreads, 0, 1, 0, 0>(sdum, xm, mdum, ldum, c.part, 1, cp.rank, cp.count);
  __shared__ double red[1];
  if (!pass_fold<kThreads>(c, cp, 1, 0, 1, 0, red)) return;
  if (threadIdx.x != 0) return;
  c.st->sbgnrm = (S)red[0];
  c.st->f = f;
  c.st->res_g = (S)red[0];
}
template <typename R, typename H, typename S>
__global__ void __launch_bounds__(kThreads) k_projgr(Ctx<R, H, S> c, const R* __restrict__ x,
                                                     const R* __restrict__ g, S f) {
  projgr_pass<R, H, S>(c, cta_here(), x, g, f);
}

// The memory reset of the reference driver (col = 0, head = 1, theta = 1, iupdat = 0,
// updatd = false), and the branch flags of the next iteration.
template <typename S>
__device__ __forceinline__ void begin_state(DevState<S>* st, int reset) {
  if (reset) {
    st->col = 0;
    st->head = 1;
    st->theta = 1;
    st->iupdat = 0;
    st->updatd = 0;
  }
  st->internal_fail = 0;
  st->uncon_branch = (!st->cnstnd && st->col > 0) ? 1 : 0;
  st->subsm_active = 0;
  st->iword = -1;
  st->free_hash = 0;
  st->ls_info = 0;
  if (st->uncon_branch) {
    // z = x, wrk = updatd, nint = 0 (lbfgsbcpu.cpp:281-284)
    st->gcp_state = GCP_SKIPPED;
    st->tsum = 0;
    st->nint = 0;
  }
}

template <typename S>
__global__ void k_begin_iteration(DevState<S>* st, int reset) {
  begin_state(st, reset);
}


// The value a history element holds once stored (the history precision H), as a double.
template <typename H, typename A, typename R>
__device__ __forceinline__ A stored_value(R v) {
  const H h = HistTraits<H>::from(v);
  if constexpr (sizeof(H) == 2) {
    return (A)__bfloat162float(h);
  } else {
    return (A)h;
  }
}

// ------------------------------------------------------------------------------------
// E+A: the post-evaluation pass fused with the next iteration's Cauchy-point scan, for
// problems with bounds.  Two warp roles cover every tile:
//   role P (consumer warps 0..7): k_post_eval's per-variable work (g'd, projgr, |dx|, y,
//     the S'y / S's sums, the (s, y) write);
//   role G (warps 8..15): cauchy's scan at the trial point xt with its gradient gt, as the
//     next iteration will need it if the line search accepts xt: iwhere codes, breakpoints,
//     and p = W'd summed over the old ring positions and over the new pair (s, y) in its
//     stored precision, so that the epilogue can form p for whichever ring the update
//     produces.
// The epilogue runs the post-evaluation epilogue; when the step is accepted and the memory
// update succeeded it starts the next iteration (the reference's loop top, 279-284) and
// runs cauchy's epilogue on the reordered sums, and marks spec_gcp so that the host skips
// the separate scan.  A rejected trial leaves codes that the next trial overwrites.
template <typename R, typename H, typename S, int CONS>
__device__ __forceinline__ void post_gcp_pass(const Ctx<R, H, S>& c, CtaPos cp, int stages,
    const R* __restrict__ t,
                                                       const R* __restrict__ z,
                                                       const R* __restrict__ xt,
                                                       const R* __restrict__ gt,
                                                       const R* __restrict__ go, S f,
                                                       int force_accept) {
  static_assert(CONS == 512, "the role split assumes 16 consumer warps");
  DevState<S>* st = c.st;
  if (c.rounds) {
    if (!(st->ev_active || st->ev_force)) return;
    t = c.X[st->xr[0]];
    z = c.X[st->xr[1]];
    xt = st->ev_is_z ? z : c.X[st->xr[2]];
    gt = c.G[st->gr[1]];
    go = c.G[st->gr[0]];
    force_accept = st->ev_force;
    f = st->ev_force ? st->f : (S)(R)*c.ev_f;
  }
  const int n = c.epi_only ? 0 : c.n, col = st->col;
  const R stp = (R)st->stp;
  const bool unit = st->stp == S(1);
  H* ysp = c.wy + (size_t)st->spare * (size_t)c.ld;
  H* ssp = c.ws + (size_t)st->spare * (size_t)c.ld;
  // With float sums (the FP32 plain form) one role does both (kOneRole): every consumer
  // thread runs role P and role G on one element per tile, reading the element's inputs
  // and history values from the stage once.
  using A = typename AccOf<S>::type;
  constexpr bool kOneRole = sizeof(A) == 4;
  static_assert(!kOneRole || CONS == kTile, "one element per consumer thread and tile");
  constexpr int kRoleWarps = kOneRole ? CONS / 32 : 8, kRoleThreads = 32 * kRoleWarps;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int role = warp < kRoleWarps ? 0 : (!kOneRole && warp < 2 * kRoleWarps) ? 1 : 2;  // 2: producer
  const int rt = (int)threadIdx.x - (role == 1 ? kRoleThreads : 0);
  // role P: acc[0] g'd, [1] |xold - x|^2, [2] y'y, [3..10] s'y_j, [11..18] s_j's;
  //   xmx |proj g|.
  // role G: acc[0] sum g^2 (movable), [1..8] / [9..16] y_j'(-g) / s_j'(-g) by old ring
  //   position, [17] / [18] y'(-g) / s'(-g) of the new pair, [19] nbreak, [20] movable
  //   without breakpoint; xmx: any of those with g != 0; mn: smallest breakpoint.
  //   kOneRole: role G's sums in accg, its xmx in xmxg.
  constexpr int NP = 19, NG = 21;
  A acc[NG];
#pragma unroll
  for (int k = 0; k < NG; k++) acc[k] = A(0);
  A accg[kOneRole ? NG : 1];
#pragma unroll
  for (int k = 0; k < (kOneRole ? NG : 1); k++) accg[k] = A(0);
  A xmx = A(0), xmxg = A(0);
  ArgMin<R> bp;  // role G: the smallest breakpoint

  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ StreamSet ss;
  __shared__ int s_hy, s_hs;
  const bool xt_is_z = xt == z;
  if (threadIdx.x == 0) {
    ss.count = 0;
    ss.stage_bytes = 0;
    add_stream(ss, t, kTile * (int)sizeof(R));
    add_stream(ss, z, kTile * (int)sizeof(R));
    add_stream(ss, gt, kTile * (int)sizeof(R));
    add_stream(ss, go, kTile * (int)sizeof(R));
    add_stream(ss, c.l, kTile * (int)sizeof(R));
    add_stream(ss, c.u, kTile * (int)sizeof(R));
    add_stream(ss, c.nbd, kTile * 4);
    if (!xt_is_z) add_stream(ss, xt, kTile * (int)sizeof(R));
    add_history(ss, c, st, s_hy, s_hs);
  }
  __syncthreads();
  const int o_t = ss.off[0], o_z = ss.off[1], o_g = ss.off[2], o_go = ss.off[3];
  const int o_l = ss.off[4], o_u = ss.off[5], o_nb = ss.off[6];
  const int o_xt = xt_is_z ? o_z : ss.off[7];
  const int hy = s_hy, hs = s_hs, hb = kTile * (int)sizeof(H);
  const int cap = stage_capacity(StageBytes<R>::post, 0, st->m, (int)sizeof(H));
  dispatch_cols(col, [&](auto cols_tag) {
    constexpr bool kFull = decltype(cols_tag)::value == kMaxM;
    auto post_elem = [&](const unsigned char* buf, long long tt, int valid, int e) {
      if (e >= valid) return;
      const int i = (int)(tt * kTile) + e;
      const R ti = stage_at<R>(buf, o_t, e), zi = stage_at<R>(buf, o_z, e);
      const R xi = stage_at<R>(buf, o_xt, e), gi = stage_at<R>(buf, o_g, e);
      const R gold = stage_at<R>(buf, o_go, e);
      const R d = rsub(zi, ti);
      acc[0] = fma((A)gi, (A)d, acc[0]);
      // projgr (1389-1414), its cases as selects
      const int nb = stage_at<int>(buf, o_nb, e);
      const bool neg = gi < R(0);
      const R tb = rsub(xi, stage_at<R>(buf, neg ? o_u : o_l, e));
      const bool clip = nb != 0 && (neg ? nb >= 2 : nb <= 2);
      const R pg = clip ? (neg ? smax<R>(tb, gi) : smin<R>(tb, gi)) : gi;
      const A apg = fabs((A)pg);
      xmx = (apg > xmx) ? apg : xmx;
      const R xd = rsub(ti, xi);
      acc[1] = fma((A)xd, (A)xd, acc[1]);
      const R y = rsub(gi, gold);
      acc[2] = fma((A)y, (A)y, acc[2]);
      const R sv = unit ? d : rmul(d, stp);
#pragma unroll
      for (int j = 0; j < kMaxM; j++) {
        if (kFull || j < col) {
          acc[3 + j] = fma((A)sv, hist_at<H, A>(buf, hy + j * hb, e), acc[3 + j]);
          acc[11 + j] = fma(hist_at<H, A>(buf, hs + j * hb, e), (A)sv, acc[11 + j]);
        }
      }
      ssp[i] = HistTraits<H>::from(sv);
      ysp[i] = HistTraits<H>::from(y);
    };
    auto gcp_elem = [&](const unsigned char* buf, long long tt, int valid, int e) {
      if (e >= valid) return;
      const int i = (int)(tt * kTile) + e;
      const R xi = stage_at<R>(buf, o_xt, e), gi = stage_at<R>(buf, o_g, e);
      const R li = stage_at<R>(buf, o_l, e), ui = stage_at<R>(buf, o_u, e);
      const int nb = stage_at<int>(buf, o_nb, e);
      bool has_bp;
      R tnum, tden;
      const int code = classify_q(xi, gi, li, ui, nb, has_bp, tnum, tden);
      c.code[i] = (int8_t)code;
      if (code == IW_FREE || code == IW_UNB) {
        const A neggi = -(A)gi;
        acc[0] = fma(neggi, neggi, acc[0]);
#pragma unroll
        for (int j = 0; j < kMaxM; j++) {
          if (kFull || j < col) {
            acc[1 + j] = fma(hist_at<H, A>(buf, hy + j * hb, e), neggi, acc[1 + j]);
            acc[9 + j] = fma(hist_at<H, A>(buf, hs + j * hb, e), neggi, acc[9 + j]);
          }
        }
        // the new pair as the ring will hold it
        const R ti = stage_at<R>(buf, o_t, e), zi = stage_at<R>(buf, o_z, e);
        const R d = rsub(zi, ti);
        const R sv = unit ? d : rmul(d, stp);
        const R y = rsub(gi, stage_at<R>(buf, o_go, e));
        acc[17] = fma(stored_value<H, A>(y), neggi, acc[17]);
        acc[18] = fma(stored_value<H, A>(sv), neggi, acc[18]);
        if (has_bp) {
          acc[19] += A(1);
          bp.offer_quotient(tnum, tden, i + c.ioff);
        } else {
          acc[20] += A(1);
          if (neggi != A(0)) xmx = A(1);
        }
      }
    };
    // kOneRole: post_elem and gcp_elem on one element, each input read from the stage once
    // fast: every column live and a unit step (the trial point is z), as constants
    // Every input of the element is read into registers first and the stage released.
    auto one_role = [&](const unsigned char* buf, long long tt, int valid, int e, auto fast,
                        auto release) {
      constexpr bool F = decltype(fast)::value;
      const bool unit_ = F ? true : unit;
      const int i = (int)(tt * kTile) + e;
      const R ti = stage_at<R>(buf, o_t, e), zi = stage_at<R>(buf, o_z, e);
      const R xi = F ? zi : stage_at<R>(buf, o_xt, e);
      const R gi = stage_at<R>(buf, o_g, e);
      const R gold = stage_at<R>(buf, o_go, e);
      const R li = stage_at<R>(buf, o_l, e), ui = stage_at<R>(buf, o_u, e);
      const int nb = stage_at<int>(buf, o_nb, e);
      A yv[kMaxM], sh[kMaxM];
#pragma unroll
      for (int j = 0; j < kMaxM; j++) {
        const bool live = kFull || j < col;
        yv[j] = live ? hist_at<H, A>(buf, hy + j * hb, e) : A(0);
        sh[j] = live ? hist_at<H, A>(buf, hs + j * hb, e) : A(0);
      }
      release();
      if (e >= valid) return;  // (stale stage bytes past the tile's end)
      // role P
      const R d = rsub(zi, ti);
      acc[0] = fma((A)gi, (A)d, acc[0]);
      const bool neg = gi < R(0);
      const R tb = rsub(xi, neg ? ui : li);
      const bool clip = nb != 0 && (neg ? nb >= 2 : nb <= 2);
      const R pg = clip ? (neg ? smax<R>(tb, gi) : smin<R>(tb, gi)) : gi;
      const A apg = fabs((A)pg);
      xmx = (apg > xmx) ? apg : xmx;
      const R xd = rsub(ti, xi);
      acc[1] = fma((A)xd, (A)xd, acc[1]);
      const R y = rsub(gi, gold);
      acc[2] = fma((A)y, (A)y, acc[2]);
      const R sv = unit_ ? d : rmul(d, stp);
#pragma unroll
      for (int j = 0; j < kMaxM; j++) {
        if (kFull || j < col) {
          acc[3 + j] = fma((A)sv, yv[j], acc[3 + j]);
          acc[11 + j] = fma(sh[j], (A)sv, acc[11 + j]);
        }
      }
      ssp[i] = HistTraits<H>::from(sv);
      ysp[i] = HistTraits<H>::from(y);
      // role G
      bool has_bp;
      R tnum, tden;
      const int code = classify_q(xi, gi, li, ui, nb, has_bp, tnum, tden);
      c.code[i] = (int8_t)code;
      if (code == IW_FREE || code == IW_UNB) {
        const A neggi = -(A)gi;
        accg[0] = fma(neggi, neggi, accg[0]);
#pragma unroll
        for (int j = 0; j < kMaxM; j++) {
          if (kFull || j < col) {
            accg[1 + j] = fma(yv[j], neggi, accg[1 + j]);
            accg[9 + j] = fma(sh[j], neggi, accg[9 + j]);
          }
        }
        accg[17] = fma(stored_value<H, A>(y), neggi, accg[17]);
        accg[18] = fma(stored_value<H, A>(sv), neggi, accg[18]);
        if (has_bp) {
          accg[19] += A(1);
          bp.offer_quotient(tnum, tden, i + c.ioff);
        } else {
          accg[20] += A(1);
          if (neggi != A(0)) xmxg = A(1);
        }
      }
    };
    auto stream_tiles = [&](auto fast) {
    run_stages<CONS>(ss, n, stages, dyn,
                     reinterpret_cast<uint64_t*>(dyn + (size_t)stages * cap), &st->device_error, cp,
                     [&](const unsigned char* buf, long long tt, int valid, auto release) {
      if constexpr (kOneRole) {
        one_role(buf, tt, valid, (int)threadIdx.x, fast, release);
        return;
      } else if (role == 0) {
#pragma unroll
        for (int h = 0; h < kTile / kRoleThreads; h++) post_elem(buf, tt, valid, rt + h * kRoleThreads);
      } else {
#pragma unroll
        for (int h = 0; h < kTile / kRoleThreads; h++) gcp_elem(buf, tt, valid, rt + h * kRoleThreads);
      }
      release();
    });
    };
    if constexpr (kOneRole) {
      if (kFull && unit && xt_is_z)
        stream_tiles(std::true_type{});
      else
        stream_tiles(std::false_type{});
    } else {
      stream_tiles(std::false_type{});
    }
  });
  // CTA row: [ role P sums (19) | role G sums (21) | role P max | role G max | min pair ]
  constexpr int NS = NP + NG, W = NS + 2 + 2;
  constexpr int kAllWarps = CONS / 32 + 1;
  if (!c.epi_only) {
    __shared__ double wsum[kAllWarps][W];
    for (int k = lane; k < W; k += 32) wsum[warp][k] = 0.0;
    __syncwarp();
    const int off = role == 0 ? 0 : NP;
    const int cnt = role == 0 ? NP : role == 1 ? NG : 0;
#pragma unroll
    for (int k = 0; k < NG; k++) {
      const double v = warp_sum((double)acc[k]);
      if (lane == 0 && k < cnt) wsum[warp][off + k] = v;
    }
    // the warps that ran role G (kOneRole: role 0 ran both)
    const int grole = kOneRole ? 0 : 1;
    if constexpr (kOneRole) {
#pragma unroll
      for (int k = 0; k < NG; k++) {
        const double v = warp_sum((double)accg[k]);
        if (lane == 0 && role == 0) wsum[warp][NP + k] = v;
      }
    }
    const double xv = warp_max((double)xmx);
    const double xvg = warp_max((double)xmxg);
    const MinPair mv = warp_min(bp.pair());
    if (lane == 0) {
      if (role < 2) wsum[warp][NS + role] = xv;
      if (kOneRole && role == 0) wsum[warp][NS + 1] = xvg;
      wsum[warp][NS + 2] = role == grole ? mv.v : INFINITY;
      wsum[warp][NS + 3] = role == grole ? (double)mv.i : (double)kNoIndex;
    }
    __syncthreads();
    double* row = c.part + cp.rank;  // entry k at row[k * cp.count] (reduce.cuh)
    for (int k = threadIdx.x; k < W; k += CONS + 32) {
      if (k < NS) {
        double a = 0.0;
        for (int w = 0; w < kAllWarps; w++) a += wsum[w][k];
        row[(size_t)k * cp.count] = a;
      } else if (k < NS + 2) {
        double a = 0.0;
        for (int w = 0; w < kAllWarps; w++) a = wsum[w][k] > a ? wsum[w][k] : a;
        row[(size_t)k * cp.count] = a;
      } else if (k == NS + 2) {
        MinPair a = MinPair{INFINITY, kNoIndex};
        for (int w = 0; w < kAllWarps; w++)
          a = minpair(a, MinPair{wsum[w][k], (long long)wsum[w][k + 1]});
        row[(size_t)k * cp.count] = a.v;
        row[(size_t)(k + 1) * cp.count] = (double)a.i;
      }
    }
  }
  __shared__ double red[W];
  if (!pass_fold<CONS + 32>(c, cp, W, NS, 2, 1, red)) return;
  __shared__ SmallWork<S> sw;
  __shared__ double rp[NP + 1], rg[22];  // epilogue temporaries (shared, as all of them)
  epilogue_on_shared_warp<S>(st, [&](DevState<S>* st, int lane) {
    if (lane == 0) {
      for (int k = 0; k < NP; k++) rp[k] = red[k];
      rp[NP] = red[NS];
      st->spec_gcp = 0;
    }
    __syncwarp();
    const int col_old = col;
    if (!post_epilogue<S>(st, rp, f, force_accept, lane) || st->internal_fail != 0) return;
    // the next iteration's loop top and cauchy epilogue (279-284, 702-747) at the accepted x
    if (lane == 0) begin_state(st, 0);
    __syncwarp();
    if (st->uncon_branch) {
      if (lane == 0) st->spec_gcp = 1;
      return;
    }
    const int ncol = st->col;
    if (lane == 0) {
      const double* g = red + NP;
      const int shifted = (st->updatd && st->iupdat > st->m) ? 1 : 0;
      rg[0] = g[0];
      for (int j = 1; j <= kMaxM; j++) {
        rg[j] = 0.0;
        rg[8 + j] = 0.0;
      }
      if (!st->updatd) {
        for (int j = 1; j <= col_old; j++) {
          rg[j] = g[j];
          rg[8 + j] = g[8 + j];
        }
      } else {
        for (int j = 1; j <= ncol - 1; j++) {
          rg[j] = g[j + shifted];
          rg[8 + j] = g[8 + j + shifted];
        }
        rg[ncol] = g[17];
        rg[8 + ncol] = g[18];
      }
      rg[17] = g[19];
      rg[18] = g[20];
      rg[19] = red[NS + 1];
      rg[20] = red[NS + 2];
      rg[21] = red[NS + 3];
    }
    __syncwarp();
    gcp_epilogue<S>(st, rg, ncol, sw, lane);
    if (lane == 0) st->spec_gcp = 1;
  });
}

template <typename R, typename H, typename S, int CONS>
__global__ void __launch_bounds__(CONS + 32) k_post_gcp(Ctx<R, H, S> c,
    const R* __restrict__ t, const R* __restrict__ z, const R* __restrict__ xt,
    const R* __restrict__ gt, const R* __restrict__ go, S f, int force_accept) {
  post_gcp_pass<R, H, S, CONS>(c, cta_here(), c.stages, t, z, xt, gt, go, f, force_accept);
}

}  // namespace lbfgsb_b200
