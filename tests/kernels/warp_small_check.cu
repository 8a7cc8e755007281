// Compares the warp-cooperative small-matrix routines of csrc/warp_small.cuh with the
// serial routines of csrc/small.cuh bit for bit: each trial builds one set of inputs,
// runs the serial routine on one copy (thread 0) and the warp routine on another (32
// lanes), and compares every output entry and the info codes.  The inputs are Gram
// matrices of random vectors over a random free set, so that most factorisations
// succeed, plus indefinite and singular cases for the failure paths:
//   formk  (every col 1..8, with and without a new pair, with and without the ring shift,
//           with and without entering/leaving corrections),
//   formt, bmv (on formt's factor), the K solves of the subspace step (job 11, negate,
//   job 1 on formk's K), dpofa on indefinite matrices, dtrsl with a zero diagonal.
// Prints the mismatch count and the number of trials that reached each stage per
// precision, and exits 1 on any mismatch.
//   argv[1] = trials per precision (default 20000)
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../lbfgsb-gpu_b200/csrc/warp_small.cuh"

using namespace lbfgsb_b200;

__device__ __forceinline__ unsigned long long sm64(unsigned long long& s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unif(unsigned long long& s) {  // [-1, 1)
  return (double)(sm64(s) >> 11) * 0x1p-52 - 1.0;
}

__device__ __forceinline__ bool bits_eq(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}
__device__ __forceinline__ bool bits_eq(float a, float b) { return __float_as_int(a) == __float_as_int(b); }

constexpr int NV = 40;  // variables of the random vectors
constexpr int L2 = 2 * kMaxM;

template <typename S>
struct Case {
  S sy[kMaxM * kMaxM], ss[kMaxM * kMaxM], wt[kMaxM * kMaxM], wm[kMaxM * kMaxM];
  S wn[L2 * L2], wn1[L2 * L2], snap[L2 * L2], a[L2 * L2];
  S work[kMaxM + 1], v[L2 + 1], p[L2 + 1], b[L2 + 1];
  FormkSums<S> fs;
};

// counters: [0] mismatches, [1] formk ok, [2] formk failed, [3] formt ok, [4] bmv run,
// [5] K solves run, [6] dpofa failed, [7] dtrsl zero diagonal
template <typename S>
__global__ void k_check(unsigned long long seed, unsigned long long* cnt) {
  __shared__ Case<S> A, B;
  __shared__ double sv[kMaxM + 1][NV], yv[kMaxM + 1][NV];
  __shared__ int freev[NV];
  __shared__ int prm[6];  // m, col, updatd, iupdat, corrections, dpofa kind
  __shared__ S s_theta;
  __shared__ int res[8];
  const int lane = threadIdx.x;
  unsigned long long s = seed * 0x9E3779B97F4A7C15ULL + blockIdx.x * 7919ULL + 1;
  if (lane == 0) {
    const int m = kMaxM;
    int col = 1 + (int)(sm64(s) % m);
    const int updatd = (int)(sm64(s) % 4 != 0);
    int iupdat = updatd ? ((sm64(s) & 1) ? col : m + 1 + (int)(sm64(s) % 5)) : col;
    if (iupdat > m) col = m;  // a shifted ring is full
    prm[0] = m; prm[1] = col; prm[2] = updatd; prm[3] = iupdat;
    prm[4] = (int)(sm64(s) % 3);
    prm[5] = (int)(sm64(s) % 4);
    s_theta = (S)(0.1 + 10.0 * (unif(s) + 1.0));
    for (int k = 0; k < NV; k++) freev[k] = (sm64(s) % 3) != 0;
    for (int v = 0; v <= m; v++)
      for (int k = 0; k < NV; k++) {
        sv[v][k] = unif(s);
        yv[v][k] = sv[v][k] + 0.3 * unif(s);
      }
  }
  __syncthreads();
  const int m = prm[0], col = prm[1], updatd = prm[2], iupdat = prm[3];
  const S theta = s_theta;
  if (lane == 0) {
    // ring position p (1..m) holds vector vec(p); the pair entering the ring is vector m
    // (a shifted ring: positions 1..m-1 hold vectors 1..m-1 after the shift, 0..m-2 before)
    auto dotv = [&](const double* a, const double* b, int which) {  // 0 all, 1 free, 2 active
      double r = 0;
      for (int k = 0; k < NV; k++)
        if (which == 0 || (which == 1) == (freev[k] != 0)) r += a[k] * b[k];
      return r;
    };
    const bool shift = updatd && iupdat > m;
    auto vec_before = [&](int p) { return p - 1; };
    memset(&A, 0, sizeof(A));
    // wn1 before the call: Gram blocks of the vectors at positions 1..m
    for (int i = 1; i <= m; i++)
      for (int j = 1; j <= m; j++) {
        const int vi = vec_before(i), vj = vec_before(j);
        LB_AT(A.wn1, L2, i, j) = (S)dotv(yv[vi], yv[vj], 1);
        LB_AT(A.wn1, L2, m + i, m + j) = (S)dotv(sv[vi], sv[vj], 2);
        LB_AT(A.wn1, L2, m + i, j) = (S)(i <= j ? dotv(sv[vi], yv[vj], 2) : dotv(sv[vi], yv[vj], 1));
      }
    // the products of the new pair with the ring after the update
    const int vnew = m;
    auto vec_after = [&](int p) { return p == col ? vnew : (shift ? p : p - 1); };
    for (int j = 1; j <= col; j++) {
      const int vj = vec_after(j);
      A.fs.yy_new[j - 1] = (S)dotv(yv[vnew], yv[vj], 1);
      A.fs.ss_new[j - 1] = (S)dotv(sv[vnew], sv[vj], 2);
      A.fs.sy_row[j - 1] = (S)dotv(sv[vnew], yv[vj], 2);
      A.fs.sy_col[j - 1] = (S)dotv(sv[vj], yv[vnew], 1);
    }
    const double ce = prm[4] == 0 ? 0.0 : prm[4] == 1 ? 1e-3 : 0.5;
    for (int a = 0; a < kMaxM; a++)
      for (int b = 0; b < kMaxM; b++) {
        A.fs.dyy[a][b] = (S)(ce * unif(s));
        A.fs.dss[a][b] = (S)(ce * unif(s));
        A.fs.dsy[a][b] = (S)(ce * unif(s));
      }
    for (int i = 1; i <= m; i++)
      for (int j = 1; j <= m; j++) {
        const int vi = vec_after(i), vj = vec_after(j);
        LB_AT(A.sy, kMaxM, i, j) = (S)dotv(sv[vi], yv[vj], 0);
        LB_AT(A.ss, kMaxM, i, j) = (S)dotv(sv[vi], sv[vj], 0);
      }
    // stale lower triangles, as the state holds them
    for (int e = 0; e < L2 * L2; e++) A.wn[e] = (S)unif(s);
    for (int e = 0; e < kMaxM * kMaxM; e++) A.wt[e] = (S)unif(s);
    for (int e = 0; e < kMaxM * kMaxM; e++) A.wm[e] = (S)unif(s);
    for (int j = 1; j <= L2; j++) A.v[j] = (S)unif(s);
    for (int j = 1; j <= L2; j++) A.b[j] = (S)unif(s);
    // a symmetric matrix for dpofa: a Gram matrix, shifted to be indefinite in some cases
    const int kind = prm[5];
    for (int i = 1; i <= L2; i++)
      for (int j = 1; j <= L2; j++) {
        double g = 0;
        for (int k = 0; k < NV; k++) {
          const double* ri = i <= kMaxM + 1 ? sv[i - 1] : yv[i - kMaxM - 2];
          const double* rj = j <= kMaxM + 1 ? sv[j - 1] : yv[j - kMaxM - 2];
          g += ri[k] * rj[k];
        }
        if (kind == 1 && i == j && i == 1 + (int)(sm64(s) % L2)) g -= 40.0;
        LB_AT(A.a, L2, i, j) = (S)g;
      }
  }
  __syncthreads();
  for (int e = lane; e < (int)(sizeof(Case<S>) / 4); e += 32)
    reinterpret_cast<unsigned int*>(&B)[e] = reinterpret_cast<const unsigned int*>(&A)[e];
  __syncthreads();
  auto same = [](const S* x, const S* y, int len) {
    for (int e = 0; e < len; e++)
      if (!bits_eq(x[e], y[e])) return false;
    return true;
  };

  // formk
  if (lane == 0) res[0] = sformk<S>(m, col, updatd, iupdat, theta, A.sy, A.wn, A.wn1, A.fs, A.work, A.wm);
  __syncthreads();
  const int kb = wformk<S>(m, col, updatd, iupdat, theta, B.sy, B.wn, B.wn1, B.fs, B.wm, B.snap, lane);
  __syncthreads();
  if (lane == 0) {
    unsigned long long bad = 0;
    if (kb != res[0]) bad++;
    if (!same(A.wn1, B.wn1, L2 * L2)) bad++;
    if (res[0] == 0) {
      if (!same(A.wn, B.wn, L2 * L2)) bad++;
      atomicAdd(&cnt[1], 1ULL);
    } else {
      atomicAdd(&cnt[2], 1ULL);
    }
    if (bad) atomicAdd(&cnt[0], bad);
  }
  // the K solves of the subspace step (job 11, negate the first col entries, job 1)
  if (res[0] == 0) {
    if (lane == 0) {
      int info = 0;
      sdtrsl(A.wn, L2, 2 * col, A.b, 11, &info);
      for (int j = 1; j <= col; j++) A.b[j] = -A.b[j];
      sdtrsl(A.wn, L2, 2 * col, A.b, 1, &info);
      res[1] = info;
    }
    __syncthreads();
    const int zb = wdiag_zero(B.wn, L2, 2 * col, lane);
    if (zb == 0) {
      wdtrsl11(B.wn, L2, 2 * col, B.b, lane);
      if (lane < col) B.b[lane + 1] = -B.b[lane + 1];
      __syncwarp();
      wdtrsl1(B.wn, L2, 2 * col, B.b, lane);
    }
    __syncthreads();
    if (lane == 0) {
      if (zb != res[1] || !same(A.b, B.b, L2 + 1)) atomicAdd(&cnt[0], 1ULL);
      atomicAdd(&cnt[5], 1ULL);
    }
  }
  // formt, then bmv on its factor
  if (lane == 0) res[2] = sformt<S>(A.wt, A.sy, A.ss, col, theta);
  __syncthreads();
  const int tb = wformt<S>(B.wt, B.sy, B.ss, col, theta, lane);
  __syncthreads();
  if (lane == 0) {
    if (tb != res[2]) atomicAdd(&cnt[0], 1ULL);
    if (res[2] == 0) {
      if (!same(A.wt, B.wt, kMaxM * kMaxM)) atomicAdd(&cnt[0], 1ULL);
      atomicAdd(&cnt[3], 1ULL);
    }
  }
  if (res[2] == 0) {
    if (lane == 0) {
      int info = 0;
      sbmv(A.sy, A.wt, col, A.v, A.p, &info, A.work);
      res[3] = info;
    }
    __syncthreads();
    const int ib = wbmv(B.sy, B.wt, col, B.v, B.p, B.work, lane);
    __syncthreads();
    if (lane == 0) {
      if (ib != res[3] || !same(A.p, B.p, L2 + 1)) atomicAdd(&cnt[0], 1ULL);
      atomicAdd(&cnt[4], 1ULL);
    }
  }
  // dpofa on the (possibly indefinite) symmetric matrix, every order 1..16
  const int na = 1 + (int)(blockIdx.x % L2);
  if (lane == 0) res[4] = sdpofa(A.a, L2, na) ? 1 : 0;
  __syncthreads();
  const int pb = wdpofa(B.a, L2, na, lane) ? 1 : 0;
  __syncthreads();
  if (lane == 0) {
    if (pb != res[4] || (res[4] && !same(A.a, B.a, L2 * L2))) atomicAdd(&cnt[0], 1ULL);
    if (!res[4]) atomicAdd(&cnt[6], 1ULL);
  }
  // dtrsl with a zero on the diagonal (info codes; b must stay as it was)
  if (lane == 0) {
    LB_AT(A.a, L2, 3, 3) = 0;
    LB_AT(B.a, L2, 3, 3) = 0;
    int info = 0;
    sdtrsl(A.a, L2, L2, A.v, 1, &info);
    res[5] = info;
  }
  __syncthreads();
  const int zz = wdiag_zero(B.a, L2, L2, lane);
  __syncthreads();
  if (lane == 0) {
    if (zz != res[5] || !same(A.v, B.v, L2 + 1)) atomicAdd(&cnt[0], 1ULL);
    if (zz != 0) atomicAdd(&cnt[7], 1ULL);
  }
}

template <typename S>
static int run(const char* name, int trials) {
  unsigned long long* d;
  cudaMalloc(&d, 8 * sizeof(unsigned long long));
  cudaMemset(d, 0, 8 * sizeof(unsigned long long));
  k_check<S><<<trials, 32>>>(12345ULL, d);
  cudaError_t e = cudaDeviceSynchronize();
  unsigned long long h[8];
  cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    printf("%s: CUDA error %s\n", name, cudaGetErrorString(e));
    return 1;
  }
  printf("%s: %llu mismatches (formk ok %llu failed %llu, K solves %llu, formt ok %llu, bmv %llu, "
         "dpofa failed %llu, zero diagonal %llu)\n",
         name, h[0], h[1], h[2], h[5], h[3], h[4], h[6], h[7]);
  return h[0] != 0 || h[1] == 0 || h[2] == 0 || h[4] == 0 || h[6] == 0 || h[7] == 0;
}

int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 20000;
  int bad = run<double>("f64", trials);
  bad |= run<float>("f32", trials);
  return bad;
}
