// small.cuh -- the 2m x 2m (<= 16 x 16) matrix algebra and the scalar line-search logic.
//
// These routines run on one device thread inside the epilogue of a streaming pass (or
// per breakpoint candidate in the Cauchy walk).  Each follows the arithmetic order of the
// reference routine it is named after, so that for the same inputs it rounds the same
// way: culbfgsb/lbfgsbcpu.cpp bmv 517-565, dpofa 1876-1908, dtrsl 1910-1986,
// formt 1105-1133, formk 907-1103 (assembly and factorisation part), dcsrch 1541-1735,
// dcstep 1737-1874.  S is the scalar type (float or double).
#pragma once

#include <math.h>

#include "common.cuh"

namespace lbfgsb_b200 {

// Every loop here is kept rolled (#pragma unroll 1).  These routines run in the epilogue
// of a pass, on one warp of the one CTA that finishes last, whose SM fetches their code
// afresh in each launch; unrolled copies make that code longer and its first run wait on
// more instruction fetches.  Rolled, the two large pass epilogues take 12-24 us less per
// launch at n = 4096^2, with every loop's operations in the same order.

// 1-based element (i, j) of a row-major matrix with leading dimension ld.
#define LB_AT(a, ld, i, j) ((a)[((i)-1) * (ld) + (j)-1])

template <typename S>
__host__ __device__ inline S smax(S a, S b) { return a > b ? a : b; }
template <typename S>
__host__ __device__ inline S smin(S a, S b) { return a > b ? b : a; }

__host__ __device__ inline double ssqrt(double v) { return sqrt(v); }
__host__ __device__ inline float ssqrt(float v) { return sqrtf(v); }
__host__ __device__ inline double sabs(double v) { return fabs(v); }
__host__ __device__ inline float sabs(float v) { return fabsf(v); }

// Dot product in groups of four, each group summed left to right and then added to the
// running sum (the order of the reference's vector helper).
template <typename S>
__host__ __device__ inline S sdot(const S* a, int sa, const S* b, int sb, int len) {
  S r = 0;
  int groups = len / 4;
  #pragma unroll 1
  for (int i = 0; i < groups; i++) {
    r += a[0] * b[0] + a[sa] * b[sb] + a[2 * sa] * b[2 * sb] + a[3 * sa] * b[3 * sb];
    a += 4 * sa;
    b += 4 * sb;
  }
  #pragma unroll 1
  for (int i = 0; i < len % 4; i++) {
    r += a[0] * b[0];
    a += sa;
    b += sb;
  }
  return r;
}

// Cholesky factor (upper, in place) of the leading n x n block; false on a non-positive
// pivot.
template <typename S>
__host__ __device__ inline bool sdpofa(S* a, int ld, int n) {
  #pragma unroll 1
  for (int j = 1; j <= n; j++) {
    S s = 0;
    #pragma unroll 1
    for (int k = 1; k <= j - 1; k++) {
      S v = sdot(&LB_AT(a, ld, 1, k), ld, &LB_AT(a, ld, 1, j), ld, k - 1);
      S t = LB_AT(a, ld, k, j) - v;
      t = t / LB_AT(a, ld, k, k);
      LB_AT(a, ld, k, j) = t;
      s = s + t * t;
    }
    s = LB_AT(a, ld, j, j) - s;
    if (s <= 0) return false;
    LB_AT(a, ld, j, j) = ssqrt(s);
  }
  return true;
}

// Triangular solve with the upper factor t: job 1 solves t x = b, job 11 solves t' x = b.
// b is 1-based (b[1..n]).  info = index of a zero diagonal, else 0.
template <typename S>
__host__ __device__ inline void sdtrsl(const S* t, int ld, int n, S* b, int job, int* info) {
  #pragma unroll 1
  for (int j = 1; j <= n; j++) {
    if (LB_AT(t, ld, j, j) == 0) {
      *info = j;
      return;
    }
  }
  *info = 0;
  if (job == 1) {
    b[n] = b[n] / LB_AT(t, ld, n, n);
    #pragma unroll 1
    for (int jj = 2; jj <= n; jj++) {
      int j = n - jj + 1;
      S temp = -b[j + 1];
      #pragma unroll 1
      for (int i = 1; i <= j; i++) b[i] += temp * LB_AT(t, ld, i, j + 1);
      b[j] = b[j] / LB_AT(t, ld, j, j);
    }
    return;
  }
  b[1] = b[1] / LB_AT(t, ld, 1, 1);
  #pragma unroll 1
  for (int j = 2; j <= n; j++) {
    S v = sdot(&LB_AT(t, ld, 1, j), ld, &b[1], 1, j - 1);
    b[j] = b[j] - v;
    b[j] = b[j] / LB_AT(t, ld, j, j);
  }
}

// p = M v for the middle matrix defined by sy (m x m, ld kMaxM) and the factor wt.
// v and p are 1-based (index 1..2col); work holds kMaxM + 1 scalars.
//
// On the device every temporary of these routines lives in shared (or global) memory
// passed in by the caller, next to the state copy the epilogues work on: a runtime-indexed
// thread-local array would be placed in local memory (the pass kernels run at 96 registers
// a thread), and keeping all operands in one place lets the warp-shared forms of
// warp_small.cuh exchange them between lanes.  No routine here declares a local array.
template <typename S>
__host__ __device__ inline void sbmv(const S* sy, const S* wt, int col, const S* v, S* p,
                                     int* info, S* work) {
  constexpr int ld = kMaxM;
  *info = 0;
  if (col == 0) return;
  p[col + 1] = v[col + 1];
  #pragma unroll 1
  for (int i = 2; i <= col; i++) {
    S s = 0;
    #pragma unroll 1
    for (int k = 1; k <= i - 1; k++) s = s + LB_AT(sy, ld, i, k) * v[k] / LB_AT(sy, ld, k, k);
    p[col + i] = v[col + i] + s;
  }
  #pragma unroll 1
  for (int i = 1; i <= col; i++) work[i] = p[col + i];
  sdtrsl(wt, ld, col, work, 11, info);
  #pragma unroll 1
  for (int i = 1; i <= col; i++) p[col + i] = work[i];
  if (*info != 0) return;
  #pragma unroll 1
  for (int i = 1; i <= col; i++) p[i] = v[i] / ssqrt(LB_AT(sy, ld, i, i));
  #pragma unroll 1
  for (int i = 1; i <= col; i++) work[i] = p[col + i];
  sdtrsl(wt, ld, col, work, 1, info);
  #pragma unroll 1
  for (int i = 1; i <= col; i++) p[col + i] = work[i];
  if (*info != 0) return;
  #pragma unroll 1
  for (int i = 1; i <= col; i++) p[i] = -p[i] / ssqrt(LB_AT(sy, ld, i, i));
  #pragma unroll 1
  for (int i = 1; i <= col; i++) {
    S s = 0;
    #pragma unroll 1
    for (int k = i + 1; k <= col; k++) s = s + LB_AT(sy, ld, k, i) * p[col + k] / LB_AT(sy, ld, i, i);
    p[i] = p[i] + s;
  }
}

// wt = chol(theta*SS + L D^-1 L'); returns 0 or -3.
template <typename S>
__host__ __device__ inline int sformt(S* wt, const S* sy, const S* ss, int col, S theta) {
  constexpr int ld = kMaxM;
  #pragma unroll 1
  for (int j = 1; j <= col; j++) LB_AT(wt, ld, 1, j) = theta * LB_AT(ss, ld, 1, j);
  #pragma unroll 1
  for (int i = 2; i <= col; i++) {
    #pragma unroll 1
    for (int j = i; j <= col; j++) {
      int k1 = (i < j ? i : j) - 1;
      S ddum = 0;
      #pragma unroll 1
      for (int k = 1; k <= k1; k++) ddum = ddum + LB_AT(sy, ld, i, k) * LB_AT(sy, ld, j, k) / LB_AT(sy, ld, k, k);
      LB_AT(wt, ld, i, j) = ddum + theta * LB_AT(ss, ld, i, j);
    }
  }
  return sdpofa(wt, ld, col) ? 0 : -3;
}

// Products that the streaming pass gathers for formk (over the current free set F and its
// complement A, positions 1..col counted from head):
//   yy_new[j] = sum_F y_col y_j, ss_new[j] = sum_A s_col s_j,
//   sy_row[j] = sum_A s_col y_j, sy_col[j] = sum_F s_j y_col,
// and the signed entering(+)/leaving(-) sums dyy[a][b], dss[a][b] (a >= b) and
// dsy[i][j] over the variables whose free/active status changed since the last freev.
template <typename S>
struct SmallWork;  // defined below

template <typename S>
struct FormkSums {
  S yy_new[kMaxM], ss_new[kMaxM], sy_row[kMaxM], sy_col[kMaxM];
  S dyy[kMaxM][kMaxM], dss[kMaxM][kMaxM], dsy[kMaxM][kMaxM];
};

// formk: update wn1 (ld 2*kMaxM, the reference's 2m x 2m layout with m = kMaxM offsets
// replaced by the actual m) from the gathered products, assemble K into wn (ld 2*kMaxM)
// and factor it.  Returns 0, -1 or -2 like the reference.
template <typename S>
__host__ __device__ inline int sformk(int m, int col, int updatd, int iupdat, S theta,
                                      const S* sy, S* wn, S* wn1, const FormkSums<S>& fs,
                                      S* work, S* wm) {
  constexpr int L2 = 2 * kMaxM;
  int upcl;
  if (updatd) {
    if (iupdat > m) {
      #pragma unroll 1
      for (int jy = 1; jy <= m - 1; jy++) {
        int js = m + jy;
        #pragma unroll 1
        for (int i = 0; i <= m - 1 - jy; i++) LB_AT(wn1, L2, jy + i, jy) = LB_AT(wn1, L2, jy + 1 + i, jy + 1);
        #pragma unroll 1
        for (int i = 0; i <= m - 1 - jy; i++) LB_AT(wn1, L2, js + i, js) = LB_AT(wn1, L2, js + 1 + i, js + 1);
        #pragma unroll 1
        for (int i = 0; i <= m - 2; i++) LB_AT(wn1, L2, m + 1 + i, jy) = LB_AT(wn1, L2, m + 2 + i, jy + 1);
      }
    }
    #pragma unroll 1
    for (int jy = 1; jy <= col; jy++) {
      LB_AT(wn1, L2, col, jy) = fs.yy_new[jy - 1];
      LB_AT(wn1, L2, m + col, m + jy) = fs.ss_new[jy - 1];
      LB_AT(wn1, L2, m + col, jy) = fs.sy_row[jy - 1];
    }
    #pragma unroll 1
    for (int i = 1; i <= col; i++) LB_AT(wn1, L2, m + i, col) = fs.sy_col[i - 1];
    upcl = col - 1;
  } else {
    upcl = col;
  }
  #pragma unroll 1
  for (int iy = 1; iy <= upcl; iy++) {
    #pragma unroll 1
    for (int jy = 1; jy <= iy; jy++) {
      LB_AT(wn1, L2, iy, jy) = LB_AT(wn1, L2, iy, jy) + fs.dyy[iy - 1][jy - 1];
      LB_AT(wn1, L2, m + iy, m + jy) = LB_AT(wn1, L2, m + iy, m + jy) - fs.dss[iy - 1][jy - 1];
    }
  }
  #pragma unroll 1
  for (int i = 1; i <= upcl; i++) {
    #pragma unroll 1
    for (int jy = 1; jy <= upcl; jy++) {
      if (i <= jy)
        LB_AT(wn1, L2, m + i, jy) = LB_AT(wn1, L2, m + i, jy) + fs.dsy[i - 1][jy - 1];
      else
        LB_AT(wn1, L2, m + i, jy) = LB_AT(wn1, L2, m + i, jy) - fs.dsy[i - 1][jy - 1];
    }
  }
  #pragma unroll 1
  for (int iy = 1; iy <= col; iy++) {
    int iis = col + iy, is1 = m + iy;
    #pragma unroll 1
    for (int jy = 1; jy <= iy; jy++) {
      int js = col + jy, js1 = m + jy;
      LB_AT(wn, L2, jy, iy) = LB_AT(wn1, L2, iy, jy) / theta;
      LB_AT(wn, L2, js, iis) = LB_AT(wn1, L2, is1, js1) * theta;
    }
    #pragma unroll 1
    for (int jy = 1; jy <= iy - 1; jy++) LB_AT(wn, L2, jy, iis) = -LB_AT(wn1, L2, is1, jy);
    #pragma unroll 1
    for (int jy = iy; jy <= col; jy++) LB_AT(wn, L2, jy, iis) = LB_AT(wn1, L2, is1, jy);
    LB_AT(wn, L2, iy, iy) = LB_AT(wn, L2, iy, iy) + LB_AT(sy, kMaxM, iy, iy);
  }
  if (!sdpofa(wn, L2, col)) return -1;
  int info = 0;
  int col2 = 2 * col;
  #pragma unroll 1
  for (int js = col + 1; js <= col2; js++) {
    #pragma unroll 1
    for (int i = 1; i <= col; i++) work[i] = LB_AT(wn, L2, i, js);
    sdtrsl(wn, L2, col, work, 11, &info);
    #pragma unroll 1
    for (int i = 1; i <= col; i++) LB_AT(wn, L2, i, js) = work[i];
  }
  #pragma unroll 1
  for (int iis = col + 1; iis <= col2; iis++) {
    #pragma unroll 1
    for (int js = iis; js <= col2; js++) {
      S v = sdot(&LB_AT(wn, L2, 1, iis), L2, &LB_AT(wn, L2, 1, js), L2, col);
      LB_AT(wn, L2, iis, js) = LB_AT(wn, L2, iis, js) + v;
    }
  }
  #pragma unroll 1
  for (int j = 1; j <= col; j++)
    #pragma unroll 1
    for (int i = 1; i <= col; i++) LB_AT(wm, kMaxM, j, i) = LB_AT(wn, L2, col + j, col + i);
  if (!sdpofa(wm, kMaxM, col)) return -2;
  #pragma unroll 1
  for (int j = 1; j <= col; j++)
    #pragma unroll 1
    for (int i = 1; i <= col; i++) LB_AT(wn, L2, col + j, col + i) = LB_AT(wm, kMaxM, j, i);
  return 0;
}

// Shared-memory workspace of one epilogue (see the note at sbmv).
template <typename S>
struct SmallWork {
  S work[kMaxM + 1];
  S wm[kMaxM * kMaxM];
  S v[2 * kMaxM + 1];
  S wv[2 * kMaxM + 1];
  FormkSums<S> fs;
};

// ---------------------------------------------------------------------------------------
// Line search (More'-Thuente as in L-BFGS-B 2.1).  dcsrch task codes: 0 start, 1 evaluate
// f and g at stp, 2 input error, 3 warning (terminate), 4 converged.
template <typename S>
struct LineSearchSave {
  int isave[3];
  S dsave[14];
};

template <typename S>
__host__ __device__ inline void sdcstep(S& stx, S& fx, S& dx, S& sty, S& fy, S& dy, S& stp,
                                        S fp, S dp, int& brackt, S stpmin, S stpmax) {
  S gamma, p, q, r, s, sgnd, stpc, stpf, stpq, theta;
  sgnd = dp * (dx / sabs(dx));
  if (fp > fx) {
    theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
    s = smax(sabs(theta), smax(sabs(dx), sabs(dp)));
    gamma = s * ssqrt((theta / s) * (theta / s) - dx / s * (dp / s));
    if (stp < stx) gamma = -gamma;
    p = gamma - dx + theta;
    q = gamma - dx + gamma + dp;
    r = p / q;
    stpc = stx + r * (stp - stx);
    stpq = stx + dx / ((fx - fp) / (stp - stx) + dx) / 2 * (stp - stx);
    if (sabs(stpc - stx) < sabs(stpq - stx))
      stpf = stpc;
    else
      stpf = stpc + (stpq - stpc) / 2;
    brackt = 1;
  } else if (sgnd < 0) {
    theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
    s = smax(sabs(theta), smax(sabs(dx), sabs(dp)));
    gamma = s * ssqrt((theta / s) * (theta / s) - dx / s * (dp / s));
    if (stp > stx) gamma = -gamma;
    p = gamma - dp + theta;
    q = gamma - dp + gamma + dx;
    r = p / q;
    stpc = stp + r * (stx - stp);
    stpq = stp + dp / (dp - dx) * (stx - stp);
    stpf = (sabs(stpc - stp) > sabs(stpq - stp)) ? stpc : stpq;
    brackt = 1;
  } else if (sabs(dp) < sabs(dx)) {
    theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
    s = smax(sabs(theta), smax(sabs(dx), sabs(dp)));
    gamma = s * ssqrt(smax((S)0, (theta / s) * (theta / s) - dx / s * (dp / s)));
    if (stp > stx) gamma = -gamma;
    p = gamma - dp + theta;
    q = gamma + (dx - dp) + gamma;
    r = p / q;
    if (r < 0 && gamma != 0)
      stpc = stp + r * (stx - stp);
    else
      stpc = (stp > stx) ? stpmax : stpmin;
    stpq = stp + dp / (dp - dx) * (stx - stp);
    if (brackt) {
      stpf = (sabs(stpc - stp) < sabs(stpq - stp)) ? stpc : stpq;
      // the 0.66 extrapolation bound is evaluated in double, as in the reference
      S bound = (S)((double)stp + 0.66 * (double)(sty - stp));
      stpf = (stp > stx) ? smin(bound, stpf) : smax(bound, stpf);
    } else {
      stpf = (sabs(stpc - stp) > sabs(stpq - stp)) ? stpc : stpq;
      stpf = smin(stpmax, stpf);
      stpf = smax(stpmin, stpf);
    }
  } else {
    if (brackt) {
      theta = 3 * (fp - fy) / (sty - stp) + dy + dp;
      s = smax(sabs(theta), smax(sabs(dy), sabs(dp)));
      gamma = s * ssqrt((theta / s) * (theta / s) - dy / s * (dp / s));
      if (stp > sty) gamma = -gamma;
      p = gamma - dp + theta;
      q = gamma - dp + gamma + dy;
      r = p / q;
      stpc = stp + r * (sty - stp);
      stpf = stpc;
    } else {
      stpf = (stp > stx) ? stpmax : stpmin;
    }
  }
  if (fp > fx) {
    sty = stp;
    fy = fp;
    dy = dp;
  } else {
    if (sgnd < 0) {
      sty = stx;
      fy = fx;
      dy = dx;
    }
    stx = stp;
    fx = fp;
    dx = dp;
  }
  stp = stpf;
}

template <typename S>
__host__ __device__ inline void sdcsrch(S f, S g, S& stp, S ftol, S gtol, S xtol, S stpmin,
                                        S stpmax, int& task, LineSearchSave<S>& sv) {
  int brackt, stage;
  S finit, ftest, fm, fx, fxm, fy, fym, ginit, gtest, gm, gx, gxm, gy, gym, stx, sty, stmin,
      stmax, width, width1;
  const S xtrapl = (S)1.1, xtrapu = (S)4.0;
  if (task == 0) {
    if (stp < stpmin) task = 2;
    if (stp > stpmax) task = 2;
    if (g >= 0) task = 2;
    if (ftol < 0) task = 2;
    if (gtol < 0) task = 2;
    if (xtol < 0) task = 2;
    if (stpmin < 0) task = 2;
    if (stpmax < stpmin) task = 2;
    if (task == 2) return;
    brackt = 0;
    stage = 1;
    finit = f;
    ginit = g;
    gtest = ftol * ginit;
    width = stpmax - stpmin;
    width1 = width / (S)0.5;
    stx = 0;
    fx = finit;
    gx = ginit;
    sty = 0;
    fy = finit;
    gy = ginit;
    stmin = 0;
    stmax = stp + xtrapu * stp;
    task = 1;
  } else {
    brackt = sv.isave[1] == 1;
    stage = sv.isave[2];
    ginit = sv.dsave[1];
    gtest = sv.dsave[2];
    gx = sv.dsave[3];
    gy = sv.dsave[4];
    finit = sv.dsave[5];
    fx = sv.dsave[6];
    fy = sv.dsave[7];
    stx = sv.dsave[8];
    sty = sv.dsave[9];
    stmin = sv.dsave[10];
    stmax = sv.dsave[11];
    width = sv.dsave[12];
    width1 = sv.dsave[13];
    ftest = finit + stp * gtest;
    if (stage == 1 && f <= ftest && g >= 0) stage = 2;
    if (brackt && (stp <= stmin || stp >= stmax)) task = 3;
    if (brackt && stmax - stmin <= xtol * stmax) task = 3;
    if (stp == stpmax && f <= ftest && g <= gtest) task = 3;
    if (stp == stpmin && (f > ftest || g >= gtest)) task = 3;
    if (f <= ftest && sabs(g) <= gtol * (-ginit)) task = 4;
    if (task != 3 && task != 4) {
      if (stage == 1 && f <= fx && f > ftest) {
        fm = f - stp * gtest;
        fxm = fx - stx * gtest;
        fym = fy - sty * gtest;
        gm = g - gtest;
        gxm = gx - gtest;
        gym = gy - gtest;
        sdcstep(stx, fxm, gxm, sty, fym, gym, stp, fm, gm, brackt, stmin, stmax);
        fx = fxm + stx * gtest;
        fy = fym + sty * gtest;
        gx = gxm + gtest;
        gy = gym + gtest;
      } else {
        sdcstep(stx, fx, gx, sty, fy, gy, stp, f, g, brackt, stmin, stmax);
      }
      if (brackt) {
        if (sabs(sty - stx) >= (S)0.66 * width1) stp = stx + (S)0.5 * (sty - stx);
        width1 = width;
        width = sabs(sty - stx);
      }
      if (brackt) {
        stmin = smin(stx, sty);
        stmax = smax(stx, sty);
      } else {
        stmin = stp + xtrapl * (stp - stx);
        stmax = stp + xtrapu * (stp - stx);
      }
      stp = smax(stp, stpmin);
      stp = smin(stp, stpmax);
      if ((brackt && (stp <= stmin || stp >= stmax)) || (brackt && stmax - stmin <= xtol * stmax))
        stp = stx;
      task = 1;
    }
  }
  sv.isave[1] = brackt ? 1 : 0;
  sv.isave[2] = stage;
  sv.dsave[1] = ginit;
  sv.dsave[2] = gtest;
  sv.dsave[3] = gx;
  sv.dsave[4] = gy;
  sv.dsave[5] = finit;
  sv.dsave[6] = fx;
  sv.dsave[7] = fy;
  sv.dsave[8] = stx;
  sv.dsave[9] = sty;
  sv.dsave[10] = stmin;
  sv.dsave[11] = stmax;
  sv.dsave[12] = width;
  sv.dsave[13] = width1;
}

}  // namespace lbfgsb_b200
