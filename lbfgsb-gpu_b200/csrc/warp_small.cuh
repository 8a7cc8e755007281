// warp_small.cuh -- warp-cooperative forms of the small-matrix routines of small.cuh.
//
// Every routine here is called by all 32 lanes of one warp, with its operands in shared
// memory.  Each output entry is computed by one lane with exactly the operations, in the
// same order, of the serial routine of small.cuh (and so of the reference routine that
// one follows: culbfgsb/lbfgsbcpu.cpp formk 907-1103, formt 1105-1133, bmv 517-565,
// dpofa 1876-1908, dtrsl 1910-1986); only entries that do not depend on one another are
// computed side by side.  The results are therefore bit-identical to the serial routines.
// Phases that read what other lanes wrote are separated by __syncwarp, which also orders
// the warp's shared-memory accesses.  Return values are the same on every lane, so the
// callers may branch on them without splitting the warp.
#pragma once

#include "small.cuh"

namespace lbfgsb_b200 {

// Every loop here is kept rolled (#pragma unroll 1).  These routines run in the epilogue
// of a pass, on one warp of the one CTA that finishes last, whose SM fetches their code
// afresh in each launch; unrolled copies make that code longer and its first run wait on
// more instruction fetches.  Rolled, the two large pass epilogues take 12-24 us less per
// launch at n = 4096^2, with every loop's operations in the same order.

constexpr unsigned kFullMask = 0xffffffffu;

// 1-based index of the first zero on the diagonal of the leading n x n block (n <= 32),
// else 0: the info code of sdtrsl.
template <typename S>
__device__ __forceinline__ int wdiag_zero(const S* t, int ld, int n, int lane) {
  const bool z = lane < n && LB_AT(t, ld, lane + 1, lane + 1) == S(0);
  const unsigned bal = __ballot_sync(kFullMask, z);
  return bal ? __ffs(bal) : 0;
}

// sdpofa as a wavefront (n <= 32): step k finishes the diagonal of column k and then
// entry (k, j) of every later column j (lane j-1).  Entry (k, j) reads column k and
// entries 1..k-1 of column j, all final after step k-1, so its dot product is formed
// while the diagonal's square root is taken; lane k-1 holds that column's sum of squares
// (accumulated over the earlier steps in the serial order) and every lane takes the same
// square root of the broadcast value, so the warp does not split.  No lane reads a(k, k)
// after step k except lane k-1, which stores it.  Lanes past n work on column n and
// discard the result.  On a non-positive pivot the columns after it are left partly
// updated; every caller discards the matrix in that case, as after a failure of the
// serial routine.
template <typename S>
__device__ bool wdpofa(S* a, int ld, int n, int lane) {
  S s = 0;
  const int j = lane + 1 <= n ? lane + 1 : n;
  const bool mine = lane + 1 <= n;
  #pragma unroll 1
  for (int k = 1; k <= n; k++) {
    const S v = sdot(&LB_AT(a, ld, 1, k), ld, &LB_AT(a, ld, 1, j), ld, k - 1);
    const S d = LB_AT(a, ld, k, k) - __shfl_sync(kFullMask, s, k - 1);
    if (d <= 0) return false;
    const S dk = ssqrt(d);
    if (mine && j > k) {
      S t = LB_AT(a, ld, k, j) - v;
      t = t / dk;
      LB_AT(a, ld, k, j) = t;
      s = s + t * t;
    }
    __syncwarp();  // every lane has read a(k, k) before it is replaced
    if (lane == k - 1) LB_AT(a, ld, k, k) = dk;
  }
  __syncwarp();
  return true;
}

// sdtrsl job 11 (t' x = b) for one right-hand side b (1-based, n <= 32).  Lane j-1 owns
// b[j] and forms the dot product of row j incrementally: at step i it receives the
// finished b[i] and adds t(i, j) b[i] exactly where sdot adds it (inside a group of four,
// then the group into the sum, or one by one past the last full group).  The caller has
// checked the diagonal.
template <typename S>
__device__ __forceinline__ void wdtrsl11(const S* t, int ld, int n, S* b, int lane) {
  const int j = lane + 1;
  const bool mine = j <= n;
  S bj = mine ? b[j] : S(0);
  if (j == 1) bj = bj / LB_AT(t, ld, 1, 1);
  const int full = 4 * ((j - 1) / 4);  // row j's indices inside full groups
  S r = 0, gp = 0;
  #pragma unroll 1
  for (int i = 1; i < n; i++) {
    const S bi = __shfl_sync(kFullMask, bj, i - 1);
    if (mine && j > i) {
      const S pr = LB_AT(t, ld, i, j) * bi;
      if (i <= full) {
        const int pos = (i - 1) & 3;
        gp = pos == 0 ? pr : gp + pr;
        if (pos == 3) r += gp;
      } else {
        r += pr;
      }
      if (i == j - 1) {
        bj = bj - r;
        bj = bj / LB_AT(t, ld, j, j);
      }
    }
  }
  __syncwarp();
  if (mine) b[j] = bj;
  __syncwarp();
}

// sdtrsl job 1 (t x = b), b 1-based, n <= 32, in its column (axpy) order: lane i-1 holds
// b[i]; step j broadcasts the finished b[j+1], every lane i <= j subtracts its multiple,
// and lane j-1 divides.  The caller has checked the diagonal.
template <typename S>
__device__ __forceinline__ void wdtrsl1(const S* t, int ld, int n, S* b, int lane) {
  S bi = lane < n ? b[lane + 1] : S(0);
  if (lane == n - 1) bi = bi / LB_AT(t, ld, n, n);
  #pragma unroll 1
  for (int jj = 2; jj <= n; jj++) {
    const int j = n - jj + 1;
    const S temp = -__shfl_sync(kFullMask, bi, j);
    if (lane < j) bi += temp * LB_AT(t, ld, lane + 1, j + 1);
    if (lane == j - 1) bi = bi / LB_AT(t, ld, j, j);
  }
  __syncwarp();
  if (lane < n) b[lane + 1] = bi;
  __syncwarp();
}

// p = M v (sbmv); returns its info.  v and p are 1-based and must not overlap.
template <typename S>
__device__ int wbmv(const S* sy, const S* wt, int col, const S* v, S* p, S* work, int lane) {
  constexpr int ld = kMaxM;
  if (col == 0) return 0;
  const int i = lane + 1;
  if (i == 1) p[col + 1] = v[col + 1];
  if (i >= 2 && i <= col) {
    S s = 0;
    #pragma unroll 1
    for (int k = 1; k <= i - 1; k++) s = s + LB_AT(sy, ld, i, k) * v[k] / LB_AT(sy, ld, k, k);
    p[col + i] = v[col + i] + s;
  }
  if (i <= col) work[i] = p[col + i];
  __syncwarp();
  const int info = wdiag_zero(wt, ld, col, lane);
  if (info == 0) wdtrsl11(wt, ld, col, work, lane);
  if (i <= col) p[col + i] = work[i];
  if (info != 0) {
    __syncwarp();
    return info;
  }
  if (i <= col) {
    p[i] = v[i] / ssqrt(LB_AT(sy, ld, i, i));
    work[i] = p[col + i];
  }
  __syncwarp();
  wdtrsl1(wt, ld, col, work, lane);
  if (i <= col) {
    p[col + i] = work[i];
    p[i] = -p[i] / ssqrt(LB_AT(sy, ld, i, i));
  }
  __syncwarp();
  if (i <= col) {
    S s = 0;
    #pragma unroll 1
    for (int k = i + 1; k <= col; k++) s = s + LB_AT(sy, ld, k, i) * p[col + k] / LB_AT(sy, ld, i, i);
    p[i] = p[i] + s;
  }
  __syncwarp();
  return 0;
}

// sformt: entry (i, j) of the upper triangle by one lane, then the wavefront factor.
template <typename S>
__device__ int wformt(S* wt, const S* sy, const S* ss, int col, S theta, int lane) {
  constexpr int ld = kMaxM;
  if (lane < col) LB_AT(wt, ld, 1, lane + 1) = theta * LB_AT(ss, ld, 1, lane + 1);
  #pragma unroll 1
  for (int q = lane; q < col * col; q += 32) {
    const int i = q / col + 1, j = q % col + 1;
    if (i < 2 || j < i) continue;
    const int k1 = (i < j ? i : j) - 1;
    S ddum = 0;
    #pragma unroll 1
    for (int k = 1; k <= k1; k++) ddum = ddum + LB_AT(sy, ld, i, k) * LB_AT(sy, ld, j, k) / LB_AT(sy, ld, k, k);
    LB_AT(wt, ld, i, j) = ddum + theta * LB_AT(ss, ld, i, j);
  }
  __syncwarp();
  return wdpofa(wt, ld, col, lane) ? 0 : -3;
}

// sformk.  snap holds 4 kMaxM^2 scalars: the shift of wn1 writes every entry from one to
// its lower right that the serial loops have not yet rewritten, so each write is a copy
// from a snapshot taken before it.  The serial loops write entry (r, c) of three regions,
// (c <= r <= m-1), (m+1 <= c <= r <= 2m-1) and (m+1 <= r <= 2m-1, c <= m-1), each from
// (r+1, c+1).  Items are dealt to the lanes by index (q = lane, lane + 32, ...), so that
// the lanes work at the same time.
template <typename S>
__device__ int wformk(int m, int col, int updatd, int iupdat, S theta, const S* sy, S* wn,
                      S* wn1, const FormkSums<S>& fs, S* wm, S* snap, int lane) {
  constexpr int L2 = 2 * kMaxM;
  int upcl;
  if (updatd) {
    if (iupdat > m) {
      #pragma unroll 1
      for (int e = lane; e < L2 * L2; e += 32) snap[e] = wn1[e];
      __syncwarp();
      #pragma unroll 1
      for (int e = lane; e < L2 * L2; e += 32) {
        const int r = e / L2 + 1, c = e % L2 + 1;
        const bool lo = c <= r && r <= m - 1;
        const bool hi = m + 1 <= c && c <= r && r <= 2 * m - 1;
        const bool mid = m + 1 <= r && r <= 2 * m - 1 && c <= m - 1;
        if (lo || hi || mid) LB_AT(wn1, L2, r, c) = LB_AT(snap, L2, r + 1, c + 1);
      }
      __syncwarp();
    }
    if (lane < col) {
      const int jy = lane + 1;
      LB_AT(wn1, L2, col, jy) = fs.yy_new[jy - 1];
      LB_AT(wn1, L2, m + col, m + jy) = fs.ss_new[jy - 1];
      LB_AT(wn1, L2, m + col, jy) = fs.sy_row[jy - 1];
    }
    __syncwarp();
    if (lane < col) LB_AT(wn1, L2, m + lane + 1, col) = fs.sy_col[lane];
    __syncwarp();
    upcl = col - 1;
  } else {
    upcl = col;
  }
  #pragma unroll 1
  for (int q = lane; q < upcl * upcl; q += 32) {
    const int iy = q / upcl + 1, jy = q % upcl + 1;
    if (jy <= iy) {
      LB_AT(wn1, L2, iy, jy) = LB_AT(wn1, L2, iy, jy) + fs.dyy[iy - 1][jy - 1];
      LB_AT(wn1, L2, m + iy, m + jy) = LB_AT(wn1, L2, m + iy, m + jy) - fs.dss[iy - 1][jy - 1];
    }
    if (iy <= jy)
      LB_AT(wn1, L2, m + iy, jy) = LB_AT(wn1, L2, m + iy, jy) + fs.dsy[iy - 1][jy - 1];
    else
      LB_AT(wn1, L2, m + iy, jy) = LB_AT(wn1, L2, m + iy, jy) - fs.dsy[iy - 1][jy - 1];
  }
  __syncwarp();
  // K's assembly: the three blocks of the upper triangle, entry by entry
  #pragma unroll 1
  for (int q = lane; q < col * col; q += 32) {
    const int iy = q / col + 1, jy = q % col + 1;
    const int iis = col + iy, is1 = m + iy;
    if (jy <= iy) {
      S v = LB_AT(wn1, L2, iy, jy) / theta;
      if (jy == iy) v = v + LB_AT(sy, kMaxM, iy, iy);
      LB_AT(wn, L2, jy, iy) = v;
      LB_AT(wn, L2, col + jy, iis) = LB_AT(wn1, L2, is1, m + jy) * theta;
    }
    LB_AT(wn, L2, jy, iis) = jy < iy ? -LB_AT(wn1, L2, is1, jy) : LB_AT(wn1, L2, is1, jy);
  }
  __syncwarp();
  if (!wdpofa(wn, L2, col, lane)) return -1;
  // L_a^{-1} of the upper right block, one column per lane (its info is not used)
  if (wdiag_zero(wn, L2, col, lane) == 0 && lane < col) {
    S* b = &LB_AT(wn, L2, 1, col + 1 + lane);
    b[0] = b[0] / LB_AT(wn, L2, 1, 1);
    #pragma unroll 1
    for (int j = 2; j <= col; j++) {
      const S v = sdot(&LB_AT(wn, L2, 1, j), L2, b, L2, j - 1);
      b[(j - 1) * L2] = b[(j - 1) * L2] - v;
      b[(j - 1) * L2] = b[(j - 1) * L2] / LB_AT(wn, L2, j, j);
    }
  }
  __syncwarp();
  #pragma unroll 1
  for (int q = lane; q < col * col; q += 32) {
    const int iis = col + 1 + q / col, js = col + 1 + q % col;
    if (js < iis) continue;
    const S v = sdot(&LB_AT(wn, L2, 1, iis), L2, &LB_AT(wn, L2, 1, js), L2, col);
    LB_AT(wn, L2, iis, js) = LB_AT(wn, L2, iis, js) + v;
  }
  __syncwarp();
  #pragma unroll 1
  for (int e = lane; e < col * col; e += 32) {
    const int j = e / col + 1, i = e % col + 1;
    LB_AT(wm, kMaxM, j, i) = LB_AT(wn, L2, col + j, col + i);
  }
  __syncwarp();
  if (!wdpofa(wm, kMaxM, col, lane)) return -2;
  #pragma unroll 1
  for (int e = lane; e < col * col; e += 32) {
    const int j = e / col + 1, i = e % col + 1;
    LB_AT(wn, L2, col + j, col + i) = LB_AT(wm, kMaxM, j, i);
  }
  __syncwarp();
  return 0;
}

}  // namespace lbfgsb_b200
