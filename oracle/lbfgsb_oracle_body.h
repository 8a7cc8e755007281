/*
 * lbfgsb_oracle_body.h -- TEST INFRASTRUCTURE (the oracle).  Type-generic body of the
 * plain-C restatement of the reference's CPU L-BFGS-B, included twice by lbfgsb_oracle.c
 * with REAL = double / float.  Only tests, smoke() and bench.py's CPU legs use it.
 *
 * Every routine restates the reference routine named in its comment
 * (culbfgsb/lbfgsbcpu.cpp, L-BFGS-B 2.1 lineage) with the same arithmetic in the same
 * order, so that, compiled by gcc -O2 for x86-64 (SSE2, no FMA contraction), it
 * reproduces the reference build bit for bit.  Arrays use 1-based index macros to keep
 * the correspondence with the reference readable; storage is 0-based C arrays.
 *
 * Required macros: REAL, SFX (f64/f32), SQRT, FABS, OPT_T, SUM_T, CB_T.
 */

#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

/* 1-based accessors.  Vectors: v[i] with i in 1..len (allocated len+1).
 * n x m history (row-major, like the reference's 2-D AP arrays): H(i, j).
 * Small square matrices of leading dimension ld: M(i, j). */
#define V1(v, i) ((v)[(i)])
#define HM(h, m, i, j) ((h)[((size_t)(i)-1) * (size_t)(m) + (size_t)(j)-1])
#define SQ(a, ld, i, j) ((a)[((i)-1) * (ld) + (j)-1])

/* ap::vdotproduct / _vdotproduct (culbfgsb/apvt.h:87-148): groups of four products
 * summed left to right, each group added to the running sum, then the tail. */
static REAL FN(dot)(const REAL* a, long sa, const REAL* b, long sb, int len) {
  REAL r = 0;
  int groups = len / 4, i;
  for (i = 0; i < groups; i++) {
    r += a[0] * b[0] + a[sa] * b[sb] + a[2 * sa] * b[2 * sb] + a[3 * sa] * b[3 * sb];
    a += 4 * sa;
    b += 4 * sb;
  }
  for (i = 0; i < len % 4; i++) {
    r += a[0] * b[0];
    a += sa;
    b += sb;
  }
  return r;
}

static REAL FN(maxr)(REAL a, REAL b) { return a > b ? a : b; } /* ap::maxreal */
static REAL FN(minr)(REAL a, REAL b) { return a > b ? b : a; } /* ap::minreal */

/* lbfgsberrclb, lbfgsbcpu.cpp:871-905 */
static void FN(errclb)(int n, int m, REAL factr, const REAL* l, const REAL* u,
                       const int* nbd, int* task, int* info, int* k) {
  int i;
  if (n <= 0) *task = 2;
  if (m <= 0) *task = 2;
  if (m > n) *task = 2;
  if (factr < 0) *task = 2;
  for (i = 1; i <= n; i++) {
    if (V1(nbd, i) < 0 || V1(nbd, i) > 3) {
      *task = 2;
      *info = -6;
      *k = i;
    }
    if (V1(nbd, i) == 2 && V1(l, i) > V1(u, i)) {
      *task = 2;
      *info = -7;
      *k = i;
    }
  }
}

/* lbfgsbactive, lbfgsbcpu.cpp:467-515: project x into the box, initial iwhere. */
static void FN(active)(int n, const REAL* l, const REAL* u, const int* nbd, REAL* x,
                       int* iwhere, int* prjctd, int* cnstnd, int* boxed) {
  int i;
  *prjctd = 0;
  *cnstnd = 0;
  *boxed = 1;
  for (i = 1; i <= n; i++) {
    int b = V1(nbd, i);
    if (b > 0) {
      if (b <= 2 && V1(x, i) <= V1(l, i)) {
        if (V1(x, i) < V1(l, i)) {
          *prjctd = 1;
          V1(x, i) = V1(l, i);
        }
      } else if (b >= 2 && V1(x, i) >= V1(u, i)) {
        if (V1(x, i) > V1(u, i)) {
          *prjctd = 1;
          V1(x, i) = V1(u, i);
        }
      }
    }
  }
  for (i = 1; i <= n; i++) {
    int b = V1(nbd, i);
    if (b != 2) *boxed = 0;
    if (b == 0) {
      V1(iwhere, i) = -1;
    } else {
      *cnstnd = 1;
      V1(iwhere, i) = (b == 2 && V1(u, i) - V1(l, i) <= 0) ? 3 : 0;
    }
  }
}

/* lbfgsbprojgr, lbfgsbcpu.cpp:1389-1414: infinity norm of the projected gradient. */
static REAL FN(projgr)(int n, const REAL* l, const REAL* u, const int* nbd,
                       const REAL* x, const REAL* g) {
  REAL sbgnrm = 0;
  int i;
  for (i = 1; i <= n; i++) {
    REAL gi = V1(g, i);
    int b = V1(nbd, i);
    if (b != 0) {
      if (gi < 0) {
        if (b >= 2) gi = FN(maxr)(V1(x, i) - V1(u, i), gi);
      } else {
        if (b <= 2) gi = FN(minr)(V1(x, i) - V1(l, i), gi);
      }
    }
    sbgnrm = FN(maxr)(sbgnrm, (REAL)FABS(gi));
  }
  return sbgnrm;
}

/* lbfgsbdpofa, lbfgsbcpu.cpp:1876-1908: Cholesky (upper factor in place) of the
 * leading n x n block of a (leading dimension ld).  Returns 0 on a non-positive pivot. */
static int FN(dpofa)(REAL* a, int ld, int n) {
  int j, k;
  for (j = 1; j <= n; j++) {
    REAL s = 0.0;
    for (k = 1; k <= j - 1; k++) {
      /* column k rows 1..k-1 against column j rows 1..k-1 */
      REAL v = FN(dot)(&SQ(a, ld, 1, k), ld, &SQ(a, ld, 1, j), ld, k - 1);
      REAL t = SQ(a, ld, k, j) - v;
      t = t / SQ(a, ld, k, k);
      SQ(a, ld, k, j) = t;
      s = s + t * t;
    }
    s = SQ(a, ld, j, j) - s;
    if (s <= 0.0) return 0;
    SQ(a, ld, j, j) = SQRT(s);
  }
  return 1;
}

/* lbfgsbdtrsl, lbfgsbcpu.cpp:1910-1986, for an upper-triangular t (the only form the
 * solver uses): job 01 solves t*x = b, job 11 solves t'*x = b.  b is 1-based. */
static void FN(dtrsl)(REAL* t, int ld, int n, REAL* b, int job, int* info) {
  int j, jj;
  for (j = 1; j <= n; j++) {
    if (SQ(t, ld, j, j) == 0.0) {
      *info = j;
      return;
    }
  }
  *info = 0;
  if (job == 1) { /* case 2: back substitution with columns */
    V1(b, n) = V1(b, n) / SQ(t, ld, n, n);
    if (n < 2) return;
    for (jj = 2; jj <= n; jj++) {
      int i;
      REAL temp;
      j = n - jj + 1;
      temp = -V1(b, j + 1);
      for (i = 1; i <= j; i++) V1(b, i) += temp * SQ(t, ld, i, j + 1);
      V1(b, j) = V1(b, j) / SQ(t, ld, j, j);
    }
    return;
  }
  /* job == 11, case 4: forward substitution with transposed columns */
  V1(b, 1) = V1(b, 1) / SQ(t, ld, 1, 1);
  if (n < 2) return;
  for (j = 2; j <= n; j++) {
    REAL v = FN(dot)(&SQ(t, ld, 1, j), ld, &V1(b, 1), 1, j - 1);
    V1(b, j) = V1(b, j) - v;
    V1(b, j) = V1(b, j) / SQ(t, ld, j, j);
  }
}

/* lbfgsbbmv, lbfgsbcpu.cpp:517-565: p = M v for the 2col x 2col middle matrix given
 * by sy and the Cholesky factor wt of T = theta*S'S + L D^-1 L'. */
static void FN(bmv)(int m, const REAL* sy, REAL* wt, int col, const REAL* v, REAL* p,
                    int* info, REAL* work) {
  int i, k;
  REAL s;
  if (col == 0) return;
  V1(p, col + 1) = V1(v, col + 1);
  for (i = 2; i <= col; i++) {
    s = 0.0;
    for (k = 1; k <= i - 1; k++)
      s = s + SQ(sy, m, i, k) * V1(v, k) / SQ(sy, m, k, k);
    V1(p, col + i) = V1(v, col + i) + s;
  }
  for (i = 1; i <= col; i++) V1(work, i) = V1(p, col + i);
  FN(dtrsl)(wt, m, col, work, 11, info);
  for (i = 1; i <= col; i++) V1(p, col + i) = V1(work, i);
  if (*info != 0) return;
  for (i = 1; i <= col; i++) V1(p, i) = V1(v, i) / SQRT(SQ(sy, m, i, i));
  for (i = 1; i <= col; i++) V1(work, i) = V1(p, col + i);
  FN(dtrsl)(wt, m, col, work, 1, info);
  for (i = 1; i <= col; i++) V1(p, col + i) = V1(work, i);
  if (*info != 0) return;
  for (i = 1; i <= col; i++) V1(p, i) = -V1(p, i) / SQRT(SQ(sy, m, i, i));
  for (i = 1; i <= col; i++) {
    s = 0;
    for (k = i + 1; k <= col; k++)
      s = s + SQ(sy, m, k, i) * V1(p, col + k) / SQ(sy, m, i, i);
    V1(p, i) = V1(p, i) + s;
  }
}

/* lbfgsbhpsolb, lbfgsbcpu.cpp:1175-1233: heap of the breakpoints t(1..n); when iheap==0
 * the heap is built first; then the least element is moved to position n. */
static void FN(hpsolb)(int n, REAL* t, int* iorder, int iheap) {
  int i, j, k, indxin, indxou;
  REAL ddum, dout;
  if (iheap == 0) {
    for (k = 2; k <= n; k++) {
      ddum = V1(t, k);
      indxin = V1(iorder, k);
      i = k;
      while (i > 1) {
        j = i / 2;
        if (!(ddum < V1(t, j))) break;
        V1(t, i) = V1(t, j);
        V1(iorder, i) = V1(iorder, j);
        i = j;
      }
      V1(t, i) = ddum;
      V1(iorder, i) = indxin;
    }
  }
  if (n > 1) {
    i = 1;
    dout = V1(t, 1);
    indxou = V1(iorder, 1);
    ddum = V1(t, n);
    indxin = V1(iorder, n);
    for (;;) {
      j = i + i;
      if (j > n - 1) break;
      if (V1(t, j + 1) < V1(t, j)) j = j + 1;
      if (!(V1(t, j) < ddum)) break;
      V1(t, i) = V1(t, j);
      V1(iorder, i) = V1(iorder, j);
      i = j;
    }
    V1(t, i) = ddum;
    V1(iorder, i) = indxin;
    V1(t, n) = dout;
    V1(iorder, n) = indxou;
  }
}

typedef struct {
  int nbreak, nint, early; /* early: returned before the walk (no breakpoints, no free) */
  REAL dtm, tsum, f1_0, f2_0;
} FN(gcp_out);

/* lbfgsbcauchy, lbfgsbcpu.cpp:567-817: generalized Cauchy point by the sequential
 * breakpoint walk.  p = wa(1..2m), c = wa(2m+1..4m), wbp = wa(4m+1..), v = wa(6m+1..). */
static void FN(cauchy)(int n, const REAL* x, const REAL* l, const REAL* u, const int* nbd,
                       const REAL* g, int* iorder, int* iwhere, REAL* t, REAL* d,
                       REAL* xcp, int m, const REAL* wy, const REAL* ws, const REAL* sy,
                       REAL* wt, REAL theta, int col, int head, REAL* p, REAL* c,
                       REAL* wbp, REAL* v, int* nint, REAL sbgnrm, int* info, REAL* work,
                       FN(gcp_out) * out) {
  int bnded = 1, i, j, col2 = 2 * col, nfree = n + 1, nbreak = 0, ibkmin = 0;
  int pointr, ibp, nleft, iter;
  REAL f1 = 0, f2, f2org, dt, dtm, tsum, dibp, zibp, dibp2, bkmin = 0, tu = 0, tl = 0;
  REAL wmc, wmp, wmw, tj, tj0, neggi;

  out->early = 0;
  out->nbreak = 0;
  if (sbgnrm <= 0) {
    for (i = 1; i <= n; i++) V1(xcp, i) = V1(x, i);
    out->early = 1;
    return;
  }
  for (i = 1; i <= col2; i++) V1(p, i) = 0;
  /* scan: iwhere update, direction d = -g on movable variables, p = W'd, breakpoints */
  for (i = 1; i <= n; i++) {
    int b = V1(nbd, i);
    neggi = -V1(g, i);
    if (V1(iwhere, i) != 3 && V1(iwhere, i) != -1) {
      int xlower, xupper;
      tl = 0;
      tu = 0;
      if (b <= 2) tl = V1(x, i) - V1(l, i);
      if (b >= 2) tu = V1(u, i) - V1(x, i);
      xlower = b <= 2 && tl <= 0;
      xupper = b >= 2 && tu <= 0;
      V1(iwhere, i) = 0;
      if (xlower) {
        if (neggi <= 0) V1(iwhere, i) = 1;
      } else if (xupper) {
        if (neggi >= 0) V1(iwhere, i) = 2;
      } else if (FABS(neggi) <= 0) {
        V1(iwhere, i) = -3;
      }
    }
    pointr = head;
    if (V1(iwhere, i) != 0 && V1(iwhere, i) != -1) {
      V1(d, i) = 0;
    } else {
      V1(d, i) = neggi;
      f1 = f1 - neggi * neggi;
      for (j = 1; j <= col; j++) {
        V1(p, j) = V1(p, j) + HM(wy, m, i, pointr) * neggi;
        V1(p, col + j) = V1(p, col + j) + HM(ws, m, i, pointr) * neggi;
        pointr = pointr % m + 1;
      }
      if (b <= 2 && b != 0 && neggi < 0) {
        nbreak = nbreak + 1;
        V1(iorder, nbreak) = i;
        V1(t, nbreak) = tl / (-neggi);
        if (nbreak == 1 || V1(t, nbreak) < bkmin) {
          bkmin = V1(t, nbreak);
          ibkmin = nbreak;
        }
      } else if (b >= 2 && neggi > 0) {
        nbreak = nbreak + 1;
        V1(iorder, nbreak) = i;
        V1(t, nbreak) = tu / neggi;
        if (nbreak == 1 || V1(t, nbreak) < bkmin) {
          bkmin = V1(t, nbreak);
          ibkmin = nbreak;
        }
      } else {
        nfree = nfree - 1;
        V1(iorder, nfree) = i;
        if (FABS(neggi) > 0) bnded = 0;
      }
    }
  }
  out->nbreak = nbreak;
  if (theta != 1) {
    for (j = col + 1; j <= col2; j++) V1(p, j) *= theta;
  }
  for (i = 1; i <= n; i++) V1(xcp, i) = V1(x, i);
  if (nbreak == 0 && nfree == n + 1) {
    out->early = 1;
    return;
  }
  for (j = 1; j <= col2; j++) V1(c, j) = 0;
  f2 = -theta * f1;
  f2org = f2;
  if (col > 0) {
    FN(bmv)(m, sy, wt, col, p, v, info, work);
    if (*info != 0) return;
    f2 = f2 - FN(dot)(&V1(v, 1), 1, &V1(p, 1), 1, col2);
  }
  dtm = -f1 / f2;
  out->f1_0 = f1;
  out->f2_0 = f2;
  tsum = 0;
  *nint = 1;
  if (nbreak != 0) {
    nleft = nbreak;
    iter = 1;
    tj = 0;
    for (;;) {
      tj0 = tj;
      if (iter == 1) {
        tj = bkmin;
        ibp = V1(iorder, ibkmin);
      } else {
        if (iter == 2 && ibkmin != nbreak) {
          V1(t, ibkmin) = V1(t, nbreak);
          V1(iorder, ibkmin) = V1(iorder, nbreak);
        }
        FN(hpsolb)(nleft, t, iorder, iter - 2);
        tj = V1(t, nleft);
        ibp = V1(iorder, nleft);
      }
      dt = tj - tj0;
      if (dtm < dt) break;
      /* the breakpoint is passed: fix variable ibp at its bound */
      tsum = tsum + dt;
      nleft = nleft - 1;
      iter = iter + 1;
      dibp = V1(d, ibp);
      V1(d, ibp) = 0;
      if (dibp > 0) {
        zibp = V1(u, ibp) - V1(x, ibp);
        V1(xcp, ibp) = V1(u, ibp);
        V1(iwhere, ibp) = 2;
      } else {
        zibp = V1(l, ibp) - V1(x, ibp);
        V1(xcp, ibp) = V1(l, ibp);
        V1(iwhere, ibp) = 1;
      }
      if (nleft == 0 && nbreak == n) {
        dtm = dt;
        if (col > 0)
          for (j = 1; j <= col2; j++) V1(c, j) += dtm * V1(p, j);
        out->dtm = dtm;
        out->tsum = tsum;
        return;
      }
      *nint = *nint + 1;
      dibp2 = dibp * dibp;
      f1 = f1 + dt * f2 + dibp2 - theta * dibp * zibp;
      f2 = f2 - theta * dibp2;
      if (col > 0) {
        for (j = 1; j <= col2; j++) V1(c, j) += dt * V1(p, j);
        pointr = head;
        for (j = 1; j <= col; j++) {
          V1(wbp, j) = HM(wy, m, ibp, pointr);
          V1(wbp, col + j) = theta * HM(ws, m, ibp, pointr);
          pointr = pointr % m + 1;
        }
        FN(bmv)(m, sy, wt, col, wbp, v, info, work);
        if (*info != 0) return;
        wmc = FN(dot)(&V1(c, 1), 1, &V1(v, 1), 1, col2);
        wmp = FN(dot)(&V1(p, 1), 1, &V1(v, 1), 1, col2);
        wmw = FN(dot)(&V1(wbp, 1), 1, &V1(v, 1), 1, col2);
        for (j = 1; j <= col2; j++) V1(p, j) += (-dibp) * V1(wbp, j);
        f1 = f1 + dibp * wmc;
        f2 = f2 + (REAL)2.0 * dibp * wmp - dibp2 * wmw;
      }
      f2 = FN(maxr)((REAL)(5E-16 * f2org), f2);
      if (nleft > 0) {
        dtm = -f1 / f2;
        continue;
      }
      if (bnded) {
        f1 = 0;
        f2 = 0;
        dtm = 0;
      } else {
        dtm = -f1 / f2;
      }
      break;
    }
  }
  if (dtm <= 0) dtm = 0;
  tsum = tsum + dtm;
  for (i = 1; i <= n; i++) V1(xcp, i) += tsum * V1(d, i);
  if (col > 0)
    for (j = 1; j <= col2; j++) V1(c, j) += dtm * V1(p, j);
  out->dtm = dtm;
  out->tsum = tsum;
}

/* lbfgsbfreev, lbfgsbcpu.cpp:1135-1173: free/active partition of iwhere, and the
 * variables that entered / left the free set since the previous call. */
static void FN(freev)(int n, int* nfree, int* index, int* nenter, int* ileave, int* indx2,
                      const int* iwhere, int* wrk, int updatd, int cnstnd, int iter) {
  int i, k, iact;
  *nenter = 0;
  *ileave = n + 1;
  if (iter > 0 && cnstnd) {
    for (i = 1; i <= *nfree; i++) {
      k = V1(index, i);
      if (V1(iwhere, k) > 0) {
        *ileave = *ileave - 1;
        V1(indx2, *ileave) = k;
      }
    }
    for (i = 1 + *nfree; i <= n; i++) {
      k = V1(index, i);
      if (V1(iwhere, k) <= 0) {
        *nenter = *nenter + 1;
        V1(indx2, *nenter) = k;
      }
    }
  }
  *wrk = *ileave < n + 1 || *nenter > 0 || updatd;
  *nfree = 0;
  iact = n + 1;
  for (i = 1; i <= n; i++) {
    if (V1(iwhere, i) <= 0) {
      *nfree = *nfree + 1;
      V1(index, *nfree) = i;
    } else {
      iact = iact - 1;
      V1(index, iact) = i;
    }
  }
}

/* lbfgsbformk, lbfgsbcpu.cpp:907-1103: the 2col x 2col matrix K of the subspace
 * problem, kept incrementally in wn1 (ld 2m) and factored into wn (ld 2m). */
static void FN(formk)(int n, int nsub, const int* ind, int nenter, int ileave,
                      const int* indx2, int iupdat, int updatd, REAL* wn, REAL* wn1,
                      int m, const REAL* ws, const REAL* wy, const REAL* sy, REAL theta,
                      int col, int head, int* info, REAL* work, REAL* workmat) {
  int m2 = 2 * m, ipntr, jpntr, iy, iis, jy, js, is1, js1, k1, i, k, col2, upcl, j;
  REAL temp1, temp2, temp3, temp4, v;

  if (updatd) {
    if (iupdat > m) {
      /* shift the old part of wn1 up and left by one position */
      for (jy = 1; jy <= m - 1; jy++) {
        js = m + jy;
        for (i = 0; i <= m - 1 - jy; i++) SQ(wn1, m2, jy + i, jy) = SQ(wn1, m2, jy + 1 + i, jy + 1);
        for (i = 0; i <= m - 1 - jy; i++) SQ(wn1, m2, js + i, js) = SQ(wn1, m2, js + 1 + i, js + 1);
        for (i = 0; i <= m - 2; i++) SQ(wn1, m2, m + 1 + i, jy) = SQ(wn1, m2, m + 2 + i, jy + 1);
      }
    }
    /* new row of Y'Y over the free set and of S'S, S'Y over the active set */
    iy = col;
    iis = m + col;
    ipntr = head + col - 1;
    if (ipntr > m) ipntr = ipntr - m;
    jpntr = head;
    for (jy = 1; jy <= col; jy++) {
      js = m + jy;
      temp1 = 0;
      temp2 = 0;
      temp3 = 0;
      for (k = 1; k <= nsub; k++) {
        k1 = V1(ind, k);
        temp1 = temp1 + HM(wy, m, k1, ipntr) * HM(wy, m, k1, jpntr);
      }
      for (k = nsub + 1; k <= n; k++) {
        k1 = V1(ind, k);
        temp2 = temp2 + HM(ws, m, k1, ipntr) * HM(ws, m, k1, jpntr);
        temp3 = temp3 + HM(ws, m, k1, ipntr) * HM(wy, m, k1, jpntr);
      }
      SQ(wn1, m2, iy, jy) = temp1;
      SQ(wn1, m2, iis, js) = temp2;
      SQ(wn1, m2, iis, jy) = temp3;
      jpntr = jpntr % m + 1;
    }
    /* new column of S'Y over the free set */
    jy = col;
    jpntr = head + col - 1;
    if (jpntr > m) jpntr = jpntr - m;
    ipntr = head;
    for (i = 1; i <= col; i++) {
      iis = m + i;
      temp3 = 0;
      for (k = 1; k <= nsub; k++) {
        k1 = V1(ind, k);
        temp3 = temp3 + HM(ws, m, k1, ipntr) * HM(wy, m, k1, jpntr);
      }
      ipntr = ipntr % m + 1;
      SQ(wn1, m2, iis, jy) = temp3;
    }
    upcl = col - 1;
  } else {
    upcl = col;
  }
  /* corrections of the older rows for the variables that entered / left the free set */
  ipntr = head;
  for (iy = 1; iy <= upcl; iy++) {
    iis = m + iy;
    jpntr = head;
    for (jy = 1; jy <= iy; jy++) {
      js = m + jy;
      temp1 = 0;
      temp2 = 0;
      temp3 = 0;
      temp4 = 0;
      for (k = 1; k <= nenter; k++) {
        k1 = V1(indx2, k);
        temp1 = temp1 + HM(wy, m, k1, ipntr) * HM(wy, m, k1, jpntr);
        temp2 = temp2 + HM(ws, m, k1, ipntr) * HM(ws, m, k1, jpntr);
      }
      for (k = ileave; k <= n; k++) {
        k1 = V1(indx2, k);
        temp3 = temp3 + HM(wy, m, k1, ipntr) * HM(wy, m, k1, jpntr);
        temp4 = temp4 + HM(ws, m, k1, ipntr) * HM(ws, m, k1, jpntr);
      }
      SQ(wn1, m2, iy, jy) = SQ(wn1, m2, iy, jy) + temp1 - temp3;
      SQ(wn1, m2, iis, js) = SQ(wn1, m2, iis, js) - temp2 + temp4;
      jpntr = jpntr % m + 1;
    }
    ipntr = ipntr % m + 1;
  }
  ipntr = head;
  for (iis = m + 1; iis <= m + upcl; iis++) {
    jpntr = head;
    for (jy = 1; jy <= upcl; jy++) {
      temp1 = 0;
      temp3 = 0;
      for (k = 1; k <= nenter; k++) {
        k1 = V1(indx2, k);
        temp1 = temp1 + HM(ws, m, k1, ipntr) * HM(wy, m, k1, jpntr);
      }
      for (k = ileave; k <= n; k++) {
        k1 = V1(indx2, k);
        temp3 = temp3 + HM(ws, m, k1, ipntr) * HM(wy, m, k1, jpntr);
      }
      if (iis <= jy + m)
        SQ(wn1, m2, iis, jy) = SQ(wn1, m2, iis, jy) + temp1 - temp3;
      else
        SQ(wn1, m2, iis, jy) = SQ(wn1, m2, iis, jy) - temp1 + temp3;
      jpntr = jpntr % m + 1;
    }
    ipntr = ipntr % m + 1;
  }
  /* assemble the upper triangle of K from wn1 */
  for (iy = 1; iy <= col; iy++) {
    iis = col + iy;
    is1 = m + iy;
    for (jy = 1; jy <= iy; jy++) {
      js = col + jy;
      js1 = m + jy;
      SQ(wn, m2, jy, iy) = SQ(wn1, m2, iy, jy) / theta;
      SQ(wn, m2, js, iis) = SQ(wn1, m2, is1, js1) * theta;
    }
    for (jy = 1; jy <= iy - 1; jy++) SQ(wn, m2, jy, iis) = -SQ(wn1, m2, is1, jy);
    for (jy = iy; jy <= col; jy++) SQ(wn, m2, jy, iis) = SQ(wn1, m2, is1, jy);
    SQ(wn, m2, iy, iy) = SQ(wn, m2, iy, iy) + SQ(sy, m, iy, iy);
  }
  /* factor: upper-left Cholesky, off-diagonal solve, Schur complement, its Cholesky */
  *info = 0;
  if (!FN(dpofa)(wn, m2, col)) {
    *info = -1;
    return;
  }
  col2 = 2 * col;
  for (js = col + 1; js <= col2; js++) {
    for (i = 1; i <= col; i++) V1(work, i) = SQ(wn, m2, i, js);
    FN(dtrsl)(wn, m2, col, work, 11, info);
    for (i = 1; i <= col; i++) SQ(wn, m2, i, js) = V1(work, i);
  }
  for (iis = col + 1; iis <= col2; iis++) {
    for (js = iis; js <= col2; js++) {
      v = FN(dot)(&SQ(wn, m2, 1, iis), m2, &SQ(wn, m2, 1, js), m2, col);
      SQ(wn, m2, iis, js) = SQ(wn, m2, iis, js) + v;
    }
  }
  for (j = 1; j <= col; j++)
    for (i = 1; i <= col; i++) SQ(workmat, m, j, i) = SQ(wn, m2, col + j, col + i);
  *info = 0;
  if (!FN(dpofa)(workmat, m, col)) {
    *info = -2;
    return;
  }
  for (j = 1; j <= col; j++)
    for (i = 1; i <= col; i++) SQ(wn, m2, col + j, col + i) = SQ(workmat, m, j, i);
}

/* lbfgsbformt, lbfgsbcpu.cpp:1105-1133: wt = chol(theta*SS + L D^-1 L'). */
static void FN(formt)(int m, REAL* wt, const REAL* sy, const REAL* ss, int col,
                      REAL theta, int* info) {
  int i, j, k;
  for (j = 1; j <= col; j++) SQ(wt, m, 1, j) = theta * SQ(ss, m, 1, j);
  for (i = 2; i <= col; i++) {
    for (j = i; j <= col; j++) {
      int k1 = (i < j ? i : j) - 1;
      REAL ddum = 0;
      for (k = 1; k <= k1; k++)
        ddum = ddum + SQ(sy, m, i, k) * SQ(sy, m, j, k) / SQ(sy, m, k, k);
      SQ(wt, m, i, j) = ddum + theta * SQ(ss, m, i, j);
    }
  }
  *info = FN(dpofa)(wt, m, col) ? 0 : -3;
}

/* lbfgsbcmprlb, lbfgsbcpu.cpp:819-869: reduced gradient r = -Z'(B(xcp - x) + g). */
static void FN(cmprlb)(int n, int m, const REAL* x, const REAL* g, const REAL* ws,
                       const REAL* wy, const REAL* sy, REAL* wt, const REAL* z, REAL* r,
                       REAL* wa, const int* index, REAL theta, int col, int head,
                       int nfree, int cnstnd, int* info, REAL* work, REAL* work2) {
  int i, j, k, pointr;
  if (!cnstnd && col > 0) {
    for (i = 1; i <= n; i++) V1(r, i) = -V1(g, i);
    return;
  }
  for (i = 1; i <= nfree; i++) {
    k = V1(index, i);
    V1(r, i) = -theta * (V1(z, k) - V1(x, k)) - V1(g, k);
  }
  for (i = 1; i <= 2 * m; i++) V1(work2, i) = V1(wa, 2 * m + i);
  FN(bmv)(m, sy, wt, col, work2, wa, info, work); /* wa(1..2col) = M c */
  for (i = 1; i <= 2 * m; i++) V1(wa, 2 * m + i) = V1(work2, i);
  if (*info != 0) {
    *info = -8;
    return;
  }
  pointr = head;
  for (j = 1; j <= col; j++) {
    REAL a1 = V1(wa, j), a2 = theta * V1(wa, col + j);
    for (i = 1; i <= nfree; i++) {
      k = V1(index, i);
      V1(r, i) = V1(r, i) + HM(wy, m, k, pointr) * a1 + HM(ws, m, k, pointr) * a2;
    }
    pointr = pointr % m + 1;
  }
}

/* lbfgsbsubsm, lbfgsbcpu.cpp:1416-1539: subspace Newton step on the free set, then the
 * L-BFGS-B 2.1 truncation of the step at the first bound it meets.  x here is xcp; xx and
 * gg are the iterate and its gradient, used by the 3.0 option only. */
static void FN(subsm)(int n, int m, int nsub, const int* ind, const REAL* l,
                      const REAL* u, const int* nbd, REAL* x, REAL* d, const REAL* ws,
                      const REAL* wy, REAL theta, int col, int head, int* iword, REAL* wv,
                      REAL* wn, int* info, const REAL* xx, const REAL* gg) {
  int pointr, col2, ibd = 0, jy, js, i, j, k;
  REAL alpha, dk, temp1, temp2;
  if (nsub <= 0) return;
  pointr = head;
  for (i = 1; i <= col; i++) {
    temp1 = 0;
    temp2 = 0;
    for (j = 1; j <= nsub; j++) {
      k = V1(ind, j);
      temp1 = temp1 + HM(wy, m, k, pointr) * V1(d, j);
      temp2 = temp2 + HM(ws, m, k, pointr) * V1(d, j);
    }
    V1(wv, i) = temp1;
    V1(wv, col + i) = theta * temp2;
    pointr = pointr % m + 1;
  }
  col2 = 2 * col;
  FN(dtrsl)(wn, 2 * m, col2, wv, 11, info);
  if (*info != 0) return;
  for (i = 1; i <= col; i++) V1(wv, i) = -V1(wv, i);
  FN(dtrsl)(wn, 2 * m, col2, wv, 1, info);
  if (*info != 0) return;
  pointr = head;
  for (jy = 1; jy <= col; jy++) {
    js = col + jy;
    for (i = 1; i <= nsub; i++) {
      k = V1(ind, i);
      V1(d, i) = V1(d, i) + HM(wy, m, k, pointr) * V1(wv, jy) / theta +
                 HM(ws, m, k, pointr) * V1(wv, js);
    }
    pointr = pointr % m + 1;
  }
  for (i = 1; i <= nsub; i++) V1(d, i) = V1(d, i) / theta;
  if (g_subsm_projection) {
    /* L-BFGS-B 3.0 (J. L. Morales and J. Nocedal, "Remark on Algorithm 778", ACM TOMS
     * 38(1), 2011): project xcp + d onto the box, variable by variable (the lower bound,
     * then the upper one).  If no variable lands on a bound, that is the step; if some do,
     * keep the projected point when (x_p - xx)'gg <= 0, a descent direction from the
     * iterate, and otherwise fall back to the 2.1 truncated step below. */
    int projected = 0;
    REAL ddp = 0;
    REAL* keep = (REAL*)malloc(sizeof(REAL) * (size_t)(nsub + 1));
    for (i = 1; i <= nsub; i++) {
      const int lo = V1(nbd, V1(ind, i)) == 1 || V1(nbd, V1(ind, i)) == 2;
      const int hi = V1(nbd, V1(ind, i)) == 2 || V1(nbd, V1(ind, i)) == 3;
      k = V1(ind, i);
      V1(keep, i) = V1(x, k);
      temp1 = V1(x, k) + V1(d, i);
      if (lo) temp1 = FN(maxr)(V1(l, k), temp1);
      if (hi) temp1 = FN(minr)(V1(u, k), temp1);
      if ((lo && temp1 == V1(l, k)) || (hi && temp1 == V1(u, k))) projected = 1;
      V1(x, k) = temp1;
    }
    if (!projected) {
      free(keep);
      *iword = 0;
      return;
    }
    for (i = 1; i <= n; i++) ddp = ddp + (V1(x, i) - V1(xx, i)) * V1(gg, i);
    if (ddp <= 0) {
      free(keep);
      *iword = 1;
      return;
    }
    for (i = 1; i <= nsub; i++) V1(x, V1(ind, i)) = V1(keep, i);
    free(keep);
  }
  /* step length to the first bound (temp1 carries across variables, as in the source) */
  alpha = 1;
  temp1 = alpha;
  for (i = 1; i <= nsub; i++) {
    k = V1(ind, i);
    dk = V1(d, i);
    if (V1(nbd, k) != 0) {
      if (dk < 0 && V1(nbd, k) <= 2) {
        temp2 = V1(l, k) - V1(x, k);
        if (temp2 >= 0)
          temp1 = 0;
        else if (dk * alpha < temp2)
          temp1 = temp2 / dk;
      } else if (dk > 0 && V1(nbd, k) >= 2) {
        temp2 = V1(u, k) - V1(x, k);
        if (temp2 <= 0)
          temp1 = 0;
        else if (dk * alpha > temp2)
          temp1 = temp2 / dk;
      }
      if (temp1 < alpha) {
        alpha = temp1;
        ibd = i;
      }
    }
  }
  if (alpha < 1) {
    dk = V1(d, ibd);
    k = V1(ind, ibd);
    if (dk > 0) {
      V1(x, k) = V1(u, k);
      V1(d, ibd) = 0;
    } else if (dk < 0) {
      V1(x, k) = V1(l, k);
      V1(d, ibd) = 0;
    }
  }
  for (i = 1; i <= nsub; i++) {
    k = V1(ind, i);
    V1(x, k) = V1(x, k) + alpha * V1(d, i);
  }
  *iword = alpha < 1 ? 1 : 0;
}

/* lbfgsbdcstep, lbfgsbcpu.cpp:1737-1874: safeguarded cubic/quadratic step. */
static void FN(dcstep)(REAL* stx, REAL* fx, REAL* dx, REAL* sty, REAL* fy, REAL* dy,
                       REAL* stp, REAL fp, REAL dp, int* brackt, REAL stpmin,
                       REAL stpmax) {
  REAL gamma, p, q, r, s, sgnd, stpc, stpf, stpq, theta;
  sgnd = dp * (*dx / (REAL)FABS(*dx));
  if (fp > *fx) {
    theta = 3 * (*fx - fp) / (*stp - *stx) + *dx + dp;
    s = FN(maxr)((REAL)FABS(theta), FN(maxr)((REAL)FABS(*dx), (REAL)FABS(dp)));
    gamma = s * SQRT((theta / s) * (theta / s) - *dx / s * (dp / s));
    if (*stp < *stx) gamma = -gamma;
    p = gamma - *dx + theta;
    q = gamma - *dx + gamma + dp;
    r = p / q;
    stpc = *stx + r * (*stp - *stx);
    stpq = *stx + *dx / ((*fx - fp) / (*stp - *stx) + *dx) / 2 * (*stp - *stx);
    if (FABS(stpc - *stx) < FABS(stpq - *stx))
      stpf = stpc;
    else
      stpf = stpc + (stpq - stpc) / 2;
    *brackt = 1;
  } else if (sgnd < 0) {
    theta = 3 * (*fx - fp) / (*stp - *stx) + *dx + dp;
    s = FN(maxr)((REAL)FABS(theta), FN(maxr)((REAL)FABS(*dx), (REAL)FABS(dp)));
    gamma = s * SQRT((theta / s) * (theta / s) - *dx / s * (dp / s));
    if (*stp > *stx) gamma = -gamma;
    p = gamma - dp + theta;
    q = gamma - dp + gamma + *dx;
    r = p / q;
    stpc = *stp + r * (*stx - *stp);
    stpq = *stp + dp / (dp - *dx) * (*stx - *stp);
    stpf = (FABS(stpc - *stp) > FABS(stpq - *stp)) ? stpc : stpq;
    *brackt = 1;
  } else if (FABS(dp) < FABS(*dx)) {
    theta = 3 * (*fx - fp) / (*stp - *stx) + *dx + dp;
    s = FN(maxr)((REAL)FABS(theta), FN(maxr)((REAL)FABS(*dx), (REAL)FABS(dp)));
    gamma = s * SQRT(FN(maxr)((REAL)0, (theta / s) * (theta / s) - *dx / s * (dp / s)));
    if (*stp > *stx) gamma = -gamma;
    p = gamma - dp + theta;
    q = gamma + (*dx - dp) + gamma;
    r = p / q;
    if (r < 0 && gamma != 0)
      stpc = *stp + r * (*stx - *stp);
    else
      stpc = (*stp > *stx) ? stpmax : stpmin;
    stpq = *stp + dp / (dp - *dx) * (*stx - *stp);
    if (*brackt) {
      stpf = (FABS(stpc - *stp) < FABS(stpq - *stp)) ? stpc : stpq;
      /* the reference evaluates stp + 0.66*(sty - stp) in double */
      if (*stp > *stx)
        stpf = FN(minr)((REAL)((double)*stp + 0.66 * (double)(*sty - *stp)), stpf);
      else
        stpf = FN(maxr)((REAL)((double)*stp + 0.66 * (double)(*sty - *stp)), stpf);
    } else {
      stpf = (FABS(stpc - *stp) > FABS(stpq - *stp)) ? stpc : stpq;
      stpf = FN(minr)(stpmax, stpf);
      stpf = FN(maxr)(stpmin, stpf);
    }
  } else {
    if (*brackt) {
      theta = 3 * (fp - *fy) / (*sty - *stp) + *dy + dp;
      s = FN(maxr)((REAL)FABS(theta), FN(maxr)((REAL)FABS(*dy), (REAL)FABS(dp)));
      gamma = s * SQRT((theta / s) * (theta / s) - *dy / s * (dp / s));
      if (*stp > *sty) gamma = -gamma;
      p = gamma - dp + theta;
      q = gamma - dp + gamma + *dy;
      r = p / q;
      stpc = *stp + r * (*sty - *stp);
      stpf = stpc;
    } else {
      stpf = (*stp > *stx) ? stpmax : stpmin;
    }
  }
  if (fp > *fx) {
    *sty = *stp;
    *fy = fp;
    *dy = dp;
  } else {
    if (sgnd < 0) {
      *sty = *stx;
      *fy = *fx;
      *dy = *dx;
    }
    *stx = *stp;
    *fx = fp;
    *dx = dp;
  }
  *stp = stpf;
}

/* lbfgsbdcsrch, lbfgsbcpu.cpp:1541-1735: More'-Thuente line search driver.  The saved
 * state lives in isave[1..2] / dsave[1..13] between calls, as in the source.  task: 0
 * start, 1 evaluate, 2 error, 3 warning, 4 converged. */
static void FN(dcsrch)(REAL f, REAL g, REAL* stp, REAL ftol, REAL gtol, REAL xtol,
                       REAL stpmin, REAL stpmax, int* task, int* isave, REAL* dsave) {
  int brackt, stage;
  REAL finit, ftest, fm, fx, fxm, fy, fym, ginit, gtest, gm, gx, gxm, gy, gym, stx, sty,
      stmin, stmax, width, width1;
  const REAL xtrapl = (REAL)1.1E0, xtrapu = (REAL)4.0E0;
  if (*task == 0) {
    if (*stp < stpmin) *task = 2;
    if (*stp > stpmax) *task = 2;
    if (g >= 0) *task = 2;
    if (ftol < 0) *task = 2;
    if (gtol < 0) *task = 2;
    if (xtol < 0) *task = 2;
    if (stpmin < 0) *task = 2;
    if (stpmax < stpmin) *task = 2;
    if (*task == 2) return;
    brackt = 0;
    stage = 1;
    finit = f;
    ginit = g;
    gtest = ftol * ginit;
    width = stpmax - stpmin;
    width1 = width / (REAL)0.5;
    stx = 0;
    fx = finit;
    gx = ginit;
    sty = 0;
    fy = finit;
    gy = ginit;
    stmin = 0;
    stmax = *stp + xtrapu * *stp;
    *task = 1;
    goto save;
  }
  brackt = isave[1] == 1;
  stage = isave[2];
  ginit = dsave[1];
  gtest = dsave[2];
  gx = dsave[3];
  gy = dsave[4];
  finit = dsave[5];
  fx = dsave[6];
  fy = dsave[7];
  stx = dsave[8];
  sty = dsave[9];
  stmin = dsave[10];
  stmax = dsave[11];
  width = dsave[12];
  width1 = dsave[13];
  ftest = finit + *stp * gtest;
  if (stage == 1 && f <= ftest && g >= 0) stage = 2;
  if (brackt && (*stp <= stmin || *stp >= stmax)) *task = 3;
  if (brackt && stmax - stmin <= xtol * stmax) *task = 3;
  if (*stp == stpmax && f <= ftest && g <= gtest) *task = 3;
  if (*stp == stpmin && (f > ftest || g >= gtest)) *task = 3;
  if (f <= ftest && FABS(g) <= gtol * (-ginit)) *task = 4;
  if (*task == 3 || *task == 4) goto save;
  if (stage == 1 && f <= fx && f > ftest) {
    fm = f - *stp * gtest;
    fxm = fx - stx * gtest;
    fym = fy - sty * gtest;
    gm = g - gtest;
    gxm = gx - gtest;
    gym = gy - gtest;
    FN(dcstep)(&stx, &fxm, &gxm, &sty, &fym, &gym, stp, fm, gm, &brackt, stmin, stmax);
    fx = fxm + stx * gtest;
    fy = fym + sty * gtest;
    gx = gxm + gtest;
    gy = gym + gtest;
  } else {
    FN(dcstep)(&stx, &fx, &gx, &sty, &fy, &gy, stp, f, g, &brackt, stmin, stmax);
  }
  if (brackt) {
    if ((REAL)FABS(sty - stx) >= (REAL)0.66 * width1) *stp = stx + (REAL)0.5 * (sty - stx);
    width1 = width;
    width = (REAL)FABS(sty - stx);
  }
  if (brackt) {
    stmin = FN(minr)(stx, sty);
    stmax = FN(maxr)(stx, sty);
  } else {
    stmin = *stp + xtrapl * (*stp - stx);
    stmax = *stp + xtrapu * (*stp - stx);
  }
  *stp = FN(maxr)(*stp, stpmin);
  *stp = FN(minr)(*stp, stpmax);
  if ((brackt && (*stp <= stmin || *stp >= stmax)) || (brackt && stmax - stmin <= xtol * stmax))
    *stp = stx;
  *task = 1;
save:
  isave[1] = brackt ? 1 : 0;
  isave[2] = stage;
  dsave[1] = ginit;
  dsave[2] = gtest;
  dsave[3] = gx;
  dsave[4] = gy;
  dsave[5] = finit;
  dsave[6] = fx;
  dsave[7] = fy;
  dsave[8] = stx;
  dsave[9] = sty;
  dsave[10] = stmin;
  dsave[11] = stmax;
  dsave[12] = width;
  dsave[13] = width1;
}

typedef struct {
  REAL f, fold, gd, gdold, stp, dnrm, dtd, xstep, stpmx;
  int iter, ifun, iback, nfgv, info, task, boxed, cnstnd, csave;
  int isave[3];
  REAL dsave[14];
} FN(lnsrch_state);

/* lbfgsblnsrlb, lbfgsbcpu.cpp:1235-1339: one step of the projected line search. */
static void FN(lnsrlb)(int n, const REAL* l, const REAL* u, const int* nbd, REAL* x,
                       const REAL* g, const REAL* d, REAL* r, REAL* t, const REAL* z,
                       FN(lnsrch_state) * s) {
  const REAL big = (REAL)1.0E10, ftol = (REAL)1.0E-3, gtol = (REAL)0.9E0,
             xtol = (REAL)0.1E0;
  int i;
  if (s->task != 1) {
    s->dtd = FN(dot)(&V1(d, 1), 1, &V1(d, 1), 1, n);
    s->dnrm = SQRT(s->dtd);
    s->stpmx = big;
    if (s->cnstnd) {
      if (s->iter == 0) {
        s->stpmx = 1;
      } else {
        for (i = 1; i <= n; i++) {
          REAL a1 = V1(d, i), a2;
          if (V1(nbd, i) != 0) {
            if (a1 < 0 && V1(nbd, i) <= 2) {
              a2 = V1(l, i) - V1(x, i);
              if (a2 >= 0)
                s->stpmx = 0;
              else if (a1 * s->stpmx < a2)
                s->stpmx = a2 / a1;
            } else if (a1 > 0 && V1(nbd, i) >= 2) {
              a2 = V1(u, i) - V1(x, i);
              if (a2 <= 0)
                s->stpmx = 0;
              else if (a1 * s->stpmx > a2)
                s->stpmx = a2 / a1;
            }
          }
        }
      }
    }
    if (s->iter == 0 && !s->boxed)
      s->stp = FN(minr)(1 / s->dnrm, s->stpmx);
    else
      s->stp = 1;
    for (i = 1; i <= n; i++) V1(t, i) = V1(x, i);
    for (i = 1; i <= n; i++) V1(r, i) = V1(g, i);
    s->fold = s->f;
    s->ifun = 0;
    s->iback = 0;
    s->csave = 0;
  }
  s->gd = FN(dot)(&V1(g, 1), 1, &V1(d, 1), 1, n);
  if (s->ifun == 0) {
    s->gdold = s->gd;
    if (s->gd >= 0) {
      s->info = -4;
      return;
    }
  }
  FN(dcsrch)(s->f, s->gd, &s->stp, ftol, gtol, xtol, 0, s->stpmx, &s->csave, s->isave,
             s->dsave);
  s->xstep = s->stp * s->dnrm;
  if (s->csave != 4 && s->csave != 3) {
    s->task = 1;
    s->ifun = s->ifun + 1;
    s->nfgv = s->nfgv + 1;
    s->iback = s->ifun - 1;
    if (s->stp == 1) {
      for (i = 1; i <= n; i++) V1(x, i) = V1(z, i);
    } else {
      for (i = 1; i <= n; i++) V1(x, i) = s->stp * V1(d, i) + V1(t, i);
    }
  } else {
    s->task = 5;
  }
}

/* lbfgsbmatupd, lbfgsbcpu.cpp:1341-1387: push (s, y) = (d, r) into the ring and update
 * the S'Y (lower) and S'S (upper) matrices. */
static void FN(matupd)(int n, int m, REAL* ws, REAL* wy, REAL* sy, REAL* ss, const REAL* d,
                       const REAL* r, int* itail, int iupdat, int* col, int* head,
                       REAL* theta, REAL rr, REAL dr, REAL stp, REAL dtd) {
  int i, j, pointr;
  if (iupdat <= m) {
    *col = iupdat;
    *itail = (*head + iupdat - 2) % m + 1;
  } else {
    *itail = *itail % m + 1;
    *head = *head % m + 1;
  }
  for (i = 1; i <= n; i++) {
    HM(ws, m, i, *itail) = V1(d, i);
    HM(wy, m, i, *itail) = V1(r, i);
  }
  *theta = rr / dr;
  if (iupdat > m) {
    for (j = 1; j <= *col - 1; j++) {
      for (i = 1; i <= j; i++) SQ(ss, m, i, j) = SQ(ss, m, i + 1, j + 1);
      for (i = j; i <= *col - 1; i++) SQ(sy, m, i, j) = SQ(sy, m, i + 1, j + 1);
    }
  }
  pointr = *head;
  for (j = 1; j <= *col - 1; j++) {
    SQ(sy, m, *col, j) = FN(dot)(&V1(d, 1), 1, &HM(wy, m, 1, pointr), m, n);
    SQ(ss, m, j, *col) = FN(dot)(&HM(ws, m, 1, pointr), m, &V1(d, 1), 1, n);
    pointr = pointr % m + 1;
  }
  SQ(ss, m, *col, *col) = (stp == 1) ? dtd : stp * stp * dtd;
  SQ(sy, m, *col, *col) = dr;
}

static unsigned long long FN(mix64)(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static void FN(copy_summary)(SUM_T* dst, const SUM_T* src) { *dst = *src; }

/* lbfgsbminimize, lbfgsbcpu.cpp:117-465: the outer loop. */
void CAT2(orc_lbfgsb_minimize, SFX)(int n, REAL* x_, const int* nbd_, const REAL* l_,
                                    const REAL* u_, const OPT_T* opt, CB_T funcgrad,
                                    CB_T after_iter, CB_T custom_stop, void* user,
                                    orc_trace_cb trace, void* trace_user, SUM_T* summary) {
  int m = opt->hessian_approximate_dimension < 8 ? opt->hessian_approximate_dimension : 8;
  int mm = m > 0 ? m : 1, m2 = 2 * mm;
  size_t n1 = (size_t)(n > 0 ? n : 0) + 1;
  REAL *x, *l, *u, *g, *xold, *xdiff, *ws, *wy, *sy, *ss, *wt, *wn, *snd, *z, *r, *d, *t;
  REAL *wa, *wa0, *wa1, *wa2, *wa3, *work, *work2, *workmat;
  int *nbd, *index, *iwhere, *indx2;
  int i, k = 0, task = 0, prjctd, cnstnd, boxed, updatd = 0, wrk = 0, head = 1, col = 0,
         iter = 0, itail = 0, iupdat = 0, nint = 0, internalinfo = 0, iword = -1,
         nfree = n, ileave = 0, nenter = 0, reset_pending = 0;
  REAL theta = 1, sbgnrm, tf, ddum, rr, dr;
  FN(lnsrch_state) ls;
  FN(gcp_out) gout;
  orc_trace_rec rec;

  memset(&ls, 0, sizeof(ls));
  memset(&rec, 0, sizeof(rec));
  /* 1-based working copies (lbfgsbcpu.cpp:122-130) */
  x = (REAL*)calloc(n1, sizeof(REAL));
  l = (REAL*)calloc(n1, sizeof(REAL));
  u = (REAL*)calloc(n1, sizeof(REAL));
  nbd = (int*)calloc(n1, sizeof(int));
  for (i = 1; i < (int)n1; i++) {
    x[i] = x_[i - 1];
    l[i] = l_[i - 1];
    u[i] = u_[i - 1];
    nbd[i] = nbd_[i - 1];
  }
  g = (REAL*)calloc(n1, sizeof(REAL));
  xold = (REAL*)calloc(n1, sizeof(REAL));
  xdiff = (REAL*)calloc(n1, sizeof(REAL));
  z = (REAL*)calloc(n1, sizeof(REAL));
  r = (REAL*)calloc(n1, sizeof(REAL));
  d = (REAL*)calloc(n1, sizeof(REAL));
  t = (REAL*)calloc(n1, sizeof(REAL));
  ws = (REAL*)calloc(n1 * mm, sizeof(REAL));
  wy = (REAL*)calloc(n1 * mm, sizeof(REAL));
  sy = (REAL*)calloc((size_t)mm * mm, sizeof(REAL));
  ss = (REAL*)calloc((size_t)mm * mm, sizeof(REAL));
  wt = (REAL*)calloc((size_t)mm * mm, sizeof(REAL));
  workmat = (REAL*)calloc((size_t)mm * mm, sizeof(REAL));
  wn = (REAL*)calloc((size_t)m2 * m2, sizeof(REAL));
  snd = (REAL*)calloc((size_t)m2 * m2, sizeof(REAL));
  wa = (REAL*)calloc(8 * (size_t)mm + 1, sizeof(REAL));
  wa0 = (REAL*)calloc(2 * (size_t)mm + 1, sizeof(REAL));
  wa1 = (REAL*)calloc(2 * (size_t)mm + 1, sizeof(REAL));
  wa2 = (REAL*)calloc(2 * (size_t)mm + 1, sizeof(REAL));
  wa3 = (REAL*)calloc(2 * (size_t)mm + 1, sizeof(REAL));
  work = (REAL*)calloc(2 * (size_t)mm + 1, sizeof(REAL));
  work2 = (REAL*)calloc(2 * (size_t)mm + 1, sizeof(REAL));
  index = (int*)calloc(n1, sizeof(int));
  iwhere = (int*)calloc(n1, sizeof(int));
  indx2 = (int*)calloc(n1, sizeof(int));

#define FINISH(code)                                         \
  do {                                                       \
    summary->info = (code);                                  \
    for (i = 1; i < (int)n1; i++) x_[i - 1] = x[i];          \
    goto cleanup;                                            \
  } while (0)

  FN(errclb)(n, m, opt->eps_f, l, u, nbd, &task, &internalinfo, &k);
  if (task == 2 || opt->max_iteration < 0 || opt->eps_g < 0 || opt->eps_x < 0) FINISH(-1);
  internalinfo = 0;
  FN(active)(n, l, u, nbd, x, iwhere, &prjctd, &cnstnd, &boxed);
  ls.cnstnd = cnstnd;
  ls.boxed = boxed;
  for (i = 1; i <= n; i++) xold[i] = x[i];
  if (funcgrad) funcgrad(user, &x[1], &ls.f, &g[1], summary);
  ls.nfgv = 1;
  sbgnrm = FN(projgr)(n, l, u, nbd, x, g);
  summary->residual_g = sbgnrm;
  if (sbgnrm <= opt->eps_g) FINISH(4);

  for (;;) {
    int gcp_skipped = 0;
    REAL* p = wa0; /* cauchy's p, c, wbp, v live in wa (lbfgsbcpu.cpp:286-296) */
    iword = -1;
    gout.nbreak = 0;
    gout.dtm = 0;
    gout.tsum = 0;
    gout.f1_0 = 0;
    gout.f2_0 = 0;
    nenter = 0;
    ileave = n + 1;
    if (!cnstnd && col > 0) {
      for (i = 1; i <= n; i++) z[i] = x[i];
      wrk = updatd;
      nint = 0;
      gcp_skipped = 1;
    } else {
      for (i = 1; i <= 2 * m; i++) {
        wa0[i] = wa[i];
        wa1[i] = wa[2 * m + i];
        wa2[i] = wa[4 * m + i];
        wa3[i] = wa[6 * m + i];
      }
      FN(cauchy)(n, x, l, u, nbd, g, indx2, iwhere, t, d, z, m, wy, ws, sy, wt, theta, col,
                 head, p, wa1, wa2, wa3, &nint, sbgnrm, &internalinfo, work, &gout);
      for (i = 1; i <= 2 * m; i++) {
        wa[i] = wa0[i];
        wa[2 * m + i] = wa1[i];
        wa[4 * m + i] = wa2[i];
        wa[6 * m + i] = wa3[i];
      }
      if (internalinfo != 0) {
        internalinfo = 0;
        col = 0;
        head = 1;
        theta = 1;
        iupdat = 0;
        updatd = 0;
        reset_pending = 1;
        continue;
      }
      FN(freev)(n, &nfree, index, &nenter, &ileave, indx2, iwhere, &wrk, updatd, cnstnd, iter);
    }
    if (nfree != 0 && col != 0) {
      if (wrk)
        FN(formk)(n, nfree, index, nenter, ileave, indx2, iupdat, updatd, wn, snd, m, ws, wy,
                  sy, theta, col, head, &internalinfo, work, workmat);
      if (internalinfo != 0) {
        internalinfo = 0;
        col = 0;
        head = 1;
        theta = 1;
        iupdat = 0;
        updatd = 0;
        reset_pending = 1;
        continue;
      }
      FN(cmprlb)(n, m, x, g, ws, wy, sy, wt, z, r, wa, index, theta, col, head, nfree, cnstnd,
                 &internalinfo, work, work2);
      if (internalinfo == 0)
        FN(subsm)(n, m, nfree, index, l, u, nbd, z, r, ws, wy, theta, col, head, &iword, wa,
                  wn, &internalinfo, x, g);
      if (internalinfo != 0) {
        internalinfo = 0;
        col = 0;
        head = 1;
        theta = 1;
        iupdat = 0;
        updatd = 0;
        reset_pending = 1;
        continue;
      }
    }
    /* trace: what this iteration's step was built from */
    rec.nint = gcp_skipped ? 0 : nint;
    rec.nbreak = gout.nbreak;
    rec.nfree = nfree;
    rec.nenter = nenter;
    rec.nleave = n + 1 - ileave;
    rec.col = col;
    rec.head = head;
    rec.theta = theta;
    rec.dtm = gout.dtm;
    rec.tsum = gout.tsum;
    rec.f1_0 = gout.f1_0;
    rec.f2_0 = gout.f2_0;
    rec.dbg[0] = col > 0 ? wa[1] : 0;
    rec.dbg[1] = col > 0 ? wa[col + 1] : 0;
    rec.dbg[2] = col > 0 ? wa[2 * m + 1] : 0;
    rec.dbg[3] = col > 0 ? wa[2 * m + col + 1] : 0;
    rec.dbg[4] = 0;
    rec.dbg[5] = 0;
    rec.dbg[6] = col > 0 ? sy[0] : 0;
    rec.dbg[7] = col > 0 ? wt[0] : 0;
    rec.iword = iword;
    rec.reset = reset_pending;
    reset_pending = 0;
    if (trace) {
      unsigned long long hsh = 0, lo = 0, up = 0;
      for (i = 1; i <= n; i++) {
        if (iwhere[i] <= 0) hsh += FN(mix64)((unsigned long long)(i - 1));
        if (iwhere[i] == 1) lo++;
        if (iwhere[i] == 2) up++;
      }
      rec.free_hash = hsh;
      rec.at_lower = lo;
      rec.at_upper = up;
    }

    for (i = 1; i <= n; i++) d[i] = z[i] - x[i];
    ls.task = 0;
    ls.iter = iter;
    ls.info = 0;
    for (;;) {
      FN(lnsrlb)(n, l, u, nbd, x, g, d, r, t, z, &ls);
      if (ls.info != 0 || ls.iback >= 20 || ls.task != 1) break;
      if (funcgrad) funcgrad(user, &x[1], &ls.f, &g[1], summary);
    }
    internalinfo = ls.info;
    if (internalinfo != 0) {
      for (i = 1; i <= n; i++) {
        x[i] = t[i];
        g[i] = r[i];
      }
      ls.f = ls.fold;
      if (col == 0) {
        iter = iter + 1;
        FINISH(-2);
      }
      internalinfo = 0;
      ls.info = 0;
      col = 0;
      head = 1;
      theta = 1;
      iupdat = 0;
      updatd = 0;
      reset_pending = 1;
      continue;
    }
    iter = iter + 1;
    summary->num_iteration = iter;
    if (trace) {
      rec.iter = iter;
      rec.f = ls.f;
      rec.stp = ls.stp;
      rec.gd = ls.gd;
      rec.gdold = ls.gdold;
      rec.dtd = ls.dtd;
      rec.stpmx = ls.stpmx;
      rec.nfgv = ls.nfgv;
      rec.ifun = ls.ifun;
      trace(trace_user, &rec);
    }
    if (after_iter) after_iter(user, &x[1], &ls.f, &g[1], summary);
    sbgnrm = FN(projgr)(n, l, u, nbd, x, g);
    summary->residual_g = sbgnrm;
    if (sbgnrm <= opt->eps_g) FINISH(4);
    for (i = 1; i <= n; i++) xdiff[i] = xold[i];
    for (i = 1; i <= n; i++) xdiff[i] -= x[i];
    tf = FN(dot)(&xdiff[1], 1, &xdiff[1], 1, n);
    tf = SQRT(tf);
    summary->residual_x = tf;
    if (tf <= opt->eps_x) FINISH(2);
    ddum = FN(maxr)((REAL)FABS(ls.fold), FN(maxr)((REAL)FABS(ls.f), (REAL)1));
    summary->residual_f = (ls.fold - ls.f) / ddum;
    if (ls.fold - ls.f <= opt->eps_f * ddum) FINISH(1);
    if (iter > opt->max_iteration && opt->max_iteration > 0) FINISH(5);
    if (custom_stop && custom_stop(user, &x[1], &ls.f, &g[1], summary)) FINISH(0);
    for (i = 1; i <= n; i++) xold[i] = x[i];
    for (i = 1; i <= n; i++) r[i] = g[i] - r[i];
    rr = FN(dot)(&r[1], 1, &r[1], 1, n);
    if (ls.stp == 1) {
      dr = ls.gd - ls.gdold;
      ddum = -ls.gdold;
    } else {
      dr = (ls.gd - ls.gdold) * ls.stp;
      for (i = 1; i <= n; i++) d[i] *= ls.stp;
      ddum = -ls.gdold * ls.stp;
    }
    if ((double)dr <= 5E-16 * (double)ddum) {
      updatd = 0;
    } else {
      updatd = 1;
      iupdat = iupdat + 1;
      FN(matupd)(n, m, ws, wy, sy, ss, d, r, &itail, iupdat, &col, &head, &theta, rr, dr,
                 ls.stp, ls.dtd);
      FN(formt)(m, wt, sy, ss, col, theta, &internalinfo);
      if (internalinfo != 0) {
        internalinfo = 0;
        col = 0;
        head = 1;
        theta = 1;
        iupdat = 0;
        updatd = 0;
        reset_pending = 1;
        continue;
      }
    }
  }
cleanup:
  free(x);
  free(l);
  free(u);
  free(nbd);
  free(g);
  free(xold);
  free(xdiff);
  free(z);
  free(r);
  free(d);
  free(t);
  free(ws);
  free(wy);
  free(sy);
  free(ss);
  free(wt);
  free(workmat);
  free(wn);
  free(snd);
  free(wa);
  free(wa0);
  free(wa1);
  free(wa2);
  free(wa3);
  free(work);
  free(work2);
  free(index);
  free(iwhere);
  free(indx2);
#undef FINISH
  (void)FN(copy_summary);
  (void)prjctd;
}

#undef FN
#undef CAT2
#undef CAT2_
#undef V1
#undef HM
#undef SQ
