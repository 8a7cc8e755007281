/*
 * objective.c -- TEST INFRASTRUCTURE: CPU evaluation of the synthetic objective that every
 * parity case and the CPU baseline minimise (the reference ships no such objective; its
 * only example is MINPACK-2 dsscfg).  On an s x s grid, k = j*s + i, h = 1/(s+1), zero
 * Dirichlet neighbours:
 *
 *   f(x) = sum_k 0.5*kappa_k*((x_{i+1,j}-x_k)^2 + (x_{i,j+1}-x_k)^2)
 *        + h^2 * sum_k [ w_k*softplus(x_k - t_k) - b_k*x_k + 0.05*cos(3*x_k) ]
 *
 * (the h^2 of the stated form multiplies the 1/h^2 of the difference quotients).  f is
 * accumulated in double in index order; the f32 variant evaluates each term in float.
 */
#include <math.h>

#include "oracle_api.h"

static double softplus_d(double z) { return (z > 0 ? z : 0.0) + log1p(exp(-fabs(z))); }
static double sigmoid_d(double z) {
  if (z >= 0) return 1.0 / (1.0 + exp(-z));
  double e = exp(z);
  return e / (1.0 + e);
}
static float softplus_f(float z) { return (z > 0 ? z : 0.0f) + log1pf(expf(-fabsf(z))); }
static float sigmoid_f(float z) {
  if (z >= 0) return 1.0f / (1.0f + expf(-z));
  float e = expf(z);
  return e / (1.0f + e);
}

void orc_synth_eval_off_f64(int s, const double* kappa, const double* w, const double* t,
                            const double* b, double f0, const double* x, double* f, double* g) {
  const double h = 1.0 / (double)(s + 1), h2 = h * h;
  double acc = 0.0;
  long k;
  int i, j;
  for (j = 0; j < s; j++) {
    for (i = 0; i < s; i++) {
      k = (long)j * s + i;
      double xk = x[k];
      double xe = (i + 1 < s) ? x[k + 1] : 0.0;
      double xn = (j + 1 < s) ? x[k + s] : 0.0;
      double de = xe - xk, dn = xn - xk;
      double z = xk - t[k];
      acc += 0.5 * kappa[k] * (de * de + dn * dn) +
             h2 * (w[k] * softplus_d(z) - b[k] * xk + 0.05 * cos(3.0 * xk));
      if (g) {
        double gk = -kappa[k] * (de + dn);
        if (i > 0) gk += kappa[k - 1] * (xk - x[k - 1]);
        if (j > 0) gk += kappa[k - s] * (xk - x[k - s]);
        gk += h2 * (w[k] * sigmoid_d(z) - b[k] - 0.15 * sin(3.0 * xk));
        g[k] = gk;
      }
    }
  }
  *f = acc - f0;
}

void orc_synth_eval_off_f32(int s, const double* kappa, const double* w, const double* t,
                            const double* b, double f0, const float* x, float* f, float* g) {
  const float h = 1.0f / (float)(s + 1), h2 = h * h;
  double acc = 0.0;
  long k;
  int i, j;
  for (j = 0; j < s; j++) {
    for (i = 0; i < s; i++) {
      k = (long)j * s + i;
      float xk = x[k];
      float xe = (i + 1 < s) ? x[k + 1] : 0.0f;
      float xn = (j + 1 < s) ? x[k + s] : 0.0f;
      float de = xe - xk, dn = xn - xk;
      float kk = (float)kappa[k], wk = (float)w[k], bk = (float)b[k];
      float z = xk - (float)t[k];
      float term = 0.5f * kk * (de * de + dn * dn) +
                   h2 * (wk * softplus_f(z) - bk * xk + 0.05f * cosf(3.0f * xk));
      acc += (double)term;
      if (g) {
        float gk = -kk * (de + dn);
        if (i > 0) gk += (float)kappa[k - 1] * (xk - x[k - 1]);
        if (j > 0) gk += (float)kappa[k - s] * (xk - x[k - s]);
        gk += h2 * (wk * sigmoid_f(z) - bk - 0.15f * sinf(3.0f * xk));
        g[k] = gk;
      }
    }
  }
  *f = (float)(acc - f0);
}

/* The objective minus a constant f0, subtracted from the double sum before f is rounded to
 * the caller's precision: the minimiser and g are unchanged, while a float f keeps the
 * resolution of the decrease near f0 (on a 4096 x 4096 grid f is about 0.45 and an
 * iteration lowers it by about 1e-8, below the spacing of floats there). */
void orc_synth_eval_f64(int s, const double* kappa, const double* w, const double* t,
                        const double* b, const double* x, double* f, double* g) {
  orc_synth_eval_off_f64(s, kappa, w, t, b, 0.0, x, f, g);
}

void orc_synth_eval_f32(int s, const double* kappa, const double* w, const double* t,
                        const double* b, const float* x, float* f, float* g) {
  orc_synth_eval_off_f32(s, kappa, w, t, b, 0.0, x, f, g);
}

/* Separable quadratic f = sum_k 0.5*a_k*(x_k - c_k)^2 (ties and zero gradients on demand:
 * equal a_k and c_k give equal breakpoints; c_k == x_k gives a zero gradient). */
void orc_quad_eval_f64(int n, const double* a, const double* c, const double* x, double* f,
                       double* g) {
  double acc = 0.0;
  int k;
  for (k = 0; k < n; k++) {
    double r = x[k] - c[k];
    acc += 0.5 * a[k] * r * r;
    if (g) g[k] = a[k] * r;
  }
  *f = acc;
}

void orc_quad_eval_f32(int n, const double* a, const double* c, const float* x, float* f,
                       float* g) {
  double acc = 0.0;
  int k;
  for (k = 0; k < n; k++) {
    float r = x[k] - (float)c[k];
    float ak = (float)a[k];
    acc += (double)(0.5f * ak * r * r);
    if (g) g[k] = ak * r;
  }
  *f = (float)acc;
}

/* ---- dsscfg: MINPACK-2 steady-state combustion (Averick, Carter, More, Xue, "The
 * MINPACK-2 test problem collection", 1992), in the variant of the reference's example
 * (examples/dsscfg/dsscfg_cpu.cpp:16-147): nx x ny nodes, k = nx*j + i, h = 1/(n+1),
 * zero values outside the grid, two triangles per node (lower: the node, its right and
 * top neighbours; upper: the node, its left and bottom neighbours),
 *
 *   f = area * (0.5 * sum dv^2 terms + fexp),  fexp = -lambda/3 * sum over triangles of
 *   the exponentials of their three corners (trapezoidal rule), area = hx*hy/2.
 *
 * f sums the triangles in the reference's order (j, then i, lower then upper).  The
 * gradient is gathered per node from the (up to) six triangles that touch it, added in
 * the reference's order: own lower + own upper, then the triangles of the nodes above,
 * right, left and below.  The f32 variant repeats the reference's float expressions
 * including their promotions to double (the literals 3.0 and 0.5 are doubles there, and
 * its unqualified exp of a float is the C library's double exp, rounded to float). */

static float expd_f(float v) { return (float)exp((double)v); }

void orc_dsscfg_start_f64(int nx, int ny, double lam, double* x) {
  const double hx = 1.0 / (double)(nx + 1), hy = 1.0 / (double)(ny + 1);
  const double c = lam / (lam + 1.0);
  int i, j;
  for (j = 0; j < ny; j++) {
    const double ty = (double)(j < ny - j ? j : ny - j) * hy;
    for (i = 0; i < nx; i++) {
      const double tx = (double)(i < nx - i ? i : nx - i) * hx;
      x[(long)nx * j + i] = c * sqrt(ty < tx ? ty : tx);
    }
  }
}

void orc_dsscfg_start_f32(int nx, int ny, float lam, float* x) {
  const float hx = (float)(1.0 / (double)(float)(nx + 1));
  const float hy = (float)(1.0 / (double)(float)(ny + 1));
  const float c = (float)((double)lam / ((double)lam + 1.0));
  int i, j;
  for (j = 0; j < ny; j++) {
    const float ty = (float)(j < ny - j ? j : ny - j) * hy;
    for (i = 0; i < nx; i++) {
      const float tx = (float)(i < nx - i ? i : nx - i) * hx;
      x[(long)nx * j + i] = c * sqrtf(ty < tx ? ty : tx);
    }
  }
}

void orc_dsscfg_eval_f64(int nx, int ny, double lam, const double* x, double* f, double* g) {
  const double hx = 1.0 / (double)(nx + 1), hy = 1.0 / (double)(ny + 1);
  const double area = 0.5 * hx * hy;
  double fquad = 0.0, fexp = 0.0;
  int i, j;
  for (j = 0; j < ny; j++) {
    for (i = 0; i < nx; i++) {
      const long k = (long)nx * j + i;
      const double v = x[k];
      const double vr = i < nx - 1 ? x[k + 1] : 0.0, vt = j < ny - 1 ? x[k + nx] : 0.0;
      const double vl = i > 0 ? x[k - 1] : 0.0, vb = j > 0 ? x[k - nx] : 0.0;
      double dx = (vr - v) / hx, dy = (vt - v) / hy;
      fquad += dx * dx + dy * dy;
      fexp = fexp - lam * (exp(v) + exp(vr) + exp(vt)) / 3.0;
      dx = (v - vl) / hx;
      dy = (v - vb) / hy;
      fquad += dx * dx + dy * dy;
      fexp = fexp - lam * (exp(vb) + exp(vl) + exp(v)) / 3.0;
      if (g) {
        const double e3 = lam * exp(v) / 3.0;
        double gk = 0.0 + (-((vr - v) / hx) / hx - ((vt - v) / hy) / hy - e3);
        gk = gk + (((v - vl) / hx) / hx + ((v - vb) / hy) / hy - e3);
        const double above = j < ny - 1 ? -((vt - v) / hy) / hy - e3 : 0.0;
        const double right = i < nx - 1 ? -((vr - v) / hx) / hx - e3 : 0.0;
        const double left = i > 0 ? ((v - vl) / hx) / hx - e3 : 0.0;
        const double below = j > 0 ? ((v - vb) / hy) / hy - e3 : 0.0;
        g[k] = ((((gk + above) + right) + left) + below) * area;
      }
    }
  }
  *f = area * (0.5 * fquad + fexp);
}

void orc_dsscfg_eval_f32(int nx, int ny, float lam, const float* x, float* f, float* g) {
  const float hx = (float)(1.0 / (double)(float)(nx + 1));
  const float hy = (float)(1.0 / (double)(float)(ny + 1));
  const float area = (float)(0.5 * (double)hx * (double)hy);
  float fquad = 0.0f, fexp = 0.0f;
  int i, j;
  for (j = 0; j < ny; j++) {
    for (i = 0; i < nx; i++) {
      const long k = (long)nx * j + i;
      const float v = x[k];
      const float vr = i < nx - 1 ? x[k + 1] : 0.0f, vt = j < ny - 1 ? x[k + nx] : 0.0f;
      const float vl = i > 0 ? x[k - 1] : 0.0f, vb = j > 0 ? x[k - nx] : 0.0f;
      float dx = (vr - v) / hx, dy = (vt - v) / hy;
      fquad += dx * dx + dy * dy;
      fexp = (float)((double)fexp - (double)(lam * (expd_f(v) + expd_f(vr) + expd_f(vt))) / 3.0);
      dx = (v - vl) / hx;
      dy = (v - vb) / hy;
      fquad += dx * dx + dy * dy;
      fexp = (float)((double)fexp - (double)(lam * (expd_f(vb) + expd_f(vl) + expd_f(v))) / 3.0);
      if (g) {
        const double e3 = (double)(lam * expd_f(v)) / 3.0;
        const float dxl = (vr - v) / hx, dyl = (vt - v) / hy;   /* own lower triangle */
        const float dxu = (v - vl) / hx, dyu = (v - vb) / hy;   /* own upper triangle */
        float gk = (float)(0.0 + ((double)(-dxl / hx - dyl / hy) - e3));
        gk = (float)((double)gk + ((double)(dxu / hx + dyu / hy) - e3));
        const float above = j < ny - 1 ? (float)((double)(-dyl / hy) - e3) : 0.0f;
        const float right = i < nx - 1 ? (float)((double)(-dxl / hx) - e3) : 0.0f;
        const float left = i > 0 ? (float)((double)(dxu / hx) - e3) : 0.0f;
        const float below = j > 0 ? (float)((double)(dyu / hy) - e3) : 0.0f;
        g[k] = ((((gk + above) + right) + left) + below) * area;
      }
    }
  }
  *f = (float)((double)area * (0.5 * (double)fquad + (double)fexp));
}
