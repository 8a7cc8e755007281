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

void orc_synth_eval_f64(int s, const double* kappa, const double* w, const double* t,
                        const double* b, const double* x, double* f, double* g) {
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
  *f = acc;
}

void orc_synth_eval_f32(int s, const double* kappa, const double* w, const double* t,
                        const double* b, const float* x, float* f, float* g) {
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
  *f = (float)acc;
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
