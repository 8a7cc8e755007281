// common.cuh -- shared definitions of the sm_100a L-BFGS-B library.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbfgsb_b200 {

// History storage types: the two vector forms keep S and Y in their own precision; the
// bf16 form stores them as bfloat16 and widens on load.
template <typename T>
struct HistTraits;
template <>
struct HistTraits<double> {
  __device__ __forceinline__ static double load(const double* p) { return __ldg(p); }
  __device__ __forceinline__ static double from(double v) { return v; }
};
template <>
struct HistTraits<float> {
  __device__ __forceinline__ static float load(const float* p) { return __ldg(p); }
  __device__ __forceinline__ static float from(double v) { return (float)v; }
  __device__ __forceinline__ static float from(float v) { return v; }
};
template <>
struct HistTraits<__nv_bfloat16> {
  __device__ __forceinline__ static float load(const __nv_bfloat16* p) {
    return __bfloat162float(*p);
  }
  __device__ __forceinline__ static __nv_bfloat16 from(double v) {
    return __float2bfloat16_rn((float)v);
  }
  __device__ __forceinline__ static __nv_bfloat16 from(float v) { return __float2bfloat16_rn(v); }
};

// Elementwise arithmetic that must round exactly like the reference's scalar C++ code:
// no FMA contraction, one rounding per operation.
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }

// Correctly rounded a / b for a divisor b that is the same over a whole pass (theta),
// from y = RN(1/b) computed once.  Markstein's theorem (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1),
// 1990; restated in Muller et al., Handbook of Floating-Point Arithmetic, ch. 4): if
// y = RN(1/b) and q is a faithful approximation of a/b, then r = a - b*q is exactly
// representable (one fma computes it) and RN(q + r*y) = RN(a/b).  q0 = RN(a*y) is within
// about 2 ulp of a/b, so one correction q1 = RN(q0 + r0*y) first makes it faithful, and a
// second one gives the correctly rounded quotient.  The theorem needs every intermediate
// in the normal range: the caller passes fast = false unless |b| is in [2^-300, 2^300]
// (double) / [2^-30, 2^30] (float), and |a| outside [2^-600, 2^600] / [2^-60, 2^60] (zero,
// subnormal, infinite, NaN included) takes the full division.
struct FixedDiv64 {
  double b, y;
  bool fast;
  __device__ __forceinline__ explicit FixedDiv64(double b_) : b(b_) {
    const double ab = fabs(b_);
    fast = ab >= 0x1p-300 && ab <= 0x1p300;
    y = __ddiv_rn(1.0, b_);
  }
  __device__ __forceinline__ double operator()(double a) const {
    if (!in_range(a)) return __ddiv_rn(a, b);
    return markstein(a);
  }
  // the two halves of operator(), for callers that form several quotients branch-free and
  // redo the (rare) out-of-range ones with the full division
  __device__ __forceinline__ bool in_range(double a) const {
    const double aa = fabs(a);
    return fast && aa >= 0x1p-600 && aa <= 0x1p600;
  }
  __device__ __forceinline__ double markstein(double a) const {
    double q = __dmul_rn(a, y);
    double r = __fma_rn(-q, b, a);
    q = __fma_rn(r, y, q);
    r = __fma_rn(-q, b, a);
    return __fma_rn(r, y, q);
  }
  __device__ __forceinline__ double full(double a) const { return __ddiv_rn(a, b); }
};
struct FixedDiv32 {
  float b, y;
  bool fast;
  __device__ __forceinline__ explicit FixedDiv32(float b_) : b(b_) {
    const float ab = fabsf(b_);
    fast = ab >= 0x1p-30f && ab <= 0x1p30f;
    y = __fdiv_rn(1.0f, b_);
  }
  __device__ __forceinline__ float operator()(float a) const {
    if (!in_range(a)) return __fdiv_rn(a, b);
    return markstein(a);
  }
  __device__ __forceinline__ bool in_range(float a) const {
    const float aa = fabsf(a);
    return fast && aa >= 0x1p-60f && aa <= 0x1p60f;
  }
  __device__ __forceinline__ float markstein(float a) const {
    float q = __fmul_rn(a, y);
    float r = __fmaf_rn(-q, b, a);
    q = __fmaf_rn(r, y, q);
    r = __fmaf_rn(-q, b, a);
    return __fmaf_rn(r, y, q);
  }
  __device__ __forceinline__ float full(float a) const { return __fdiv_rn(a, b); }
};
// Filter for arg-min reductions of quotients num/den (breakpoints, steps to a bound):
// true when the correctly rounded num/den certainly exceeds the running minimum `best`, so
// that it need not be formed.  thr = next_up(best) is the least value of the quotients'
// type T above best; the exact quotient above thr rounds to thr or more, so above best.  num/den > thr is tested as num > thr*den (den > 0) or num < thr*den
// (den < 0), the product rounded toward the side that keeps the candidate (up, or down),
// so that no candidate whose rounded quotient could equal or undercut best is skipped.  A
// NaN operand or den = 0 compares false (kept).  One multiplication, no reciprocal.  A
// filtered candidate is strictly larger than the minimum, so it can change neither the
// minimum nor its (lowest) index.
__device__ __forceinline__ double next_up(double v) {  // least double above v (NaN, +inf: v)
  if (!(v < INFINITY)) return v;
  if (v == 0.0) return __longlong_as_double(1LL);
  const long long b = __double_as_longlong(v);
  return __longlong_as_double(v > 0.0 ? b + 1 : b - 1);
}
__device__ __forceinline__ float next_up(float v) {
  if (!(v < INFINITY)) return v;
  if (v == 0.0f) return __int_as_float(1);
  const int b = __float_as_int(v);
  return __int_as_float(v > 0.0f ? b + 1 : b - 1);
}
__device__ __forceinline__ bool quotient_exceeds(double num, double den, double thr) {
  if (den > 0.0) return num > __dmul_ru(thr, den);
  if (den < 0.0) return num < __dmul_rd(thr, den);
  return false;
}
__device__ __forceinline__ bool quotient_exceeds(float num, float den, float thr) {
  if (den > 0.0f) return num > __fmul_ru(thr, den);
  if (den < 0.0f) return num < __fmul_rd(thr, den);
  return false;
}

// Per-thread accumulators of the streaming sums: float in the plain FP32 form (S = float;
// each thread sums a few hundred terms, the CTA and grid levels sum in double), double
// otherwise.
template <typename S>
struct AccOf {
  using type = double;
};
template <>
struct AccOf<float> {
  using type = float;
};

template <typename S>
struct FixedDiv;
template <>
struct FixedDiv<double> : FixedDiv64 {
  using FixedDiv64::FixedDiv64;
};
template <>
struct FixedDiv<float> : FixedDiv32 {
  using FixedDiv32::FixedDiv32;
};

// A CTA's place among the CTAs that share one problem instance: rank 0..count-1.  A
// single-instance launch is the whole grid; a batched launch gives each instance its own
// contiguous range of CTAs (batch.cuh).
struct CtaPos {
  int rank;
  int count;
};
__device__ __forceinline__ CtaPos cta_here() { return CtaPos{(int)blockIdx.x, (int)gridDim.x}; }

// Splitmix64 finaliser: the order-free hash of the free set used by the trace.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// iwhere codes, one byte per variable (the reference keeps an int per variable).
// 0 free, -1 unbounded, -3 zero gradient, 1/2 at the lower/upper bound, 3 l == u,
// 4/5 fixed at the lower/upper bound by the breakpoint walk of this iteration's
// generalized Cauchy point (the reference stores these as 1/2; the distinct codes let
// later passes rebuild the Cauchy point without storing it).
enum : int8_t {
  IW_FREE = 0,
  IW_UNB = -1,
  IW_ZERO = -3,
  IW_LOW = 1,
  IW_UPP = 2,
  IW_FIX = 3,
  IW_WALK_LOW = 4,
  IW_WALK_UPP = 5
};
__host__ __device__ __forceinline__ bool iw_free(int c) { return c <= 0; }

constexpr int kMaxM = 8;          // L-BFGS memory (the reference fixes m = 8)
constexpr int kSlots = kMaxM + 1; // ring slots plus one spare for speculative writes
constexpr int kThreads = 256;     // threads per CTA of the streaming passes

}  // namespace lbfgsb_b200
