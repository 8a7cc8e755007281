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
};
template <>
struct HistTraits<__nv_bfloat16> {
  __device__ __forceinline__ static float load(const __nv_bfloat16* p) {
    return __bfloat162float(*p);
  }
  __device__ __forceinline__ static __nv_bfloat16 from(double v) {
    return __float2bfloat16_rn((float)v);
  }
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
