// Compares the fixed-divisor quotient of csrc/common.cuh (FixedDiv64 / FixedDiv32) with
// CUDA's correctly rounded division (__ddiv_rn / __fdiv_rn) bit for bit on random and
// constructed inputs, and checks that the arg-min filter
// quotient_exceeds(num, den, next_up(best)) never reports a quotient whose correctly
// rounded value is <= best (with best at, just below and just above that value, and far
// from it).  Prints the number of mismatches /
// violations per family and exits 1 if any.
//   argv[1] = millions of random pairs per family (default 64)
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "../../lbfgsb-gpu_b200/csrc/common.cuh"

using namespace lbfgsb_b200;

__device__ __forceinline__ unsigned long long sm64(unsigned long long& s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// a double with random mantissa, exponent uniform in [elo, ehi], random sign
__device__ double rand_double(unsigned long long& s, int elo, int ehi) {
  const unsigned long long r = sm64(s);
  const int e = elo + (int)(sm64(s) % (unsigned long long)(ehi - elo + 1));
  const unsigned long long bits = ((unsigned long long)(e + 1023) << 52) | (r & ((1ULL << 52) - 1));
  const double v = __longlong_as_double((long long)bits);
  return (r >> 63) ? -v : v;
}
__device__ float rand_float(unsigned long long& s, int elo, int ehi) {
  const unsigned long long r = sm64(s);
  const int e = elo + (int)(sm64(s) % (unsigned long long)(ehi - elo + 1));
  const unsigned int bits = ((unsigned int)(e + 127) << 23) | (unsigned int)(r & ((1u << 23) - 1));
  const float v = __int_as_float((int)bits);
  return (r >> 63) ? -v : v;
}

// family 0: random a, b (theta-like and wide);  1: a = q*b rounded (quotient near a
// representable value);  2: a such that a/b is near a midpoint between two doubles;
// 3: divisors with all-ones / all-zero mantissas and powers of two;  4: a outside the fast
// range (zero, subnormal, huge, inf, nan)
__global__ void k_check64(long long count, unsigned long long seed, unsigned long long* bad) {
  unsigned long long s = seed + 0x1234567ULL * (blockIdx.x * blockDim.x + threadIdx.x);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x) {
    const int fam = (int)(k % 5);
    double b = (sm64(s) & 1) ? rand_double(s, -12, 12) : rand_double(s, -290, 290);
    double a;
    if (fam == 0) {
      a = rand_double(s, -580, 580);
    } else if (fam == 1) {
      const double q = rand_double(s, -200, 200);
      a = __dmul_rn(q, b);
    } else if (fam == 2) {
      const double q = rand_double(s, -200, 200);
      const double half = __longlong_as_double(__double_as_longlong(fabs(q)) + 1) - fabs(q);
      a = __fma_rn(q, b, copysign(0.5 * half, q) * b);  // (q + ulp/2) * b, rounded once
      if (sm64(s) & 1) a = __longlong_as_double(__double_as_longlong(a) + ((sm64(s) & 2) ? 1 : -1));
    } else if (fam == 3) {
      const int e = (int)(sm64(s) % 41) - 20;
      const unsigned long long m = (sm64(s) & 1) ? ((1ULL << 52) - 1) : 0ULL;
      b = __longlong_as_double((long long)(((unsigned long long)(e + 1023) << 52) | m));
      a = rand_double(s, -100, 100);
    } else {
      const unsigned long long r = sm64(s) % 6;
      a = r == 0 ? 0.0 : r == 1 ? -0.0 : r == 2 ? 4.9e-320
        : r == 3 ? rand_double(s, 700, 1000) : r == 4 ? __longlong_as_double(0x7FF0000000000000LL)
        : __longlong_as_double(0x7FF8000000000000LL);
    }
    const FixedDiv64 fd(b);
    const double want = __ddiv_rn(a, b), got = fd(a);
    const bool same = __double_as_longlong(want) == __double_as_longlong(got) ||
                      (want != want && got != got);
    if (!same) atomicAdd(&bad[fam], 1ULL);
  }
}

__global__ void k_check32(long long count, unsigned long long seed, unsigned long long* bad) {
  unsigned long long s = seed + 0x7654321ULL * (blockIdx.x * blockDim.x + threadIdx.x);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x) {
    const int fam = (int)(k % 5);
    float b = (sm64(s) & 1) ? rand_float(s, -12, 12) : rand_float(s, -29, 29);
    float a;
    if (fam == 0) {
      a = rand_float(s, -58, 58);
    } else if (fam == 1) {
      a = __fmul_rn(rand_float(s, -25, 25), b);
    } else if (fam == 2) {
      const float q = rand_float(s, -25, 25);
      const float half = __int_as_float(__float_as_int(fabsf(q)) + 1) - fabsf(q);
      a = __fmaf_rn(q, b, copysignf(0.5f * half, q) * b);
      if (sm64(s) & 1) a = __int_as_float(__float_as_int(a) + ((sm64(s) & 2) ? 1 : -1));
    } else if (fam == 3) {
      const int e = (int)(sm64(s) % 41) - 20;
      const unsigned int m = (sm64(s) & 1) ? ((1u << 23) - 1) : 0u;
      b = __int_as_float((int)(((unsigned int)(e + 127) << 23) | m));
      a = rand_float(s, -20, 20);
    } else {
      const unsigned long long r = sm64(s) % 6;
      a = r == 0 ? 0.0f : r == 1 ? -0.0f : r == 2 ? 1e-40f : r == 3 ? rand_float(s, 70, 127)
        : r == 4 ? __int_as_float(0x7F800000) : __int_as_float(0x7FC00000);
    }
    const FixedDiv32 fd(b);
    const float want = __fdiv_rn(a, b), got = fd(a);
    const bool same = __float_as_int(want) == __float_as_int(got) || (want != want && got != got);
    if (!same) atomicAdd(&bad[fam], 1ULL);
  }
}

template <typename T>
__device__ T rand_real(unsigned long long& s, int elo, int ehi);
template <>
__device__ double rand_real<double>(unsigned long long& s, int elo, int ehi) { return rand_double(s, elo, ehi); }
template <>
__device__ float rand_real<float>(unsigned long long& s, int elo, int ehi) { return rand_float(s, elo, ehi); }

// bad[0]: filtered although q <= best; bad[1]: number filtered (for information)
template <typename T>
__global__ void k_check_filter(long long count, unsigned long long seed, unsigned long long* bad) {
  unsigned long long s = seed + 0x2468aceULL * (blockIdx.x * blockDim.x + threadIdx.x);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x) {
    const int wide = (sizeof(T) == 8) ? 120 : 25;
    const T num = rand_real<T>(s, -wide, wide);
    const T den = rand_real<T>(s, -wide, wide);
    const T q = num / den;  // correctly rounded
    // the running minimum in the quotients' type, as the passes keep it
    T best;
    const int mode = (int)(k % 6);
    if (mode == 0) best = q;
    else if (mode == 1) best = -next_up(-q);  // the value just below q
    else if (mode == 2) best = next_up(q);
    else if (mode == 3) best = q * T(0.5);
    else if (mode == 4) best = q * T(2);
    else best = (T)((double)q * (1.0 - 1e-6));
    if (quotient_exceeds(num, den, next_up(best))) {
      atomicAdd(&bad[1], 1ULL);
      if (!(q > best)) atomicAdd(&bad[0], 1ULL);
    }
  }
}

int main(int argc, char** argv) {
  const long long count = (argc > 1 ? atoll(argv[1]) : 64) * 1000000LL;
  unsigned long long* bad = nullptr;
  if (cudaMalloc(&bad, 10 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  cudaMemset(bad, 0, 10 * sizeof(unsigned long long));
  k_check64<<<148 * 8, 256>>>(count, 1, bad);
  k_check32<<<148 * 8, 256>>>(count, 2, bad + 5);
  unsigned long long h[10];
  if (cudaMemcpy(h, bad, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
  cudaMemset(bad, 0, 4 * sizeof(unsigned long long));
  k_check_filter<double><<<148 * 8, 256>>>(count, 3, bad);
  k_check_filter<float><<<148 * 8, 256>>>(count, 4, bad + 2);
  unsigned long long hf[4];
  if (cudaMemcpy(hf, bad, sizeof(hf), cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
  cudaFree(bad);
  printf("filter f64: %llu violations, %llu of %lld filtered\n", hf[0], hf[1], count);
  printf("filter f32: %llu violations, %llu of %lld filtered\n", hf[2], hf[3], count);
  unsigned long long total = 0;
  for (int k = 0; k < 10; k++) {
    printf("%s family %d: %llu mismatches of %lld\n", k < 5 ? "f64" : "f32", k % 5, h[k], count / 5);
    total += h[k];
  }
  total += hf[0] + hf[2];
  return total == 0 ? 0 : 1;
}
