// Device helpers for the sm_100a ORB kernels: exact-rounding arithmetic that
// reproduces the reference build's floating-point results, and small utilities.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace orbx {

// dealBorder (cuda_utils.h:145-152): reflect-101.  The clamp only matters for
// octaves narrower than the reflected reach, whose outputs are never used.
__device__ __forceinline__ int reflect101(int i, int n) {
  if (i < 0) i = -i;
  if (i >= n) i = n + n - 2 - i;
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// "w = k[0]*t0; w += k[1]*t1; w += k[2]*t2; w += k[3]*t3" as the reference build
// evaluates it (orbd.cu:1292-1296, 1309-1319): the first add fuses the k0
// product, the next two adds are fused multiply-adds.
__device__ __forceinline__ float gauss_dot4(const float* k, float t0, float t1, float t2, float t3) {
  float acc = __fmaf_rn(k[0], t0, __fmul_rn(k[1], t1));
  acc = __fmaf_rn(k[2], t2, acc);
  return __fmaf_rn(k[3], t3, acc);
}

// Round-to-nearest-even of a 64-bit fixed-point value to a multiple of 2^sh.
__host__ __device__ __forceinline__ uint64_t rne_shift(uint64_t v, int sh) {
  const uint64_t one = 1ull << sh;
  const uint64_t low = v & (one - 1);
  const uint64_t half = one >> 1;
  v -= low;
  if (low > half || (low == half && ((v >> sh) & 1ull))) v += one;
  return v;
}

// (float)(M_PI - (double)r) for 0 <= r < 2 without double arithmetic.  The
// reference computes the quadrant fold of dFastAtan2 (orbd.cu:995) in double
// because M_PI is the double macro; here the difference is formed exactly in
// 64-bit fixed point (2^-62 units), rounded to 53 significant bits (the double
// result), then to 24 (the float conversion), both to nearest-even.
__host__ __device__ __forceinline__ float pi_minus_as_double(float r) {
  // M_PI as a double: mantissa 0x1921FB54442D18 with exponent 1, i.e.
  // 0x1921FB54442D18 * 2^-51 = 0x1921FB54442D18 << 11 in 2^-62 units.
  const uint64_t kPi62 = 0x1921FB54442D18ull << 11;
  uint32_t bits;
#ifdef __CUDA_ARCH__
  bits = __float_as_uint(r);
#else
  __builtin_memcpy(&bits, &r, 4);
#endif
  const int e = (int)((bits >> 23) & 0xFF);
  if (e < 127 - 39) {
    // r < 2^-39: the difference rounds to the float nearest M_PI
    const uint32_t pi_f = 0x40490FDBu;
#ifdef __CUDA_ARCH__
    return __uint_as_float(pi_f);
#else
    float out;
    __builtin_memcpy(&out, &pi_f, 4);
    return out;
#endif
  }
  // r = m * 2^(e - 150) with the hidden bit; in 2^-62 units: m << (e - 150 + 62)
  const uint64_t m = (uint64_t)((bits & 0x7FFFFFu) | 0x800000u);
  const uint64_t r62 = m << (e - 88);
  uint64_t d = kPi62 - r62;
  d = rne_shift(d, (d >> 63) ? 11 : 10);  // to double: 53 significant bits
  d = rne_shift(d, (d >> 63) ? 40 : 39);  // to float: 24 significant bits
  uint32_t out_bits;
  if (d >> 63)
    out_bits = (128u << 23) | (uint32_t)((d >> 40) & 0x7FFFFFu);  // [2, 4)
  else
    out_bits = (127u << 23) | (uint32_t)((d >> 39) & 0x7FFFFFu);  // [1, 2)
#ifdef __CUDA_ARCH__
  return __uint_as_float(out_bits);
#else
  float out;
  __builtin_memcpy(&out, &out_bits, 4);
  return out;
#endif
}

#ifdef __CUDACC__
// dFastAtan2 (orbd.cu:986-998): a 3-term odd polynomial of min/max with an
// IEEE division and explicit FMAs, then the quadrant folds.
__device__ __forceinline__ float fast_atan2(float y, float x) {
  const float ax = fabsf(x);
  const float ay = fabsf(y);
  const float a = __fdiv_rn(fminf(ax, ay), fmaxf(ax, ay));
  const float s = __fmul_rn(a, a);
  float r = __fmaf_rn(__fmaf_rn(__fmaf_rn(-0.0464964749f, s, 0.15931422f), s, -0.327622764f), __fmul_rn(s, a), a);
  r = (ay > ax) ? __fsub_rn(1.5707963267948966f, r) : r;
  r = (x < 0.f) ? pi_minus_as_double(r) : r;
  r = (y < 0.f) ? -r : r;
  return r;
}

// Strong relaxed load and store (at the device's coherence point, no ordering
// of other accesses), for words that carry all the data their reader needs.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Index of the frame whose tile range [base[f], base[f+1]) holds t.
__device__ __forceinline__ int find_frame(const int* base, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(base + mid) <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}
#endif

}  // namespace orbx
