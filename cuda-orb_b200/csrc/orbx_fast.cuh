// FAST-9 segment test, FAST corner score and the Harris combine step, shared by
// the reference-exact detector (orbx_detect.cu) and the OpenCV-style pyramid
// (orbx_ocv.cu).
#pragma once
#include <stdint.h>

namespace orbx {

// FAST ring (makeOffsets, orbd.cu:463-496), as (dx, dy) of ring position k.
// Functions of a compile-time k fold to immediates in the unrolled loops.
__host__ __device__ constexpr int ring_dx(int k) {
  switch (k & 15) {
    case 0: return 0;   case 1: return 1;   case 2: return 2;   case 3: return 3;
    case 4: return 3;   case 5: return 3;   case 6: return 2;   case 7: return 1;
    case 8: return 0;   case 9: return -1;  case 10: return -2; case 11: return -3;
    case 12: return -3; case 13: return -3; case 14: return -2; default: return -1;
  }
}
__host__ __device__ constexpr int ring_dy(int k) { return ring_dx(k + 4); }

__device__ __forceinline__ bool has_arc9(uint32_t m16) {
  uint32_t m = m16 | (m16 << 16);  // circular
  uint32_t a = m & (m >> 1);       // runs of 2
  a &= a >> 2;                     // runs of 4
  a &= a >> 4;                     // runs of 8
  a &= m >> 8;                     // runs of 9
  return (a & 0xFFFFu) != 0u;
}

// Final step of dHarrisScore (orbd.cu:667-668) as the reference build evaluates it.
__device__ __forceinline__ float harris_combine(int dxx, int dyy, int dxy, float scale4) {
  const unsigned dsxy = (unsigned)dxx + (unsigned)dyy;
  const int A = (int)((unsigned)dxx * (unsigned)dyy - (unsigned)dxy * (unsigned)dxy);
  const unsigned Bq = dsxy * dsxy;
  const float u = __fmaf_rn(-0.04f, __uint2float_rn(Bq), __int2float_rn(A));
  return __fmul_rn(u, scale4);
}


// dFastScore (orbd.cu:538-586, FAST_PATTERN 16).
__device__ __forceinline__ float fast_score(const int* d, int threshold) {
  int a0 = threshold;
#pragma unroll
  for (int k = 0; k < 16; k += 2) {
    int a = min(d[k + 1], d[k + 2]);
    a = min(a, d[k + 3]);
    if (a <= a0) continue;
    a = min(a, d[k + 4]);
    a = min(a, d[k + 5]);
    a = min(a, d[k + 6]);
    a = min(a, d[k + 7]);
    a = min(a, d[k + 8]);
    a0 = max(a0, min(a, d[k]));
    a0 = max(a0, min(a, d[k + 9]));
  }
  int b0 = -a0;
#pragma unroll
  for (int k = 0; k < 16; k += 2) {
    int b = max(d[k + 1], d[k + 2]);
    b = max(b, d[k + 3]);
    b = max(b, d[k + 4]);
    b = max(b, d[k + 5]);
    if (b >= b0) continue;
    b = max(b, d[k + 6]);
    b = max(b, d[k + 7]);
    b = max(b, d[k + 8]);
    b0 = min(b0, max(b, d[k]));
    b0 = min(b0, max(b, d[k + 9]));
  }
  return (float)(-b0 - 1);
}

// FAST-9 segment test on a shared-memory tile of row stride sw: a run of 9
// contiguous ring pixels all darker than v - t or all brighter than v + t (the
// reference's LUT pre-test and arc loop, orbd.cu:683-740, decide exactly this).
__device__ __forceinline__ bool fast9_full(const uint8_t* c, int sw, int lo, int hi) {
  uint32_t dark = 0, bright = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    const int p = c[ring_dy(k) * sw + ring_dx(k)];
    dark |= (uint32_t)(p < lo) << k;
    bright |= (uint32_t)(p > hi) << k;
  }
  return has_arc9(dark) || has_arc9(bright);
}

}  // namespace orbx
