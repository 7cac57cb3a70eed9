// OpenCV-compatible mode (include/orbx.h, orbx_ocv_*): cv::ORB's published
// algorithm on the GPU, for callers who want OpenCV-like keypoints rather than
// the reference's.  The reference exposes retain_topn but never uses it
// (orb.cpp:41); this mode is where a Harris top-N retain lives.
//
//   pyramid   level 0 = the image; level l = level l-1 resized by 1/scale_factor
//             (bilinear, pixel centres aligned), one launch per level
//   blur      every level, separable 7x7 Gaussian (sigma 2), reflect-101 border
//   FAST      9-arc segment test and FAST score on every level pixel
//   NMS       3x3 strict maximum of the FAST score, outside edge_threshold;
//             survivors appended as unique 64-bit keys (score, ~position)
//   retain    per level, the best 2 * budget keys by FAST score, then (Harris
//             mode) the best budget keys by Harris score: an exact 8-pass radix
//             select on the unique keys (ties cannot split the set), then a
//             bitonic sort so the output order is deterministic
//   describe  one warp per keypoint: intensity-centroid angle on the level,
//             rBRIEF with the rotated pattern on the blurred level
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "orb_pattern31.h"
#include "orbx_fast.cuh"
#include "orbx_internal.cuh"

namespace orbx {

constexpr int kOcvMaxLevels = 16;
constexpr int kOcvCandCap = 1 << 17;  // NMS survivors kept per level
constexpr int kOcvSelCap = 8192;      // keys per level after the first retain
constexpr int kOcvHarrisBlock = 7;    // Harris window (blockSize)

struct OcvLevel {
  int w, h, pitch, n_keep;
  long long off;   // byte offset of the level in the level buffers
  long long pix0;  // first flattened pixel index of the level
  float scale;     // scale_factor^level
};

struct OcvArgs {
  int L, edge, fast_thr, harris, patch;
  long long total_pix;
  OcvLevel lv[kOcvMaxLevels];
  float g[7];  // Gaussian taps
  float harris_s4;
  uint8_t* img;
  uint8_t* blr;
  uint8_t* score;
  unsigned long long* cand;  // [L][kOcvCandCap]
  int* ncand;
  unsigned long long* sel;   // [L][kOcvSelCap]: after the FAST retain
  int* nsel;
  unsigned long long* hkey;  // [L][kOcvSelCap]: Harris keys of sel
  unsigned long long* fin;   // [L][kOcvSelCap]: final keys, descending
  int* nfin;
  const int* umax;
  const int8_t* pattern;
  orbx_ocv_keypoint* out;
  uint8_t* desc;
  int* count;
  int cap;
};

struct OcvWork {
  int w = 0, h = 0, L = 0;
  float scale = 0.f;
  size_t level_bytes = 0;
  uint8_t *img = nullptr, *blr = nullptr, *score = nullptr;
  unsigned long long *cand = nullptr, *sel = nullptr, *hkey = nullptr, *fin = nullptr;
  int* counts = nullptr;  // ncand, nsel, nfin: 3 * kOcvMaxLevels
  int* umax = nullptr;
  int8_t* pattern = nullptr;
};

void ocv_free(OcvWork* w) {
  if (!w) return;
  cudaFree(w->img);
  cudaFree(w->blr);
  cudaFree(w->score);
  cudaFree(w->cand);
  cudaFree(w->sel);
  cudaFree(w->hkey);
  cudaFree(w->fin);
  cudaFree(w->counts);
  cudaFree(w->umax);
  cudaFree(w->pattern);
  delete w;
}

namespace {

__device__ __forceinline__ int ocv_level_of(const OcvArgs& a, long long i) {
  int l = 0;
  while (l + 1 < a.L && i >= a.lv[l + 1].pix0) l++;
  return l;
}

__device__ __forceinline__ int reflect101(int i, int n) {
  if (i < 0) i = -i;
  if (i >= n) i = 2 * n - 2 - i;
  return min(max(i, 0), n - 1);
}

// Order-preserving image of a float in 32 bits.
__device__ __forceinline__ uint32_t ocv_order(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ocv_unorder(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

__global__ void k_ocv_copy0(OcvArgs a, const uint8_t* __restrict__ src, int src_pitch) {
  const OcvLevel& L0 = a.lv[0];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)L0.w * L0.h) return;
  const int y = (int)(i / L0.w), x = (int)(i - (long long)y * L0.w);
  a.img[L0.off + (long long)y * L0.pitch + x] = src[(long long)y * src_pitch + x];
}

// Level l from level l - 1, bilinear with pixel centres aligned.
__global__ void k_ocv_resize(OcvArgs a, int l) {
  const OcvLevel& D = a.lv[l];
  const OcvLevel& S = a.lv[l - 1];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)D.w * D.h) return;
  const int y = (int)(i / D.w), x = (int)(i - (long long)y * D.w);
  const float fxs = (float)S.w / (float)D.w, fys = (float)S.h / (float)D.h;
  const float sx = fmaxf((x + 0.5f) * fxs - 0.5f, 0.f), sy = fmaxf((y + 0.5f) * fys - 0.5f, 0.f);
  int x0 = (int)sx, y0 = (int)sy;
  const float fx = sx - (float)x0, fy = sy - (float)y0;
  x0 = min(x0, S.w - 1);
  y0 = min(y0, S.h - 1);
  const int x1 = min(x0 + 1, S.w - 1), y1 = min(y0 + 1, S.h - 1);
  const uint8_t* s = a.img + S.off;
  const float p00 = s[(long long)y0 * S.pitch + x0], p01 = s[(long long)y0 * S.pitch + x1];
  const float p10 = s[(long long)y1 * S.pitch + x0], p11 = s[(long long)y1 * S.pitch + x1];
  const float v = (1.f - fy) * ((1.f - fx) * p00 + fx * p01) + fy * ((1.f - fx) * p10 + fx * p11);
  a.img[D.off + (long long)y * D.pitch + x] = (uint8_t)min(max(__float2int_rn(v), 0), 255);
}

__global__ void k_ocv_blur(OcvArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.total_pix) return;
  const int l = ocv_level_of(a, i);
  const OcvLevel& V = a.lv[l];
  const long long k = i - V.pix0;
  const int y = (int)(k / V.w), x = (int)(k - (long long)y * V.w);
  const uint8_t* s = a.img + V.off;
  int xs[7];
#pragma unroll
  for (int d = 0; d < 7; d++) xs[d] = reflect101(x + d - 3, V.w);
  float acc = 0.f;
#pragma unroll
  for (int dy = 0; dy < 7; dy++) {
    const uint8_t* row = s + (long long)reflect101(y + dy - 3, V.h) * V.pitch;
    float hs = 0.f;
#pragma unroll
    for (int dx = 0; dx < 7; dx++) hs += a.g[dx] * (float)row[xs[dx]];
    acc += a.g[dy] * hs;
  }
  a.blr[V.off + (long long)y * V.pitch + x] = (uint8_t)min(max(__float2int_rn(acc), 0), 255);
}

// FAST score of every level pixel (0 where it is not a corner).
__global__ void k_ocv_fast(OcvArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.total_pix) return;
  const int l = ocv_level_of(a, i);
  const OcvLevel& V = a.lv[l];
  const long long k = i - V.pix0;
  const int y = (int)(k / V.w), x = (int)(k - (long long)y * V.w);
  uint8_t sc = 0;
  if (x >= 3 && x < V.w - 3 && y >= 3 && y < V.h - 3) {
    const uint8_t* c = a.img + V.off + (long long)y * V.pitch + x;
    const int v = c[0];
    if (fast9_full(c, V.pitch, v - a.fast_thr, v + a.fast_thr)) {
      int d[25];
#pragma unroll
      for (int r = 0; r < 25; r++) d[r] = (int)(short)(v - c[ring_dy(r) * V.pitch + ring_dx(r)]);
      sc = (uint8_t)min(max((int)fast_score(d, a.fast_thr), 1), 255);
    }
  }
  a.score[V.off + (long long)y * V.pitch + x] = sc;
}

// 3x3 strict maxima of the FAST score outside the edge band, as unique keys.
__global__ void k_ocv_nms(OcvArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.total_pix) return;
  const int l = ocv_level_of(a, i);
  const OcvLevel& V = a.lv[l];
  const long long k = i - V.pix0;
  const int y = (int)(k / V.w), x = (int)(k - (long long)y * V.w);
  if (x < a.edge || x >= V.w - a.edge || y < a.edge || y >= V.h - a.edge) return;
  const uint8_t* s = a.score + V.off + (long long)y * V.pitch + x;
  const int c = s[0];
  if (!c) return;
  const int p = V.pitch;
  if (c <= s[-p - 1] || c <= s[-p] || c <= s[-p + 1] || c <= s[-1] || c <= s[1] || c <= s[p - 1] || c <= s[p] ||
      c <= s[p + 1])
    return;
  const int pos = atomicAdd(&a.ncand[l], 1);
  if (pos < kOcvCandCap)
    a.cand[(size_t)l * kOcvCandCap + pos] =
        ((unsigned long long)c << 32) | (0xFFFFFFFFu - (uint32_t)((long long)y * V.w + x));
}

// Per level (one block of 1024 threads): the k largest of n unique keys, by an
// 8-pass radix select on bytes from the top, then sorted in decreasing order.
__global__ void __launch_bounds__(1024) k_ocv_select(OcvArgs a, const unsigned long long* src, int src_stride,
                                                     const int* src_n, int src_cap, int mult,
                                                     unsigned long long* dst, int* dst_n) {
  extern __shared__ unsigned long long s_keys[];  // kOcvSelCap
  __shared__ int s_hist[256];
  __shared__ int s_digit, s_above, s_cnt;
  const int l = blockIdx.x;
  const unsigned long long* in = src + (size_t)l * src_stride;
  const int n = min(src_n[l], src_cap);
  const int k = min(a.lv[l].n_keep * mult, kOcvSelCap);
  unsigned long long prefix = 0ull, mask = 0ull;
  if (n > k) {
    int remaining = k;
    for (int byte = 7; byte >= 0; byte--) {
      for (int d = threadIdx.x; d < 256; d += blockDim.x) s_hist[d] = 0;
      __syncthreads();
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const unsigned long long key = in[j];
        if ((key & mask) == prefix) atomicAdd(&s_hist[(int)((key >> (8 * byte)) & 0xFFu)], 1);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int above = 0, d = 255;
        for (; d > 0; d--) {
          if (above + s_hist[d] >= remaining) break;
          above += s_hist[d];
        }
        s_digit = d;
        s_above = above;
      }
      __syncthreads();
      remaining -= s_above;
      prefix |= (unsigned long long)s_digit << (8 * byte);
      mask |= 0xFFull << (8 * byte);
      __syncthreads();
    }
  }
  // keys >= prefix (all keys when n <= k): exactly min(n, k) of them
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const unsigned long long key = in[j];
    if (key >= prefix) {
      const int pos = atomicAdd(&s_cnt, 1);
      if (pos < kOcvSelCap) s_keys[pos] = key;
    }
  }
  __syncthreads();
  const int cnt = min(s_cnt, kOcvSelCap);
  int P = 1;
  while (P < cnt) P <<= 1;
  for (int j = cnt + threadIdx.x; j < P; j += blockDim.x) s_keys[j] = 0ull;
  __syncthreads();
  // bitonic sort, decreasing
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int j = threadIdx.x; j < P; j += blockDim.x) {
        const int partner = j ^ stride;
        if (partner > j) {
          const bool desc = (j & size) == 0;
          const unsigned long long x = s_keys[j], y = s_keys[partner];
          if (desc ? (x < y) : (x > y)) {
            s_keys[j] = y;
            s_keys[partner] = x;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) dst[(size_t)l * kOcvSelCap + j] = s_keys[j];
  if (threadIdx.x == 0) dst_n[l] = cnt;
}

// Harris score (blockSize 7, k = 0.04, derivatives of the 3x3 Sobel form) of
// the keys kept by the FAST retain; the Harris key keeps the position bits.
__global__ void k_ocv_harris(OcvArgs a) {
  const int l = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.nsel[l]) return;
  const OcvLevel& V = a.lv[l];
  const unsigned long long key = a.sel[(size_t)l * kOcvSelCap + j];
  const uint32_t low = (uint32_t)key;
  const uint32_t idx = 0xFFFFFFFFu - low;
  const int y = (int)(idx / (uint32_t)V.w), x = (int)(idx - (uint32_t)y * (uint32_t)V.w);
  const int p = V.pitch;
  const uint8_t* c = a.img + V.off + (long long)y * p + x;
  int sa = 0, sb = 0, sc = 0;
  for (int wy = -3; wy <= 3; wy++)
    for (int wx = -3; wx <= 3; wx++) {
      const uint8_t* q = c + wy * p + wx;
      const int ix = ((int)q[1] - (int)q[-1]) * 2 + ((int)q[-p + 1] - (int)q[-p - 1]) + ((int)q[p + 1] - (int)q[p - 1]);
      const int iy = ((int)q[p] - (int)q[-p]) * 2 + ((int)q[p - 1] - (int)q[-p - 1]) + ((int)q[p + 1] - (int)q[-p + 1]);
      sa += ix * ix;
      sb += iy * iy;
      sc += ix * iy;
    }
  const float fa = (float)sa, fb = (float)sb, fc = (float)sc;
  const float r = (fa * fb - fc * fc - 0.04f * (fa + fb) * (fa + fb)) * a.harris_s4;
  a.hkey[(size_t)l * kOcvSelCap + j] = ((unsigned long long)ocv_order(r) << 32) | low;
}

// One warp per final keypoint: angle, descriptor, output entry.
__global__ void __launch_bounds__(256) k_ocv_describe(OcvArgs a) {
  const int l = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * 8 + warp;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    int tot = 0;
    for (int m = 0; m < a.L; m++) tot += a.nfin[m];
    *a.count = min(tot, a.cap);
  }
  if (j >= a.nfin[l]) return;
  int base = 0;
  for (int m = 0; m < l; m++) base += a.nfin[m];
  const int o = base + j;
  if (o >= a.cap) return;
  const OcvLevel& V = a.lv[l];
  const unsigned long long key = a.fin[(size_t)l * kOcvSelCap + j];
  const uint32_t idx = 0xFFFFFFFFu - (uint32_t)key;
  const int y = (int)(idx / (uint32_t)V.w), x = (int)(idx - (uint32_t)y * (uint32_t)V.w);
  const int p = V.pitch;
  // intensity centroid over the disc of radius patch / 2
  const int half = a.patch / 2;
  const uint8_t* c = a.img + V.off + (long long)y * p + x;
  int m10 = 0, m01 = 0;
  const int u = lane - half;
  if (lane <= 2 * half) {
    m10 = u * (int)c[u];
    for (int v = 1; v <= half; v++) {
      const int d = a.umax[v];
      if (u >= -d && u <= d) {
        const int vp = c[u + v * p], vm = c[u - v * p];
        m10 += u * (vp + vm);
        m01 += v * (vp - vm);
      }
    }
  }
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    m10 += __shfl_xor_sync(0xffffffffu, m10, s);
    m01 += __shfl_xor_sync(0xffffffffu, m01, s);
  }
  float ang = atan2f((float)m01, (float)m10) * (180.f / 3.14159265358979f);
  if (ang < 0.f) ang += 360.f;
  // rBRIEF on the blurred level: lane t computes byte t from 8 point pairs
  const float th = ang * (3.14159265358979f / 180.f);
  const float ca = cosf(th), sa = sinf(th);
  const uint8_t* b = a.blr + V.off + (long long)y * p + x;
  uint32_t byte = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int t = 8 * lane + k;
    const float x0 = a.pattern[4 * t], y0 = a.pattern[4 * t + 1];
    const float x1 = a.pattern[4 * t + 2], y1 = a.pattern[4 * t + 3];
    const int i0 = b[__float2int_rn(x0 * sa + y0 * ca) * p + __float2int_rn(x0 * ca - y0 * sa)];
    const int i1 = b[__float2int_rn(x1 * sa + y1 * ca) * p + __float2int_rn(x1 * ca - y1 * sa)];
    byte |= (uint32_t)(i0 < i1) << k;
  }
  a.desc[(size_t)o * 32 + lane] = (uint8_t)byte;
  if (lane == 0) {
    orbx_ocv_keypoint kp;
    kp.x = (float)x * V.scale;
    kp.y = (float)y * V.scale;
    kp.size = (float)a.patch * V.scale;
    kp.angle = ang;
    kp.response = a.harris ? ocv_unorder((uint32_t)(key >> 32)) : (float)(uint32_t)(key >> 32);
    kp.octave = l;
    a.out[o] = kp;
  }
}

}  // namespace
}  // namespace orbx

using namespace orbx;

namespace {
struct OGuard {
  int prev = -1;
  explicit OGuard(int d) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != d)
      cudaSetDevice(d);
    else
      prev = -1;
  }
  ~OGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
#define OCHK(x)                                                             \
  do {                                                                      \
    cudaError_t _e = (x);                                                   \
    if (_e != cudaSuccess) {                                                \
      (void)cudaGetLastError();                                             \
      return _e == cudaErrorMemoryAllocation ? ORBX_ERR_NOMEM : ORBX_ERR_CUDA; \
    }                                                                       \
  } while (0)
unsigned ogrid(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }
}  // namespace

ORBX_API int orbx_ocv_default_params(orbx_ocv_params* p) {
  if (!p) return ORBX_ERR_ARG;
  // cv::ORB defaults except the budget (500 there)
  p->nfeatures = 5000;
  p->scale_factor = 1.2f;
  p->nlevels = 8;
  p->edge_threshold = 31;
  p->score_type = 0;
  p->patch_size = 31;
  p->fast_threshold = 20;
  return ORBX_OK;
}

ORBX_API int orbx_ocv_detect_and_compute(orbx_ctx* ctx, const orbx_ocv_params* p, const uint8_t* d_image, int w, int h,
                                         int pitch, orbx_ocv_keypoint* d_keypoints, uint8_t* d_desc, int* d_n,
                                         int cap) {
  if (!ctx || !p || !d_image || !d_keypoints || !d_desc || !d_n || cap < 0 || w < 16 || h < 16 || pitch < w)
    return ORBX_ERR_ARG;
  if (p->nfeatures < 1 || p->nfeatures > 16000 || !(p->scale_factor > 1.f && p->scale_factor <= 2.f) ||
      p->nlevels < 1 || p->nlevels > kOcvMaxLevels || p->edge_threshold < 19 || p->patch_size != 31 ||
      p->fast_threshold < 0 || p->fast_threshold > 255 || (p->score_type != 0 && p->score_type != 1))
    return ORBX_ERR_ARG;
  if ((long long)w * h >= (1ll << 31)) return ORBX_ERR_SIZE;
  OGuard g(ctx_device(ctx));
  cudaStream_t s = ctx_stream(ctx);
  OcvArgs a{};
  a.L = p->nlevels;
  a.edge = p->edge_threshold;
  a.fast_thr = p->fast_threshold;
  a.harris = p->score_type == 0 ? 1 : 0;
  a.patch = p->patch_size;
  // levels: sizes rounded from the previous scale, budgets geometric in 1 / scale
  {
    const double f = 1.0 / p->scale_factor;
    double per = p->nfeatures * (1.0 - f) / (1.0 - std::pow(f, (double)p->nlevels));
    int used = 0;
    long long off = 0, pix = 0;
    for (int l = 0; l < a.L; l++) {
      const double sc = std::pow((double)p->scale_factor, (double)l);
      OcvLevel& V = a.lv[l];
      V.w = std::max(1, (int)std::lround(w / sc));
      V.h = std::max(1, (int)std::lround(h / sc));
      V.pitch = (V.w + 127) / 128 * 128;
      V.off = off;
      V.pix0 = pix;
      V.scale = (float)sc;
      if (l < a.L - 1) {
        V.n_keep = (int)std::lround(per);
        used += V.n_keep;
        per *= f;
      } else {
        V.n_keep = std::max(p->nfeatures - used, 0);
      }
      if (V.n_keep * (a.harris ? 2 : 1) > kOcvSelCap) return ORBX_ERR_SIZE;
      off += (long long)V.pitch * (V.h + 1);
      pix += (long long)V.w * V.h;
    }
    a.total_pix = pix;
    // Gaussian taps for sigma 2
    double gs[7], sum = 0.0;
    for (int i = 0; i < 7; i++) {
      gs[i] = std::exp(-(double)((i - 3) * (i - 3)) / (2.0 * 4.0));
      sum += gs[i];
    }
    for (int i = 0; i < 7; i++) a.g[i] = (float)(gs[i] / sum);
    const double hs = 1.0 / (4.0 * kOcvHarrisBlock * 255.0);
    a.harris_s4 = (float)(hs * hs * hs * hs);
    // workspace
    OcvWork*& W = ctx_ocv(ctx);
    if (!W) W = new OcvWork();
    const size_t lb = (size_t)off;
    if (W->level_bytes < lb) {
      cudaFree(W->img);
      cudaFree(W->blr);
      cudaFree(W->score);
      W->img = W->blr = W->score = nullptr;
      W->level_bytes = 0;
      OCHK(cudaMalloc(&W->img, lb));
      OCHK(cudaMalloc(&W->blr, lb));
      OCHK(cudaMalloc(&W->score, lb));
      W->level_bytes = lb;
    }
    if (!W->cand) {
      OCHK(cudaMalloc(&W->cand, sizeof(unsigned long long) * (size_t)kOcvMaxLevels * kOcvCandCap));
      OCHK(cudaMalloc(&W->sel, sizeof(unsigned long long) * (size_t)kOcvMaxLevels * kOcvSelCap));
      OCHK(cudaMalloc(&W->hkey, sizeof(unsigned long long) * (size_t)kOcvMaxLevels * kOcvSelCap));
      OCHK(cudaMalloc(&W->fin, sizeof(unsigned long long) * (size_t)kOcvMaxLevels * kOcvSelCap));
      OCHK(cudaMalloc(&W->counts, sizeof(int) * 3 * kOcvMaxLevels));
      int umax[64] = {0};
      umax_table(p->patch_size, umax);
      OCHK(cudaMalloc(&W->umax, sizeof(umax)));
      OCHK(cudaMemcpy(W->umax, umax, sizeof(umax), cudaMemcpyHostToDevice));
      OCHK(cudaMalloc(&W->pattern, sizeof(kOrbPattern31)));
      OCHK(cudaMemcpy(W->pattern, kOrbPattern31, sizeof(kOrbPattern31), cudaMemcpyHostToDevice));
      OCHK(cudaFuncSetAttribute(k_ocv_select, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(unsigned long long) * kOcvSelCap)));
    }
    a.img = W->img;
    a.blr = W->blr;
    a.score = W->score;
    a.cand = W->cand;
    a.sel = W->sel;
    a.hkey = W->hkey;
    a.fin = W->fin;
    a.ncand = W->counts;
    a.nsel = W->counts + kOcvMaxLevels;
    a.nfin = W->counts + 2 * kOcvMaxLevels;
    a.umax = W->umax;
    a.pattern = W->pattern;
  }
  a.out = d_keypoints;
  a.desc = d_desc;
  a.count = d_n;
  a.cap = cap;
  OCHK(cudaMemsetAsync(a.ncand, 0, sizeof(int) * 3 * kOcvMaxLevels, s));
  k_ocv_copy0<<<ogrid((long long)w * h, 256), 256, 0, s>>>(a, d_image, pitch);
  for (int l = 1; l < a.L; l++)
    k_ocv_resize<<<ogrid((long long)a.lv[l].w * a.lv[l].h, 256), 256, 0, s>>>(a, l);
  k_ocv_blur<<<ogrid(a.total_pix, 256), 256, 0, s>>>(a);
  k_ocv_fast<<<ogrid(a.total_pix, 256), 256, 0, s>>>(a);
  k_ocv_nms<<<ogrid(a.total_pix, 256), 256, 0, s>>>(a);
  const size_t smem = sizeof(unsigned long long) * kOcvSelCap;
  if (a.harris) {
    k_ocv_select<<<a.L, 1024, smem, s>>>(a, a.cand, kOcvCandCap, a.ncand, kOcvCandCap, 2, a.sel, a.nsel);
    k_ocv_harris<<<dim3(kOcvSelCap / 256, a.L), 256, 0, s>>>(a);
    k_ocv_select<<<a.L, 1024, smem, s>>>(a, a.hkey, kOcvSelCap, a.nsel, kOcvSelCap, 1, a.fin, a.nfin);
  } else {
    k_ocv_select<<<a.L, 1024, smem, s>>>(a, a.cand, kOcvCandCap, a.ncand, kOcvCandCap, 1, a.fin, a.nfin);
  }
  k_ocv_describe<<<dim3(kOcvSelCap / 8, a.L), 256, 0, s>>>(a);
  OCHK(cudaGetLastError());
  return ORBX_OK;
}
