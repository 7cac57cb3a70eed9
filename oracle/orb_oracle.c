/* CPU restatement of the CUDA-ORB detect / describe / match path.
 *
 * TEST INFRASTRUCTURE ONLY (see orb_oracle.h).  Each function cites the
 * reference lines (file:line in the CUDA-ORB tree) whose arithmetic it
 * restates.  Floating-point steps whose fusing into FMA by nvcc is not visible
 * in the source take a variant selector; the variant the reference build uses
 * is fixed by comparing against its outputs (tests/test_oracle_golden.py).
 *
 * Built with gcc -ffp-contract=off: a plain float expression here rounds after
 * every operation, and every fused multiply-add is an explicit fmaf().
 */
#include "orb_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../cuda-orb_b200/csrc/orb_pattern31.h"

#define MAX_OCTAVE 5 /* orbd.cu:18 */

static inline int align_up(int a, int b) { return (a % b != 0) ? (a - a % b + b) : a; } /* cuda_utils.h:170-173 */

int oo_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Orbor::updateParam (orb.cpp:145-191): level count and the back-to-back octave layout. */
int oo_layout(int w, int h, int noctaves, int* oszp) {
  int m = (w < h ? w : h) / 80;
  if (m <= 0) return 0;
  int n = (int)log2f((float)m) + 1;
  if (noctaves < n) n = noctaves;
  int* osizes = oszp;
  int* widths = osizes + n;
  int* heights = widths + n;
  int* pitchs = heights + n;
  int* offsets = pitchs + n;
  widths[0] = w;
  heights[0] = h;
  pitchs[0] = align_up(w, 128);
  osizes[0] = h * pitchs[0];
  offsets[0] = 0;
  offsets[1] = osizes[0];
  for (int j = 1; j < n; j++) {
    widths[j] = widths[j - 1] >> 1;
    heights[j] = heights[j - 1] >> 1;
    pitchs[j] = align_up(widths[j], 128);
    osizes[j] = heights[j] * pitchs[j];
    offsets[j + 1] = offsets[j] + osizes[j];
  }
  return n;
}

/* setFastThresholdLUT (orbd.cu:57-63). */
void oo_fast_lut(int t, uint8_t* lut) {
  for (int i = -255, j = 0; i <= 255; i++, j++) lut[j] = (uint8_t)(i < -t ? 1 : i > t ? 2 : 0);
  lut[511] = 0;
}

/* setUmax (orbd.cu:66-92): disc half-widths for the intensity centroid. */
void oo_umax(int patch_size, int* umax) {
  int half = patch_size / 2;
  umax[half + 1] = 0;
  float v = half * sqrtf(2.f) / 2;
  int vmax = (int)floorf(v + 1);
  int vmin = (int)ceilf(v);
  for (int i = 0; i <= vmax; i++) umax[i] = (int)roundf(sqrtf((float)(half * half - i * i)));
  for (int i = half, v0 = 0; i >= vmin; --i) {
    while (umax[v0] == umax[v0 + 1]) ++v0;
    umax[i] = v0;
    ++v0;
  }
}

/* setGaussianKernel (orbd.cu:413-433): 7-tap sigma 2, host expf, normalised. */
void oo_gauss_kernel(float* k) {
  const float sigma = 2.f;
  const float svar = -1.f / (2.f * sigma * sigma);
  float kersum = 0.f;
  for (int i = 0; i <= 3; i++) {
    k[i] = expf(i * i * svar);
    kersum = kersum + (k[i] + (i == 0 ? 0 : k[i]));
  }
  kersum = 1.f / kersum;
  for (int i = 0; i <= 3; i++) k[i] *= kersum;
}

/* setScaleSqSq (orbd.cu:436-441). */
float oo_harris_scale(void) {
  float scale = 1.f / (4 * 7 * 255.f);
  return scale * scale * scale * scale;
}

/* setPattern (orbd.cu:95-410): the fixed 31x31 table, the libc rand() pattern for
 * other patch sizes (with its offset bug, orbd.cu:366-367), and the WTA_K 3/4
 * tuple selection.  pattern_xy receives up to 512 (x, y) pairs; returns the count. */
int oo_pattern(int patch_size, int wta_k, int* out) {
  int base[1024];
  for (int i = 0; i < 512; i++) {
    base[2 * i] = kOrbPattern31[i][0];
    base[2 * i + 1] = kOrbPattern31[i][1];
  }
  if (patch_size != 31) {
    srand(0x34985739);
    for (int i = 0; i < 512; i++) {
      base[2 * i] = rand() % patch_size - -patch_size / 2;
      base[2 * i + 1] = rand() % patch_size - -patch_size / 2;
    }
  }
  if (wta_k == 2) {
    memcpy(out, base, sizeof(base));
    return 512;
  }
  srand(0x12345678);
  const int ntuples = 128;
  for (int i = 0; i < ntuples; i++) {
    for (int k = 0; k < wta_k; k++) {
      for (;;) {
        int idx = rand() % 512;
        int px = base[2 * idx], py = base[2 * idx + 1];
        int k1;
        for (k1 = 0; k1 < k; k1++) {
          if (px == out[2 * (wta_k * i + k1)] && py == out[2 * (wta_k * i + k1) + 1]) break;
        }
        if (k1 == k) {
          out[2 * (wta_k * i + k)] = px;
          out[2 * (wta_k * i + k) + 1] = py;
          break;
        }
      }
    }
  }
  return ntuples * wta_k;
}

/* dFastAtan2 (orbd.cu:986-998).  The quadrant step uses the double constant
 * M_PI (cuda_utils.h:7 leaves the float one commented out), so it is computed
 * in double and rounded to float, as here. */
float oo_fast_atan2(float y, float x) {
  const float absx = fabsf(x);
  const float absy = fabsf(y);
  const float a = fminf(absx, absy) / fmaxf(absx, absy);
  const float s = a * a;
  float r = fmaf(fmaf(fmaf(-0.0464964749f, s, 0.15931422f), s, -0.327622764f), s * a, a);
  r = (absy > absx ? 1.5707963267948966f - r : r);
  r = (x < 0 ? (float)(3.14159265358979323846 - (double)r) : r);
  r = (y < 0 ? -r : r);
  return r;
}

/* hFastDectectWithNMS pyramid (orbd.cu:1584-1600 with gDownSampleUnroll4,
 * orbd.cu:514-535): octave 0 is a copy of h*pitch0 input bytes; octave o is the
 * nearest sample img[y<<o][x<<o] of the input, with no blur. */
void oo_pyramid(const uint8_t* img, int pitch_in, uint8_t* pyr, const int* oszp, int n) {
  const int* osizes = oszp;
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  (void)pitch_in;
  memcpy(pyr, img, (size_t)osizes[0]);
  for (int o = 1; o < n; o++) {
    uint8_t* dst = pyr + offsets[o];
    for (int y = 0; y < heights[o]; y++)
      for (int x = 0; x < widths[o]; x++)
        dst[(size_t)y * pitchs[o] + x] = img[((size_t)y * pitchs[0] + x) << o];
  }
}

/* FAST ring (makeOffsets, orbd.cu:463-496): (dx, dy) for k = 0..15. */
static const int kRing[16][2] = {{0, 3},  {1, 3},  {2, 2},  {3, 1},  {3, 0},  {3, -1}, {2, -2}, {1, -3},
                                 {0, -3}, {-1, -3}, {-2, -2}, {-3, -1}, {-3, 0}, {-3, 1}, {-2, 2}, {-1, 3}};

/* dHarrisScore (orbd.cu:651-669): 7x7 window of 3x3 Sobel sums in int32 (the
 * products wrap as the GPU's 32-bit integer multiply does), then an FP32
 * combine.  harris_fma selects whether f(A) - 0.04f*f(B) is one fused op. */
static float harris(const uint8_t* ptr, int p, int harris_fma, float scale4) {
  int dxx = 0, dyy = 0, dxy = 0;
  for (int i = 0; i < 7; i++) {
    for (int j = 0; j < 7; j++) {
      const uint8_t* c = ptr + (i - 3) * p + (j - 3);
      int dx = ((int)c[1] - (int)c[-1]) * 2 + ((int)c[-p + 1] - (int)c[-p - 1]) + ((int)c[p + 1] - (int)c[p - 1]);
      int dy = ((int)c[p] - (int)c[-p]) * 2 + ((int)c[p - 1] - (int)c[-p - 1]) + ((int)c[p + 1] - (int)c[-p + 1]);
      dxx += dx * dx;
      dyy += dy * dy;
      dxy += dx * dy;
    }
  }
  int dsxy = dxx + dyy;
  int32_t A = (int32_t)((uint32_t)dxx * (uint32_t)dyy - (uint32_t)dxy * (uint32_t)dxy);
  uint32_t Bu = (uint32_t)dsxy * (uint32_t)dsxy;
  /* bit 1 of harris_fma: the square is converted as an unsigned 32-bit value
   * (a square cannot be negative without signed overflow, which is undefined,
   * so the compiler may pick the unsigned conversion). */
  float fB = (harris_fma & 2) ? (float)Bu : (float)(int32_t)Bu;
  float u;
  if (harris_fma & 1)
    u = fmaf(-0.04f, fB, (float)A);
  else
    u = (float)A - 0.04f * fB;
  return u * scale4;
}

/* dFastScore (orbd.cu:538-586, FAST_PATTERN 16). */
static float fast_score(const uint8_t* ptr, const int* pix, int threshold) {
  int v = ptr[0];
  short d[25];
  for (int k = 0; k < 25; k++) d[k] = (short)(v - ptr[pix[k]]);
  int a0 = threshold;
  for (int k = 0; k < 16; k += 2) {
    int a = d[k + 1] < d[k + 2] ? d[k + 1] : d[k + 2];
    if (d[k + 3] < a) a = d[k + 3];
    if (a <= a0) continue;
    for (int j = 4; j <= 8; j++)
      if (d[k + j] < a) a = d[k + j];
    int t = a < d[k] ? a : d[k];
    if (t > a0) a0 = t;
    t = a < d[k + 9] ? a : d[k + 9];
    if (t > a0) a0 = t;
  }
  int b0 = -a0;
  for (int k = 0; k < 16; k += 2) {
    int b = d[k + 1] > d[k + 2] ? d[k + 1] : d[k + 2];
    for (int j = 3; j <= 5; j++)
      if (d[k + j] > b) b = d[k + j];
    if (b >= b0) continue;
    for (int j = 6; j <= 8; j++)
      if (d[k + j] > b) b = d[k + j];
    int t = b > d[k] ? b : d[k];
    if (t < b0) b0 = t;
    t = b > d[k + 9] ? b : d[k + 9];
    if (t < b0) b0 = t;
  }
  return (float)(-b0 - 1);
}

/* gCalcExtramaMap (orbd.cu:672-756) for every octave in order 0..n-1
 * (orbd.cu:1616-1634): FAST-9 segment test, score, and the level-0 keyed
 * score map update "if (vmap < score) { vmap = score; layer = octave; }".
 * vmap/layer must be zeroed by the caller (orb.cpp:67-68). */
void oo_score_map(const uint8_t* pyr, const int* oszp, int n, int threshold, int harris_score, int harris_fma,
                  float* vmap, int* layer) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  const int p0 = pitchs[0];
  const float scale4 = oo_harris_scale();
  uint8_t lut[512];
  oo_fast_lut(threshold, lut);
  for (int o = 0; o < n; o++) {
    const int w = widths[o], h = heights[o], p = pitchs[o];
    const uint8_t* img = pyr + offsets[o];
    int pix[25];
    for (int k = 0; k < 16; k++) pix[k] = kRing[k][0] + kRing[k][1] * p;
    for (int k = 16; k < 25; k++) pix[k] = pix[k - 16];
#pragma omp parallel for schedule(static)
    for (int iy = 3; iy < h - 3; iy++) {
      for (int ix = 3; ix < w - 3; ix++) {
        const uint8_t* ptr = img + (size_t)iy * p + ix;
        const uint8_t* tab = lut + 255 - ptr[0];
        int d = tab[ptr[pix[0]]] | tab[ptr[pix[8]]];
        if (d == 0) continue;
        d &= tab[ptr[pix[2]]] | tab[ptr[pix[10]]];
        d &= tab[ptr[pix[4]]] | tab[ptr[pix[12]]];
        d &= tab[ptr[pix[6]]] | tab[ptr[pix[14]]];
        if (d == 0) continue;
        d &= tab[ptr[pix[1]]] | tab[ptr[pix[9]]];
        d &= tab[ptr[pix[3]]] | tab[ptr[pix[11]]];
        d &= tab[ptr[pix[5]]] | tab[ptr[pix[13]]];
        d &= tab[ptr[pix[7]]] | tab[ptr[pix[15]]];
        int corner = 0;
        if (d & 1) {
          int vt = ptr[0] - threshold, count = 0;
          for (int k = 0; k < 25; k++) {
            if (ptr[pix[k]] < vt) {
              if (++count > 8) { corner = 1; break; }
            } else {
              count = 0;
            }
          }
        } else if (d & 2) {
          int vt = ptr[0] + threshold, count = 0;
          for (int k = 0; k < 25; k++) {
            if (ptr[pix[k]] > vt) {
              if (++count > 8) { corner = 1; break; }
            } else {
              count = 0;
            }
          }
        }
        if (!corner) continue;
        float score = harris_score ? harris(ptr, p, harris_fma, scale4) : fast_score(ptr, pix, threshold);
        size_t idx = (size_t)(iy << o) * p0 + (ix << o);
        if (vmap[idx] < score) {
          vmap[idx] = score;
          layer[idx] = o;
        }
      }
    }
  }
}

/* gNmsUnroll4 (orbd.cu:919-983): a centre with score > 0 at octave o survives
 * unless a neighbour in the square of radius 2^o has a larger score, or an equal
 * score at dx <= 0 && dy <= 0.  Border: max(edge, 3) (orbd.cu:1567-1568).
 * Survivors are written in raster order (the reference appends them in
 * atomicInc order); returns the survivor count, writes at most cap. */
int oo_nms(const float* vmap, const int* layer, const int* oszp, int n, int border, oo_point* out, int cap) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int w = widths[0], h = heights[0], p = pitchs[0];
  if (border < 3) border = 3;
  int count = 0;
  for (int iy = border; iy < h - border; iy++) {
    for (int ix = border; ix < w - border; ix++) {
      const size_t vidx = (size_t)iy * p + ix;
      const float v = vmap[vidx];
      if (!(v > 0)) continue;
      const int o = layer[vidx];
      const int r = 1 << o;
      int sup = 0;
      for (int dy = -r; dy <= r && !sup; dy++) {
        for (int dx = -r; dx <= r; dx++) {
          if (dx == 0 && dy == 0) continue;
          const float u = vmap[vidx + (ptrdiff_t)dy * p + dx];
          if (u > 0 && (u > v || (u == v && dx <= 0 && dy <= 0))) {
            sup = 1;
            break;
          }
        }
      }
      if (sup) continue;
      if (count < cap) {
        oo_point* q = &out[count];
        q->x = ix;
        q->y = iy;
        q->octave = o;
        q->score = v;
        q->angle = 0.f;
        q->match = 0;
        q->distance = 0;
      }
      count++;
    }
  }
  return count;
}

/* angleIC (orbd.cu:1001-1036): intensity centroid over the umax disc on the
 * unblurred octave, then dFastAtan2 of the float moments. */
void oo_angle(const uint8_t* pyr, const int* oszp, int n, oo_point* pts, int npts, int patch_size) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  int umax[32];
  oo_umax(patch_size, umax);
  const int half_k = patch_size / 2;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < npts; i++) {
    oo_point* q = &pts[i];
    const int o = q->octave;
    const int pitch = pitchs[o];
    const uint8_t* center = pyr + offsets[o] + (ptrdiff_t)(q->y >> o) * pitch + (q->x >> o);
    int m01 = 0, m10 = 0;
    for (int u = -half_k; u <= half_k; ++u) m10 += u * center[u];
    for (int v = 1; v <= half_k; ++v) {
      int v_sum = 0;
      const int pofs = v * pitch;
      for (int u = -umax[v]; u <= umax[v]; ++u) {
        int vp = center[u + pofs], vm = center[u - pofs];
        v_sum += vp - vm;
        m10 += u * (vp + vm);
      }
      m01 += v * v_sum;
    }
    q->angle = oo_fast_atan2((float)m01, (float)m10);
  }
}

static inline int reflect101(int i, int sz) { /* dealBorder, cuda_utils.h:145-152 */
  if (i < 0) return -i;
  if (i >= sz) return sz + sz - 2 - i;
  return i;
}

static inline int rint_i(float v) { /* __float2int_rn: ties to even, NaN -> 0 */
  if (v != v) return 0;
  return (int)lrintf(v);
}

/* k0*t0 + k1*t1 + k2*t2 + k3*t3 summed left to right, as "wsum = k[0]*x;
 * wsum += k[i]*(...)" (orbd.cu:1292-1296).  mode bits 0-1 pick the first add:
 * 0 rounds both products, 1 fuses the k1 product, 2 fuses the k0 product;
 * bit 2 fuses the k2 and k3 products into their adds. */
static inline float dot4(const float* k, const float* t, int mode) {
  float acc;
  switch (mode & 3) {
    case 1: acc = fmaf(k[1], t[1], k[0] * t[0]); break;
    case 2: acc = fmaf(k[0], t[0], k[1] * t[1]); break;
    default: acc = k[0] * t[0] + k[1] * t[1]; break;
  }
  for (int i = 2; i <= 3; i++) acc = (mode & 4) ? fmaf(k[i], t[i], acc) : acc + k[i] * t[i];
  return acc;
}

/* gConv2dUnroll (orbd.cu:1273-1338) written out of place: separable 7-tap blur,
 * horizontal FP32 sums of integer pixels with reflect-101 columns, vertical FP32
 * sums of those rows with reflect-101 rows, then round-to-nearest-even to u8.
 * fma_h / fma_v are dot4 modes of the horizontal and vertical sums. */
void oo_blur(const uint8_t* pyr, uint8_t* out, const int* oszp, int n, int fma_h, int fma_v) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  float k[4];
  oo_gauss_kernel(k);
  for (int o = 0; o < n; o++) {
    const int w = widths[o], h = heights[o], p = pitchs[o];
    const uint8_t* src = pyr + offsets[o];
    uint8_t* dst = out + offsets[o];
    float* rows = (float*)malloc(sizeof(float) * (size_t)w * h);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++) {
      const uint8_t* s = src + (size_t)y * p;
      for (int x = 0; x < w; x++) {
        float t[4];
        t[0] = (float)(int)s[reflect101(x, w)];
        for (int i = 1; i <= 3; i++) t[i] = (float)((int)s[reflect101(x - i, w)] + (int)s[reflect101(x + i, w)]);
        rows[(size_t)y * w + x] = dot4(k, t, fma_h);
      }
    }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++) {
      for (int x = 0; x < w; x++) {
        float t[4];
        t[0] = rows[(size_t)reflect101(y, h) * w + x];
        for (int i = 1; i <= 3; i++)
          t[i] = rows[(size_t)reflect101(y - i, h) * w + x] + rows[(size_t)reflect101(y + i, h) * w + x];
        dst[(size_t)y * p + x] = (uint8_t)rint_i(dot4(k, t, fma_v));
      }
    }
    free(rows);
  }
}

/* getValue (orbd.cu:1341-1348): rotate a pattern point and sample.  The two
 * rotated coordinates are a*b -/+ c*d; rot = 0 rounds both products, 1 fuses the
 * first product into the add, 2 fuses the second. */
static inline uint8_t sample(const uint8_t* center, const int* pat, int idx, float s, float c, int pitch, int rot_x,
                             int rot_y) {
  const float x = (float)pat[2 * idx];
  const float y = (float)pat[2 * idx + 1];
  float fx, fy;
  if (rot_x == 1)
    fx = fmaf(x, c, -(y * s));
  else if (rot_x == 2)
    fx = fmaf(-y, s, x * c);
  else
    fx = x * c - y * s;
  if (rot_y == 1)
    fy = fmaf(x, s, y * c);
  else if (rot_y == 2)
    fy = fmaf(y, c, x * s);
  else
    fy = x * s + y * c;
  const int ix = rint_i(fx), iy = rint_i(fy);
  return center[(ptrdiff_t)iy * pitch + ix];
}

/* gDescrible + feature2/3/4 (orbd.cu:1351-1468): 32 bytes per keypoint on the
 * blurred octave; byte t is built from pattern points [pstep*t, pstep*t+pstep). */
void oo_describe(const uint8_t* blurred, const int* oszp, int n, const oo_point* pts, int npts, const float* sinv,
                 const float* cosv, const int* pat, int wta_k, int rot_x, int rot_y, uint8_t* desc) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  const int pstep = (wta_k == 2 || wta_k == 4) ? 16 : 12;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < npts; i++) {
    const oo_point* q = &pts[i];
    const int o = q->octave;
    const int pitch = pitchs[o];
    const uint8_t* center = blurred + offsets[o] + (ptrdiff_t)(q->y >> o) * pitch + (q->x >> o);
    const float s = sinv[i], c = cosv[i];
    for (int t = 0; t < 32; t++) {
      const int* pt = pat + 2 * pstep * t;
#define G(j) sample(center, pt, (j), s, c, pitch, rot_x, rot_y)
      uint8_t val = 0;
      if (wta_k == 2) {
        for (int j = 0; j < 8; j++) val |= (uint8_t)((G(2 * j) < G(2 * j + 1)) << j);
      } else if (wta_k == 3) {
        static const int idx3[4][3] = {{0, 1, 2}, {3, 4, 5}, {6, 7, 8}, {8, 9, 11}}; /* orbd.cu:1382-1384 */
        for (int g = 0; g < 4; g++) {
          int t0 = G(idx3[g][0]), t1 = G(idx3[g][1]), t2 = G(idx3[g][2]);
          int v = t2 > t1 ? (t2 > t0 ? 2 : 0) : (t1 > t0);
          val |= (uint8_t)(v << (2 * g));
        }
      } else {
        for (int g = 0; g < 4; g++) {
          int t0 = G(4 * g), t1 = G(4 * g + 1), t2 = G(4 * g + 2), t3 = G(4 * g + 3);
          int u = 0, v = 2;
          if (t1 > t0) t0 = t1, u = 1;
          if (t3 > t2) t2 = t3, v = 3;
          int kk = t0 > t2 ? u : v;
          val |= (uint8_t)(kk << (2 * g));
        }
      }
#undef G
      desc[(size_t)i * 32 + t] = val;
    }
  }
}

static inline int hamming256(const uint8_t* a, const uint8_t* b) {
  int s = 0;
  for (int j = 0; j < 4; j++) {
    uint64_t x, y;
    memcpy(&x, a + 8 * j, 8);
    memcpy(&y, b + 8 * j, 8);
    s += __builtin_popcountll(x ^ y);
  }
  return s;
}

/* gHammingMatch (orbd.cu:1471-1559): best and second-best distance over the
 * train set (both start at 256); match = argmin and distance = best when the
 * best is unique (best < second) and below MAX_DIST = 64, else -1 / -1. */
void oo_match(const uint8_t* d1, int n1, const uint8_t* d2, int n2, int* match, int* dist) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n1; i++) {
    int b1 = 256, b2 = 256, i1 = 0;
    for (int j = 0; j < n2; j++) {
      int s = hamming256(d1 + (size_t)32 * i, d2 + (size_t)32 * j);
      if (s < b1) {
        b2 = b1;
        b1 = s;
        i1 = j;
      } else if (s < b2) {
        b2 = s;
      }
    }
    if (b1 < b2 && b1 < 64) {
      match[i] = i1;
      dist[i] = b1;
    } else {
      match[i] = -1;
      dist[i] = -1;
    }
  }
}

/* k = 2 nearest neighbours, ordered by (distance, index); missing entries are
 * (0xFFFFFFFF, -1).  The reference-semantics match above follows from it. */
void oo_knn2(const uint8_t* q, int nq, const uint8_t* db, int ndb, uint32_t* dist2, int32_t* idx2) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nq; i++) {
    uint32_t b1 = 0xFFFFFFFFu, b2 = 0xFFFFFFFFu;
    int32_t i1 = -1, i2 = -1;
    for (int j = 0; j < ndb; j++) {
      uint32_t s = (uint32_t)hamming256(q + (size_t)32 * i, db + (size_t)32 * j);
      if (s < b1) {
        b2 = b1;
        i2 = i1;
        b1 = s;
        i1 = j;
      } else if (s < b2) {
        b2 = s;
        i2 = j;
      }
    }
    dist2[2 * i] = b1;
    dist2[2 * i + 1] = b2;
    idx2[2 * i] = i1;
    idx2[2 * i + 1] = i2;
  }
}

/* ------------------------------------------------------------------------ */
/* FP64 side-oracle and per-keypoint exception flags.                        */
/* ------------------------------------------------------------------------ */

/* The wrapped integer Harris sums of dHarrisScore (orbd.cu:651-669) at one
 * octave pixel: A = int32(dxx*dyy - dxy*dxy), B = uint32((dxx+dyy)^2), both
 * with the GPU's 32-bit wrap. */
static void harris_terms(const uint8_t* ptr, int p, int32_t* A, uint32_t* B) {
  int dxx = 0, dyy = 0, dxy = 0;
  for (int i = 0; i < 7; i++) {
    for (int j = 0; j < 7; j++) {
      const uint8_t* c = ptr + (i - 3) * p + (j - 3);
      int dx = ((int)c[1] - (int)c[-1]) * 2 + ((int)c[-p + 1] - (int)c[-p - 1]) + ((int)c[p + 1] - (int)c[p - 1]);
      int dy = ((int)c[p] - (int)c[-p]) * 2 + ((int)c[p - 1] - (int)c[-p - 1]) + ((int)c[p + 1] - (int)c[-p + 1]);
      dxx += dx * dx;
      dyy += dy * dy;
      dxy += dx * dy;
    }
  }
  int dsxy = dxx + dyy;
  *A = (int32_t)((uint32_t)dxx * (uint32_t)dyy - (uint32_t)dxy * (uint32_t)dxy);
  *B = (uint32_t)dsxy * (uint32_t)dsxy;
}

/* FP64 restatement of the Harris combine (orbd.cu:651-669) at each keypoint's
 * own octave pixel (x >> o, y >> o): the same wrapped integer terms, combined
 * as (A - 0.04 B) * (1 / (4*7*255))^4 in double with exact decimal constants.
 * terms[2i] = |A| and terms[2i+1] = 0.04 B (the magnitudes that cancel), so a
 * caller can scale an absolute floor by them. */
void oo_harris_f64(const uint8_t* pyr, const int* oszp, int n, const oo_point* pts, int npts, double* score,
                   double* terms) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  const double s = 1.0 / (4.0 * 7.0 * 255.0);
  const double scale4 = s * s * s * s;
  (void)widths;
  (void)heights;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < npts; i++) {
    const int o = pts[i].octave;
    const int p = pitchs[o];
    const uint8_t* ptr = pyr + offsets[o] + (ptrdiff_t)(pts[i].y >> o) * p + (pts[i].x >> o);
    int32_t A;
    uint32_t B;
    harris_terms(ptr, p, &A, &B);
    score[i] = ((double)A - 0.04 * (double)B) * scale4;
    if (terms) {
      terms[2 * i] = fabs((double)A) * scale4;
      terms[2 * i + 1] = 0.04 * (double)B * scale4;
    }
  }
}

/* FP64 restatement of angleIC + dFastAtan2 (orbd.cu:1001-1036, 986-998): the
 * same integer moments, then the same 3-term polynomial and quadrant folds in
 * double (not libm atan2: the polynomial itself is about 1e-5 rad from atan2).
 * Zero moments give NaN, as 0/0 does in the reference. */
void oo_angle_f64(const uint8_t* pyr, const int* oszp, int n, const oo_point* pts, int npts, int patch_size,
                  double* angle) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  const int* pitchs = heights + n;
  const int* offsets = pitchs + n;
  int umax[32];
  oo_umax(patch_size, umax);
  const int half_k = patch_size / 2;
  (void)widths;
  (void)heights;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < npts; i++) {
    const int o = pts[i].octave;
    const int pitch = pitchs[o];
    const uint8_t* center = pyr + offsets[o] + (ptrdiff_t)(pts[i].y >> o) * pitch + (pts[i].x >> o);
    int m01 = 0, m10 = 0;
    for (int u = -half_k; u <= half_k; ++u) m10 += u * center[u];
    for (int v = 1; v <= half_k; ++v) {
      int v_sum = 0;
      const int pofs = v * pitch;
      for (int u = -umax[v]; u <= umax[v]; ++u) {
        int vp = center[u + pofs], vm = center[u - pofs];
        v_sum += vp - vm;
        m10 += u * (vp + vm);
      }
      m01 += v * v_sum;
    }
    const double x = (double)m10, y = (double)m01;
    const double ax = fabs(x), ay = fabs(y);
    const double a = fmin(ax, ay) / fmax(ax, ay);
    const double q = a * a;
    double r = ((-0.0464964749 * q + 0.15931422) * q - 0.327622764) * q * a + a;
    if (ay > ax) r = 1.5707963267948966 - r;
    if (x < 0) r = 3.14159265358979323846 - r;
    if (y < 0) r = -r;
    angle[i] = r;
  }
}

/* Per-keypoint exception flags for the parity report:
 *  bit 0 (ORACLE_TIE): a rotated pattern coordinate x*c - y*s or x*s + y*c,
 *        evaluated in double from the float sin/cos the descriptor used, lies
 *        within tie_eps of a .5 rounding tie (getValue, orbd.cu:1341-1348), so
 *        the sampled pixel depends on the last bits of sin/cos and on FMA
 *        contraction;
 *  bit 1 (ORACLE_STRADDLE_ANGLE): the umax disc of angleIC (orbd.cu:1001-1036)
 *        reaches outside its octave's w x h rectangle;
 *  bit 2 (ORACLE_STRADDLE_DESC): a rotated, rounded pattern point of the
 *        descriptor (orbd.cu:1437-1468, rounding as the reference build)
 *        lands outside its octave's w x h rectangle.
 * Pixels outside the rectangle are pitch padding, a neighbouring octave or the
 * zero guard after the last one: the reference's result there depends on its
 * memory layout. */
void oo_exception_flags(const int* oszp, int n, const oo_point* pts, int npts, const float* sinv, const float* cosv,
                        const int* pat, int npat, int patch_size, double tie_eps, int* flags) {
  const int* widths = oszp + n;
  const int* heights = widths + n;
  int umax[32];
  oo_umax(patch_size, umax);
  const int half_k = patch_size / 2;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < npts; i++) {
    const int o = pts[i].octave;
    const int w = widths[o], h = heights[o];
    const int cx = pts[i].x >> o, cy = pts[i].y >> o;
    int f = 0;
    /* the disc: rows cy-half_k..cy+half_k; row v spans +-umax[|v|] (row 0 spans +-half_k) */
    for (int v = -half_k; v <= half_k && !(f & 2); v++) {
      const int u = v == 0 ? half_k : umax[v < 0 ? -v : v];
      if (cy + v < 0 || cy + v >= h || cx - u < 0 || cx + u >= w) f |= 2;
    }
    const float s = sinv[i], c = cosv[i];
    for (int k = 0; k < npat; k++) {
      const double px = (double)pat[2 * k], py = (double)pat[2 * k + 1];
      const double fx = px * (double)c - py * (double)s;
      const double fy = px * (double)s + py * (double)c;
      const double tx = fx - floor(fx), ty = fy - floor(fy);
      if (fabs(tx - 0.5) < tie_eps || fabs(ty - 0.5) < tie_eps) f |= 1;
      const float gx = fmaf((float)pat[2 * k], c, -((float)pat[2 * k + 1] * s));
      const float gy = fmaf((float)pat[2 * k], s, (float)pat[2 * k + 1] * c);
      const int ix = cx + rint_i(gx), iy = cy + rint_i(gy);
      if (ix < 0 || ix >= w || iy < 0 || iy >= h) f |= 4;
    }
    flags[i] = f;
  }
}
