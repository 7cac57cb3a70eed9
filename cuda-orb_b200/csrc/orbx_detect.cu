// Pyramid, blur, FAST-9 + Harris score map and NMS for sm_100a.
//
// Each launch covers a batch of frames; a block finds its frame through a
// prefix table of tile counts.  Pyramid layout, guards and the score-map
// format follow the reference (orb.cpp:145-191, orbd.cu:1576-1577) so that
// reads that leave an octave see the same bytes the reference sees.
#include "orbx_device.cuh"
#include "orbx_internal.cuh"
#include "orbx_fast.cuh"

namespace orbx {

// ---------------------------------------------------------------------------
// Pyramid + blur
//
// Octave o is the nearest-neighbour decimation img[y<<o][x<<o] of level 0
// (gDownSampleUnroll4, orbd.cu:514-535; octave 0 is a copy, orbd.cu:1584).
// The blurred pyramid is the separable 7-tap sigma-2 filter of each octave with
// reflect-101 borders (gConv2dUnroll, orbd.cu:1273-1338), computed here out of
// place, so it has no dependence on block scheduling.  One block owns a
// kPyrTW x kPyrTH octave tile: it stages the tile plus a 3-pixel reflected
// halo in shared memory, writes the raw tile, and blurs it.  With pyr_src set
// the octaves are read from an existing pyramid instead (hGassianBlur on a
// caller's buffer, orbd.cu:1732-1773).
// ---------------------------------------------------------------------------
constexpr int kPyrSW = kPyrTW + 8;  // 3-pixel halo each side, padded to a multiple of 4
constexpr int kPyrSH = kPyrTH + 6;

// Exact small-integer <-> float conversions on the full-rate pipes: a float
// whose exponent field is 2^23 holds the integer in its mantissa.
__device__ __forceinline__ float u8_to_float(uint32_t x) {  // 0 <= x < 2^23
  return __fsub_rn(__uint_as_float(0x4B000000u | x), 8388608.0f);
}
__device__ __forceinline__ uint32_t float_to_u8_rne(float v) {  // 0 <= v < 2^22: round to nearest, ties to even
  return (uint32_t)(__float_as_int(__fadd_rn(v, 12582912.0f)) - 0x4B400000);
}

__global__ void __launch_bounds__(256) k_pyramid_blur(Batch b) {
  __shared__ __align__(16) float s_src[kPyrSH * kPyrSW];
  __shared__ __align__(16) uint8_t s_byte[kPyrSH * kPyrSW];
  __shared__ __align__(16) float s_row[kPyrSH * kPyrTW];

  const int t = blockIdx.x;
  const int f = find_frame(b.pyr_base, b.n_frames, t);
  const Frame& F = b.frames[f];
  int lt = t - b.pyr_base[f];
  int o = 0;
  while (o + 1 < F.n_oct && lt >= F.pyr_tile_base[o + 1]) o++;
  lt -= F.pyr_tile_base[o];
  const int tiles_x = F.pyr_tiles_x[o];
  const int x0 = (lt % tiles_x) * kPyrTW;
  const int y0 = (lt / tiles_x) * kPyrTH;
  const int ow = F.ow[o], oh = F.oh[o], op = F.op[o];
  const uint8_t* __restrict__ img = F.img;
  const int pitch_in = F.pitch_in;

  // Per-frame housekeeping for the later stages of the same batch.
  if (o == 0 && lt == 0) {
    for (int i = threadIdx.x; i < F.nms_strips; i += blockDim.x) F.nms_status[i] = 0ull;
    if (threadIdx.x == 0) {
      *F.count = 0;
      if (F.total) *F.total = 0;
    }
  }
  if (t == 0 && threadIdx.x == 0) *b.nms_ticket = 0u;

  // stage: source rows y0-3 .. y0+34, columns x0-3 .. x0+132, reflect-101 at
  // the octave edges, as floats and as bytes
  const uint8_t* __restrict__ psrc = F.pyr_src ? F.pyr_src + F.ooff[o] : nullptr;
  // octave 0 read from a 4-byte aligned image: interior groups take two aligned
  // words (the group starts one byte past a word boundary, x0 being a multiple of 4)
  const bool words0 = (o == 0) && !psrc && ((reinterpret_cast<uintptr_t>(img) | (uintptr_t)pitch_in) & 3u) == 0;
  constexpr int kGroups = kPyrSW / 4;
  for (int it = threadIdx.x; it < kPyrSH * kGroups; it += blockDim.x) {
    const int r = it / kGroups;
    const int g = it - r * kGroups;
    const int y = reflect101(y0 - 3 + r, oh);
    const uint8_t* rowp = psrc ? psrc + (size_t)y * op : img + (size_t)(y << o) * pitch_in;
    const int sh = psrc ? 0 : o;
    const int cx = x0 - 3 + 4 * g;
    uint32_t v[4];
    if (words0 && cx >= 1 && cx + 3 < ow) {
      // bytes cx-1 .. cx+6 lie in [0, pitch_in): cx + 3 < ow <= pitch_in and both words are aligned
      const uint32_t* wp = reinterpret_cast<const uint32_t*>(rowp + (cx - 1));
      const uint32_t word = __byte_perm(__ldg(wp), __ldg(wp + 1), 0x4321);
#pragma unroll
      for (int j = 0; j < 4; j++) v[j] = (word >> (8 * j)) & 0xFFu;
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) v[j] = __ldg(rowp + (reflect101(cx + j, ow) << sh));
    }
    reinterpret_cast<float4*>(s_src)[it] = make_float4(u8_to_float(v[0]), u8_to_float(v[1]), u8_to_float(v[2]),
                                                       u8_to_float(v[3]));
    reinterpret_cast<uint32_t*>(s_byte)[it] = v[0] | (v[1] << 8) | (v[2] << 16) | (v[3] << 24);
  }
  __syncthreads();

  const float* k = b.gauss;
  // horizontal pass: 4 consecutive outputs per thread; integer tap sums are
  // exact in float, so they are summed as floats
  for (int it = threadIdx.x; it < kPyrSH * (kPyrTW / 4); it += blockDim.x) {
    const int r = it / (kPyrTW / 4);
    const int g = it - r * (kPyrTW / 4);
    const float4* q = reinterpret_cast<const float4*>(s_src + r * kPyrSW) + g;
    const float4 a0 = q[0], a1 = q[1], a2 = q[2];
    const float p[12] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w};
    float4 out;
    float* op4 = &out.x;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float t1 = __fadd_rn(p[j + 2], p[j + 4]);
      const float t2 = __fadd_rn(p[j + 1], p[j + 5]);
      const float t3 = __fadd_rn(p[j], p[j + 6]);
      op4[j] = gauss_dot4(k, p[j + 3], t1, t2, t3);
    }
    reinterpret_cast<float4*>(s_row + r * kPyrTW)[g] = out;
  }
  __syncthreads();

  // vertical pass and stores: 4 consecutive columns of one row per thread
  uint8_t* P = F.pyr + F.ooff[o];
  uint8_t* B = F.blr + F.ooff[o];
  const bool copy_pad = (o == 0) && (pitch_in == op);
  for (int it = threadIdx.x; it < kPyrTH * (kPyrTW / 4); it += blockDim.x) {
    const int r = it / (kPyrTW / 4);
    const int g = it - r * (kPyrTW / 4);
    const int y = y0 + r;
    const int x = x0 + 4 * g;
    if (y >= oh || x >= op) continue;
    float4 h[7];
#pragma unroll
    for (int j = 0; j < 7; j++) h[j] = reinterpret_cast<const float4*>(s_row + (r + j) * kPyrTW)[g];
    const float* hf = reinterpret_cast<const float*>(h);
    uint32_t bw = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float t1 = __fadd_rn(hf[8 + j], hf[16 + j]);
      const float t2 = __fadd_rn(hf[4 + j], hf[20 + j]);
      const float t3 = __fadd_rn(hf[j], hf[24 + j]);
      bw |= (float_to_u8_rne(gauss_dot4(k, hf[12 + j], t1, t2, t3)) & 0xFFu) << (8 * j);
    }
    // raw bytes of the same 4 pixels: staged columns 4g+3 .. 4g+6 of row r+3
    const uint32_t* sb = reinterpret_cast<const uint32_t*>(s_byte + (r + 3) * kPyrSW) + g;
    const uint32_t pw = __byte_perm(sb[0], sb[1], 0x6543);
    const size_t a = (size_t)y * op + x;
    if (x + 4 <= ow) {
      *reinterpret_cast<uint32_t*>(B + a) = bw;
      *reinterpret_cast<uint32_t*>(P + a) = pw;
    } else {
      // the group reaches into the row padding: octave 0 carries the caller's
      // padding bytes (the reference copies h * pitch0 bytes, orbd.cu:1584),
      // other octaves hold zeros
#pragma unroll
      for (int j = 0; j < 4; j++) {
        if (x + j < ow) {
          B[a + j] = (uint8_t)(bw >> (8 * j));
          P[a + j] = (uint8_t)(pw >> (8 * j));
        } else {
          const uint8_t v = psrc ? __ldg(psrc + a + j)
                                 : (copy_pad ? __ldg(img + (size_t)y * pitch_in + x + j) : (uint8_t)0);
          B[a + j] = v;
          P[a + j] = v;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FAST-9 + score -> level-0 keyed score map
//
// gCalcExtramaMap (orbd.cu:672-756) run for octaves 0..n-1 in order
// (orbd.cu:1616-1634): a pixel is a corner when 9 contiguous ring pixels are
// all darker than v - t or all brighter than v + t (the reference's LUT pre-test
// and arc loop decide exactly this).  Its score lands at level-0 position
// (x << o, y << o) if strictly greater than what a lower octave put there.
// One block owns a kDetTW x kDetTH level-0 tile and all octave pixels that map
// into it; it stages each octave's pixels with a 4-pixel halo (the Harris
// window with its Sobel reach) in shared memory using the pyramid's linear
// addressing, so reads past an octave edge return the same neighbouring bytes
// as in the reference, merges the octaves in shared memory, and writes the
// tile's occupancy bits densely and its scores sparsely (no clearing pass).
// ---------------------------------------------------------------------------
constexpr int kHalo = 4;
__host__ __device__ constexpr int det_stage_off(int octave) {
  int s = 0;
  for (int o = 0; o < octave; o++) s += ((kDetTW >> o) + 2 * kHalo) * ((kDetTH >> o) + 2 * kHalo);
  return s;
}
__host__ __device__ constexpr int det_stage_bytes() { return det_stage_off(kMaxOctaves); }

// dHarrisScore (orbd.cu:651-669) on a shared-memory tile of row stride sw.
// Integer sums wrap as 32-bit; the final combine is
// fma(-0.04f, (float)(uint32)(dsxy*dsxy), (float)(int32)(dxx*dyy - dxy*dxy)) * scale^4,
// which is how the reference build evaluates
// (dxx*dyy - dxy*dxy - HARRIS_K*(dsxy*dsxy)) * d_scale_sq_sq.
__device__ __forceinline__ float harris_score(const uint8_t* c, int sw, float scale4) {
  int dxx = 0, dyy = 0, dxy = 0;
#pragma unroll 1
  for (int i = -3; i <= 3; i++) {
#pragma unroll
    for (int j = -3; j <= 3; j++) {
      const uint8_t* q = c + i * sw + j;
      const int dx = ((int)q[1] - (int)q[-1]) * 2 + ((int)q[-sw + 1] - (int)q[-sw - 1]) +
                     ((int)q[sw + 1] - (int)q[sw - 1]);
      const int dy = ((int)q[sw] - (int)q[-sw]) * 2 + ((int)q[sw - 1] - (int)q[-sw - 1]) +
                     ((int)q[sw + 1] - (int)q[-sw + 1]);
      dxx += dx * dx;
      dyy += dy * dy;
      dxy += dx * dy;
    }
  }
  return harris_combine(dxx, dyy, dxy, scale4);
}

// Byte-wise arithmetic on packed words with plain integer operations (the
// byte-SIMD intrinsics are several instructions each on this architecture).
constexpr uint32_t kB7 = 0x80808080u, kLo7 = 0x7F7F7F7Fu;
// bit 7 of each byte set where x < y (unsigned): the 7-bit differences cannot
// borrow across bytes, and the top bits decide when they differ
__device__ __forceinline__ uint32_t swar_lt(uint32_t x, uint32_t y) {
  const uint32_t t = (x | kB7) - (y & kLo7);
  return ((~x & y) | (~(x ^ y) & ~t)) & kB7;
}
// max(v - t, 0) and min(v + t, 255) per byte, t given in every byte
__device__ __forceinline__ uint32_t swar_sub_sat(uint32_t v, uint32_t t4) {
  const uint32_t d = ((v | kB7) - (t4 & kLo7)) ^ ((v ^ ~t4) & kB7);
  return d & ~((swar_lt(v, t4) >> 7) * 0xFFu);
}
__device__ __forceinline__ uint32_t swar_add_sat(uint32_t v, uint32_t t4) {
  const uint32_t s = ((v & kLo7) + (t4 & kLo7)) ^ ((v ^ t4) & kB7);
  const uint32_t carry = ((v & t4) | ((v | t4) & ~s)) & kB7;
  return s | ((carry >> 7) * 0xFFu);
}

// Necessary condition for FAST-9: every run of 9 ring pixels contains two
// neighbouring cardinal points (ring positions k and k+4, k = 0, 4, 8, 12), so
// both of some such pair must be darker than v - t, or both brighter than
// v + t.  It never changes a result.  Evaluated for four horizontally adjacent
// centres at once on packed bytes: w points at the aligned word holding them
// (row stride sw bytes, a multiple of 4); returns bit 7 of each byte whose
// centre passes.  Saturating v - t and v + t (t <= 255) give the same answers
// as the signed comparisons p < v - t and p > v + t.
__device__ __forceinline__ uint32_t fast9_pretest4(const uint8_t* w, int sw, uint32_t t4) {
  const uint32_t c = *reinterpret_cast<const uint32_t*>(w);
  const uint32_t cl = *reinterpret_cast<const uint32_t*>(w - 4);
  const uint32_t cr = *reinterpret_cast<const uint32_t*>(w + 4);
  const uint32_t p0 = *reinterpret_cast<const uint32_t*>(w + 3 * sw);   // ring 0: (x, y + 3)
  const uint32_t p8 = *reinterpret_cast<const uint32_t*>(w - 3 * sw);   // ring 8: (x, y - 3)
  const uint32_t p4 = __byte_perm(c, cr, 0x6543);                       // ring 4: (x + 3, y)
  const uint32_t p12 = __byte_perm(cl, c, 0x4321);                      // ring 12: (x - 3, y)
  const uint32_t lo = swar_sub_sat(c, t4), hi = swar_add_sat(c, t4);
  const uint32_t d0 = swar_lt(p0, lo), d4 = swar_lt(p4, lo), d8 = swar_lt(p8, lo), d12 = swar_lt(p12, lo);
  const uint32_t b0 = swar_lt(hi, p0), b4 = swar_lt(hi, p4), b8 = swar_lt(hi, p8), b12 = swar_lt(hi, p12);
  return ((d0 | d8) & (d4 | d12)) | ((b0 | b8) & (b4 | b12));
}

__device__ __forceinline__ float corner_score(const Batch& b, const uint8_t* c, int sw) {
  if (b.harris) return harris_score(c, sw, b.harris_scale4);
  const int v = c[0];
  int d[25];
#pragma unroll
  for (int k = 0; k < 25; k++) d[k] = (int)(short)(v - c[c_ring[k & 15][1] * sw + c_ring[k & 15][0]]);
  return fast_score(d, b.fast_thr);
}

// Tile-level candidate lists hold (octave, row, column) of the octave tile as
// o << 11 | ly << 6 | lx; a tile has at most 2048 + 512 + 128 + 32 + 8 pixels.
constexpr int kDetMaxCand = 2728;
__device__ __forceinline__ uint16_t det_item(int o, int ly, int lx) { return (uint16_t)((o << 11) | (ly << 6) | lx); }

// Merge key of a level-0 position: the larger score wins and, between equal
// scores, the lower octave (the reference visits octaves in increasing order
// and replaces only on a strictly larger score).  Only scores > 0 are stored.
__device__ __forceinline__ unsigned long long det_key(float score, int o) {
  return ((unsigned long long)__float_as_uint(score) << 32) | (unsigned)(7 - o);
}

__global__ void __launch_bounds__(256, 4) k_detect(Batch b) {
  __shared__ __align__(16) uint8_t s_stage[det_stage_bytes()];
  __shared__ __align__(16) unsigned long long s_key[kDetTH * kDetTW];
  __shared__ uint16_t s_cand[kDetMaxCand];
  __shared__ uint16_t s_corner[kDetMaxCand];
  __shared__ int s_n[2];
  __shared__ uint32_t s_occ[kDetTH * kDetTW / 32];
  __shared__ int s_ow[kMaxOctaves], s_oh[kMaxOctaves];

  const int t = blockIdx.x;
  const int f = find_frame(b.det_base, b.n_frames, t);
  const Frame& F = b.frames[f];
  const int lt = t - b.det_base[f];
  const int X0 = (lt % F.det_tiles_x) * kDetTW;
  const int Y0 = (lt / F.det_tiles_x) * kDetTH;
  const int n_oct = F.n_oct;
  const uint8_t* __restrict__ pyr = F.pyr;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int thr = b.fast_thr;

  for (int i = threadIdx.x; i < kDetTH * kDetTW / 2; i += blockDim.x)
    reinterpret_cast<ulonglong2*>(s_key)[i] = make_ulonglong2(0ull, 0ull);
  if (threadIdx.x < kDetTH * kDetTW / 32) s_occ[threadIdx.x] = 0u;
  if (threadIdx.x < 2) s_n[threadIdx.x] = 0;
  if (threadIdx.x < kMaxOctaves) {
    s_ow[threadIdx.x] = threadIdx.x < n_oct ? F.ow[threadIdx.x] : 0;
    s_oh[threadIdx.x] = threadIdx.x < n_oct ? F.oh[threadIdx.x] : 0;
  }
  // Stage every octave's tile with its halo, 4 bytes per load, one row per warp
  // and step: octave offsets and pitches are multiples of 128 and (X0 >> o) - 4
  // is a multiple of 4; a staged row is at most 18 words.
  for (int o = 0; o < n_oct; o++) {
    const int sw = (kDetTW >> o) + 2 * kHalo;
    const int sh = (kDetTH >> o) + 2 * kHalo;
    const int sw4 = sw >> 2;
    const int op = F.op[o];
    const long long base = F.ooff[o] + (long long)((Y0 >> o) - kHalo) * op + ((X0 >> o) - kHalo);
    uint32_t* dst = reinterpret_cast<uint32_t*>(s_stage + det_stage_off(o));
    if (lane < sw4)
      for (int r = warp; r < sh; r += 8)
        dst[r * sw4 + lane] = __ldg(reinterpret_cast<const uint32_t*>(pyr + base + (long long)r * op) + lane);
  }
  __syncthreads();

  // 1. cardinal pre-test, four centres per word, words of every octave spread
  //    over the whole block (octave o has (32 >> o) rows of (16 >> o) words)
  {
    const uint32_t t4 = (uint32_t)min(max(thr, 0), 255) * 0x01010101u;
    int total = 0;
    for (int o = 0; o < n_oct; o++) total += 512 >> (2 * o);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      int o = 0, w = i;
      while (w >= (512 >> (2 * o))) {
        w -= 512 >> (2 * o);
        o++;
      }
      const int nwl = 4 - o;  // log2 words per row
      const int ly = w >> nwl, lx = (w & ((1 << nwl) - 1)) << 2;
      const int x = (X0 >> o) + lx, y = (Y0 >> o) + ly;
      const int ow = s_ow[o], oh = s_oh[o];
      uint32_t m = 0u;
      if (y >= 3 && y < oh - 3 && x < ow - 3) {
        const int sw = (kDetTW >> o) + 2 * kHalo;
        m = fast9_pretest4(s_stage + det_stage_off(o) + (ly + kHalo) * sw + (lx + kHalo), sw, t4);
        if (x < 3 || x + 3 >= ow - 3) {  // border word: keep the centres with 3 <= x + k < ow - 3
          uint32_t vm = 0u;
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (x + k >= 3 && x + k < ow - 3) vm |= 0xFFu << (8 * k);
          m &= vm;
        }
      }
      m &= 0x80808080u;
      if (m) {
        int pos = atomicAdd(&s_n[0], __popc(m));
        while (m) {
          const int k = (__ffs(m) >> 3) - 1;
          m &= m - 1u;
          s_cand[pos++] = det_item(o, ly, lx + k);
        }
      }
    }
  }
  __syncthreads();

  // 2. full 9-arc segment test of the candidates
  {
    const int n1 = s_n[0];
    for (int j = threadIdx.x; j < n1; j += blockDim.x) {
      const int e = s_cand[j];
      const int o = e >> 11, ly = (e >> 6) & 31, lx = e & 63;
      const int sw = (kDetTW >> o) + 2 * kHalo;
      const uint8_t* c = s_stage + det_stage_off(o) + (ly + kHalo) * sw + (lx + kHalo);
      const int v = c[0];
      if (fast9_full(c, sw, v - thr, v + thr)) s_corner[atomicAdd(&s_n[1], 1)] = (uint16_t)e;
    }
  }
  __syncthreads();

  // 3. scores of the corners, merged into the level-0 map
  {
    const int n2 = s_n[1];
    if (b.harris) {
      // 32 groups of 8 lanes, one corner per group; lane s of a group takes
      // window positions s, s + 8, ... of the 7x7 Harris window (the 32-bit sums
      // wrap, so their order is free)
      const int gid = threadIdx.x >> 3, sub = threadIdx.x & 7;
      for (int j0 = 0; j0 < n2; j0 += 32) {
        if (j0 + 4 * warp >= n2) break;  // this warp's four groups have no corner (warp-uniform)
        const int j = j0 + gid;
        int dxx = 0, dyy = 0, dxy = 0;
        int e = 0;
        if (j < n2) {
          e = s_corner[j];
          const int o = e >> 11, ly = (e >> 6) & 31, lx = e & 63;
          const int sw = (kDetTW >> o) + 2 * kHalo;
          const uint8_t* c = s_stage + det_stage_off(o) + (ly + kHalo) * sw + (lx + kHalo);
          for (int pos = sub; pos < 49; pos += 8) {
            const int wy = pos / 7 - 3, wx = pos % 7 - 3;
            const uint8_t* q = c + wy * sw + wx;
            const int dx = ((int)q[1] - (int)q[-1]) * 2 + ((int)q[-sw + 1] - (int)q[-sw - 1]) +
                           ((int)q[sw + 1] - (int)q[sw - 1]);
            const int dy = ((int)q[sw] - (int)q[-sw]) * 2 + ((int)q[sw - 1] - (int)q[-sw - 1]) +
                           ((int)q[sw + 1] - (int)q[-sw + 1]);
            dxx += dx * dx;
            dyy += dy * dy;
            dxy += dx * dy;
          }
        }
#pragma unroll
        for (int d = 4; d >= 1; d >>= 1) {
          dxx += __shfl_xor_sync(0xffffffffu, dxx, d);
          dyy += __shfl_xor_sync(0xffffffffu, dyy, d);
          dxy += __shfl_xor_sync(0xffffffffu, dxy, d);
        }
        if (j < n2 && sub == 0) {
          const int o = e >> 11, ly = (e >> 6) & 31, lx = e & 63;
          const float score = harris_combine(dxx, dyy, dxy, b.harris_scale4);
          if (score > 0.f) {
            const int m = (ly << o) * kDetTW + (lx << o);
            if (atomicMax(&s_key[m], det_key(score, o)) == 0ull) atomicOr(&s_occ[m >> 5], 1u << (m & 31));
          }
        }
      }
    } else {
      for (int j = threadIdx.x; j < n2; j += blockDim.x) {
        const int e = s_corner[j];
        const int o = e >> 11, ly = (e >> 6) & 31, lx = e & 63;
        const int sw = (kDetTW >> o) + 2 * kHalo;
        const float score = corner_score(b, s_stage + det_stage_off(o) + (ly + kHalo) * sw + (lx + kHalo), sw);
        if (score > 0.f) {
          const int m = (ly << o) * kDetTW + (lx << o);
          if (atomicMax(&s_key[m], det_key(score, o)) == 0ull) atomicOr(&s_occ[m >> 5], 1u << (m & 31));
        }
      }
    }
  }
  __syncthreads();

  // Output: the tile's occupancy words (every word written, so no clearing
  // pass), then score and octave only where a bit is set.  The tile's 64
  // columns are two aligned 32-bit words of each row (pitch0 is a multiple of 128).
  if (threadIdx.x < kDetTH * kDetTW / 32) {
    const int r = threadIdx.x >> 1, half = threadIdx.x & 1;
    const int Y = Y0 + r;
    if (Y < F.h) {
      uint32_t m = s_occ[threadIdx.x];
      const size_t a0 = (size_t)Y * F.op[0] + X0 + 32 * half;
      F.occ[a0 >> 5] = m;
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1u;
        const unsigned long long key = s_key[r * kDetTW + 32 * half + k];
        F.vmap[a0 + k] = __uint_as_float((uint32_t)(key >> 32));
        F.oct8[a0 + k] = (uint8_t)(7 - (int)(key & 0xFFu));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// NMS + ordered compaction
//
// gNmsUnroll4 (orbd.cu:919-983): a level-0 position with score v > 0 from
// octave o survives unless a neighbour in the square of radius 2^o has a larger
// score, or an equal one at dx <= 0 && dy <= 0.  The reference appends
// survivors with atomicInc (order and, past max_pts, the kept subset depend on
// scheduling).  Here each block takes a full-width strip of F.nms_rows rows in
// ticket order, ranks its survivors with warp ballots, and chains strip totals
// with a decoupled look-back, so keypoints come out in raster order and the cap
// keeps the first max_pts of them.
// ---------------------------------------------------------------------------
constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagPre = 2ull << 32;
constexpr int kLookbackSpinLimit = 1 << 22;

// Warp 0 of a strip's block resolves the strip's exclusive prefix: it reads the
// look-back words of up to 32 predecessors per round with acquire loads, and
// stops at the nearest one that already carries an inclusive prefix.
__device__ __forceinline__ int nms_lookback(unsigned long long* st, int s, int lane, int* err) {
  int excl = 0;
  int j = s - 1;
  int spins = 0;
  while (j >= 0) {
    const int idx = j - lane;
    const unsigned long long wv = (idx >= 0) ? ld_acquire_u64(&st[idx]) : kFlagPre;
    const unsigned long long flag = wv & (3ull << 32);
    const unsigned pre = __ballot_sync(0xffffffffu, flag == kFlagPre);
    const unsigned notready = __ballot_sync(0xffffffffu, flag == 0ull);
    const int first_pre = pre ? (__ffs(pre) - 1) : 32;
    const unsigned need = (first_pre >= 31) ? 0xffffffffu : ((2u << first_pre) - 1u);
    if (notready & need) {
      if (++spins > kLookbackSpinLimit) {
        if (lane == 0) atomicOr(err, kErrLookbackTimeout);
        break;
      }
      __nanosleep(20);
      continue;
    }
    int v = ((need >> lane) & 1u) ? (int)(unsigned)wv : 0;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    excl += v;
    if (first_pre < 32) break;
    j -= 32;
  }
  return excl;
}

// Neighbour rule of gNmsUnroll4 (orbd.cu:938-956) for the centre at linear
// index idx (score v, octave o), checked by a group of kNmsGroup lanes: lane
// `sub` of the group takes window rows dy = sub - r, sub + kNmsGroup - r, ...;
// each row is at most two occupancy words, and scores are read only where a
// bit is set.  Returns whether this lane's rows hold a suppressing position.
// Positions are linear like the reference's (a column past the edge is the
// adjacent row's entry); positions outside the map, reachable only with an
// edge threshold below 2^o, are empty.
constexpr int kNmsGroup = 8;
constexpr int kNmsChunkWords = 128;  // occupancy words compacted per round: at most 4096 centres

__device__ __forceinline__ bool nms_suppressed_rows(const Frame& F, long long idx, float v, int o, int p0,
                                                    long long npx, int sub) {
  const int r = 1 << o;
  for (int dyi = sub; dyi <= 2 * r; dyi += kNmsGroup) {
    const int dy = dyi - r;
    const long long rc = idx + (long long)dy * p0;
    long long lo = rc - r, hi = rc + r;
    if (hi < 0 || lo >= npx) continue;
    if (lo < 0) lo = 0;
    if (hi >= npx) hi = npx - 1;
    for (long long wi = lo >> 5; wi <= (hi >> 5); wi++) {
      const long long base = wi << 5;
      uint32_t m = __ldg(F.occ + wi);
      if (base < lo) m &= ~0u << (int)(lo - base);
      if (hi - base < 31) m &= (2u << (int)(hi - base)) - 1u;
      while (m) {
        const int bb = __ffs(m) - 1;
        m &= m - 1u;
        const long long li = base + bb;
        if (li == idx) continue;
        const int dx = (int)(li - rc);
        const float u = __ldg(F.vmap + li);
        if (u > v || (u == v && dx <= 0 && dy <= 0)) return true;
      }
    }
  }
  return false;
}

__global__ void __launch_bounds__(256) k_nms(Batch b) {
  __shared__ uint32_t s_sur[kNmsMaxWords];
  __shared__ int s_pref[kNmsMaxWords];
  __shared__ uint16_t s_cand[kNmsChunkWords * 32];
  __shared__ float s_cv[kNmsChunkWords * 32];
  __shared__ uint8_t s_co[kNmsChunkWords * 32];
  __shared__ int s_ncand[2];
  __shared__ int s_warp_tot[8];
  __shared__ int s_ticket, s_base;

  if (threadIdx.x == 0) s_ticket = (int)atomicAdd(b.nms_ticket, 1u);
  __syncthreads();
  const int ticket = s_ticket;
  const int f = find_frame(b.nms_base, b.n_frames, ticket);
  const Frame& F = b.frames[f];
  const int s = ticket - b.nms_base[f];
  const int border = F.border;
  const int row0 = border + s * F.nms_rows;
  const int row1 = min(row0 + F.nms_rows, F.h - border);
  const int xlo = border, xhi = F.w - border;  // columns [xlo, xhi)
  const int wlo = xlo >> 5, whi = (xhi - 1) >> 5;
  const int nw = whi - wlo + 1;
  const int nwords = (row1 - row0) * nw;
  const int p0 = F.op[0];
  const int wpr = p0 >> 5;  // occupancy words per row
  const long long npx = (long long)F.h * p0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // pass 1: survivor bits of every occupancy word of the strip.  In rounds of
  // kNmsChunkWords words: the centres of the round (with their scores) are
  // compacted into shared memory, then checked by 32 groups of 8 lanes, so a
  // textured patch of the strip spreads over every warp.
  for (int k = threadIdx.x; k < nwords; k += blockDim.x) s_sur[k] = 0u;
  if (threadIdx.x == 0) s_ncand[0] = 0;
  const int gid = warp * (32 / kNmsGroup) + (lane / kNmsGroup), sub = lane % kNmsGroup;
  const uint32_t gmask = ((1u << kNmsGroup) - 1u) << (lane & ~(kNmsGroup - 1));
  for (int c0 = 0, round = 0; c0 < nwords; c0 += kNmsChunkWords, round++) {
    int* cnt = &s_ncand[round & 1];
    __syncthreads();  // the previous round's checks are done; its counter is free
    if (threadIdx.x == 0) s_ncand[(round + 1) & 1] = 0;
    const int k = c0 + (int)threadIdx.x;
    if (threadIdx.x < kNmsChunkWords && k < nwords) {
      const int row = row0 + k / nw;
      const int wj = wlo + k % nw;
      const int cbase = wj << 5;
      uint32_t m = __ldg(F.occ + (long long)row * wpr + wj);
      if (cbase < xlo) m &= ~0u << (xlo - cbase);
      if (xhi - cbase < 32) m &= (xhi - cbase <= 0) ? 0u : ((xhi - cbase == 32) ? ~0u : ((1u << (xhi - cbase)) - 1u));
      if (m) {
        int pos = atomicAdd(cnt, __popc(m));
        while (m) {
          const int bit = __ffs(m) - 1;
          m &= m - 1u;
          const long long idx = (long long)row * p0 + cbase + bit;
          s_cand[pos] = (uint16_t)(((k - c0) << 5) | bit);
          s_cv[pos] = __ldg(F.vmap + idx);
          s_co[pos] = __ldg(F.oct8 + idx);
          pos++;
        }
      }
    }
    __syncthreads();
    const int nc = *cnt;
    for (int j0 = 0; j0 < nc; j0 += 32 * 8 / kNmsGroup) {
      const int j = j0 + gid;
      bool sup = false;
      int kk = 0, bit = 0;
      if (j < nc) {
        const int e = s_cand[j];
        kk = c0 + (e >> 5);
        bit = e & 31;
        const int row = row0 + kk / nw;
        const int cbase = (wlo + kk % nw) << 5;
        sup = nms_suppressed_rows(F, (long long)row * p0 + cbase + bit, s_cv[j], s_co[j], p0, npx, sub);
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, sup);
      if (j < nc && sub == 0 && !(bal & gmask)) atomicOr(&s_sur[kk], 1u << bit);
    }
  }
  __syncthreads();

  // exclusive scan of the survivor counts, in word order
  const int per = (nwords + 255) >> 8;
  const int beg = min((int)threadIdx.x * per, nwords), end = min(beg + per, nwords);
  int local = 0;
  for (int i = beg; i < end; i++) local += __popc(s_sur[i]);
  int incl = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += n;
  }
  if (lane == 31) s_warp_tot[warp] = incl;
  __syncthreads();
  int warp_off = 0;
  for (int w2 = 0; w2 < warp; w2++) warp_off += s_warp_tot[w2];
  int run = warp_off + incl - local;
  for (int i = beg; i < end; i++) {
    s_pref[i] = run;
    run += __popc(s_sur[i]);
  }
  int strip_total = 0;
  for (int w2 = 0; w2 < 8; w2++) strip_total += s_warp_tot[w2];

  // decoupled look-back over the frame's strips (warp 0)
  if (warp == 0) {
    unsigned long long* st = F.nms_status;
    int excl = 0;
    if (s == 0) {
      if (lane == 0) st_release_u64(&st[0], kFlagPre | (unsigned)strip_total);
    } else {
      if (lane == 0) st_release_u64(&st[s], kFlagAgg | (unsigned)strip_total);
      __syncwarp();
      excl = nms_lookback(st, s, lane, b.err);
      if (lane == 0) st_release_u64(&st[s], kFlagPre | (unsigned)(excl + strip_total));
    }
    if (lane == 0) {
      s_base = excl;
      if (s == F.nms_strips - 1) {
        const int tot = excl + strip_total;
        *F.count = min(tot, F.max_pts);
        if (F.total) *F.total = tot;
      }
    }
  }
  __syncthreads();
  const int base = s_base;
  if (base >= F.max_pts) return;

  // pass 2: write the survivors
  for (int k = threadIdx.x; k < nwords; k += blockDim.x) {
    uint32_t m = s_sur[k];
    if (!m) continue;
    const int row = row0 + k / nw;
    const int cbase = (wlo + k % nw) << 5;
    int rank = base + s_pref[k];
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1u;
      if (rank >= F.max_pts) break;
      const long long idx = (long long)row * p0 + cbase + bit;
      orbx_point q;
      q.x = cbase + bit;
      q.y = row;
      q.octave = F.oct8[idx];
      q.score = F.vmap[idx];
      q.angle = 0.f;
      q.match = 0;
      q.distance = 0;
      F.pts[rank] = q;
      rank++;
    }
  }
}

// Dense reference-layout maps (vmem: f32 scores then i32 octaves,
// orbd.cu:1576-1577) from the sparse ones, for orbd.h callers and debugging.
__global__ void k_expand_score_map(const Frame* __restrict__ fr, float* vmap_dense, int* layer_dense,
                                   long long npx) {
  const Frame& F = fr[0];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npx;
       i += (long long)gridDim.x * blockDim.x) {
    const bool on = (__ldg(F.occ + (i >> 5)) >> (i & 31)) & 1u;
    vmap_dense[i] = on ? F.vmap[i] : 0.f;
    layer_dense[i] = on ? (int)F.oct8[i] : 0;
  }
}

cudaError_t launch_expand_score_map(const Frame* d_frame, float* vmap_dense, int* layer_dense, long long npx,
                                    cudaStream_t s) {
  k_expand_score_map<<<4 * 148, 256, 0, s>>>(d_frame, vmap_dense, layer_dense, npx);
  return cudaGetLastError();
}

cudaError_t launch_pyramid_blur(const Batch& b, int total_tiles, cudaStream_t s) {
  if (total_tiles <= 0) return cudaSuccess;
  k_pyramid_blur<<<total_tiles, 256, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_detect(const Batch& b, int total_tiles, cudaStream_t s) {
  if (total_tiles <= 0) return cudaSuccess;
  k_detect<<<total_tiles, 256, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_nms(const Batch& b, int total_strips, cudaStream_t s) {
  if (total_strips <= 0) return cudaSuccess;
  k_nms<<<total_strips, 256, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace orbx
