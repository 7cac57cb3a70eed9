// Stage bodies of the sm_100a ORB pipeline as device functions: pyramid +
// blur tiles, FAST-9 + score tiles and NMS strips.  Each kernel of the
// five-launch form (orbx_detect.cu) runs one of them per block, and the
// persistent batch kernel (orbx_persist.cu) runs them per claimed work item.
#pragma once
#include "orbx_device.cuh"
#include "orbx_internal.cuh"
#include "orbx_fast.cuh"

namespace orbx {

// Loads of data a stage reads.  Standalone kernels read their inputs through
// the read-only path; in the persistent kernel a stage reads what an earlier
// stage wrote in the same launch, after an acquire, so it uses plain
// (coherent) cached loads instead.
template <bool P, class T>
__device__ __forceinline__ T ldx(const T* p) {
  if constexpr (P)
    return __ldca(p);
  else
    return __ldg(p);
}

// The frame table of a launch: from the launch parameters (INL, batches of up
// to kInlineFrames frames, constant-bank reads) or from global memory.
template <bool INL>
__device__ __forceinline__ const Frame& batch_frame(const Batch& b, int f) {
  if constexpr (INL)
    return b.inl[f];
  else
    return b.frames[f];
}
// Index of the frame whose range [base[f], base[f+1]) holds t (base in the
// launch parameters when INL).
template <bool INL>
__device__ __forceinline__ int find_frame_in(const int* base, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    int v;
    if constexpr (INL)
      v = base[mid];
    else
      v = __ldg(base + mid);
    if (v <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

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

// Exact small-integer <-> float conversions on the full-rate pipes: a float
// whose exponent field is 2^23 holds the integer in its mantissa.  byte_bits:
// the byte of `word` that selector `sel` (0x754j, j = 0..3) picks, in the low
// mantissa byte of 2^23, i.e. the float bits of 2^23 + byte.
__device__ __forceinline__ float byte_bits(uint32_t word, uint32_t sel) {
  return __uint_as_float(__byte_perm(word, 0x4B000000u, sel));
}
// Low bytes of four 32-bit words packed into one word (a | b << 8 | c << 16 | d << 24).
__device__ __forceinline__ uint32_t pack_low_bytes(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}
__device__ __forceinline__ float2 pair2(float v) { return make_float2(v, v); }
// gauss_dot4 on both lanes of a pair: the same operations in the same order,
// each lane rounded as the scalar form (one packed sm_100 FP32 instruction per step).
__device__ __forceinline__ float2 gauss_dot4x2(const float2* k, float2 t0, float2 t1, float2 t2, float2 t3) {
  float2 acc = __ffma2_rn(k[0], t0, __fmul2_rn(k[1], t1));
  acc = __ffma2_rn(k[2], t2, acc);
  return __ffma2_rn(k[3], t3, acc);
}
// One 4-byte group of staged source columns cx .. cx+3 of a row (reflect-101 at
// the octave edges).  words: the row is level 0 of a 4-byte aligned image, so
// interior groups take two aligned words (cx is one past a multiple of 4).
template <bool PL>
__device__ __forceinline__ uint32_t pyr_stage_word(const uint8_t* rowp, int cx, int ow, int sh, bool words,
                                                   BoundsRec* rec, Span src) {
  if (words && cx >= 1 && cx + 3 < ow) {
    // bytes cx-1 .. cx+6 lie in [0, pitch_in): cx + 3 < ow <= pitch_in and both words are aligned
    const uint32_t* wp = reinterpret_cast<const uint32_t*>(rowp + (cx - 1));
    if (!ORBX_IN(rec, kSitePyrLoad, src, wp, 8)) return 0u;
    return __byte_perm(ldx<PL>(wp), ldx<PL>(wp + 1), 0x4321);
  }
  uint32_t v[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const uint8_t* p = rowp + (reflect101(cx + j, ow) << sh);
    v[j] = ORBX_IN(rec, kSitePyrLoad, src, p, 1) ? ldx<PL>(p) : 0u;
  }
  return pack_low_bytes(v[0], v[1], v[2], v[3]);
}
// Row-major walk over items (r, g) with W items per row: item threadIdx.x +
// k * T for k = 0, 1, .. in a block of T threads, stepped without a division.
template <int W, int T>
struct RowWalk {
  int r, g;
  __device__ __forceinline__ RowWalk() : r(threadIdx.x / W), g(threadIdx.x % W) {}
  __device__ __forceinline__ void next() {
    r += T / W;
    g += T % W;
    if (g >= W) {
      g -= W;
      r++;
    }
  }
};

// Staged source of a TW x TH tile.  The filters run on column pairs: pair k of a
// row holds column k of the tile's left half and column k of its right half
// (each half with its 3-pixel halo on both sides), so one packed instruction
// filters two output columns.  Pairs are grouped two to a 16-byte slot, and a
// row's even slots are stored before its odd slots: a thread that works on
// slots 2g, 2g+1, .. reads slot 2g+m of its row at (m odd) * half + g + m/2,
// so the lanes of a warp read consecutive 16-byte words for every m.  The raw
// bytes are staged linearly.
template <int TW, int TH>
struct PyrSmem {
  static constexpr int HW = TW / 2;   // columns per half
  static constexpr int SW = TW + 8;   // staged bytes per row
  static constexpr int SW2 = HW + 8;  // staged column pairs per row (3 + HW + 3, padded to 4)
  static constexpr int SH = TH + 6;
  __align__(16) float2 src[SH * SW2];
  __align__(16) uint8_t byte[SH * SW];
  __align__(16) float2 row[SH * HW];
};

// Position of pyramid tile t (tile index over the batch) of shape TW x TH.
struct PyrTile {
  int f;       // frame
  int o;       // octave
  int lt;      // tile index within the octave
  int x0, y0;  // octave-pixel origin
};
template <bool INL, int TW, int TH>
__device__ __forceinline__ PyrTile pyr_tile_at(const Batch& b, int t) {
  const int* base = INL ? b.inl_pyr_base : b.pyr_base;
  PyrTile g;
  g.f = find_frame_in<INL>(base, b.n_frames, t);
  const Frame& F = batch_frame<INL>(b, g.f);
  int lt = t - (INL ? base[g.f] : __ldg(base + g.f));
  int o = 0;
  while (o + 1 < F.n_oct && lt >= F.pyr_tile_base[o + 1]) o++;
  lt -= F.pyr_tile_base[o];
  const int tiles_x = F.pyr_tiles_x[o];
  g.o = o;
  g.lt = lt;
  g.x0 = (lt % tiles_x) * TW;
  g.y0 = (lt / tiles_x) * TH;
  return g;
}

template <int TW, int TH>
__host__ __device__ constexpr int pyr_stage_items() {
  return (PyrSmem<TW, TH>::SH * (PyrSmem<TW, TH>::SW2 / 4) + kPyrThreads - 1) / kPyrThreads;
}

// Staging loads of tile g: source rows y0-3 .. y0+TH+2; item (r, g) takes
// columns 4g-3 .. 4g of the left half and of the right half (tile-relative),
// reflect-101 at the octave edges.  All of a thread's loads are issued before
// any is used (blocks have kPyrThreads threads).
template <bool PL, int TW, int TH, bool INL>
__device__ __forceinline__ void pyr_tile_load(const Batch& b, const PyrTile& g, uint32_t* wa, uint32_t* wb) {
  using S = PyrSmem<TW, TH>;
  constexpr int kHW = S::HW, kSH = S::SH, kGroups = S::SW2 / 4;
  const Frame& F = batch_frame<INL>(b, g.f);
  const int o = g.o, ow = F.ow[o], oh = F.oh[o], op = F.op[o];
  const uint8_t* __restrict__ img = F.img;
  const int pitch_in = F.pitch_in;
  const uint8_t* __restrict__ psrc = F.pyr_src ? F.pyr_src + F.ooff[o] : nullptr;
  const bool words0 = (o == 0) && !psrc && ((reinterpret_cast<uintptr_t>(img) | (uintptr_t)pitch_in) & 3u) == 0;
  const int sh = psrc ? 0 : o;
  const Span src = psrc ? Span{F.pyr_src, F.ooff[F.n_oct]} : img_span(F);
  RowWalk<kGroups, kPyrThreads> w;
#pragma unroll
  for (int q = 0; q < pyr_stage_items<TW, TH>(); q++) {
    wa[q] = wb[q] = 0u;
    if (w.r < kSH) {
      const int y = reflect101(g.y0 - 3 + w.r, oh);
      const uint8_t* rowp = psrc ? psrc + (size_t)y * op : img + (size_t)(y << o) * pitch_in;
      const int cx = g.x0 - 3 + 4 * w.g;
      wa[q] = pyr_stage_word<PL>(rowp, cx, ow, sh, words0, b.bounds, src);
      wb[q] = pyr_stage_word<PL>(rowp, cx + kHW, ow, sh, words0, b.bounds, src);
    }
    w.next();
  }
}

// The staged words of tile g into shared memory, as float pairs and as bytes,
// plus the per-frame housekeeping of the frame's first tile.  No barrier.
template <int TW, int TH, bool INL>
__device__ __forceinline__ void pyr_tile_stage(const Batch& b, int t, const PyrTile& g, const uint32_t* wa,
                                               const uint32_t* wb, PyrSmem<TW, TH>& sm) {
  using S = PyrSmem<TW, TH>;
  constexpr int kHW = S::HW, kSW = S::SW, kSH = S::SH;
  constexpr int kRowSlots = S::SW2 / 2;  // 16-byte slots per staged pair row (two planes)
  constexpr int kGroups = S::SW2 / 4;    // staging items per row = slots per plane of a staged row
  static_assert(TW % 16 == 0 && S::SW2 % 4 == 0, "pyramid tile width");
  float4* s_src = reinterpret_cast<float4*>(sm.src);
  uint8_t* s_byte = sm.byte;
  const Frame& F = batch_frame<INL>(b, g.f);
  if (g.o == 0 && g.lt == 0) {
    for (int i = threadIdx.x; i < F.nms_strips; i += blockDim.x)
      if (ORBX_IN_ROWS(b.bounds, kSiteFrameState, i, F.nms_strips)) F.nms_status[i] = 0ull;
    if (threadIdx.x == 0) {
      *F.count = 0;
      if (F.total) *F.total = 0;
    }
  }
  if (t == 0 && threadIdx.x == 0) *b.nms_ticket = 0u;
  const float2 m23 = pair2(-8388608.0f);
  RowWalk<kGroups, kPyrThreads> w;
#pragma unroll
  for (int q = 0; q < pyr_stage_items<TW, TH>(); q++, w.next()) {
    const int r = w.r, gg = w.g;
    if (r >= kSH) break;
    // pair j = (byte j of wa, byte j of wb) as floats: 2^23 + byte, minus 2^23
    const float2 p0 = __fadd2_rn(make_float2(byte_bits(wa[q], 0x7540u), byte_bits(wb[q], 0x7540u)), m23);
    const float2 p1 = __fadd2_rn(make_float2(byte_bits(wa[q], 0x7541u), byte_bits(wb[q], 0x7541u)), m23);
    const float2 p2 = __fadd2_rn(make_float2(byte_bits(wa[q], 0x7542u), byte_bits(wb[q], 0x7542u)), m23);
    const float2 p3 = __fadd2_rn(make_float2(byte_bits(wa[q], 0x7543u), byte_bits(wb[q], 0x7543u)), m23);
    // pairs 4g .. 4g+3 = slots 2g (even plane) and 2g+1 (odd plane) of row r
    float4* row = s_src + r * kRowSlots + gg;
    row[0] = make_float4(p0.x, p0.y, p1.x, p1.y);
    row[kGroups] = make_float4(p2.x, p2.y, p3.x, p3.y);
    // the halves' halos overlap in the middle: both writes there store the same bytes
    *reinterpret_cast<uint32_t*>(s_byte + r * kSW + 4 * gg) = wa[q];
    *reinterpret_cast<uint32_t*>(s_byte + r * kSW + kHW + 4 * gg) = wb[q];
  }
}

// Blur of the staged tile g and the stores of its raw and blurred bytes:
// a barrier, the horizontal pass, a barrier, the vertical pass.  PL: the
// level-0 image was written earlier in the same launch.
template <bool PL, int TW, int TH, bool INL>
__device__ __forceinline__ void pyr_tile_filter(const Batch& b, const PyrTile& g, PyrSmem<TW, TH>& sm) {
  using S = PyrSmem<TW, TH>;
  constexpr int kHW = S::HW, kSW = S::SW, kSH = S::SH;
  constexpr int kRowSlots = S::SW2 / 2;
  constexpr int kOutSlots = kHW / 2;     // 16-byte slots per filtered pair row (two planes)
  constexpr int kGroups = S::SW2 / 4;
  float4* s_src = reinterpret_cast<float4*>(sm.src);
  float4* s_row = reinterpret_cast<float4*>(sm.row);
  uint8_t* s_byte = sm.byte;
  const Frame& F = batch_frame<INL>(b, g.f);
  const int o = g.o, x0 = g.x0, y0 = g.y0;
  const int ow = F.ow[o], oh = F.oh[o], op = F.op[o];
  const uint8_t* __restrict__ img = F.img;
  const int pitch_in = F.pitch_in;
  const uint8_t* __restrict__ psrc = F.pyr_src ? F.pyr_src + F.ooff[o] : nullptr;
  __syncthreads();

  float2 k[4];
#pragma unroll
  for (int i = 0; i < 4; i++) k[i] = pair2(b.gauss[i]);
  // horizontal pass: 4 consecutive output pairs per thread; integer tap sums
  // are exact in float, so they are summed as floats
  constexpr int kHG = kHW / 4;  // items per row = slots per plane of a filtered row
  for (RowWalk<kHG, kPyrThreads> w; w.r < kSH; w.next()) {
    const int r = w.r, g = w.g;
    const float4* row = s_src + r * kRowSlots + g;
    // slots 2g .. 2g+4: even plane g, g+1, g+2 and odd plane g, g+1
    const float4 e0 = row[0], o0 = row[kGroups], e1 = row[1], o1 = row[kGroups + 1], e2 = row[2];
    const float2 p[10] = {make_float2(e0.x, e0.y), make_float2(e0.z, e0.w), make_float2(o0.x, o0.y),
                          make_float2(o0.z, o0.w), make_float2(e1.x, e1.y), make_float2(e1.z, e1.w),
                          make_float2(o1.x, o1.y), make_float2(o1.z, o1.w), make_float2(e2.x, e2.y),
                          make_float2(e2.z, e2.w)};
    float2 q[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
      q[j] = gauss_dot4x2(k, p[j + 3], __fadd2_rn(p[j + 2], p[j + 4]), __fadd2_rn(p[j + 1], p[j + 5]),
                          __fadd2_rn(p[j], p[j + 6]));
    float4* out = s_row + r * kOutSlots + g;
    out[0] = make_float4(q[0].x, q[0].y, q[1].x, q[1].y);
    out[kHG] = make_float4(q[2].x, q[2].y, q[3].x, q[3].y);
  }
  __syncthreads();

  // vertical pass and stores: 4 consecutive column pairs of one row per thread
  uint8_t* P = F.pyr + F.ooff[o];
  uint8_t* B = F.blr + F.ooff[o];
  const bool copy_pad = (o == 0) && (pitch_in == op);
  const float2 rne = pair2(12582912.0f);
  for (RowWalk<kHG, kPyrThreads> w; w.r < TH; w.next()) {
    const int r = w.r, g = w.g;
    const int y = y0 + r;
    if (y >= oh) continue;
    float2 h[7][4];
    const float4* col = s_row + r * kOutSlots + g;
#pragma unroll
    for (int i = 0; i < 7; i++) {
      const float4 v0 = col[i * kOutSlots], v1 = col[i * kOutSlots + kHG];
      h[i][0] = make_float2(v0.x, v0.y);
      h[i][1] = make_float2(v0.z, v0.w);
      h[i][2] = make_float2(v1.x, v1.y);
      h[i][3] = make_float2(v1.z, v1.w);
    }
    // rounded to the nearest integer, ties to even, by adding 1.5 * 2^23: the
    // result's low byte is the blurred pixel (0 <= v <= 255)
    uint32_t ua[4], ub[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float2 v = __fadd2_rn(gauss_dot4x2(k, h[3][j], __fadd2_rn(h[2][j], h[4][j]),
                                               __fadd2_rn(h[1][j], h[5][j]), __fadd2_rn(h[0][j], h[6][j])),
                                  rne);
      ua[j] = __float_as_uint(v.x);
      ub[j] = __float_as_uint(v.y);
    }
    const uint8_t* sb = s_byte + (r + 3) * kSW + 4 * g;
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int x = x0 + half * kHW + 4 * g;
      if (x >= op) continue;
      const uint32_t bw = half ? pack_low_bytes(ub[0], ub[1], ub[2], ub[3]) : pack_low_bytes(ua[0], ua[1], ua[2], ua[3]);
      // raw bytes of the same 4 pixels: staged columns 4g+3 .. 4g+6 of the half
      const uint32_t* sw = reinterpret_cast<const uint32_t*>(sb + half * kHW);
      const uint32_t pw = __byte_perm(sw[0], sw[1], 0x6543);
      const size_t a = (size_t)y * op + x;
      if (x + 4 <= ow) {
        if (ORBX_IN(b.bounds, kSitePyrStore, octave_span(F.blr, F, o), B + a, 4))
          *reinterpret_cast<uint32_t*>(B + a) = bw;
        if (ORBX_IN(b.bounds, kSitePyrStore, octave_span(F.pyr, F, o), P + a, 4))
          *reinterpret_cast<uint32_t*>(P + a) = pw;
      } else {
        // the group reaches into the row padding: octave 0 carries the caller's
        // padding bytes (the reference copies h * pitch0 bytes, orbd.cu:1584),
        // other octaves hold zeros
#pragma unroll
        for (int j = 0; j < 4; j++) {
          if (x + j < ow) {
            if (ORBX_IN(b.bounds, kSitePyrStore, octave_span(F.blr, F, o), B + a + j, 1))
              B[a + j] = (uint8_t)(bw >> (8 * j));
            if (ORBX_IN(b.bounds, kSitePyrStore, octave_span(F.pyr, F, o), P + a + j, 1))
              P[a + j] = (uint8_t)(pw >> (8 * j));
          } else {
            const uint8_t v =
                psrc ? (ORBX_IN(b.bounds, kSitePyrPadLoad, (Span{F.pyr_src, F.ooff[F.n_oct]}), psrc + a + j, 1)
                            ? ldx<PL>(psrc + a + j)
                            : (uint8_t)0)
                     : (copy_pad ? (ORBX_IN(b.bounds, kSitePyrPadLoad, img_span(F), img + (size_t)y * pitch_in + x + j, 1)
                                        ? ldx<PL>(img + (size_t)y * pitch_in + x + j)
                                        : (uint8_t)0)
                                 : (uint8_t)0);
            if (ORBX_IN(b.bounds, kSitePyrStore, octave_span(F.blr, F, o), B + a + j, 1)) B[a + j] = v;
            if (ORBX_IN(b.bounds, kSitePyrStore, octave_span(F.pyr, F, o), P + a + j, 1)) P[a + j] = v;
          }
        }
      }
    }
  }
}


// One pyramid tile (tile index t over the batch) of shape TW x TH: it stages
// the tile plus a 3-pixel reflected halo in shared memory, writes the raw
// tile, and blurs it.  PL: the level-0 image is copied in during the same
// launch (coherent loads instead of the read-only path).
template <bool PL, int TW = kPyrTW, int TH = kPyrTH, bool INL = false>
__device__ __forceinline__ void pyr_tile(const Batch& b, int t, PyrSmem<TW, TH>& sm) {
  uint32_t wa[pyr_stage_items<TW, TH>()], wb[pyr_stage_items<TW, TH>()];
  const PyrTile g = pyr_tile_at<INL, TW, TH>(b, t);
  pyr_tile_load<PL, TW, TH, INL>(b, g, wa, wb);
  pyr_tile_stage<TW, TH, INL>(b, t, g, wa, wb, sm);
  pyr_tile_filter<PL, TW, TH, INL>(b, g, sm);
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
  for (int k = 0; k < 25; k++) d[k] = (int)(short)(v - c[ring_dy(k) * sw + ring_dx(k)]);
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

struct DetSmem {
  __align__(16) uint8_t stage[det_stage_bytes()];
  __align__(16) unsigned long long key[kDetTH * kDetTW];
  uint16_t cand[kDetMaxCand];
  uint16_t corner[kDetMaxCand];
  int n[2];
  uint32_t occ[kDetTH * kDetTW / 32];
  int ow[kMaxOctaves], oh[kMaxOctaves];
};

// Stages octave O of a detect tile with its halo: (32 >> O) + 8 rows of
// (64 >> O) + 8 bytes starting 4 rows above and 4 bytes left of the tile's
// octave origin, in the pyramid's linear addressing.
template <int O, bool P>
__device__ __forceinline__ void stage_octave(const Frame& F, const uint8_t* pyr, int X0, int Y0, uint8_t* s_stage,
                                             BoundsRec* rec) {
  constexpr int sw4 = ((kDetTW >> O) + 2 * kHalo) / 4;
  constexpr int sh = (kDetTH >> O) + 2 * kHalo;
  const int op = F.op[O];
  const uint32_t* src =
      reinterpret_cast<const uint32_t*>(pyr + F.ooff[O] + (long long)((Y0 >> O) - kHalo) * op + ((X0 >> O) - kHalo));
  const int op4 = op >> 2;
  uint32_t* dst = reinterpret_cast<uint32_t*>(s_stage + det_stage_off(O));
#pragma unroll 4
  for (int i = threadIdx.x; i < sh * sw4; i += 256) {
    const int r = i / sw4, w = i - r * sw4;
    const uint32_t* sp = src + r * op4 + w;
    dst[i] = ORBX_IN(rec, kSiteDetLoad, guarded_span(pyr, F), sp, 4) ? ldx<P>(sp) : 0u;
  }
}

// Pre-test of word w (four centres) of octave O of a detect tile: octave O
// has (32 >> O) rows of (16 >> O) words.  Centres that pass are appended to
// the tile's candidate list.
template <int O>
__device__ __forceinline__ void pretest_word(int w, int X0, int Y0, const uint8_t* s_stage, int ow, int oh,
                                             uint32_t t4, int* s_n, uint16_t* s_cand) {
  static_assert(kDetTW == 64 && kDetTH == 32, "word layout assumes 64 x 32 detect tiles");
  constexpr int nwl = 4 - O;  // log2 words per row
  constexpr int sw = (kDetTW >> O) + 2 * kHalo;
  constexpr int off = det_stage_off(O);
  const int ly = w >> nwl, lx = (w & ((1 << nwl) - 1)) << 2;
  const int x = (X0 >> O) + lx, y = (Y0 >> O) + ly;
  uint32_t m = 0u;
  if (y >= 3 && y < oh - 3 && x < ow - 3) {
    m = fast9_pretest4(s_stage + off + (ly + kHalo) * sw + (lx + kHalo), sw, t4);
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
      s_cand[pos++] = det_item(O, ly, lx + k);
    }
  }
}

// One detect tile (tile index t over the batch).  P: the raw pyramid was
// written earlier in the same launch (coherent loads instead of the read-only path).
template <bool P, bool INL = false>
__device__ __forceinline__ void det_tile(const Batch& b, int t, DetSmem& sm) {
  uint8_t* s_stage = sm.stage;
  unsigned long long* s_key = sm.key;
  uint16_t* s_cand = sm.cand;
  uint16_t* s_corner = sm.corner;
  int* s_n = sm.n;
  uint32_t* s_occ = sm.occ;
  int* s_ow = sm.ow;
  int* s_oh = sm.oh;
  const int* base = INL ? b.inl_det_base : b.det_base;
  const int f = find_frame_in<INL>(base, b.n_frames, t);
  const Frame& F = batch_frame<INL>(b, f);
  const int lt = t - (INL ? base[f] : __ldg(base + f));
  const int X0 = (lt % F.det_tiles_x) * kDetTW;
  const int Y0 = (lt / F.det_tiles_x) * kDetTH;
  const int n_oct = F.n_oct;
  const uint8_t* __restrict__ pyr = F.pyr;
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
  // Stage every octave's tile with its halo, 4 bytes per load (octave offsets
  // and pitches are multiples of 128 and (X0 >> o) - 4 is a multiple of 4):
  // the words of each octave are spread over the whole block.
  stage_octave<0, P>(F, pyr, X0, Y0, s_stage, b.bounds);
  if (n_oct > 1) stage_octave<1, P>(F, pyr, X0, Y0, s_stage, b.bounds);
  if (n_oct > 2) stage_octave<2, P>(F, pyr, X0, Y0, s_stage, b.bounds);
  if (n_oct > 3) stage_octave<3, P>(F, pyr, X0, Y0, s_stage, b.bounds);
  if (n_oct > 4) stage_octave<4, P>(F, pyr, X0, Y0, s_stage, b.bounds);
  __syncthreads();

  // 1. cardinal pre-test, four centres per word: the 512 words of octave 0 take
  //    two passes of the block, the 128 + 32 + 8 + 2 words of octaves 1..4 one
  {
    const uint32_t t4 = (uint32_t)min(max(thr, 0), 255) * 0x01010101u;
    const int t = threadIdx.x;
    pretest_word<0>(t, X0, Y0, s_stage, s_ow[0], s_oh[0], t4, s_n, s_cand);
    pretest_word<0>(t + 256, X0, Y0, s_stage, s_ow[0], s_oh[0], t4, s_n, s_cand);
    if (t < 128) {
      if (n_oct > 1) pretest_word<1>(t, X0, Y0, s_stage, s_ow[1], s_oh[1], t4, s_n, s_cand);
    } else if (t < 160) {
      if (n_oct > 2) pretest_word<2>(t - 128, X0, Y0, s_stage, s_ow[2], s_oh[2], t4, s_n, s_cand);
    } else if (t < 168) {
      if (n_oct > 3) pretest_word<3>(t - 160, X0, Y0, s_stage, s_ow[3], s_oh[3], t4, s_n, s_cand);
    } else if (t < 170) {
      if (n_oct > 4) pretest_word<4>(t - 168, X0, Y0, s_stage, s_ow[4], s_oh[4], t4, s_n, s_cand);
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
      // 32 groups of 8 lanes, one corner per group; lanes 0..6 of a group take
      // one row each of the 7x7 Harris window (the 32-bit sums wrap, so their
      // order is free)
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
          if (sub < 7) {  // lane `sub` of the group takes window row sub - 3, its 7 columns unrolled
            const uint8_t* r = c + (sub - 3) * sw;
            const uint8_t* ru = r - sw;
            const uint8_t* rd = r + sw;
#pragma unroll
            for (int wx = -3; wx <= 3; wx++) {
              const int dx = ((int)r[wx + 1] - (int)r[wx - 1]) * 2 + ((int)ru[wx + 1] - (int)ru[wx - 1]) +
                             ((int)rd[wx + 1] - (int)rd[wx - 1]);
              const int dy = ((int)rd[wx] - (int)ru[wx]) * 2 + ((int)rd[wx - 1] - (int)ru[wx - 1]) +
                             ((int)rd[wx + 1] - (int)ru[wx + 1]);
              dxx += dx * dx;
              dyy += dy * dy;
              dxy += dx * dy;
            }
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
      if (ORBX_IN_ROWS(b.bounds, kSiteDetStore, (long long)(a0 >> 5), map_px(F) >> 5)) F.occ[a0 >> 5] = m;
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1u;
        const unsigned long long key = s_key[r * kDetTW + 32 * half + k];
        if (!ORBX_IN_ROWS(b.bounds, kSiteDetStore, (long long)(a0 + k), map_px(F))) continue;
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
constexpr int kLookPerLane = 8;  // look-back words read per lane and round: 256 predecessors

// Warp 0 of a strip's block resolves the strip's exclusive prefix.  In each
// round lane l reads the look-back words of predecessors j - l - 32u, u = 0..7
// (each of the eight loads is 32 consecutive words, so a round touches 64
// sectors), and the warp stops at the nearest predecessor that already carries
// an inclusive prefix.  A look-back word holds its flag and its count together
// and nothing else is read on its strength, so plain relaxed loads and stores
// suffice (a release store would wait for a fence).  A published word only ever
// changes from an aggregate to an inclusive prefix of the same strip, and
// summing aggregates back to any prefix gives the same total, so words already
// seen published are kept and only the pending ones are read again, after a
// back-off that doubles from 32 ns to 256 ns: the words of a frame share a few
// L2 sectors, and a store to them completes only after the reads queued there.
// The wait is bounded by wait_cycles of clock64(); on expiry it sets
// kErrLookbackTimeout and returns the prefix found so far.
__device__ __forceinline__ int nms_lookback(unsigned long long* st, int s, int lane, int* err,
                                            long long wait_cycles) {
  int excl = 0;
  int j = s - 1;
  const long long t0 = clock64();
  while (j >= 0) {
    unsigned long long wv[kLookPerLane];
#pragma unroll
    for (int u = 0; u < kLookPerLane; u++) {
      const int idx = j - lane - 32 * u;
      wv[u] = (idx >= 0) ? ld_relaxed_u64(&st[idx]) : kFlagPre;
    }
    unsigned sleep_ns = 32;
    bool timed_out = false;
    for (;;) {
      // the nearest inclusive prefix: smallest distance lane + 32u
      int first_u = kLookPerLane, first_lane = 32;
#pragma unroll
      for (int u = kLookPerLane - 1; u >= 0; u--) {
        const unsigned pre = __ballot_sync(0xffffffffu, (wv[u] & (3ull << 32)) == kFlagPre);
        if (pre) {
          first_u = u;
          first_lane = __ffs(pre) - 1;
        }
      }
      // words up to and including that prefix must all be published
      bool notready = false;
#pragma unroll
      for (int u = 0; u < kLookPerLane; u++) {
        const bool need = u < first_u || (u == first_u && lane <= first_lane);
        if (need && (wv[u] & (3ull << 32)) == 0ull) notready = true;
      }
      if (!__any_sync(0xffffffffu, notready)) {
        int v = 0;
#pragma unroll
        for (int u = 0; u < kLookPerLane; u++) {
          const bool need = u < first_u || (u == first_u && lane <= first_lane);
          if (need) v += (int)(unsigned)wv[u];
        }
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        excl += v;
        j = (first_u < kLookPerLane) ? -1 : j - 32 * kLookPerLane;
        break;
      }
      if (__any_sync(0xffffffffu, clock64() - t0 > wait_cycles)) {  // warp-uniform decision
        timed_out = true;
        break;
      }
      __nanosleep(sleep_ns);
      if (sleep_ns < 256) sleep_ns <<= 1;
#pragma unroll
      for (int u = 0; u < kLookPerLane; u++) {
        const int idx = j - lane - 32 * u;
        if (idx >= 0 && (wv[u] & (3ull << 32)) == 0ull) wv[u] = ld_relaxed_u64(&st[idx]);
      }
    }
    if (timed_out) {
      if (lane == 0) atomicOr(err, kErrLookbackTimeout);
      break;
    }
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
// edge threshold below 2^o, are empty.  Occ(wi) gives occupancy word wi and
// Score(wi, word, bit) the score of a set bit.
constexpr int kNmsGroup = 8;
constexpr int kNmsChunkWords = 128;  // occupancy words compacted per round: at most 4096 centres

template <class Occ, class Score>
__device__ __forceinline__ bool nms_window_suppressed(long long idx, float v, int o, int p0, long long npx, int sub,
                                                      Occ occ, Score score) {
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
      const uint32_t word = occ(wi);
      uint32_t m = word;
      if (base < lo) m &= ~0u << (int)(lo - base);
      if (hi - base < 31) m &= (2u << (int)(hi - base)) - 1u;
      while (m) {
        const int bb = __ffs(m) - 1;
        m &= m - 1u;
        const long long li = base + bb;
        if (li == idx) continue;
        const int dx = (int)(li - rc);
        const float u = score(wi, word, bb);
        if (u > v || (u == v && dx <= 0 && dy <= 0)) return true;
      }
    }
  }
  return false;
}

// Staged form of a strip (kNmsStageWords occupancy words: the strip's rows with
// a halo of R + 1 rows on each side; kNmsStageBits set bits with their scores
// and octaves gathered next to them).
constexpr int kNmsStageWords = 2048;
constexpr int kNmsStageBits = 2048;

struct NmsSmem {
  uint32_t sur[kNmsMaxWords];
  int pref[kNmsMaxWords];
  union {
    struct {  // rounds over the maps in global memory
      uint16_t cand[kNmsChunkWords * 32];
      float cv[kNmsChunkWords * 32];
      uint8_t co[kNmsChunkWords * 32];
    } g;
    struct {  // staged strip
      uint32_t occ[kNmsStageWords];
      float score[kNmsStageBits];
      uint16_t pfx[kNmsStageWords + 1];  // set bits before each staged word
      uint16_t idx[kNmsStageBits];       // bit offset of each set bit from the first staged word
      uint8_t oct[kNmsStageBits];
    } w;
  } u;
  int ncand[2];
  int warp_tot[8];
  int base;
};

// Exclusive scan over the block (256 threads) of one count per thread; *total
// gets the sum.  Every thread must call it.
__device__ __forceinline__ int block_scan_excl(int local, int* s_warp_tot, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += n;
  }
  if (lane == 31) s_warp_tot[warp] = incl;
  __syncthreads();
  int warp_off = 0, tot = 0;
#pragma unroll
  for (int w2 = 0; w2 < 8; w2++) {
    const int t = s_warp_tot[w2];
    if (w2 < warp) warp_off += t;
    tot += t;
  }
  __syncthreads();
  total = tot;
  return warp_off + incl - local;
}

// One NMS strip; `ticket` is the strip's index over the batch, and strips must
// start in ticket order (the look-back waits only on smaller tickets).  P: the
// score map was written earlier in the same launch.
template <bool P, bool INL = false>
__device__ __forceinline__ void nms_strip(const Batch& b, int ticket, NmsSmem& sm) {
  uint32_t* s_sur = sm.sur;
  int* s_pref = sm.pref;
  int* s_ncand = sm.ncand;
  int* s_warp_tot = sm.warp_tot;
  int& s_base = sm.base;
  const int* strip_base = INL ? b.inl_nms_base : b.nms_base;
  const int f = find_frame_in<INL>(strip_base, b.n_frames, ticket);
  const Frame& F = batch_frame<INL>(b, f);
  const int s = ticket - (INL ? strip_base[f] : __ldg(strip_base + f));
  const int border = F.border;
  const int row0 = border + s * F.nms_rows;
  const int row1 = min(row0 + F.nms_rows, F.h - border);
  const int xlo = border, xhi = F.w - border;  // columns [xlo, xhi)
  const int wlo = xlo >> 5, whi = (xhi - 1) >> 5;
  const int nw = whi - wlo + 1;
  const int nwords = (row1 - row0) * nw;
  const int p0 = F.op[0];  // a multiple of 128
  const int wpr = p0 >> 5;  // occupancy words per row
  const long long npx = (long long)F.h * p0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = warp * (32 / kNmsGroup) + (lane / kNmsGroup), sub = lane % kNmsGroup;
  const uint32_t gmask = ((1u << kNmsGroup) - 1u) << (lane & ~(kNmsGroup - 1));
  const uint32_t* occ_map = F.occ;
  const float* score_map = F.vmap;
  [[maybe_unused]] BoundsRec* rec = b.bounds;
  auto g_occ = [=](long long wi) {
    return ORBX_IN_ROWS(rec, kSiteNmsOcc, wi, npx >> 5) ? ldx<P>(occ_map + wi) : 0u;
  };
  auto g_score = [=](long long wi, uint32_t, int bb) {
    return ORBX_IN_ROWS(rec, kSiteNmsScore, (wi << 5) + bb, npx) ? ldx<P>(score_map + ((wi << 5) + bb)) : 0.f;
  };

  for (int k = threadIdx.x; k < nwords; k += blockDim.x) s_sur[k] = 0u;

  // Staged pass 1.  The halo R is the largest window radius present (2^(n_oct-1)),
  // halved until the strip fits the staging buffer; centres of octaves with a
  // larger radius read their windows from global memory.
  int R = 1 << (F.n_oct - 1);
  while (R >= 1 && (min(F.h, row1 + R + 1) - max(0, row0 - R - 1)) * wpr > kNmsStageWords) R >>= 1;
  const int srow0 = max(0, row0 - R - 1), srow1 = min(F.h, row1 + R + 1);
  const int ns = (srow1 - srow0) * wpr;
  const long long W0 = (long long)srow0 * wpr;  // first staged word
  bool staged = R >= 1;
  uint32_t* s_occ = sm.u.w.occ;
  uint16_t* s_pfx = sm.u.w.pfx;
  uint16_t* s_idx = sm.u.w.idx;
  float* s_score = sm.u.w.score;
  uint8_t* s_oct = sm.u.w.oct;
  // a staged word, or the global one for a word outside the stage (not reached
  // for radii up to R; kept so that no index leaves the buffers)
  auto w_occ = [=](long long wi) {
    const long long sw = wi - W0;
    return (sw >= 0 && sw < ns) ? s_occ[sw] : g_occ(wi);
  };
  auto w_score = [=](long long wi, uint32_t word, int bb) {
    const long long sw = wi - W0;
    return (sw >= 0 && sw < ns) ? s_score[s_pfx[sw] + __popc(word & ((1u << bb) - 1u))]
                                : g_score(wi, word, bb);
  };
  if (staged) {
    for (int i = threadIdx.x; i < ns; i += blockDim.x) s_occ[i] = g_occ(W0 + i);
    __syncthreads();
    // set bits before each word (contiguous runs of words per thread), and the
    // list of set bits in raster order
    const int per = (ns + 255) >> 8;
    const int beg = min((int)threadIdx.x * per, ns), end = min(beg + per, ns);
    int local = 0;
    for (int i = beg; i < end; i++) local += __popc(s_occ[i]);
    int total;
    int run = block_scan_excl(local, s_warp_tot, total);
    if (total <= kNmsStageBits) {
      for (int i = beg; i < end; i++) {
        s_pfx[i] = (uint16_t)run;
        uint32_t m = s_occ[i];
        while (m) {
          const int bb = __ffs(m) - 1;
          m &= m - 1u;
          s_idx[run++] = (uint16_t)((i << 5) | bb);
        }
      }
      if (threadIdx.x == 0) s_pfx[ns] = (uint16_t)total;
      __syncthreads();
      // scores and octaves of the set bits, four loads in flight per thread
      for (int r0 = threadIdx.x; r0 < total; r0 += 4 * blockDim.x) {
        long long li[4];
        bool ok[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int r = r0 + q * blockDim.x;
          ok[q] = r < total;
          li[q] = (W0 << 5) + (ok[q] ? s_idx[r] : 0);
        }
        float v[4];
        uint8_t o[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const bool in = ok[q] && ORBX_IN_ROWS(rec, kSiteNmsScore, li[q], npx);
          v[q] = in ? ldx<P>(F.vmap + li[q]) : 0.f;
          o[q] = in ? ldx<P>(F.oct8 + li[q]) : (uint8_t)0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (ok[q]) {
            s_score[r0 + q * blockDim.x] = v[q];
            s_oct[r0 + q * blockDim.x] = o[q];
          }
        }
      }
      __syncthreads();
      // the centres are the set bits of the strip's own rows (ranks c_lo ..
      // c_hi - 1) in columns [xlo, xhi), checked by 32 groups of 8 lanes
      const int c_lo = s_pfx[(row0 - srow0) * wpr], c_hi = s_pfx[(row1 - srow0) * wpr];
      for (int j0 = c_lo; j0 < c_hi; j0 += 32 * 8 / kNmsGroup) {
        const int j = j0 + gid;
        bool sup = false;
        int kk = -1, bit = 0;
        if (j < c_hi) {
          const int rel = s_idx[j];
          const int rr = rel / p0, c = rel - rr * p0;
          if (c >= xlo && c < xhi) {
            const int row = srow0 + rr;
            const long long idx = (long long)row * p0 + c;
            const int o = s_oct[j];
            sup = (1 << o) <= R ? nms_window_suppressed(idx, s_score[j], o, p0, npx, sub, w_occ, w_score)
                                : nms_window_suppressed(idx, s_score[j], o, p0, npx, sub, g_occ, g_score);
            kk = (row - row0) * nw + ((c >> 5) - wlo);
            bit = c & 31;
          }
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, sup);
        if (kk >= 0 && sub == 0 && !(bal & gmask)) atomicOr(&s_sur[kk], 1u << bit);
      }
    } else {
      staged = false;
    }
  }

  if (!staged) {
    // pass 1 over global memory, in rounds of kNmsChunkWords words: the centres
    // of the round (with their scores) are compacted into shared memory, then
    // checked by 32 groups of 8 lanes, so a textured patch of the strip spreads
    // over every warp
    uint16_t* s_cand = sm.u.g.cand;
    float* s_cv = sm.u.g.cv;
    uint8_t* s_co = sm.u.g.co;
    if (threadIdx.x == 0) s_ncand[0] = 0;
    for (int c0 = 0, round = 0; c0 < nwords; c0 += kNmsChunkWords, round++) {
      int* cnt = &s_ncand[round & 1];
      __syncthreads();  // the previous round's checks are done; its counter is free
      if (threadIdx.x == 0) s_ncand[(round + 1) & 1] = 0;
      const int k = c0 + (int)threadIdx.x;
      if (threadIdx.x < kNmsChunkWords && k < nwords) {
        const int row = row0 + k / nw;
        const int wj = wlo + k % nw;
        const int cbase = wj << 5;
        uint32_t m = g_occ((long long)row * wpr + wj);
        if (cbase < xlo) m &= ~0u << (xlo - cbase);
        if (xhi - cbase < 32) m &= (xhi - cbase <= 0) ? 0u : ((xhi - cbase == 32) ? ~0u : ((1u << (xhi - cbase)) - 1u));
        if (m) {
          int pos = atomicAdd(cnt, __popc(m));
          while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1u;
            const long long idx = (long long)row * p0 + cbase + bit;
            s_cand[pos] = (uint16_t)(((k - c0) << 5) | bit);
            const bool in = ORBX_IN_ROWS(rec, kSiteNmsScore, idx, npx);
            s_cv[pos] = in ? ldx<P>(F.vmap + idx) : 0.f;
            s_co[pos] = in ? ldx<P>(F.oct8 + idx) : (uint8_t)0;
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
          sup = nms_window_suppressed((long long)row * p0 + cbase + bit, s_cv[j], s_co[j], p0, npx, sub, g_occ,
                                      g_score);
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, sup);
        if (j < nc && sub == 0 && !(bal & gmask)) atomicOr(&s_sur[kk], 1u << bit);
      }
    }
  }
  __syncthreads();

  // exclusive scan of the survivor counts, in word order
  const int per = (nwords + 255) >> 8;
  const int beg = min((int)threadIdx.x * per, nwords), end = min(beg + per, nwords);
  int local = 0;
  for (int i = beg; i < end; i++) local += __popc(s_sur[i]);
  int strip_total;
  int run = block_scan_excl(local, s_warp_tot, strip_total);
  for (int i = beg; i < end; i++) {
    s_pref[i] = run;
    run += __popc(s_sur[i]);
  }

  // decoupled look-back over the frame's strips (warp 0)
  if (warp == 0 && ORBX_IN_ROWS(rec, kSiteFrameState, s, F.nms_strips)) {
    unsigned long long* st = F.nms_status;
    int excl = 0;
    if (s == 0) {
      if (lane == 0) st_relaxed_u64(&st[0], kFlagPre | (unsigned)strip_total);
    } else {
      if (lane == 0) st_relaxed_u64(&st[s], kFlagAgg | (unsigned)strip_total);
      __syncwarp();
      excl = nms_lookback(st, s, lane, b.err, b.wait_cycles);
      if (lane == 0) st_relaxed_u64(&st[s], kFlagPre | (unsigned)(excl + strip_total));
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

  // pass 2: write the survivors (score and octave from the stage when staged)
  for (int k = threadIdx.x; k < nwords; k += blockDim.x) {
    uint32_t m = s_sur[k];
    if (!m) continue;
    const int row = row0 + k / nw;
    const int cbase = (wlo + k % nw) << 5;
    const long long wi = ((long long)row * p0 + cbase) >> 5;
    int rank = base + s_pref[k];
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1u;
      if (rank >= F.max_pts) break;
      const long long idx = (long long)row * p0 + cbase + bit;
      orbx_point q;
      q.x = cbase + bit;
      q.y = row;
      if (staged) {
        const int sw = (int)(wi - W0);
        const int sr = s_pfx[sw] + __popc(s_occ[sw] & ((1u << bit) - 1u));
        q.octave = s_oct[sr];
        q.score = s_score[sr];
      } else {
        const bool in = ORBX_IN_ROWS(rec, kSiteNmsScore, idx, npx);
        q.octave = in ? F.oct8[idx] : 0;
        q.score = in ? F.vmap[idx] : 0.f;
      }
      q.angle = 0.f;
      q.match = 0;
      q.distance = 0;
      if (ORBX_IN_ROWS(rec, kSiteNmsPts, rank, F.max_pts)) F.pts[rank] = q;
      rank++;
    }
  }
}

// ---------------------------------------------------------------------------
// Orientation and rBRIEF (orbx_describe.cu and the persistent kernel)
// ---------------------------------------------------------------------------
// Plain loads of data written earlier in the same launch (PL) or by earlier
// launches; PL uses the coherent cached path explicitly.
template <bool PL, class T>
__device__ __forceinline__ T ldc(const T* p) {
  if constexpr (PL)
    return __ldca(p);
  else
    return *p;
}

constexpr int kDescWarps = 8;

// getValue (orbd.cu:1341-1348): the rotated point is
// (rint(x*c - y*s), rint(x*s + y*c)), evaluated by the reference build as
// fma(x, c, -(y*s)) and fma(x, s, y*c).
template <bool PL>
__device__ __forceinline__ int sample_at(const uint8_t* center, int pitch, float x, float y, float s, float c,
                                         BoundsRec* rec, Span blr) {
  const int ix = __float2int_rn(__fmaf_rn(x, c, -__fmul_rn(y, s)));
  const int iy = __float2int_rn(__fmaf_rn(x, s, __fmul_rn(y, c)));
  const uint8_t* p = center + (ptrdiff_t)iy * pitch + ix;
  return ORBX_IN(rec, kSiteDescSample, blr, p, 1) ? ldc<PL>(p) : 0;
}

template <int WTA, bool PL>
__device__ __forceinline__ uint8_t describe_byte(const uint8_t* center, int pitch, const float* px, const float* py,
                                                 float s, float c, BoundsRec* rec, Span blr) {
#define G(j) sample_at<PL>(center, pitch, px[j], py[j], s, c, rec, blr)
  uint8_t val = 0;
  if (WTA == 2) {  // feature2 (orbd.cu:1351-1361)
#pragma unroll
    for (int j = 0; j < 8; j++) val |= (uint8_t)((G(2 * j) < G(2 * j + 1)) << j);
  } else if (WTA == 3) {  // feature3 (orbd.cu:1364-1388), including its index reuse of 8 and skip of 10
    const int idx[4][3] = {{0, 1, 2}, {3, 4, 5}, {6, 7, 8}, {8, 9, 11}};
#pragma unroll
    for (int g = 0; g < 4; g++) {
      const int t0 = G(idx[g][0]), t1 = G(idx[g][1]), t2 = G(idx[g][2]);
      const int v = t2 > t1 ? (t2 > t0 ? 2 : 0) : (t1 > t0);
      val |= (uint8_t)(v << (2 * g));
    }
  } else {  // feature4 (orbd.cu:1391-1434)
#pragma unroll
    for (int g = 0; g < 4; g++) {
      int t0 = G(4 * g), t1 = G(4 * g + 1), t2 = G(4 * g + 2), t3 = G(4 * g + 3);
      int u = 0, v = 2;
      if (t1 > t0) t0 = t1, u = 1;
      if (t3 > t2) t2 = t3, v = 3;
      val |= (uint8_t)((t0 > t2 ? u : v) << (2 * g));
    }
  }
#undef G
  return val;
}

// This lane's pattern points of descriptor byte `lane` (setPattern,
// orbd.cu:95-410): PSTEP (x, y) int8 pairs, contiguous per lane, fetched as
// raw words (load_pattern_raw) so that the loads can be in flight with other
// work, then converted (pattern_points).
template <int WTA>
struct PatternRaw {
  static constexpr int PSTEP = (WTA == 3) ? 12 : 16;
  static constexpr int WORDS = PSTEP / 2;  // 2 * PSTEP bytes
  uint32_t w[WORDS];
};
template <int WTA>
__device__ __forceinline__ PatternRaw<WTA> load_pattern_raw(const Batch& b, int lane) {
  PatternRaw<WTA> r;
  constexpr int W = PatternRaw<WTA>::WORDS;
  // 2 * PSTEP * lane bytes in: a multiple of 8 (WTA 3) or 16, and the table is 16-byte aligned
  const uint32_t* src = reinterpret_cast<const uint32_t*>(b.pattern) + W * lane;
  if constexpr (W % 4 == 0) {
#pragma unroll
    for (int i = 0; i < W / 4; i++) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(src) + i);
      r.w[4 * i] = v.x, r.w[4 * i + 1] = v.y, r.w[4 * i + 2] = v.z, r.w[4 * i + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < W / 2; i++) {
      const uint2 v = __ldg(reinterpret_cast<const uint2*>(src) + i);
      r.w[2 * i] = v.x, r.w[2 * i + 1] = v.y;
    }
  }
  return r;
}
template <int WTA>
__device__ __forceinline__ void pattern_points(const PatternRaw<WTA>& r, float* px, float* py) {
#pragma unroll
  for (int j = 0; j < PatternRaw<WTA>::PSTEP; j++) {
    const uint32_t word = r.w[j >> 1];
    const int sh = 16 * (j & 1);
    px[j] = (float)(int)(int8_t)((word >> sh) & 0xFFu);
    py[j] = (float)(int)(int8_t)((word >> (sh + 8)) & 0xFFu);
  }
}
template <int WTA>
__device__ __forceinline__ void load_pattern(const Batch& b, int lane, float* px, float* py) {
  pattern_points<WTA>(load_pattern_raw<WTA>(b, lane), px, py);
}

template <int WTA, bool PL>
__device__ __forceinline__ void describe_keypoint(const Batch& b, const Frame& F, int k, const float* px,
                                                  const float* py, const int* s_umax, int lane) {
  const int half_k = b.half_k;
  if (!ORBX_IN_ROWS(b.bounds, kSiteDescPts, k, F.max_pts)) return;
  orbx_point* P = F.pts + k;
  const int x = ldc<PL>(&P->x), y = ldc<PL>(&P->y), o = ldc<PL>(&P->octave);
  const int pitch = F.op[o];
  const long long coff = F.ooff[o] + (long long)(y >> o) * pitch + (x >> o);

  float angle;
  if (b.describe_mode != kDescribeDescOnly) {
    // intensity centroid on the raw octave: lane v + half_k owns disc row v
    // and reads it as nine aligned words at once (octave pitches are multiples
    // of 128, so every row has the same alignment); the integer sums are exact
    // in any order
    const uint8_t* center = F.pyr + coff;
    int m10 = 0, m01 = 0;
    if (lane <= 2 * half_k) {
      const int v = lane - half_k;
      const int um = s_umax[v < 0 ? -v : v];
      const uintptr_t ra = reinterpret_cast<uintptr_t>(center + (ptrdiff_t)v * pitch - half_k);  // column -half_k
      const uint32_t* wp = reinterpret_cast<const uint32_t*>(ra & ~(uintptr_t)3);
      const unsigned sh = 8u * (unsigned)(ra & 3);
      uint32_t w[9];
      const bool in = ORBX_IN(b.bounds, kSiteDescMoment, guarded_span(F.pyr, F), wp, 36);
#pragma unroll
      for (int i = 0; i < 9; i++) w[i] = in ? ldc<PL>(wp + i) : 0u;
      int sum = 0;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const uint32_t r = __funnelshift_r(w[i], w[i + 1], sh);  // columns 4i - half_k .. 4i + 3 - half_k
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int uu = 4 * i + k - half_k;
          if ((unsigned)(uu + um) <= (unsigned)(2 * um)) {  // |uu| <= um
            const int val = (int)((r >> (8 * k)) & 0xFFu);
            m10 += uu * val;
            sum += val;
          }
        }
      }
      m01 = v * sum;
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      m10 += __shfl_xor_sync(0xffffffffu, m10, d);
      m01 += __shfl_xor_sync(0xffffffffu, m01, d);
    }
    angle = fast_atan2(__int2float_rn(m01), __int2float_rn(m10));
    if (lane == 0) P->angle = angle;
    if (b.describe_mode == kDescribeAngleOnly) return;
  } else {
    angle = ldc<PL>(&P->angle);
  }

  // rBRIEF on the blurred octave
  const float sn = __sinf(angle);
  const float cs = __cosf(angle);
  const uint8_t byte = describe_byte<WTA, PL>(F.blr + coff, pitch, px, py, sn, cs, b.bounds, guarded_span(F.blr, F));
  F.desc[(size_t)k * 32 + lane] = byte;
}

// ---------------------------------------------------------------------------
// k = 2 XOR-popcount matching (orbx_match.cu and the persistent kernel)
// ---------------------------------------------------------------------------
constexpr int kMQ = 128;      // queries per block
constexpr int kMChunk = 512;  // train rows per shared-memory chunk (16 KB)
constexpr int kIdxBits = kIdxBitsShared;
constexpr uint32_t kNoKey = kNoKeyShared;

__device__ __forceinline__ void top2_push(uint32_t& k1, uint32_t& k2, uint32_t key) { top2_push_shared(k1, k2, key); }
__device__ __forceinline__ void finish_query(const MatchArgs& a, int q, uint32_t k1, uint32_t k2) {
  finish_query_shared(a, q, k1, k2);
}

// One block's share of a k = 2 search with QPB queries per block (QPB =
// blockDim.x); bid / nblk replace blockIdx.x / gridDim.x so that a batch launch
// or a work item of the persistent kernel can run one search each.  P: the
// descriptors and counts were written earlier in the same launch.
template <int QPB, bool P>
__device__ __forceinline__ void match_popc_block(const MatchArgs& a, const MatchWork& w, int bid, int nblk,
                                                 uint4* s_db, unsigned int& s_last) {

  const int nq = min(a.d_nq ? ldx<P>(a.d_nq) : a.nq, w.nq_cap);
  const int ndb = a.d_ndb ? ldx<P>(a.d_ndb) : a.ndb;
  // Spread (query tile, train split) pairs over the launched blocks using the
  // actual counts, which may be far below the capacities the grid was sized for.
  const int tiles = (nq + QPB - 1) / QPB;
  if (tiles == 0) return;
  int splits = nblk / tiles;
  splits = min(splits, w.splits_cap);
  splits = min(splits, max(1, (ndb + 63) / 64));
  splits = max(splits, 1);
  const int tile = bid / splits;
  const int split = bid - tile * splits;
  if (tile >= tiles) return;
  const int q = tile * QPB + threadIdx.x;
  const bool active = q < nq;

  uint32_t qw[8];
  {
    const uint4* qp = reinterpret_cast<const uint4*>(a.q) + 2 * (size_t)(active ? q : 0);
    const bool in = ORBX_IN_ROWS(a.bounds, kSiteMatchQ, active ? q : 0, a.q_cap);
    const uint4 v0 = in ? ldx<P>(qp) : uint4{}, v1 = in ? ldx<P>(qp + 1) : uint4{};
    qw[0] = v0.x; qw[1] = v0.y; qw[2] = v0.z; qw[3] = v0.w;
    qw[4] = v1.x; qw[5] = v1.y; qw[6] = v1.z; qw[7] = v1.w;
  }

  const int r_beg = (int)((long long)ndb * split / splits);
  const int r_end = (int)((long long)ndb * (split + 1) / splits);
  uint32_t k1 = kNoKey, k2 = kNoKey;
  const uint4* db4 = reinterpret_cast<const uint4*>(a.db);
  for (int r0 = r_beg; r0 < r_end; r0 += kMChunk) {
    const int rows = min(kMChunk, r_end - r0);
    __syncthreads();
    for (int i = threadIdx.x; i < rows * 2; i += QPB)
      s_db[i] = ORBX_IN_ROWS(a.bounds, kSiteMatchDb, r0 + (i >> 1), a.db_cap) ? ldx<P>(db4 + 2 * (size_t)r0 + i)
                                                                             : uint4{};
    __syncthreads();
    for (int j = 0; j < rows; j++) {
      const uint4 t0 = s_db[2 * j], t1 = s_db[2 * j + 1];
      const uint32_t d = __popc(qw[0] ^ t0.x) + __popc(qw[1] ^ t0.y) + __popc(qw[2] ^ t0.z) +
                         __popc(qw[3] ^ t0.w) + __popc(qw[4] ^ t1.x) + __popc(qw[5] ^ t1.y) +
                         __popc(qw[6] ^ t1.z) + __popc(qw[7] ^ t1.w);
      top2_push(k1, k2, (d << kIdxBits) | (uint32_t)(r0 + j));
    }
  }

  if (splits == 1) {
    if (active) finish_query(a, q, k1, k2);
    return;
  }
  // publish this split's partial top-2; the last split to finish the tile merges
  if (active) {
    uint2* part = reinterpret_cast<uint2*>(w.part);
    part[(size_t)split * w.nq_cap + q] = make_uint2(k1, k2);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&w.tile_done[tile], 1u) == (unsigned)(splits - 1)) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) w.tile_done[tile] = 0u;  // ready for the next launch
  if (!active) return;
  const uint2* part = reinterpret_cast<const uint2*>(w.part);
  uint32_t m1 = kNoKey, m2 = kNoKey;
  for (int sp = 0; sp < splits; sp++) {
    const uint2 pk = __ldcg(part + (size_t)sp * w.nq_cap + q);
    top2_push(m1, m2, pk.x);
    top2_push(m1, m2, pk.y);
  }
  finish_query(a, q, m1, m2);
}

}  // namespace orbx
