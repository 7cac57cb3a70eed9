// Pyramid, blur, FAST-9 + Harris score map and NMS for sm_100a.
//
// Each launch covers a batch of frames; a block finds its frame through a
// prefix table of tile counts.  Pyramid layout, guards and the score-map
// format follow the reference (orb.cpp:145-191, orbd.cu:1576-1577) so that
// reads that leave an octave see the same bytes the reference sees.
#include "orbx_device.cuh"
#include "orbx_internal.cuh"

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
constexpr int kPyrSW = kPyrTW + 6;
constexpr int kPyrSH = kPyrTH + 6;

__global__ void __launch_bounds__(256) k_pyramid_blur(Batch b) {
  __shared__ uint8_t s_src[kPyrSH * kPyrSW];
  __shared__ float s_row[kPyrSH * kPyrTW];

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

  const uint8_t* __restrict__ psrc = F.pyr_src ? F.pyr_src + F.ooff[o] : nullptr;
  for (int i = threadIdx.x; i < kPyrSH * kPyrSW; i += blockDim.x) {
    const int r = i / kPyrSW;
    const int c = i - r * kPyrSW;
    const int y = reflect101(y0 - 3 + r, oh);
    const int x = reflect101(x0 - 3 + c, ow);
    s_src[i] = psrc ? __ldg(psrc + (size_t)y * op + x) : __ldg(img + (size_t)(y << o) * pitch_in + (x << o));
  }
  __syncthreads();

  const float* k = b.gauss;
  for (int i = threadIdx.x; i < kPyrSH * kPyrTW; i += blockDim.x) {
    const int r = i / kPyrTW;
    const int c = i - r * kPyrTW;
    const uint8_t* s = s_src + r * kPyrSW + c + 3;
    const float t0 = (float)(int)s[0];
    const float t1 = (float)((int)s[-1] + (int)s[1]);
    const float t2 = (float)((int)s[-2] + (int)s[2]);
    const float t3 = (float)((int)s[-3] + (int)s[3]);
    s_row[i] = gauss_dot4(k, t0, t1, t2, t3);
  }
  __syncthreads();

  uint8_t* P = F.pyr + F.ooff[o];
  uint8_t* B = F.blr + F.ooff[o];
  const bool copy_pad = (o == 0) && (pitch_in == op);
  for (int i = threadIdx.x; i < kPyrTH * kPyrTW; i += blockDim.x) {
    const int r = i / kPyrTW;
    const int c = i - r * kPyrTW;
    const int y = y0 + r;
    const int x = x0 + c;
    if (y >= oh || x >= op) continue;
    const size_t a = (size_t)y * op + x;
    if (x < ow) {
      const float* col = s_row + (r + 3) * kPyrTW + c;
      const float t0 = col[0];
      const float t1 = __fadd_rn(col[-kPyrTW], col[kPyrTW]);
      const float t2 = __fadd_rn(col[-2 * kPyrTW], col[2 * kPyrTW]);
      const float t3 = __fadd_rn(col[-3 * kPyrTW], col[3 * kPyrTW]);
      B[a] = (uint8_t)__float2int_rn(gauss_dot4(k, t0, t1, t2, t3));
      P[a] = s_src[(r + 3) * kPyrSW + c + 3];
    } else {
      // Row padding: octave 0 carries the caller's padding bytes (the reference
      // copies h * pitch0 bytes, orbd.cu:1584); other octaves hold zeros.
      const uint8_t v = psrc ? __ldg(psrc + a) : (copy_pad ? __ldg(img + (size_t)y * pitch_in + x) : (uint8_t)0);
      P[a] = v;
      B[a] = v;
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
// as in the reference, merges the octaves in shared memory, and writes its
// region of the score map densely (no clearing pass is needed).
// ---------------------------------------------------------------------------
constexpr int kHalo = 4;
__host__ __device__ constexpr int det_stage_bytes() {
  int s = 0;
  for (int o = 0; o < kMaxOctaves; o++) s += ((kDetTW >> o) + 2 * kHalo) * ((kDetTH >> o) + 2 * kHalo);
  return s;
}

// FAST ring (makeOffsets, orbd.cu:463-496), as (dx, dy).
__constant__ int8_t c_ring[16][2] = {{0, 3},  {1, 3},   {2, 2},   {3, 1},   {3, 0},  {3, -1}, {2, -2}, {1, -3},
                                     {0, -3}, {-1, -3}, {-2, -2}, {-3, -1}, {-3, 0}, {-3, 1}, {-2, 2}, {-1, 3}};

__device__ __forceinline__ bool has_arc9(uint32_t m16) {
  uint32_t m = m16 | (m16 << 16);  // circular
  uint32_t a = m & (m >> 1);       // runs of 2
  a &= a >> 2;                     // runs of 4
  a &= a >> 4;                     // runs of 8
  a &= m >> 8;                     // runs of 9
  return (a & 0xFFFFu) != 0u;
}

// dHarrisScore (orbd.cu:651-669) on a shared-memory tile of row stride sw.
// Integer sums wrap as 32-bit; the final combine is
// fma(-0.04f, (float)(uint32)(dsxy*dsxy), (float)(int32)(dxx*dyy - dxy*dxy)) * scale^4,
// which is how the reference build evaluates
// (dxx*dyy - dxy*dxy - HARRIS_K*(dsxy*dsxy)) * d_scale_sq_sq.
__device__ __forceinline__ float harris_score(const uint8_t* c, int sw, float scale4) {
  int dxx = 0, dyy = 0, dxy = 0;
#pragma unroll
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
  const unsigned dsxy = (unsigned)(dxx + dyy);
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

__global__ void __launch_bounds__(256) k_detect(Batch b) {
  __shared__ uint8_t s_stage[det_stage_bytes()];
  __shared__ float s_map[kDetTH * kDetTW];
  __shared__ int s_oct[kDetTH * kDetTW];

  const int t = blockIdx.x;
  const int f = find_frame(b.det_base, b.n_frames, t);
  const Frame& F = b.frames[f];
  const int lt = t - b.det_base[f];
  const int X0 = (lt % F.det_tiles_x) * kDetTW;
  const int Y0 = (lt / F.det_tiles_x) * kDetTH;
  const int n_oct = F.n_oct;
  const uint8_t* __restrict__ pyr = F.pyr;

  for (int i = threadIdx.x; i < kDetTH * kDetTW; i += blockDim.x) {
    s_map[i] = 0.f;
    s_oct[i] = 0;
  }
  // Stage every octave's tile with its halo (linear pyramid addressing).
  {
    int off = 0;
    for (int o = 0; o < n_oct; o++) {
      const int sw = (kDetTW >> o) + 2 * kHalo;
      const int sh = (kDetTH >> o) + 2 * kHalo;
      const long long base = F.ooff[o] + (long long)((Y0 >> o) - kHalo) * F.op[o] + ((X0 >> o) - kHalo);
      for (int i = threadIdx.x; i < sw * sh; i += blockDim.x) {
        const int r = i / sw;
        const int c = i - r * sw;
        s_stage[off + i] = __ldg(pyr + base + (long long)r * F.op[o] + c);
      }
      off += sw * sh;
    }
  }
  __syncthreads();

  const int thr = b.fast_thr;
  int off = 0;
  for (int o = 0; o < n_oct; o++) {
    const int tw = kDetTW >> o;
    const int th = kDetTH >> o;
    const int sw = tw + 2 * kHalo;
    const int ow = F.ow[o], oh = F.oh[o];
    const int xb = X0 >> o, yb = Y0 >> o;
    for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
      const int ly = i / tw;
      const int lx = i - ly * tw;
      const int x = xb + lx, y = yb + ly;
      if (x < 3 || x >= ow - 3 || y < 3 || y >= oh - 3) continue;
      const uint8_t* c = s_stage + off + (ly + kHalo) * sw + (lx + kHalo);
      const int v = c[0];
      uint32_t dark = 0, bright = 0;
      int ring[16];
#pragma unroll
      for (int k = 0; k < 16; k++) {
        const int p = c[c_ring[k][1] * sw + c_ring[k][0]];
        ring[k] = p;
        dark |= (uint32_t)(p < v - thr) << k;
        bright |= (uint32_t)(p > v + thr) << k;
      }
      if (!has_arc9(dark) && !has_arc9(bright)) continue;
      float score;
      if (b.harris) {
        score = harris_score(c, sw, b.harris_scale4);
      } else {
        int d[25];
#pragma unroll
        for (int k = 0; k < 25; k++) d[k] = (int)(short)(v - ring[k & 15]);
        score = fast_score(d, thr);
      }
      const int m = (ly << o) * kDetTW + (lx << o);
      if (s_map[m] < score) {
        s_map[m] = score;
        s_oct[m] = o;
      }
    }
    off += sw * ((kDetTH >> o) + 2 * kHalo);
    __syncthreads();
  }

  const int p0 = F.op[0];
  for (int i = threadIdx.x; i < kDetTH * kDetTW; i += blockDim.x) {
    const int r = i / kDetTW;
    const int c = i - r * kDetTW;
    const int X = X0 + c, Y = Y0 + r;
    if (X < F.w && Y < F.h) {
      const size_t a = (size_t)Y * p0 + X;
      F.vmap[a] = s_map[i];
      F.layer[a] = s_oct[i];
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
// scheduling).  Here each block takes a full-width strip of kNmsRows rows in
// ticket order, ranks its survivors with warp ballots, and chains strip totals
// with a decoupled look-back, so keypoints come out in raster order and the cap
// keeps the first max_pts of them.
// ---------------------------------------------------------------------------
constexpr int kNmsMaxChunks = 256;
constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagPre = 2ull << 32;
constexpr int kLookbackSpinLimit = 1 << 22;

// Neighbours are addressed linearly like the reference (a column past the
// edge is the adjacent row's entry); positions outside the map, reachable only
// with an edge threshold below the window radius 2^o, read as 0.
__device__ __forceinline__ bool nms_survives(const float* __restrict__ vmap, const int* __restrict__ layer, size_t idx,
                                             int p0, long long npx, float* v_out, int* o_out) {
  const float v = vmap[idx];
  if (!(v > 0.f)) return false;
  const int o = layer[idx];
  const int r = 1 << o;
  for (int dy = -r; dy <= r; dy++) {
    const long long rowi = (long long)idx + (long long)dy * p0;
    for (int dx = -r; dx <= r; dx++) {
      if (dx == 0 && dy == 0) continue;
      const long long li = rowi + dx;
      const float u = (li >= 0 && li < npx) ? vmap[li] : 0.f;
      if (u > 0.f && (u > v || (u == v && dx <= 0 && dy <= 0))) return false;
    }
  }
  *v_out = v;
  *o_out = o;
  return true;
}

__global__ void __launch_bounds__(256) k_nms(Batch b) {
  __shared__ uint32_t s_mask[kNmsMaxChunks * 8];
  __shared__ int s_pref[kNmsMaxChunks * 8];
  __shared__ int s_warp_tot[8];
  __shared__ int s_ticket, s_base;

  if (threadIdx.x == 0) s_ticket = (int)atomicAdd(b.nms_ticket, 1u);
  __syncthreads();
  const int ticket = s_ticket;
  const int f = find_frame(b.nms_base, b.n_frames, ticket);
  const Frame& F = b.frames[f];
  const int s = ticket - b.nms_base[f];
  const int border = F.border;
  const int row0 = border + s * kNmsRows;
  const int row1 = min(row0 + kNmsRows, F.h - border);
  const int ncols = F.w - 2 * border;
  const int npx = (row1 - row0) * ncols;
  const int nchunks = (npx + 255) >> 8;
  const int p0 = F.op[0];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // pass 1: survivor masks in raster order
  for (int k = 0; k < nchunks; k++) {
    const int p = (k << 8) + threadIdx.x;
    bool sur = false;
    if (p < npx) {
      const int y = row0 + p / ncols;
      const int x = border + p % ncols;
      float v;
      int o;
      sur = nms_survives(F.vmap, F.layer, (size_t)y * p0 + x, p0, (long long)F.h * p0, &v, &o);
    }
    const uint32_t m = __ballot_sync(0xffffffffu, sur);
    if (lane == 0) s_mask[k * 8 + warp] = m;
  }
  __syncthreads();

  // exclusive scan of the mask popcounts, in (chunk, warp) order
  const int nent = nchunks * 8;
  const int per = (nent + 255) >> 8;
  const int beg = min(threadIdx.x * per, nent), end = min(beg + per, nent);
  int local = 0;
  for (int i = beg; i < end; i++) local += __popc(s_mask[i]);
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
    run += __popc(s_mask[i]);
  }
  int strip_total = 0;
  for (int w2 = 0; w2 < 8; w2++) strip_total += s_warp_tot[w2];

  // decoupled look-back over the frame's strips
  if (threadIdx.x == 0) {
    unsigned long long* st = F.nms_status;
    int excl = 0;
    if (s == 0) {
      st_release_u64(&st[0], kFlagPre | (unsigned)strip_total);
    } else {
      st_release_u64(&st[s], kFlagAgg | (unsigned)strip_total);
      int j = s - 1;
      int spins = 0;
      while (j >= 0) {
        const unsigned long long wv = ld_acquire_u64(&st[j]);
        const unsigned long long flag = wv & (3ull << 32);
        if (flag == kFlagPre) {
          excl += (int)(unsigned)wv;
          break;
        }
        if (flag == kFlagAgg) {
          excl += (int)(unsigned)wv;
          j--;
          continue;
        }
        if (++spins > kLookbackSpinLimit) {
          atomicOr(b.err, kErrLookbackTimeout);
          break;
        }
        __nanosleep(32);
      }
      st_release_u64(&st[s], kFlagPre | (unsigned)(excl + strip_total));
    }
    s_base = excl;
    if (s == F.nms_strips - 1) {
      const int tot = excl + strip_total;
      *F.count = min(tot, F.max_pts);
      if (F.total) *F.total = tot;
    }
  }
  __syncthreads();
  const int base = s_base;
  if (base >= F.max_pts) return;

  // pass 2: write survivors
  for (int k = 0; k < nchunks; k++) {
    const uint32_t m = s_mask[k * 8 + warp];
    if (!((m >> lane) & 1u)) continue;
    const int rank = base + s_pref[k * 8 + warp] + __popc(m & ((1u << lane) - 1u));
    if (rank >= F.max_pts) continue;
    const int p = (k << 8) + threadIdx.x;
    const int y = row0 + p / ncols;
    const int x = border + p % ncols;
    const size_t idx = (size_t)y * p0 + x;
    orbx_point q;
    q.x = x;
    q.y = y;
    q.octave = F.layer[idx];
    q.score = F.vmap[idx];
    q.angle = 0.f;
    q.match = 0;
    q.distance = 0;
    F.pts[rank] = q;
  }
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
