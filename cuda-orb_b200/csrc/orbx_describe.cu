// Orientation and rBRIEF descriptors for sm_100a: one warp per keypoint.
//
// angleIC (orbd.cu:1001-1036) and gDescrible (orbd.cu:1437-1468) fused.  The
// warp loads the 31x31 disc row by row (lane u+15 owns column u, so each row is
// one coalesced 31-byte read), reduces the integer moments with shuffles, and
// every lane then evaluates the angle; lane t builds descriptor byte t from its
// pattern points, which it keeps in registers for all keypoints it visits.
#include "orbx_device.cuh"
#include "orbx_internal.cuh"

namespace orbx {

constexpr int kDescWarps = 8;

// getValue (orbd.cu:1341-1348): the rotated point is
// (rint(x*c - y*s), rint(x*s + y*c)), evaluated by the reference build as
// fma(x, c, -(y*s)) and fma(x, s, y*c).
__device__ __forceinline__ int sample_at(const uint8_t* center, int pitch, float x, float y, float s, float c) {
  const int ix = __float2int_rn(__fmaf_rn(x, c, -__fmul_rn(y, s)));
  const int iy = __float2int_rn(__fmaf_rn(x, s, __fmul_rn(y, c)));
  return center[(ptrdiff_t)iy * pitch + ix];
}

template <int WTA>
__device__ __forceinline__ uint8_t describe_byte(const uint8_t* center, int pitch, const float* px, const float* py,
                                                 float s, float c) {
#define G(j) sample_at(center, pitch, px[j], py[j], s, c)
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

template <int WTA>
__global__ void __launch_bounds__(kDescWarps * 32) k_describe(Batch b) {
  __shared__ int s_pref[kMaxFramesPerLaunch + 1];
  __shared__ int s_umax[32];

  __shared__ int s_wsum[kDescWarps];
  const int lane = threadIdx.x & 31;
  const int nf = b.n_frames;
  // exclusive prefix of the per-frame keypoint counts (written by k_nms):
  // thread t scans frames [t*per, (t+1)*per)
  {
    const int per = (nf + kDescWarps * 32 - 1) / (kDescWarps * 32);
    const int beg = min((int)threadIdx.x * per, nf), end = min(beg + per, nf);
    int local = 0;
    for (int f = beg; f < end; f++) local += *b.frames[f].count;
    int incl = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int n = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += n;
    }
    if (lane == 31) s_wsum[threadIdx.x >> 5] = incl;
    __syncthreads();
    int run = incl - local;
    for (int w2 = 0; w2 < (int)(threadIdx.x >> 5); w2++) run += s_wsum[w2];
    for (int f = beg; f < end; f++) {
      s_pref[f] = run;
      run += *b.frames[f].count;
    }
    if (threadIdx.x == kDescWarps * 32 - 1) s_pref[nf] = run;
  }
  const int half_k = b.half_k;
  if (threadIdx.x < half_k + 1) s_umax[threadIdx.x] = b.umax[threadIdx.x];
  __syncthreads();
  const int total = s_pref[nf];

  constexpr int PSTEP = (WTA == 3) ? 12 : 16;
  float px[PSTEP], py[PSTEP];
#pragma unroll
  for (int j = 0; j < PSTEP; j++) {
    px[j] = (float)b.pattern[2 * (PSTEP * lane + j)];
    py[j] = (float)b.pattern[2 * (PSTEP * lane + j) + 1];
  }

  const int u = lane - 15;
  const int gw = blockIdx.x * kDescWarps + (threadIdx.x >> 5);
  const int nw = gridDim.x * kDescWarps;
  for (int i = gw; i < total; i += nw) {
    int lo = 0, hi = nf - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_pref[mid] <= i)
        lo = mid;
      else
        hi = mid - 1;
    }
    const Frame& F = b.frames[lo];
    const int k = i - s_pref[lo];
    orbx_point* P = F.pts + k;
    const int x = P->x, y = P->y, o = P->octave;
    const int pitch = F.op[o];
    const long long coff = F.ooff[o] + (long long)(y >> o) * pitch + (x >> o);

    float angle;
    if (b.describe_mode != kDescribeDescOnly) {
      // intensity centroid on the raw octave
      const uint8_t* center = F.pyr + coff;
      int m10 = 0, m01 = 0;
      for (int v = -half_k; v <= half_k; v++) {
        const int um = s_umax[v < 0 ? -v : v];
        if (lane < 31 && u >= -um && u <= um) {
          const int val = center[(ptrdiff_t)v * pitch + u];
          m10 += u * val;
          m01 += v * val;
        }
      }
#pragma unroll
      for (int d = 16; d >= 1; d >>= 1) {
        m10 += __shfl_xor_sync(0xffffffffu, m10, d);
        m01 += __shfl_xor_sync(0xffffffffu, m01, d);
      }
      angle = fast_atan2(__int2float_rn(m01), __int2float_rn(m10));
      if (lane == 0) P->angle = angle;
      if (b.describe_mode == kDescribeAngleOnly) continue;
    } else {
      angle = P->angle;
    }

    // rBRIEF on the blurred octave
    const float sn = __sinf(angle);
    const float cs = __cosf(angle);
    const uint8_t byte = describe_byte<WTA>(F.blr + coff, pitch, px, py, sn, cs);
    F.desc[(size_t)k * 32 + lane] = byte;
  }
}

cudaError_t launch_describe(const Batch& b, int total_max_pts, cudaStream_t s, int blocks_per_sm) {
  if (total_max_pts <= 0) return cudaSuccess;
  int warps_needed = total_max_pts;
  int blocks = (warps_needed + kDescWarps - 1) / kDescWarps;
  const int cap = 148 * (blocks_per_sm > 0 ? blocks_per_sm : 8);
  if (blocks > cap) blocks = cap;
  if (b.wta_k == 3)
    k_describe<3><<<blocks, kDescWarps * 32, 0, s>>>(b);
  else if (b.wta_k == 4)
    k_describe<4><<<blocks, kDescWarps * 32, 0, s>>>(b);
  else
    k_describe<2><<<blocks, kDescWarps * 32, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace orbx
