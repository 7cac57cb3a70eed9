// Orientation and rBRIEF descriptors for sm_100a: one warp per keypoint.
//
// angleIC (orbd.cu:1001-1036) and gDescrible (orbd.cu:1437-1468) fused.  The
// warp loads the 31x31 disc row by row (lane u+15 owns column u, so each row is
// one coalesced 31-byte read), reduces the integer moments with shuffles, and
// every lane then evaluates the angle; lane t builds descriptor byte t from its
// pattern points, which it keeps in registers for all keypoints it visits.
#include "orbx_stages.cuh"

namespace orbx {

template <int WTA, bool INL>
__global__ void __launch_bounds__(kDescWarps * 32) k_describe(const __grid_constant__ Batch b) {
  __shared__ int s_pref[kMaxFramesPerLaunch + 1];
  __shared__ int s_umax[32];

  __shared__ int s_wsum[kDescWarps];
  const int lane = threadIdx.x & 31;
  const int nf = b.n_frames;
  // set at init: the pattern words (in flight while the counts are read) and
  // the disc table; the frame descriptors are pulled into L1 for the keypoints
  const PatternRaw<WTA> praw = load_pattern_raw<WTA>(b, lane);
  const int half_k = b.half_k;
  if (threadIdx.x < half_k + 1) s_umax[threadIdx.x] = b.umax[threadIdx.x];
  constexpr int kFrameLines = (int)((sizeof(Frame) + 127) / 128);
  if (!INL && nf <= 8 && (int)threadIdx.x < nf * kFrameLines)
    asm volatile("prefetch.global.L1 [%0];" ::"l"(reinterpret_cast<const char*>(b.frames + threadIdx.x / kFrameLines) +
                                                  128 * (threadIdx.x % kFrameLines)));
  // exclusive prefix of the per-frame keypoint counts (written by k_nms):
  // thread t scans frames [t*per, (t+1)*per)
  {
    const int per = (nf + kDescWarps * 32 - 1) / (kDescWarps * 32);
    const int beg = min((int)threadIdx.x * per, nf), end = min(beg + per, nf);
    int local = 0;
    for (int f = beg; f < end; f++) local += *batch_frame<INL>(b, f).count;
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
      run += *batch_frame<INL>(b, f).count;
    }
    if (threadIdx.x == kDescWarps * 32 - 1) s_pref[nf] = run;
  }
  __syncthreads();
  const int total = s_pref[nf];

  constexpr int PSTEP = PatternRaw<WTA>::PSTEP;
  float px[PSTEP], py[PSTEP];
  pattern_points<WTA>(praw, px, py);

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
    describe_keypoint<WTA, false>(b, batch_frame<INL>(b, lo), i - s_pref[lo], px, py, s_umax, lane);
  }
}

cudaError_t launch_describe(const Batch& b, int total_max_pts, cudaStream_t s, int blocks_per_sm) {
  if (total_max_pts <= 0) return cudaSuccess;
  int warps_needed = total_max_pts;
  int blocks = (warps_needed + kDescWarps - 1) / kDescWarps;
  const int cap = 148 * (blocks_per_sm > 0 ? blocks_per_sm : 8);
  if (blocks > cap) blocks = cap;
  const dim3 g(blocks), t(kDescWarps * 32);
  if (b.n_inline > 0) {
    if (b.wta_k == 3)
      k_describe<3, true><<<g, t, 0, s>>>(b);
    else if (b.wta_k == 4)
      k_describe<4, true><<<g, t, 0, s>>>(b);
    else
      k_describe<2, true><<<g, t, 0, s>>>(b);
  } else {
    if (b.wta_k == 3)
      k_describe<3, false><<<g, t, 0, s>>>(b);
    else if (b.wta_k == 4)
      k_describe<4, false><<<g, t, 0, s>>>(b);
    else
      k_describe<2, false><<<g, t, 0, s>>>(b);
  }
  return cudaGetLastError();
}

}  // namespace orbx
