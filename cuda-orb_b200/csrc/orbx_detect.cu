// Pyramid, blur, FAST-9 + Harris score map and NMS for sm_100a.
//
// Each launch covers a batch of frames; a block finds its frame through a
// prefix table of tile counts.  Pyramid layout, guards and the score-map
// format follow the reference (orb.cpp:145-191, orbd.cu:1576-1577) so that
// reads that leave an octave see the same bytes the reference sees.
#include "orbx_stages.cuh"

namespace orbx {

// Kernels take the batch as a grid constant so that, for batches whose frame
// table travels in the launch parameters (INL), the stages read it in place.
template <int TW, int TH, bool INL>
__global__ void __launch_bounds__(kPyrThreads, 5) k_pyramid_blur(const __grid_constant__ Batch b) {
  __shared__ PyrSmem<TW, TH> sm;
  pyr_tile<false, TW, TH, INL>(b, blockIdx.x, sm);
}

template <bool INL>
__global__ void __launch_bounds__(256, 6) k_detect(const __grid_constant__ Batch b) {
  __shared__ DetSmem sm;
  det_tile<false, INL>(b, blockIdx.x, sm);
}

template <bool INL>
__global__ void __launch_bounds__(256, 4) k_nms(const __grid_constant__ Batch b) {
  __shared__ NmsSmem sm;
  __shared__ int s_ticket;
  if (threadIdx.x == 0) s_ticket = (int)atomicAdd(b.nms_ticket, 1u);
  __syncthreads();
  nms_strip<false, INL>(b, s_ticket, sm);
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
  const bool inl = b.n_inline > 0;
  switch (b.pyr_shape) {
    case 1:
      if (inl) k_pyramid_blur<kPyrShapeTW[1], kPyrShapeTH[1], true><<<total_tiles, kPyrThreads, 0, s>>>(b);
      else k_pyramid_blur<kPyrShapeTW[1], kPyrShapeTH[1], false><<<total_tiles, kPyrThreads, 0, s>>>(b);
      break;
    case 2:
      if (inl) k_pyramid_blur<kPyrShapeTW[2], kPyrShapeTH[2], true><<<total_tiles, kPyrThreads, 0, s>>>(b);
      else k_pyramid_blur<kPyrShapeTW[2], kPyrShapeTH[2], false><<<total_tiles, kPyrThreads, 0, s>>>(b);
      break;
    case 3:
      if (inl) k_pyramid_blur<kPyrShapeTW[3], kPyrShapeTH[3], true><<<total_tiles, kPyrThreads, 0, s>>>(b);
      else k_pyramid_blur<kPyrShapeTW[3], kPyrShapeTH[3], false><<<total_tiles, kPyrThreads, 0, s>>>(b);
      break;
    default:
      if (inl) k_pyramid_blur<kPyrShapeTW[0], kPyrShapeTH[0], true><<<total_tiles, kPyrThreads, 0, s>>>(b);
      else k_pyramid_blur<kPyrShapeTW[0], kPyrShapeTH[0], false><<<total_tiles, kPyrThreads, 0, s>>>(b);
  }
  return cudaGetLastError();
}

cudaError_t launch_detect(const Batch& b, int total_tiles, cudaStream_t s) {
  if (total_tiles <= 0) return cudaSuccess;
  if (b.n_inline > 0)
    k_detect<true><<<total_tiles, 256, 0, s>>>(b);
  else
    k_detect<false><<<total_tiles, 256, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_nms(const Batch& b, int total_strips, cudaStream_t s) {
  if (total_strips <= 0) return cudaSuccess;
  if (b.n_inline > 0)
    k_nms<true><<<total_strips, 256, 0, s>>>(b);
  else
    k_nms<false><<<total_strips, 256, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace orbx
