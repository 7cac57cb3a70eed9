// Host I/O boundary: image upload with pitch conversion and keypoint export.
//
// The reference uploads nothing itself (its callers hand it device images with
// row pitch align_up(w, 128)) and copies keypoints back with strided
// cudaMemcpy2D calls of 20 or 8 bytes per 28-byte OrbPoint (orb.cpp:95-100,
// 108-111).  Here:
//  - orbx_upload_image takes a host image of any row pitch, pinned or pageable,
//    to a device image of the caller's pitch with zero padding.  Pinned sources
//    go by one 2D DMA; pageable rows are packed into a pinned staging buffer
//    (two buffers, alternating, each reused only after its DMA completed) and
//    sent as one contiguous DMA;
//  - orbx_download_points packs the requested fields of the first n device
//    keypoints into a contiguous buffer on the device, moves it with one DMA,
//    and scatters it into the host OrbPoint array on the CPU, leaving the other
//    fields of each host entry untouched (what the strided copies do).
#include <cuda_runtime.h>

#include <cstring>

#include "orbx_internal.cuh"

namespace orbx {

struct HostIO {
  uint8_t* stage[2] = {nullptr, nullptr};  // pinned upload staging
  size_t stage_bytes[2] = {0, 0};
  cudaEvent_t stage_done[2] = {nullptr, nullptr};
  int next = 0;
  int* pack = nullptr;  // device [n][k] packed fields
  int* pack_host = nullptr;  // pinned copy
  size_t pack_ints = 0;
  uint8_t* map = nullptr;      // pinned, mapped: orbx_pair_host results written by the device
  uint8_t* map_dev = nullptr;  // its device address
  size_t map_bytes = 0;
};

void hostio_free(HostIO* io) {
  if (!io) return;
  for (int i = 0; i < 2; i++) {
    if (io->stage_done[i]) cudaEventSynchronize(io->stage_done[i]);
    cudaFreeHost(io->stage[i]);
    if (io->stage_done[i]) cudaEventDestroy(io->stage_done[i]);
  }
  cudaFree(io->pack);
  cudaFreeHost(io->pack_host);
  cudaFreeHost(io->map);
  delete io;
}

// Result block of a pair in mapped host memory: a 16-byte header (counts of
// A and B, then the context's error word, which is cleared here), then the
// keypoints of A and B (max_pts each), then optionally the descriptors.
__global__ void k_export_pair(const orbx_point* __restrict__ pa, const orbx_point* __restrict__ pb,
                              const uint8_t* __restrict__ da, const uint8_t* __restrict__ db,
                              const int* __restrict__ count, int max_pts, int with_desc, int* err,
                              uint8_t* __restrict__ out) {
  const int na = min(count[0], max_pts), nb = min(count[1], max_pts);
  if (blockIdx.x == 0 && threadIdx.x < 2) reinterpret_cast<int*>(out)[threadIdx.x] = threadIdx.x ? nb : na;
  if (blockIdx.x == 0 && threadIdx.x == 2) {
    reinterpret_cast<int*>(out)[2] = *err;
    *err = 0;
  }
  const size_t pts_words = (size_t)max_pts * 7;  // one image's keypoint block, in 32-bit words
  int* o = reinterpret_cast<int*>(out + 16);
  const long long wa = (long long)na * 7, wb = (long long)nb * 7;
  const long long qa = with_desc ? (long long)na * 8 : 0, qb = with_desc ? (long long)nb * 8 : 0;
  const long long total = wa + wb + qa + qb;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    if (i < wa) {
      o[i] = reinterpret_cast<const int*>(pa)[i];
    } else if (i < wa + wb) {
      o[pts_words + (i - wa)] = reinterpret_cast<const int*>(pb)[i - wa];
    } else if (i < wa + wb + qa) {
      o[2 * pts_words + (i - wa - wb)] = reinterpret_cast<const int*>(da)[i - wa - wb];
    } else {
      o[2 * pts_words + (size_t)max_pts * 8 + (i - wa - wb - qa)] = reinterpret_cast<const int*>(db)[i - wa - wb - qa];
    }
  }
}

// Queues k_export_pair on the context stream; *host points at the result block,
// readable once the stream has been synchronised.
int hostio_map(orbx_ctx* c, int max_pts, const uint8_t** host, const uint8_t** dev) {
  HostIO*& io = ctx_hostio(c);
  if (!io) io = new HostIO();
  const size_t bytes = 16 + (size_t)max_pts * (2 * sizeof(orbx_point) + 64);
  if (io->map_bytes < bytes) {
    cudaFreeHost(io->map);
    io->map = nullptr;
    io->map_dev = nullptr;
    io->map_bytes = 0;
    if (cudaHostAlloc(&io->map, bytes, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&io->map_dev), io->map, 0) != cudaSuccess) {
      (void)cudaGetLastError();
      cudaFreeHost(io->map);
      io->map = nullptr;
      return ORBX_ERR_NOMEM;
    }
    io->map_bytes = bytes;
  }
  *host = io->map;
  if (dev) *dev = io->map_dev;
  return ORBX_OK;
}

int hostio_export_pair(orbx_ctx* c, const orbx_point* pa, const orbx_point* pb, const uint8_t* da, const uint8_t* db,
                       const int* d_count, int max_pts, bool with_desc, const uint8_t** host) {
  const uint8_t* dev = nullptr;
  const int rc = hostio_map(c, max_pts, host, &dev);
  if (rc) return rc;
  k_export_pair<<<2 * 148, 256, 0, ctx_stream(c)>>>(pa, pb, da, db, d_count, max_pts, with_desc ? 1 : 0,
                                                     ctx_err(c), const_cast<uint8_t*>(dev));
  if (cudaGetLastError() != cudaSuccess) return ORBX_ERR_CUDA;
  return ORBX_OK;
}

// fields: bit 0 = x, y, octave, score, angle (ints 0..4); bit 1 = match, distance (ints 5..6)
__global__ void k_pack_points(const orbx_point* __restrict__ pts, int n, int first, int k, int* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int i = t / k, f = t - i * k;
  out[t] = reinterpret_cast<const int*>(pts + i)[first + f];
}

}  // namespace orbx

using namespace orbx;

#define HCHK(x)                                                             \
  do {                                                                      \
    cudaError_t _e = (x);                                                   \
    if (_e != cudaSuccess) {                                                \
      (void)cudaGetLastError();                                             \
      return _e == cudaErrorMemoryAllocation ? ORBX_ERR_NOMEM : ORBX_ERR_CUDA; \
    }                                                                       \
  } while (0)

namespace {
struct Guard {
  int prev = -1;
  explicit Guard(int d) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != d)
      cudaSetDevice(d);
    else
      prev = -1;
  }
  ~Guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

HostIO* hostio(orbx_ctx* c) {
  HostIO*& io = ctx_hostio(c);
  if (!io) io = new HostIO();
  return io;
}
}  // namespace

ORBX_API int orbx_upload_image(orbx_ctx* c, const uint8_t* h_img, int w, int h, int h_pitch, uint8_t* d_img,
                               int d_pitch) {
  if (!c || !h_img || !d_img || w <= 0 || h <= 0 || h_pitch < w || d_pitch < w) return ORBX_ERR_ARG;
  Guard g(ctx_device(c));
  cudaStream_t s = ctx_stream(c);
  if (is_pinned(h_img)) {
    HCHK(cudaMemcpy2DAsync(d_img, (size_t)d_pitch, h_img, (size_t)h_pitch, (size_t)w, (size_t)h,
                           cudaMemcpyHostToDevice, s));
    if (d_pitch > w) HCHK(cudaMemset2DAsync(d_img + w, (size_t)d_pitch, 0, (size_t)(d_pitch - w), (size_t)h, s));
    return ORBX_OK;
  }
  HostIO* io = hostio(c);
  const int b = io->next;
  io->next ^= 1;
  const size_t bytes = (size_t)d_pitch * h;
  if (io->stage_done[b]) HCHK(cudaEventSynchronize(io->stage_done[b]));  // its previous DMA has finished
  if (io->stage_bytes[b] < bytes) {
    cudaFreeHost(io->stage[b]);
    io->stage[b] = nullptr;
    io->stage_bytes[b] = 0;
    HCHK(cudaMallocHost(&io->stage[b], bytes));
    io->stage_bytes[b] = bytes;
  }
  if (!io->stage_done[b]) HCHK(cudaEventCreateWithFlags(&io->stage_done[b], cudaEventDisableTiming));
  uint8_t* st = io->stage[b];
  for (int y = 0; y < h; y++) {
    std::memcpy(st + (size_t)y * d_pitch, h_img + (size_t)y * h_pitch, (size_t)w);
    if (d_pitch > w) std::memset(st + (size_t)y * d_pitch + w, 0, (size_t)(d_pitch - w));
  }
  HCHK(cudaMemcpyAsync(d_img, st, bytes, cudaMemcpyHostToDevice, s));
  HCHK(cudaEventRecord(io->stage_done[b], s));
  return ORBX_OK;
}

ORBX_API int orbx_download_points(orbx_ctx* c, const orbx_point* d_pts, int n, orbx_point* h_pts, int fields) {
  if (!c || n < 0 || (n > 0 && (!d_pts || !h_pts)) || fields < 1 || fields > 3) return ORBX_ERR_ARG;
  if (n == 0) return ORBX_OK;
  Guard g(ctx_device(c));
  cudaStream_t s = ctx_stream(c);
  if (fields == (ORBX_FIELDS_KEYPOINT | ORBX_FIELDS_MATCH)) {
    // whole records: one contiguous copy
    HCHK(cudaMemcpyAsync(h_pts, d_pts, sizeof(orbx_point) * (size_t)n, cudaMemcpyDeviceToHost, s));
    HCHK(cudaStreamSynchronize(s));
    return ORBX_OK;
  }
  const int first = fields == ORBX_FIELDS_KEYPOINT ? 0 : 5;
  const int k = fields == ORBX_FIELDS_KEYPOINT ? 5 : 2;
  HostIO* io = hostio(c);
  const size_t need = (size_t)n * k;
  if (io->pack_ints < need) {
    cudaFree(io->pack);
    cudaFreeHost(io->pack_host);
    io->pack = nullptr;
    io->pack_host = nullptr;
    io->pack_ints = 0;
    HCHK(cudaMalloc(&io->pack, need * sizeof(int)));
    HCHK(cudaMallocHost(&io->pack_host, need * sizeof(int)));
    io->pack_ints = need;
  }
  k_pack_points<<<(unsigned)((need + 255) / 256), 256, 0, s>>>(d_pts, n, first, k, io->pack);
  HCHK(cudaGetLastError());
  HCHK(cudaMemcpyAsync(io->pack_host, io->pack, need * sizeof(int), cudaMemcpyDeviceToHost, s));
  HCHK(cudaStreamSynchronize(s));
  const int* src = io->pack_host;
  for (int i = 0; i < n; i++) std::memcpy(reinterpret_cast<int*>(h_pts + i) + first, src + (size_t)i * k, sizeof(int) * k);
  return ORBX_OK;
}
