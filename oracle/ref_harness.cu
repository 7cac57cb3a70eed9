// Test harness around the reference CUDA-ORB build (oracle A / A').
//
// THIS FILE IS TEST INFRASTRUCTURE.  It is linked with the reference's own
// orbd.cu and orb.cpp, compiled unmodified for sm_100a by oracle/Makefile into
// oracle/_ref/libref_orb.so, and is only ever called by tests/, by
// tests/golden/make_golden.py and by bench.py's reference arm.  Nothing in the
// product links or loads it.
//
// What it adds around the reference:
//  * a plain C ABI (ctypes-friendly) over orb::Orbor (orb.h:11-31) and the
//    lower orbd.h API (orbd.h:10-48);
//  * guarded allocations: every cudaMalloc made by the reference is wrapped
//    (linker --wrap) to carry 256 KiB of zeroed memory before and after the
//    block and to be zero-filled itself.  The reference reads outside its
//    buffers by design (Harris window at octave-0 row 3 reads one row before
//    omem, orbd.cu:651-669; angleIC/gDescrible read past the last octave,
//    orbd.cu:1001-1036,1437-1468; angleIC may write past max_pts,
//    orbd.cu:1004,1722).  The guards keep those accesses inside mapped,
//    deterministic (zero) memory, and zero-filling makes the first call after a
//    size change deterministic too (orb.cpp:187-188 leaves omem/vmem
//    uninitialised).
//  * a race-free variant (A'): the same pipeline driven through the lower API,
//    except that the reference's own blur kernel gConv2dUnroll
//    (orbd.cu:1273-1338) is launched out of place (source = a copy of the
//    pyramid) with the reference's own launch shape (orbd.cu:1741-1758),
//    removing the in-place cross-block race of hGassianBlur (orbd.cu:1756).
#include <cuda_runtime.h>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <mutex>
#include <unordered_map>
#include <vector>

#define private public
#include "orb.h"
#undef private
#include "orbd.h"

namespace orb {
// Defined in orbd.cu with external linkage; launched here out of place.
__global__ void gConv2dUnroll(unsigned char* src, unsigned char* dst, int width, int height, int pitch);
}

// ---------------------------------------------------------------------------
// Guarded allocations
// ---------------------------------------------------------------------------
static const size_t kGuard = 256 * 1024;
static std::mutex g_alloc_mu;
static std::unordered_map<void*, void*> g_alloc_base;

extern "C" cudaError_t __real_cudaMalloc(void** p, size_t n);
extern "C" cudaError_t __real_cudaFree(void* p);

extern "C" cudaError_t __wrap_cudaMalloc(void** p, size_t n) {
  void* base = nullptr;
  cudaError_t e = __real_cudaMalloc(&base, n + 2 * kGuard);
  if (e != cudaSuccess) return e;
  e = cudaMemset(base, 0, n + 2 * kGuard);
  if (e != cudaSuccess) return e;
  *p = (char*)base + kGuard;
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  g_alloc_base[*p] = base;
  return cudaSuccess;
}

extern "C" cudaError_t __wrap_cudaFree(void* p) {
  if (!p) return cudaSuccess;
  void* base = p;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = g_alloc_base.find(p);
    if (it != g_alloc_base.end()) {
      base = it->second;
      g_alloc_base.erase(it);
    }
  }
  return __real_cudaFree(base);
}

// ---------------------------------------------------------------------------
// State
// ---------------------------------------------------------------------------
#define RCHECK(x)                                                                   \
  do {                                                                              \
    cudaError_t _e = (x);                                                           \
    if (_e != cudaSuccess) {                                                        \
      fprintf(stderr, "ref_harness: %s failed: %s\n", #x, cudaGetErrorString(_e)); \
      return -(int)_e - 1000;                                                       \
    }                                                                               \
  } while (0)

struct Slot {
  orb::OrbData data{};
  unsigned char* d_img = nullptr;
  size_t img_bytes = 0;
  unsigned char* d_desc = nullptr;
};

static orb::Orbor* g_orb = nullptr;
static Slot g_slots[2];

__global__ void kSinCos(const float* a, float* s, float* c, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    s[i] = __sinf(a[i]);
    c[i] = __cosf(a[i]);
  }
}

static int upload(Slot& s, const unsigned char* h_img, int w, int h) {
  const int pitch = iAlignUp(w, 128);
  const size_t bytes = (size_t)h * pitch;
  if (s.img_bytes != bytes) {
    if (s.d_img) RCHECK(cudaFree(s.d_img));
    RCHECK(cudaMalloc((void**)&s.d_img, bytes));
    s.img_bytes = bytes;
  }
  RCHECK(cudaMemcpy(s.d_img, h_img, bytes, cudaMemcpyHostToDevice));
  return 0;
}

extern "C" {

int ref_init(int noctaves, int edge, int wta_k, int score_type, int patch, int fast_thr, int retain_topn,
             int max_pts) {
  RCHECK(cudaSetDevice(0));
  if (!g_orb) g_orb = new orb::Orbor();
  g_orb->init(noctaves, edge, wta_k, (orb::ScoreType)score_type, patch, fast_thr, retain_topn, max_pts);
  for (auto& s : g_slots) {
    if (s.data.d_data || s.data.h_data) g_orb->freeOrbData(s.data);
    g_orb->initOrbData(s.data, max_pts, true, true);
  }
  return 0;
}

// Layout of the current pyramid: oszp = [osizes|widths|heights|pitchs|offsets] (orb.cpp:151-156).
int ref_layout(int* n_octaves, int* oszp_out, int cap) {
  if (!g_orb) return -1;
  *n_octaves = g_orb->max_octave;
  const int n = (int)g_orb->oszp.size();
  for (int i = 0; i < n && i < cap; i++) oszp_out[i] = g_orb->oszp[i];
  return n;
}

// Stock path: Orbor::detectAndCompute (orb.cpp:57-101) on image slot `slot`.
// Outputs num_pts, the raw counter, the points (host copy, 28 B each) and descriptors.
int ref_detect(int slot, const unsigned char* h_img, int w, int h, int* num_pts, unsigned int* raw_counter,
               orb::OrbPoint* h_points, unsigned char* h_desc) {
  if (!g_orb || slot < 0 || slot > 1) return -1;
  Slot& s = g_slots[slot];
  int rc = upload(s, h_img, w, h);
  if (rc) return rc;
  int3 whp = make_int3(w, h, iAlignUp(w, 128));
  g_orb->detectAndCompute(s.d_img, s.data, whp, (void**)&s.d_desc, true);
  RCHECK(cudaDeviceSynchronize());
  *num_pts = s.data.num_pts;
  RCHECK(cudaMemcpy(raw_counter, g_orb->d_point_counter_addr, 4, cudaMemcpyDeviceToHost));
  if (s.data.num_pts > 0) {
    RCHECK(cudaMemcpy(h_points, s.data.d_data, sizeof(orb::OrbPoint) * s.data.num_pts, cudaMemcpyDeviceToHost));
    if (h_desc) RCHECK(cudaMemcpy(h_desc, s.d_desc, 32 * (size_t)s.data.num_pts, cudaMemcpyDeviceToHost));
  }
  return 0;
}

// Orbor::match (orb.cpp:104-113) of slot 0 against slot 1; writes match/distance of slot 0.
int ref_match_slots(int* h_match, int* h_dist) {
  if (!g_orb) return -1;
  Slot& a = g_slots[0];
  Slot& b = g_slots[1];
  g_orb->match(a.data, b.data, a.d_desc, b.d_desc);
  RCHECK(cudaDeviceSynchronize());
  for (int i = 0; i < a.data.num_pts; i++) {
    h_match[i] = a.data.h_data[i].match;
    h_dist[i] = a.data.h_data[i].distance;
  }
  return 0;
}

// Staged path (lower API, orbd.h) on slot 0 with intermediate dumps.
// race_free = 0 reproduces Orbor::detectAndCompute exactly; 1 blurs out of place (A').
// Buffers: pyr_raw (obytes, before blur), vmem_out (vbytes), pyr_blur (obytes),
// points (num_pts), desc (num_pts*32), sinv/cosv (num_pts).
int ref_stages(const unsigned char* h_img, int w, int h, int race_free, int* num_pts, unsigned int* raw_counter,
               unsigned char* pyr_raw, float* vmem_out, unsigned char* pyr_blur, orb::OrbPoint* h_points,
               unsigned char* h_desc, float* sinv, float* cosv, long long* sizes_out) {
  if (!g_orb) return -1;
  Slot& s = g_slots[0];
  int rc = upload(s, h_img, w, h);
  if (rc) return rc;
  orb::Orbor* o = g_orb;
  int3 whp = make_int3(w, h, iAlignUp(w, 128));
  const bool reused = (whp.x == o->width) && (whp.y == o->height);
  if ((reused && !o->omem) || !reused) {
    o->updateParam(whp);
  } else {
    RCHECK(cudaMemset(o->omem, 0, o->obytes));
    RCHECK(cudaMemset(o->vmem, 0, o->vbytes));
  }
  sizes_out[0] = (long long)o->obytes;
  sizes_out[1] = (long long)o->vbytes;
  sizes_out[2] = o->max_octave;
  o->detect(s.d_img, s.data);
  RCHECK(cudaDeviceSynchronize());
  *num_pts = s.data.num_pts;
  RCHECK(cudaMemcpy(raw_counter, o->d_point_counter_addr, 4, cudaMemcpyDeviceToHost));
  if (pyr_raw) RCHECK(cudaMemcpy(pyr_raw, o->omem, o->obytes, cudaMemcpyDeviceToHost));
  if (vmem_out) RCHECK(cudaMemcpy(vmem_out, o->vmem, o->vbytes, cudaMemcpyDeviceToHost));
  const int n = s.data.num_pts;
  if (n > 0) {
    orb::hComputeAngle(o->omem, s.data, o->oszp.data(), o->max_octave, o->patch_size);
    if (!race_free) {
      orb::hGassianBlur(o->omem, o->oszp.data(), o->max_octave);
    } else {
      unsigned char* src = nullptr;
      RCHECK(cudaMalloc((void**)&src, o->obytes));
      RCHECK(cudaMemcpy(src, o->omem, o->obytes, cudaMemcpyDeviceToDevice));
      const int no = o->max_octave;
      const int* widths = o->oszp.data() + no;
      const int* heights = widths + no;
      const int* pitchs = heights + no;
      const int* offsets = pitchs + no;
      for (int i = 0; i < no; i++) {
        dim3 block(32, 3);
        dim3 grid((widths[i] + 26 - 1) / 26, (heights[i] + 32 - 1) / 32);
        orb::gConv2dUnroll<<<grid, block>>>(src + offsets[i], o->omem + offsets[i], widths[i], heights[i],
                                            pitchs[i]);
      }
      RCHECK(cudaGetLastError());
      RCHECK(cudaDeviceSynchronize());
      RCHECK(cudaFree(src));
    }
    if (s.d_desc) RCHECK(cudaFree(s.d_desc));
    RCHECK(cudaMalloc((void**)&s.d_desc, 32 * (size_t)n));
    orb::hDescribe(o->omem, s.data, s.d_desc, o->wta_k, o->max_octave);
    RCHECK(cudaDeviceSynchronize());
    RCHECK(cudaMemcpy(h_points, s.data.d_data, sizeof(orb::OrbPoint) * n, cudaMemcpyDeviceToHost));
    if (h_desc) RCHECK(cudaMemcpy(h_desc, s.d_desc, 32 * (size_t)n, cudaMemcpyDeviceToHost));
    if (sinv && cosv) {
      float *da = nullptr, *ds = nullptr, *dc = nullptr;
      std::vector<float> ang(n);
      for (int i = 0; i < n; i++) ang[i] = h_points[i].angle;
      RCHECK(cudaMalloc((void**)&da, 4 * (size_t)n));
      RCHECK(cudaMalloc((void**)&ds, 4 * (size_t)n));
      RCHECK(cudaMalloc((void**)&dc, 4 * (size_t)n));
      RCHECK(cudaMemcpy(da, ang.data(), 4 * (size_t)n, cudaMemcpyHostToDevice));
      kSinCos<<<(n + 127) / 128, 128>>>(da, ds, dc, n);
      RCHECK(cudaGetLastError());
      RCHECK(cudaMemcpy(sinv, ds, 4 * (size_t)n, cudaMemcpyDeviceToHost));
      RCHECK(cudaMemcpy(cosv, dc, 4 * (size_t)n, cudaMemcpyDeviceToHost));
      cudaFree(da);
      cudaFree(ds);
      cudaFree(dc);
    }
  }
  if (pyr_blur) RCHECK(cudaMemcpy(pyr_blur, o->omem, o->obytes, cudaMemcpyDeviceToHost));
  return 0;
}

// __sinf/__cosf of arbitrary angles (what gDescrible uses, orbd.cu:1446-1447).
int ref_sincos(const float* angles, int n, float* sinv, float* cosv) {
  if (n <= 0) return 0;
  float *da = nullptr, *ds = nullptr, *dc = nullptr;
  RCHECK(cudaMalloc((void**)&da, 4 * (size_t)n));
  RCHECK(cudaMalloc((void**)&ds, 4 * (size_t)n));
  RCHECK(cudaMalloc((void**)&dc, 4 * (size_t)n));
  RCHECK(cudaMemcpy(da, angles, 4 * (size_t)n, cudaMemcpyHostToDevice));
  kSinCos<<<(n + 127) / 128, 128>>>(da, ds, dc, n);
  RCHECK(cudaGetLastError());
  RCHECK(cudaMemcpy(sinv, ds, 4 * (size_t)n, cudaMemcpyDeviceToHost));
  RCHECK(cudaMemcpy(cosv, dc, 4 * (size_t)n, cudaMemcpyDeviceToHost));
  cudaFree(da);
  cudaFree(ds);
  cudaFree(dc);
  return 0;
}

// hMatch (orbd.cu:1786-1793) on arbitrary descriptor sets.
int ref_hmatch(const unsigned char* h_d1, int n1, const unsigned char* h_d2, int n2, int* h_match, int* h_dist) {
  if (n1 <= 0) return 0;
  orb::OrbData r1{}, r2{};
  unsigned char *d1 = nullptr, *d2 = nullptr;
  RCHECK(cudaMalloc((void**)&r1.d_data, sizeof(orb::OrbPoint) * (size_t)n1));
  RCHECK(cudaMalloc((void**)&d1, 32 * (size_t)n1));
  RCHECK(cudaMalloc((void**)&d2, 32 * (size_t)(n2 > 0 ? n2 : 1)));
  RCHECK(cudaMemcpy(d1, h_d1, 32 * (size_t)n1, cudaMemcpyHostToDevice));
  if (n2 > 0) RCHECK(cudaMemcpy(d2, h_d2, 32 * (size_t)n2, cudaMemcpyHostToDevice));
  r1.num_pts = n1;
  r2.num_pts = n2;
  orb::hMatch(r1, r2, d1, d2);
  std::vector<orb::OrbPoint> pts(n1);
  RCHECK(cudaMemcpy(pts.data(), r1.d_data, sizeof(orb::OrbPoint) * (size_t)n1, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n1; i++) {
    h_match[i] = pts[i].match;
    h_dist[i] = pts[i].distance;
  }
  cudaFree(r1.d_data);
  cudaFree(d1);
  cudaFree(d2);
  return 0;
}

// Time `iters` pair steps through the stock Orbor API, images already on the
// device: detectAndCompute(A), detectAndCompute(B), match(A, B) -- the demo's
// protocol (main.cpp:231-251) applied to one pair per step.  Returns the mean
// milliseconds per pair measured with CUDA events around the timed loop.
int ref_time_pair(const unsigned char* hA, const unsigned char* hB, int w, int h, int warmup, int iters,
                  float* ms_per_pair, int* n_a, int* n_b) {
  if (!g_orb) return -1;
  int rc = upload(g_slots[0], hA, w, h);
  if (rc) return rc;
  rc = upload(g_slots[1], hB, w, h);
  if (rc) return rc;
  int3 whp = make_int3(w, h, iAlignUp(w, 128));
  Slot& a = g_slots[0];
  Slot& b = g_slots[1];
  for (int i = 0; i < warmup; i++) {
    g_orb->detectAndCompute(a.d_img, a.data, whp, (void**)&a.d_desc, true);
    g_orb->detectAndCompute(b.d_img, b.data, whp, (void**)&b.d_desc, true);
    g_orb->match(a.data, b.data, a.d_desc, b.d_desc);
  }
  RCHECK(cudaDeviceSynchronize());
  cudaEvent_t e0, e1;
  RCHECK(cudaEventCreate(&e0));
  RCHECK(cudaEventCreate(&e1));
  RCHECK(cudaEventRecord(e0, 0));
  for (int i = 0; i < iters; i++) {
    g_orb->detectAndCompute(a.d_img, a.data, whp, (void**)&a.d_desc, true);
    g_orb->detectAndCompute(b.d_img, b.data, whp, (void**)&b.d_desc, true);
    g_orb->match(a.data, b.data, a.d_desc, b.d_desc);
  }
  RCHECK(cudaEventRecord(e1, 0));
  RCHECK(cudaEventSynchronize(e1));
  float ms = 0.f;
  RCHECK(cudaEventElapsedTime(&ms, e0, e1));
  *ms_per_pair = ms / (float)(iters > 0 ? iters : 1);
  *n_a = a.data.num_pts;
  *n_b = b.data.num_pts;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}

// Time hMatch alone on (n1 x n2) descriptor sets resident on the device.
int ref_time_hmatch(const unsigned char* h_d1, int n1, const unsigned char* h_d2, int n2, int warmup, int iters,
                    float* ms_per_call) {
  orb::OrbData r1{}, r2{};
  unsigned char *d1 = nullptr, *d2 = nullptr;
  RCHECK(cudaMalloc((void**)&r1.d_data, sizeof(orb::OrbPoint) * (size_t)n1));
  RCHECK(cudaMalloc((void**)&d1, 32 * (size_t)n1));
  RCHECK(cudaMalloc((void**)&d2, 32 * (size_t)n2));
  RCHECK(cudaMemcpy(d1, h_d1, 32 * (size_t)n1, cudaMemcpyHostToDevice));
  RCHECK(cudaMemcpy(d2, h_d2, 32 * (size_t)n2, cudaMemcpyHostToDevice));
  r1.num_pts = n1;
  r2.num_pts = n2;
  for (int i = 0; i < warmup; i++) orb::hMatch(r1, r2, d1, d2);
  cudaEvent_t e0, e1;
  RCHECK(cudaEventCreate(&e0));
  RCHECK(cudaEventCreate(&e1));
  RCHECK(cudaEventRecord(e0, 0));
  for (int i = 0; i < iters; i++) orb::hMatch(r1, r2, d1, d2);
  RCHECK(cudaEventRecord(e1, 0));
  RCHECK(cudaEventSynchronize(e1));
  float ms = 0.f;
  RCHECK(cudaEventElapsedTime(&ms, e0, e1));
  *ms_per_call = ms / (float)(iters > 0 ? iters : 1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(r1.d_data);
  cudaFree(d1);
  cudaFree(d2);
  return 0;
}

}  // extern "C"
