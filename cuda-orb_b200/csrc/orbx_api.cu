// C ABI of the sm_100a ORB library: contexts, constant tables, workspaces,
// batch descriptors and the per-call launch sequences.
#include <cuda.h>
#include <chrono>
#include <mutex>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "orb_pattern31.h"
#include "orbx_device.cuh"
#include "orbx_internal.cuh"
#include "orbx_persist.cuh"

using namespace orbx;

namespace {

struct Workspace {
  int w = 0, h = 0, noct_req = 0, n = 0;
  int oszp[5 * kMaxOctaves + 1] = {0};
  size_t obytes = 0;
  size_t guard = 0;              // zeroed bytes before and after each pyramid
  uint8_t* pyr_alloc = nullptr;  // guard + obytes + guard
  uint8_t* blr_alloc = nullptr;
  float* vmap = nullptr;     // scores, valid where occ is set
  uint8_t* oct8 = nullptr;   // octaves, valid where occ is set
  uint32_t* occ = nullptr;   // occupancy bits
  unsigned long long* nms_status = nullptr;
  int* total = nullptr;
  int nms_strips = 0;
};

struct BatchSlot {
  Frame* d_frames = nullptr;
  int* d_bases = nullptr;  // 3 * (cap + 1)
  unsigned int* d_ticket = nullptr;
  uint8_t* h_stage = nullptr;  // pinned staging for the upload
  int cap = 0;
  cudaEvent_t uploaded = nullptr;
  std::vector<uint8_t> last;
};

struct PairGraph {
  bool valid = false;
  std::vector<uint8_t> key;
  cudaGraphExec_t exec = nullptr;
  MatchWork mw{};
};

// Device tables of one persistent launch (orbx_persist.cu), reused while
// their content is unchanged.
struct PersistBufs {
  unsigned long long* items = nullptr;  // [tickets] packed work items in claim order
  int* desc_base = nullptr;  // [frames + 1]
  int* done = nullptr;       // [4 * frames + 1 + frames]: stage counters, item counter, upload flags
  MatchJob* jobs = nullptr;
  PersistRows* rows = nullptr;  // [frames] row-counter offsets (row-level dependencies)
  size_t items_cap = 0, frames_cap = 0, jobs_cap = 0, done_cap = 0;
  size_t done_ints = 0;       // counters to clear before each launch
  std::vector<uint8_t> last;  // content of the last upload
};

static void persist_free(PersistBufs& pb) {
  cudaFree(pb.items);
  cudaFree(pb.desc_base);
  cudaFree(pb.done);
  cudaFree(pb.jobs);
  cudaFree(pb.rows);
  pb = PersistBufs();
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) {
      cudaSetDevice(dev);
    } else {
      prev = -1;
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

struct orbx_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool inited = false;
  orbx_params p{};
  float gauss[4] = {0, 0, 0, 0};
  float scale4 = 0.f;
  int half_k = 15;
  int8_t* d_pattern = nullptr;
  int* d_umax = nullptr;
  int* d_err = nullptr;
  BoundsRec* d_bounds = nullptr;  // bounds-checked build only: record of skipped accesses
  long long bounds_slack = 0;     // bytes taken off each image's checked extent (orbx_bounds_set_slack)
  Workspace ws[2];
  BatchSlot single, pair;
  MatchWork mw{};  // for orbx_match / orbx_match_knn2
  PairGraph pg;
  // int8 tensor-core matcher scratch: +-1 expanded queries / database
  int8_t* imma_q = nullptr;
  int8_t* imma_db = nullptr;
  size_t imma_q_bytes = 0, imma_db_bytes = 0;
  // orbx_pair_host device buffers
  uint8_t* io_img[2] = {nullptr, nullptr};
  size_t io_img_bytes = 0;
  orbx_point* io_pts[2] = {nullptr, nullptr};
  uint8_t* io_desc[2] = {nullptr, nullptr};
  int* io_count = nullptr;  // [2]
  int* io_count_host = nullptr;  // pinned [2]
  int io_max_pts = 0;
  cudaEvent_t prof_ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  HostIO* hostio = nullptr;  // orbx_upload_image / orbx_download_points staging
  OcvWork* ocv = nullptr;    // orbx_ocv_detect_and_compute workspace
  // launch shapes (orbx_tuning)
  int nms_rows = kNmsRows;
  int describe_bps = 4;  // one wave: 64 registers x 256 threads leave room for 4 blocks per SM
  int match_bps = 8;
  int match_blocks_per_pair = 0;
  // batched pairs
  std::vector<Workspace> bws;
  BatchSlot batch;
  MatchJob* d_jobs = nullptr;
  int jobs_cap = 0;
  uint32_t* batch_part = nullptr;
  unsigned int* batch_tile_done = nullptr;
  size_t batch_part_words = 0, batch_tile_words = 0;
  std::vector<uint8_t> batch_key;
  cudaGraphExec_t batch_exec = nullptr;
  // persistent batch form: run table, describe slices, completion counters
  int batch_form = 0;
  int persist_group = 0;
  int persist_bps = 0;
  PersistBufs pbatch;  // orbx_batch_pairs, persistent form
  PersistBufs ppair;   // orbx_pair_host with overlapped uploads
  PairGraph pho;       // its graph: persistent launch + export
  PairGraph phs;       // orbx_pair_host on two streams from pinned images: copies, kernels, match, export
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_reset = nullptr;
  int upload_bands = 0;  // orbx_pair_host: 0 = copy then run; 1..16 = bands overlapped with the persistent launch
  int pair_form = 0;     // orbx_pair: 0 = five graph-replayed launches, 1 = one persistent launch
  int pyr_shape = 0;     // pyramid tile shape of the five-launch forms (kPyrShapeTW/TH)
  int row_deps = 0;      // persistent launches: detect waits per pyramid tile row, not per frame
  int host_overlap = 1;  // orbx_pair_host: 1 = image B uploads while frame A's kernels run (two streams)
  BatchSlot pair_b;      // frame B's tables for host_overlap
  MatchWork hmw{};       // its matcher scratch
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  PairGraph ppg;         // orbx_pair's persistent graph
  int memops = -1;       // stream write-value support: -1 unknown, 0 no, 1 yes
  // device-side waits
  int wait_us = 1000000;
  long long wait_cycles = 0;
  int clock_khz = 2000000;
};

// The popcount matcher's record and row capacities (bounds-checked build; the
// normal build leaves them null and zero, and its kernels test nothing).
static void match_bounds(orbx_ctx* c, MatchArgs& a, int q_cap, int db_cap, int out_cap) {
  a.bounds = c->d_bounds;
  a.q_cap = q_cap;
  a.db_cap = db_cap;
  a.out_cap = out_cap;
}

#define ORBX_CUDA(x)                   \
  do {                                 \
    cudaError_t _e = (x);              \
    if (_e != cudaSuccess) {           \
      (void)cudaGetLastError();        \
      return _e == cudaErrorMemoryAllocation ? ORBX_ERR_NOMEM : ORBX_ERR_CUDA; \
    }                                  \
  } while (0)

static double host_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static inline int align_up(int a, int b) { return (a % b != 0) ? (a - a % b + b) : a; }
static inline int div_up(int a, int b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// Tables (Orbor::init, orb.cpp:32-54)
// ---------------------------------------------------------------------------

// setUmax (orbd.cu:66-92).
static void make_umax(int patch_size, int* umax) {
  const int half = patch_size / 2;
  umax[half + 1] = 0;
  const float v = half * sqrtf(2.f) / 2;
  const int vmax = (int)floorf(v + 1);
  const int vmin = (int)ceilf(v);
  for (int i = 0; i <= vmax; i++) umax[i] = (int)roundf(sqrtf((float)(half * half - i * i)));
  for (int i = half, v0 = 0; i >= vmin; --i) {
    while (umax[v0] == umax[v0 + 1]) ++v0;
    umax[i] = v0;
    ++v0;
  }
}

// setPattern (orbd.cu:95-410).  The 31x31 table is fixed; other patch sizes and
// WTA_K 3/4 draw from the C library's rand() with the reference's seeds, so the
// sampling points agree with a reference process on the same C library.
static int make_pattern(int patch_size, int wta_k, int8_t* out /* [512][2] */) {
  int base[512][2];
  for (int i = 0; i < 512; i++) {
    base[i][0] = kOrbPattern31[i][0];
    base[i][1] = kOrbPattern31[i][1];
  }
  if (patch_size != 31) {
    srand(0x34985739);
    for (int i = 0; i < 512; i++) {
      // the reference's offset is "- -patch_size / 2", i.e. + patch_size / 2 (orbd.cu:366-367)
      base[i][0] = rand() % patch_size + patch_size / 2;
      base[i][1] = rand() % patch_size + patch_size / 2;
    }
  }
  if (wta_k == 2) {
    for (int i = 0; i < 512; i++) {
      out[2 * i] = (int8_t)base[i][0];
      out[2 * i + 1] = (int8_t)base[i][1];
    }
    return 512;
  }
  srand(0x12345678);
  const int ntuples = 128;
  int sel[512][2];
  for (int i = 0; i < ntuples; i++) {
    for (int k = 0; k < wta_k; k++) {
      for (;;) {
        const int idx = rand() % 512;
        int k1 = 0;
        for (; k1 < k; k1++) {
          if (base[idx][0] == sel[wta_k * i + k1][0] && base[idx][1] == sel[wta_k * i + k1][1]) break;
        }
        if (k1 == k) {
          sel[wta_k * i + k][0] = base[idx][0];
          sel[wta_k * i + k][1] = base[idx][1];
          break;
        }
      }
    }
  }
  std::memset(out, 0, 1024);
  for (int i = 0; i < ntuples * wta_k; i++) {
    out[2 * i] = (int8_t)sel[i][0];
    out[2 * i + 1] = (int8_t)sel[i][1];
  }
  return ntuples * wta_k;
}

// setGaussianKernel (orbd.cu:413-433): host expf, sigma 2, normalised.
static void make_gauss(float* k) {
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

// setScaleSqSq (orbd.cu:436-441).
static float make_scale4() {
  const float scale = 1.f / (4 * 7 * 255.f);
  return scale * scale * scale * scale;
}

// Orbor::updateParam (orb.cpp:145-191).  Returns the octave count, or a negative status.
static int compute_layout(int w, int h, int noctaves, int* oszp) {
  const int m = (w < h ? w : h) / 80;
  if (m <= 0) return -ORBX_ERR_SIZE;
  int n = (int)log2f((float)m) + 1;
  if (noctaves < n) n = noctaves;
  if (n <= 0 || n > kMaxOctaves) return -ORBX_ERR_SIZE;
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

// ---------------------------------------------------------------------------
// Workspaces and batches
// ---------------------------------------------------------------------------
// Zeroed bytes kept before octave 0 and after the last octave.  The reference
// reads past octave edges by design: the Harris window one row above octave 0
// (orbd.cu:651-669), the detect halo and the sampling patterns several rows
// beyond the last octave (orbd.cu:1001-1036, 1341-1348; with the rand() pattern
// of patch sizes other than 31 up to 64 rows).  72 rows of the widest pitch
// cover every such read.
static size_t pyramid_guard(int pitch0) {
  size_t g = (size_t)72 * pitch0 + 4096;
  if (g < kGuard) g = kGuard;
  return (g + 255) & ~(size_t)255;
}

static void ws_free(Workspace& ws) {
  cudaFree(ws.pyr_alloc);
  cudaFree(ws.blr_alloc);
  cudaFree(ws.vmap);
  cudaFree(ws.oct8);
  cudaFree(ws.occ);
  cudaFree(ws.nms_status);
  cudaFree(ws.total);
  ws = Workspace();
}

static int ws_ensure(orbx_ctx* c, Workspace& ws, int w, int h, int noct_req = -1) {
  if (noct_req < 0) noct_req = c->p.noctaves;
  if (ws.pyr_alloc && ws.w == w && ws.h == h && ws.noct_req == noct_req) return ORBX_OK;
  ws_free(ws);
  const int n = compute_layout(w, h, noct_req, ws.oszp);
  if (n < 0) return -n;
  ws.n = n;
  ws.w = w;
  ws.h = h;
  ws.noct_req = noct_req;
  ws.obytes = (size_t)ws.oszp[4 * n + n];
  ws.guard = pyramid_guard(ws.oszp[3 * n]);
  const size_t alloc = ws.obytes + 2 * ws.guard;
  const size_t npx = (size_t)h * ws.oszp[3 * n];
  const int border = c->p.edge_threshold < 3 ? 3 : c->p.edge_threshold;
  ws.nms_strips = (h - 2 * border > 0 && w - 2 * border > 0) ? div_up(h - 2 * border, c->nms_rows) : 0;
  ORBX_CUDA(cudaMalloc(&ws.pyr_alloc, alloc));
  ORBX_CUDA(cudaMalloc(&ws.blr_alloc, alloc));
  ORBX_CUDA(cudaMalloc(&ws.vmap, npx * sizeof(float)));
  ORBX_CUDA(cudaMalloc(&ws.oct8, npx));
  ORBX_CUDA(cudaMalloc(&ws.occ, npx / 8));
  // look-back words for the smallest border (3) and one-row strips, so any fits
  const int strips_max = (h - 6 > 0) ? h - 6 : 1;
  ORBX_CUDA(cudaMalloc(&ws.nms_status, sizeof(unsigned long long) * strips_max));
  ORBX_CUDA(cudaMalloc(&ws.total, sizeof(int)));
  ORBX_CUDA(cudaMemsetAsync(ws.pyr_alloc, 0, alloc, c->stream));
  ORBX_CUDA(cudaMemsetAsync(ws.blr_alloc, 0, alloc, c->stream));
  ORBX_CUDA(cudaMemsetAsync(ws.vmap, 0, npx * sizeof(float), c->stream));
  ORBX_CUDA(cudaMemsetAsync(ws.oct8, 0, npx, c->stream));
  // words past the detect tiles (row padding) are never written: they stay empty
  ORBX_CUDA(cudaMemsetAsync(ws.occ, 0, npx / 8, c->stream));
  return ORBX_OK;
}

// NMS border, strip height (within the shared-memory budget of occupancy words
// per strip) and strip count of a frame.
static void set_nms_shape(Frame& F, int border, int rows_req) {
  F.border = border < 3 ? 3 : border;
  const int nw = (F.w - 2 * F.border > 0) ? ((F.w - F.border - 1) >> 5) - (F.border >> 5) + 1 : 1;
  int rows = rows_req < 1 ? 1 : rows_req;
  if (rows * nw > kNmsMaxWords) rows = kNmsMaxWords / nw > 0 ? kNmsMaxWords / nw : 1;
  F.nms_rows = rows;
  F.nms_strips = (F.h - 2 * F.border > 0 && F.w - 2 * F.border > 0) ? div_up(F.h - 2 * F.border, rows) : 0;
}

static void fill_frame(const orbx_ctx* c, const Workspace& ws, const uint8_t* img, int pitch_in, orbx_point* pts,
                       uint8_t* desc, int* count, Frame& F, int max_pts = -1, int pyr_shape = 0) {
  std::memset(&F, 0, sizeof(F));
  const int n = ws.n;
  F.img = img;
  F.w = ws.w;
  F.h = ws.h;
  F.pitch_in = pitch_in;
  F.img_bytes = std::max(0LL, (long long)ws.h * pitch_in - c->bounds_slack);
  F.n_oct = n;
  for (int o = 0; o < n; o++) {
    F.ow[o] = ws.oszp[n + o];
    F.oh[o] = ws.oszp[2 * n + o];
    F.op[o] = ws.oszp[3 * n + o];
  }
  for (int o = 0; o <= n; o++) F.ooff[o] = ws.oszp[4 * n + o];
  F.pyr = ws.pyr_alloc + ws.guard;
  F.blr = ws.blr_alloc + ws.guard;
  F.vmap = ws.vmap;
  F.oct8 = ws.oct8;
  F.occ = ws.occ;
  F.layer = nullptr;
  F.pts = pts;
  F.desc = desc;
  F.count = count;
  F.total = ws.total;
  F.max_pts = max_pts > 0 ? max_pts : c->p.max_pts;
  F.border = c->p.edge_threshold < 3 ? 3 : c->p.edge_threshold;
  int acc = 0;
  for (int o = 0; o < n; o++) {
    F.pyr_tiles_x[o] = div_up(F.ow[o], kPyrShapeTW[pyr_shape]);
    F.pyr_tiles_y[o] = div_up(F.oh[o], kPyrShapeTH[pyr_shape]);
    F.pyr_tile_base[o] = acc;
    acc += F.pyr_tiles_x[o] * F.pyr_tiles_y[o];
  }
  F.pyr_tile_base[n] = acc;
  F.pyr_shape = pyr_shape;
  F.det_tiles_x = div_up(F.w, kDetTW);
  F.det_tiles_y = div_up(F.h, kDetTH);
  set_nms_shape(F, F.border, c->nms_rows);
  F.nms_status = ws.nms_status;
}

struct LaunchPlan {
  Batch b{};
  int pyr_tiles = 0, det_tiles = 0, nms_strips = 0, total_max_pts = 0;
};

static int upload_batch(orbx_ctx* c, BatchSlot& bs, const std::vector<Frame>& frames, LaunchPlan* plan) {
  const int nf = (int)frames.size();
  if (nf <= 0 || nf > kMaxFramesPerLaunch) return ORBX_ERR_SIZE;
  std::vector<int> bases(3 * (nf + 1));
  int* pb = bases.data();
  int* db = pb + nf + 1;
  int* nb = db + nf + 1;
  pb[0] = db[0] = nb[0] = 0;
  long long tmp = 0;
  for (int f = 0; f < nf; f++) {
    const Frame& F = frames[f];
    pb[f + 1] = pb[f] + F.pyr_tile_base[F.n_oct];
    db[f + 1] = db[f] + F.det_tiles_x * F.det_tiles_y;
    nb[f + 1] = nb[f] + F.nms_strips;
    tmp += F.max_pts;
  }
  const size_t fbytes = sizeof(Frame) * nf;
  const size_t bbytes = sizeof(int) * bases.size();
  std::vector<uint8_t> blob(fbytes + bbytes);
  std::memcpy(blob.data(), frames.data(), fbytes);
  std::memcpy(blob.data() + fbytes, bases.data(), bbytes);
  if (nf > bs.cap) {
    if (bs.uploaded) cudaEventSynchronize(bs.uploaded);
    cudaFree(bs.d_frames);
    cudaFree(bs.d_bases);
    cudaFreeHost(bs.h_stage);
    bs.d_frames = nullptr;
    bs.d_bases = nullptr;
    bs.h_stage = nullptr;
    bs.last.clear();
    const int cap = nf < 4 ? 4 : nf;
    ORBX_CUDA(cudaMalloc(&bs.d_frames, sizeof(Frame) * cap));
    ORBX_CUDA(cudaMalloc(&bs.d_bases, sizeof(int) * 3 * (cap + 1)));
    ORBX_CUDA(cudaMallocHost(&bs.h_stage, sizeof(Frame) * cap + sizeof(int) * 3 * (cap + 1)));
    if (!bs.d_ticket) ORBX_CUDA(cudaMalloc(&bs.d_ticket, sizeof(unsigned int)));
    if (!bs.uploaded) ORBX_CUDA(cudaEventCreateWithFlags(&bs.uploaded, cudaEventDisableTiming));
    bs.cap = cap;
  }
  if (bs.last != blob) {
    ORBX_CUDA(cudaEventSynchronize(bs.uploaded));  // the previous upload has left the staging buffer
    std::memcpy(bs.h_stage, blob.data(), blob.size());
    ORBX_CUDA(cudaMemcpyAsync(bs.d_frames, bs.h_stage, fbytes, cudaMemcpyHostToDevice, c->stream));
    ORBX_CUDA(cudaMemcpyAsync(bs.d_bases, bs.h_stage + fbytes, bbytes, cudaMemcpyHostToDevice, c->stream));
    ORBX_CUDA(cudaEventRecord(bs.uploaded, c->stream));
    bs.last.swap(blob);
  }
  Batch& b = plan->b;
  b.frames = bs.d_frames;
  b.n_frames = nf;
  b.pyr_base = bs.d_bases;
  b.det_base = bs.d_bases + (nf + 1);
  b.nms_base = bs.d_bases + 2 * (nf + 1);
  b.nms_ticket = bs.d_ticket;
  b.err = c->d_err;
  b.bounds = c->d_bounds;
  b.wait_cycles = c->wait_cycles;
  b.pyr_shape = frames[0].pyr_shape;
  b.fast_thr = c->p.fast_threshold;
  b.harris = c->p.score_type == 0 ? 1 : 0;
  b.wta_k = c->p.wta_k;
  b.half_k = c->half_k;
  for (int i = 0; i < 4; i++) b.gauss[i] = c->gauss[i];
  b.harris_scale4 = c->scale4;
  b.pattern = c->d_pattern;
  b.umax = c->d_umax;
  b.n_inline = nf <= kInlineFrames ? nf : 0;
  for (int i = 0; i < kInlineFrames + 1; i++) {
    const bool in = b.n_inline && i <= nf;
    b.inl_pyr_base[i] = in ? pb[i] : 0;
    b.inl_det_base[i] = in ? db[i] : 0;
    b.inl_nms_base[i] = in ? nb[i] : 0;
  }
  std::memset(b.inl, 0, sizeof(b.inl));
  for (int i = 0; i < b.n_inline; i++) b.inl[i] = frames[i];
  plan->pyr_tiles = pb[nf];
  plan->det_tiles = db[nf];
  plan->nms_strips = nb[nf];
  plan->total_max_pts = (int)(tmp > (1 << 30) ? (1 << 30) : tmp);
  return ORBX_OK;
}

static int launch_frames(orbx_ctx* c, const LaunchPlan& pl, bool compute_desc, cudaStream_t s = nullptr) {
  if (!s) s = c->stream;
  ORBX_CUDA(launch_pyramid_blur(pl.b, pl.pyr_tiles, s));
  ORBX_CUDA(launch_detect(pl.b, pl.det_tiles, s));
  ORBX_CUDA(launch_nms(pl.b, pl.nms_strips, s));
  if (compute_desc) ORBX_CUDA(launch_describe(pl.b, pl.total_max_pts, s, c->describe_bps));
  return ORBX_OK;
}

static constexpr int kSplitsCap = 64;

static int mw_ensure(MatchWork& mw, int nq_cap) {
  if (mw.part && mw.nq_cap >= nq_cap) return ORBX_OK;
  cudaFree(mw.part);
  cudaFree(mw.tile_done);
  mw = MatchWork();
  const int cap = nq_cap < 128 ? 128 : nq_cap;
  ORBX_CUDA(cudaMalloc(&mw.part, sizeof(uint32_t) * 2 * (size_t)kSplitsCap * cap));
  ORBX_CUDA(cudaMalloc(&mw.tile_done, sizeof(unsigned int) * (size_t)div_up(cap, 128)));
  ORBX_CUDA(cudaMemset(mw.tile_done, 0, sizeof(unsigned int) * (size_t)div_up(cap, 128)));
  mw.nq_cap = cap;
  mw.splits_cap = kSplitsCap;
  return ORBX_OK;
}

static int check_image(const orbx_ctx* c, const uint8_t* img, int w, int h, int pitch) {
  if (!c) return ORBX_ERR_ARG;
  if (!c->inited) return ORBX_ERR_STATE;
  if (!img || w <= 0 || h <= 0 || pitch < w) return ORBX_ERR_ARG;
  if (w > 16384 || h > 16384) return ORBX_ERR_SIZE;
  return ORBX_OK;
}

// ---------------------------------------------------------------------------
// Lower-level entry points of orbd.h (orbd.cu:1564-1793) on caller-owned
// pyramid buffers.  The caller's buffers have no guard bytes, so each call
// runs on the context's guarded workspace and copies between the two.
// ---------------------------------------------------------------------------
namespace orbx {

static int lower_workspace(orbx_ctx* c, const int* oszp, int noctaves, Workspace** out) {
  if (!c || !oszp || noctaves < 1 || noctaves > kMaxOctaves) return ORBX_ERR_ARG;
  if (!c->inited) return ORBX_ERR_STATE;
  const int w = oszp[noctaves], h = oszp[2 * noctaves];
  int rc = ws_ensure(c, c->ws[0], w, h, noctaves);
  if (rc) return rc;
  Workspace& ws = c->ws[0];
  if (ws.n != noctaves || std::memcmp(ws.oszp, oszp, sizeof(int) * (5 * noctaves + 1)) != 0) return ORBX_ERR_SIZE;
  *out = &ws;
  return ORBX_OK;
}

static int lower_run(orbx_ctx* c, Workspace& ws, Frame& F, int stage, int describe_mode, int threshold, int harris,
                     int wta_k, int half_k, int n_pts) {
  std::vector<Frame> frames(1, F);
  LaunchPlan pl;
  int rc = upload_batch(c, c->single, frames, &pl);
  if (rc) return rc;
  pl.b.fast_thr = threshold;
  pl.b.harris = harris;
  pl.b.wta_k = wta_k;
  pl.b.half_k = half_k;
  pl.b.describe_mode = describe_mode;
  if (stage == 0) {
    ORBX_CUDA(launch_pyramid_blur(pl.b, pl.pyr_tiles, c->stream));
    ORBX_CUDA(launch_detect(pl.b, pl.det_tiles, c->stream));
    ORBX_CUDA(launch_nms(pl.b, pl.nms_strips, c->stream));
  } else if (stage == 1) {
    ORBX_CUDA(launch_pyramid_blur(pl.b, pl.pyr_tiles, c->stream));
  } else {
    ORBX_CUDA(launch_describe(pl.b, n_pts, c->stream));
  }
  (void)ws;
  return ORBX_OK;
}

int lower_detect(orbx_ctx* c, const uint8_t* image, uint8_t* octave_images, float* vmem, orbx_point* pts,
                 int* d_count, const int* oszp, int noctaves, int threshold, int border, bool harris) {
  Workspace* ws = nullptr;
  int rc = lower_workspace(c, oszp, noctaves, &ws);
  if (rc) return rc;
  if (!image || !pts || !d_count || threshold < 0) return ORBX_ERR_ARG;
  // above 255 no pixel can differ from its centre by more than the threshold
  threshold = std::min(threshold, 255);
  Frame F;
  fill_frame(c, *ws, image, ws->oszp[3 * noctaves], pts, nullptr, d_count, F);
  set_nms_shape(F, border, c->nms_rows);
  rc = lower_run(c, *ws, F, 0, kDescribeBoth, threshold, harris ? 1 : 0, c->p.wta_k, c->half_k, 0);
  if (rc) return rc;
  const size_t npx = (size_t)ws->h * ws->oszp[3 * noctaves];
  if (octave_images)
    ORBX_CUDA(cudaMemcpyAsync(octave_images, ws->pyr_alloc + ws->guard, ws->obytes, cudaMemcpyDeviceToDevice, c->stream));
  if (vmem)
    ORBX_CUDA(launch_expand_score_map(c->single.d_frames, vmem, reinterpret_cast<int*>(vmem + npx), (long long)npx,
                                      c->stream));
  return ORBX_OK;
}

int lower_angle(orbx_ctx* c, const uint8_t* octave_images, orbx_point* pts, int n_pts, const int* oszp,
                int noctaves, int patch_size, int* d_tmp_count) {
  Workspace* ws = nullptr;
  int rc = lower_workspace(c, oszp, noctaves, &ws);
  if (rc) return rc;
  if (n_pts <= 0) return ORBX_OK;
  if (!octave_images || !pts || patch_size / 2 != c->half_k) return ORBX_ERR_ARG;
  ORBX_CUDA(cudaMemcpyAsync(ws->pyr_alloc + ws->guard, octave_images, ws->obytes, cudaMemcpyDeviceToDevice, c->stream));
  ORBX_CUDA(cudaMemcpyAsync(d_tmp_count, &n_pts, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  Frame F;
  fill_frame(c, *ws, octave_images, ws->oszp[3 * noctaves], pts, nullptr, d_tmp_count, F);
  return lower_run(c, *ws, F, 2, kDescribeAngleOnly, c->p.fast_threshold, 1, c->p.wta_k, c->half_k, n_pts);
}

int lower_blur(orbx_ctx* c, uint8_t* octave_images, const int* oszp, int noctaves, int* d_tmp_count) {
  Workspace* ws = nullptr;
  int rc = lower_workspace(c, oszp, noctaves, &ws);
  if (rc) return rc;
  if (!octave_images) return ORBX_ERR_ARG;
  ORBX_CUDA(cudaMemcpyAsync(ws->pyr_alloc + ws->guard, octave_images, ws->obytes, cudaMemcpyDeviceToDevice, c->stream));
  Frame F;
  fill_frame(c, *ws, octave_images, ws->oszp[3 * noctaves], nullptr, nullptr, d_tmp_count, F);
  F.pyr_src = ws->pyr_alloc + ws->guard;
  rc = lower_run(c, *ws, F, 1, kDescribeBoth, c->p.fast_threshold, 1, c->p.wta_k, c->half_k, 0);
  if (rc) return rc;
  ORBX_CUDA(cudaMemcpyAsync(octave_images, ws->blr_alloc + ws->guard, ws->obytes, cudaMemcpyDeviceToDevice, c->stream));
  return ORBX_OK;
}

int lower_last_layout(orbx_ctx* c, int* oszp, int noctaves) {
  if (!c || !oszp) return ORBX_ERR_ARG;
  const Workspace& ws = c->ws[0];
  if (!ws.pyr_alloc || ws.n != noctaves) return ORBX_ERR_STATE;
  std::memcpy(oszp, ws.oszp, sizeof(int) * (5 * noctaves + 1));
  return ORBX_OK;
}

int lower_describe(orbx_ctx* c, const uint8_t* octave_images, orbx_point* pts, int n_pts, uint8_t* desc, int wta_k,
                   const int* oszp, int noctaves, int* d_tmp_count) {
  Workspace* ws = nullptr;
  int rc = lower_workspace(c, oszp, noctaves, &ws);
  if (rc) return rc;
  if (n_pts <= 0) return ORBX_OK;
  if (!octave_images || !pts || !desc || wta_k < 2 || wta_k > 4) return ORBX_ERR_ARG;
  ORBX_CUDA(cudaMemcpyAsync(ws->blr_alloc + ws->guard, octave_images, ws->obytes, cudaMemcpyDeviceToDevice, c->stream));
  ORBX_CUDA(cudaMemcpyAsync(d_tmp_count, &n_pts, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  Frame F;
  fill_frame(c, *ws, octave_images, ws->oszp[3 * noctaves], pts, desc, d_tmp_count, F);
  return lower_run(c, *ws, F, 2, kDescribeDescOnly, c->p.fast_threshold, 1, wta_k, c->half_k, n_pts);
}

}  // namespace orbx

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

ORBX_API const char* orbx_version(void) { return "orbx 0.1 (sm_100a)"; }

ORBX_API const char* orbx_status_string(int status) {
  switch (status) {
    case ORBX_OK: return "ok";
    case ORBX_ERR_ARG: return "invalid argument";
    case ORBX_ERR_CUDA: return "CUDA runtime error";
    case ORBX_ERR_SIZE: return "size out of supported range";
    case ORBX_ERR_STATE: return "context not initialised";
    case ORBX_ERR_TIMEOUT: return "device-side wait timed out";
    case ORBX_ERR_NOMEM: return "device out of memory";
    default: return "unknown status";
  }
}

ORBX_API int orbx_create(orbx_ctx** out, int device) {
  if (!out) return ORBX_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    (void)cudaGetLastError();
    return ORBX_ERR_CUDA;
  }
  DeviceGuard g(device);
  orbx_ctx* c = new orbx_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_pattern, 1024) != cudaSuccess || cudaMalloc(&c->d_umax, 32 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess || cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return ORBX_ERR_CUDA;
  }
#ifdef ORBX_BOUNDS_CHECK
  if (cudaMalloc(&c->d_bounds, sizeof(BoundsRec)) != cudaSuccess ||
      cudaMemset(c->d_bounds, 0, sizeof(BoundsRec)) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return ORBX_ERR_CUDA;
  }
#endif
  c->own_stream = true;
  int khz = 0;
  if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device) != cudaSuccess || khz <= 0) {
    (void)cudaGetLastError();
    khz = 2000000;
  }
  c->clock_khz = khz;
  c->wait_cycles = (long long)c->wait_us * khz / 1000;
  *out = c;
  return ORBX_OK;
}

ORBX_API int orbx_destroy(orbx_ctx* c) {
  if (!c) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& ws : c->ws) ws_free(ws);
  for (BatchSlot* bs : {&c->single, &c->pair}) {
    cudaFree(bs->d_frames);
    cudaFree(bs->d_bases);
    cudaFree(bs->d_ticket);
    cudaFreeHost(bs->h_stage);
    if (bs->uploaded) cudaEventDestroy(bs->uploaded);
  }
  if (c->pg.exec) cudaGraphExecDestroy(c->pg.exec);
  cudaFree(c->pg.mw.part);
  cudaFree(c->pg.mw.tile_done);
  cudaFree(c->mw.part);
  cudaFree(c->mw.tile_done);
  for (int i = 0; i < 2; i++) {
    cudaFree(c->io_img[i]);
    cudaFree(c->io_pts[i]);
    cudaFree(c->io_desc[i]);
  }
  cudaFree(c->io_count);
  cudaFreeHost(c->io_count_host);
  hostio_free(c->hostio);
  ocv_free(c->ocv);
  for (auto& e : c->prof_ev)
    if (e) cudaEventDestroy(e);
  cudaFree(c->imma_q);
  cudaFree(c->imma_db);
  for (auto& ws : c->bws) ws_free(ws);
  cudaFree(c->batch.d_frames);
  cudaFree(c->batch.d_bases);
  cudaFree(c->batch.d_ticket);
  cudaFreeHost(c->batch.h_stage);
  if (c->batch.uploaded) cudaEventDestroy(c->batch.uploaded);
  cudaFree(c->d_jobs);
  cudaFree(c->batch_part);
  cudaFree(c->batch_tile_done);
  if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
  persist_free(c->pbatch);
  persist_free(c->ppair);
  if (c->pho.exec) cudaGraphExecDestroy(c->pho.exec);
  if (c->phs.exec) cudaGraphExecDestroy(c->phs.exec);
  if (c->ppg.exec) cudaGraphExecDestroy(c->ppg.exec);
  cudaFree(c->pho.mw.part);
  cudaFree(c->pho.mw.tile_done);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  cudaFree(c->hmw.part);
  cudaFree(c->hmw.tile_done);
  cudaFree(c->pair_b.d_frames);
  cudaFree(c->pair_b.d_bases);
  cudaFree(c->pair_b.d_ticket);
  cudaFreeHost(c->pair_b.h_stage);
  if (c->pair_b.uploaded) cudaEventDestroy(c->pair_b.uploaded);
  if (c->ev_reset) cudaEventDestroy(c->ev_reset);
  cudaFree(c->d_pattern);
  cudaFree(c->d_umax);
  cudaFree(c->d_err);
  cudaFree(c->d_bounds);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
  return ORBX_OK;
}

ORBX_API int orbx_set_stream(orbx_ctx* c, void* stream) {
  if (!c) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  if (c->pg.exec) {
    cudaGraphExecDestroy(c->pg.exec);
    c->pg.exec = nullptr;
    c->pg.valid = false;
  }
  return ORBX_OK;
}

ORBX_API void* orbx_get_stream(orbx_ctx* c) { return c ? (void*)c->stream : nullptr; }

ORBX_API int orbx_bounds_checked(void) {
#ifdef ORBX_BOUNDS_CHECK
  return 1;
#else
  return 0;
#endif
}

ORBX_API int orbx_bounds_report(orbx_ctx* c, long long* out) {
  if (!c || !out) return ORBX_ERR_ARG;
  if (!c->d_bounds) return ORBX_ERR_STATE;
  DeviceGuard g(c->device);
  ORBX_CUDA(cudaStreamSynchronize(c->stream));
  if (c->copy_stream) ORBX_CUDA(cudaStreamSynchronize(c->copy_stream));
  BoundsRec r{};
  ORBX_CUDA(cudaMemcpy(&r, c->d_bounds, sizeof(r), cudaMemcpyDeviceToHost));
  ORBX_CUDA(cudaMemset(c->d_bounds, 0, sizeof(r)));
  out[0] = (long long)r.n;
  out[1] = r.site;
  out[2] = r.off;
  out[3] = r.extent;
  return ORBX_OK;
}

ORBX_API int orbx_bounds_set_slack(orbx_ctx* c, long long bytes) {
  if (!c || bytes < 0) return ORBX_ERR_ARG;
  if (!c->d_bounds) return ORBX_ERR_STATE;
  c->bounds_slack = bytes;
  return ORBX_OK;
}

ORBX_API int orbx_sync(orbx_ctx* c) {
  if (!c) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  ORBX_CUDA(cudaStreamSynchronize(c->stream));
  int err = 0;
  ORBX_CUDA(cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    ORBX_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
    return ORBX_ERR_TIMEOUT;
  }
  return ORBX_OK;
}

ORBX_API int orbx_default_params(orbx_params* p) {
  if (!p) return ORBX_ERR_ARG;
  // Orbor::init defaults (orb.h:18-19)
  p->noctaves = 5;
  p->edge_threshold = 31;
  p->wta_k = 2;
  p->score_type = 0;
  p->patch_size = 31;
  p->fast_threshold = 20;
  p->retain_topn = -1;
  p->max_pts = 1000;
  return ORBX_OK;
}

ORBX_API int orbx_init(orbx_ctx* c, const orbx_params* p) {
  if (!c || !p) return ORBX_ERR_ARG;
  if (p->wta_k < 2 || p->wta_k > 4 || (p->score_type != 0 && p->score_type != 1) || p->patch_size < 3 ||
      p->patch_size > 31 || p->max_pts < 1 || p->max_pts > (1 << 22) || p->fast_threshold < 0 ||
      p->fast_threshold > 255 || p->noctaves < 1 || p->edge_threshold < 0)
    return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  ORBX_CUDA(cudaStreamSynchronize(c->stream));
  const bool shape_change = !c->inited || c->p.noctaves != p->noctaves || c->p.edge_threshold != p->edge_threshold;
  c->p = *p;
  int8_t pat[1024];
  make_pattern(p->patch_size, p->wta_k, pat);
  int umax[32] = {0};
  make_umax(p->patch_size, umax);
  make_gauss(c->gauss);
  c->scale4 = make_scale4();
  c->half_k = p->patch_size / 2;
  ORBX_CUDA(cudaMemcpy(c->d_pattern, pat, sizeof(pat), cudaMemcpyHostToDevice));
  ORBX_CUDA(cudaMemcpy(c->d_umax, umax, sizeof(umax), cudaMemcpyHostToDevice));
  if (shape_change)
    for (auto& ws : c->ws) ws_free(ws);
  for (PairGraph* g : {&c->pg, &c->ppg, &c->pho, &c->phs}) {
    if (g->exec) {
      cudaGraphExecDestroy(g->exec);
      g->exec = nullptr;
    }
    g->valid = false;
  }
  c->single.last.clear();
  c->pair.last.clear();
  c->inited = true;
  return ORBX_OK;
}

ORBX_API int orbx_layout(int w, int h, int noctaves, int* oszp, int cap) {
  if (!oszp || w <= 0 || h <= 0 || noctaves < 1) return -ORBX_ERR_ARG;
  int buf[5 * kMaxOctaves + 1];
  const int n = compute_layout(w, h, noctaves, buf);
  if (n < 0) return n;
  if (cap < 5 * n + 1) return -ORBX_ERR_ARG;
  std::memcpy(oszp, buf, sizeof(int) * (5 * n + 1));
  return n;
}

ORBX_API int orbx_detect_and_compute(orbx_ctx* c, const uint8_t* d_image, int w, int h, int pitch,
                                     orbx_point* d_points, uint8_t* d_desc, int* d_num_pts, int compute_desc) {
  int rc = check_image(c, d_image, w, h, pitch);
  if (rc) return rc;
  if (!d_points || !d_num_pts || (compute_desc && !d_desc)) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  rc = ws_ensure(c, c->ws[0], w, h);
  if (rc) return rc;
  std::vector<Frame> frames(1);
  fill_frame(c, c->ws[0], d_image, pitch, d_points, d_desc, d_num_pts, frames[0], -1, c->pyr_shape);
  LaunchPlan pl;
  rc = upload_batch(c, c->single, frames, &pl);
  if (rc) return rc;
  return launch_frames(c, pl, compute_desc != 0);
}

static int imma_ensure(orbx_ctx* c, int nq_cap, int ndb_cap) {
  const size_t qb = (size_t)imma_rows_q(nq_cap < 1 ? 1 : nq_cap) * 256;
  const size_t db = (size_t)imma_rows_db(ndb_cap < 1 ? 1 : ndb_cap) * 256;
  if (c->imma_q_bytes < qb) {
    cudaFree(c->imma_q);
    c->imma_q = nullptr;
    c->imma_q_bytes = 0;
    ORBX_CUDA(cudaMalloc(&c->imma_q, qb));
    c->imma_q_bytes = qb;
  }
  if (c->imma_db_bytes < db) {
    cudaFree(c->imma_db);
    c->imma_db = nullptr;
    c->imma_db_bytes = 0;
    ORBX_CUDA(cudaMalloc(&c->imma_db, db));
    c->imma_db_bytes = db;
  }
  return ORBX_OK;
}

// AUTO picks the tensor-core form once the pair count pays for its expansion
// pass and fixed tile cost.
static int resolve_mode(int mode, long long nq, long long ndb) {
  if (mode == ORBX_MATCH_AUTO) return (nq * ndb >= (1ll << 24) && nq >= 128) ? ORBX_MATCH_IMMA : ORBX_MATCH_POPC;
  return mode;
}

static int launch_match(orbx_ctx* c, MatchWork& mw, const MatchArgs& a, int nq_cap, int ndb_cap, int mode) {
  mode = resolve_mode(mode, nq_cap, ndb_cap);
  if (mode != ORBX_MATCH_POPC && mode != ORBX_MATCH_IMMA) return ORBX_ERR_ARG;
  int rc = mw_ensure(mw, nq_cap);
  if (rc) return rc;
  if (mode == ORBX_MATCH_POPC) {
    ORBX_CUDA(launch_match_popc(a, mw, c->stream, c->match_bps));
    return ORBX_OK;
  }
  if ((rc = imma_ensure(c, nq_cap, ndb_cap)) != 0) return rc;
  ImmaLaunch L{};
  L.args = a;
  L.work = mw;
  L.q_pm1 = c->imma_q;
  L.db_pm1 = c->imma_db;
  L.nq_cap = nq_cap;
  L.ndb_cap = ndb_cap;
  L.splits = imma_default_splits(nq_cap);
  if (L.splits > mw.splits_cap) L.splits = mw.splits_cap;
  L.err = c->d_err;
  ORBX_CUDA(launch_match_imma(L, c->stream));
  return ORBX_OK;
}

static int match_common(orbx_ctx* c, MatchWork& mw, const MatchArgs& a, int nq_cap, int ndb_cap, int mode) {
  return launch_match(c, mw, a, nq_cap, ndb_cap, mode);
}

ORBX_API int orbx_match(orbx_ctx* c, orbx_point* d_points1, const int* d_n1, const uint8_t* d_desc1,
                        const int* d_n2, const uint8_t* d_desc2, int n1_cap, int n2_cap, int mode) {
  if (!c || !d_points1 || !d_n1 || !d_desc1 || !d_n2 || (!d_desc2 && n2_cap > 0) || n1_cap < 0 || n2_cap < 0)
    return ORBX_ERR_ARG;
  if (n2_cap > (1 << 22) - 1) return ORBX_ERR_SIZE;
  if (n1_cap == 0) return ORBX_OK;
  DeviceGuard g(c->device);
  MatchArgs a{};
  a.q = d_desc1;
  a.db = d_desc2;
  a.nq = n1_cap;
  a.ndb = n2_cap;
  a.d_nq = d_n1;
  a.d_ndb = d_n2;
  a.pts = d_points1;
  match_bounds(c, a, n1_cap, n2_cap, n1_cap);
  return match_common(c, c->mw, a, n1_cap, n2_cap, mode);
}

ORBX_API int orbx_match_knn2(orbx_ctx* c, const uint8_t* d_q, int nq, const uint8_t* d_db, int ndb,
                             uint32_t* d_dist2, int32_t* d_idx2, int mode) {
  if (!c || nq < 0 || ndb < 0 || (nq > 0 && (!d_q || !d_dist2 || !d_idx2)) || (ndb > 0 && !d_db))
    return ORBX_ERR_ARG;
  if (ndb > (1 << 22) - 1) return ORBX_ERR_SIZE;
  if (nq == 0) return ORBX_OK;
  DeviceGuard g(c->device);
  MatchArgs a{};
  a.q = d_q;
  a.db = d_db;
  a.nq = nq;
  a.ndb = ndb;
  a.dist2 = d_dist2;
  a.idx2 = d_idx2;
  match_bounds(c, a, nq, ndb, nq);
  return match_common(c, c->mw, a, nq, ndb, mode);
}

static int persist_prepare(orbx_ctx* c, PersistBufs& pb, const LaunchPlan& pl, const std::vector<Frame>& frames,
                           const std::vector<MatchJob>& jobs, int blocks_per_pair, int group, PersistArgs* out,
                           int* grid_out);

// orbx_pair as one persistent launch (orbx_persist.cu) over the pair's two
// frames: a graph of a counter reset and the launch.
static int pair_persistent(orbx_ctx* c, const LaunchPlan& pl, const std::vector<Frame>& frames,
                           const MatchArgs& m) {
  PairGraph& pg = c->ppg;
  int rc;
  if ((rc = mw_ensure(pg.mw, c->p.max_pts)) != 0) return rc;
  std::vector<MatchJob> jobs(1);
  std::memset(jobs.data(), 0, sizeof(MatchJob));
  jobs[0].args = m;
  jobs[0].work = pg.mw;
  PersistArgs a;
  int grid = 0;
  if ((rc = persist_prepare(c, c->ppair, pl, frames, jobs, 2 * 148, 0, &a, &grid)) != 0) return rc;
  std::vector<uint8_t> key(sizeof(PersistArgs) + sizeof(int) + sizeof(size_t));
  std::memcpy(key.data(), &a, sizeof(PersistArgs));
  std::memcpy(key.data() + sizeof(PersistArgs), &grid, sizeof(int));
  std::memcpy(key.data() + sizeof(PersistArgs) + sizeof(int), &c->ppair.done_ints, sizeof(size_t));
  if (!(pg.valid && pg.key == key)) {
    if (pg.exec) {
      cudaGraphExecDestroy(pg.exec);
      pg.exec = nullptr;
    }
    pg.valid = false;
    cudaGraph_t graph = nullptr;
    ORBX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaMemsetAsync(a.done, 0, sizeof(int) * c->ppair.done_ints, c->stream);
    if (le == cudaSuccess) le = launch_batch_persistent(a, grid, c->stream);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (le != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      return ORBX_ERR_CUDA;
    }
    ORBX_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&pg.exec, graph, 0);
    cudaGraphDestroy(graph);
    ORBX_CUDA(ie);
    pg.key.swap(key);
    pg.valid = true;
  }
  ORBX_CUDA(cudaGraphLaunch(pg.exec, c->stream));
  return ORBX_OK;
}

ORBX_API int orbx_pair(orbx_ctx* c, const uint8_t* d_img_a, const uint8_t* d_img_b, int w, int h, int pitch,
                       orbx_point* d_pts_a, uint8_t* d_desc_a, int* d_n_a, orbx_point* d_pts_b, uint8_t* d_desc_b,
                       int* d_n_b, int mode) {
  int rc = check_image(c, d_img_a, w, h, pitch);
  if (rc) return rc;
  if (!d_img_b || !d_pts_a || !d_desc_a || !d_n_a || !d_pts_b || !d_desc_b || !d_n_b) return ORBX_ERR_ARG;
  if (mode != ORBX_MATCH_POPC && mode != ORBX_MATCH_AUTO && mode != ORBX_MATCH_IMMA) return ORBX_ERR_ARG;
  // frame pairs hold at most max_pts keypoints each: the popcount form unless asked
  if (mode == ORBX_MATCH_AUTO) mode = ORBX_MATCH_POPC;
  DeviceGuard g(c->device);
  if ((rc = ws_ensure(c, c->ws[0], w, h)) != 0) return rc;
  if ((rc = ws_ensure(c, c->ws[1], w, h)) != 0) return rc;
  if (mode == ORBX_MATCH_IMMA && (rc = imma_ensure(c, c->p.max_pts, c->p.max_pts)) != 0) return rc;
  std::vector<Frame> frames(2);
  const int shape = (c->pair_form == 1 && mode == ORBX_MATCH_POPC) ? 0 : c->pyr_shape;
  fill_frame(c, c->ws[0], d_img_a, pitch, d_pts_a, d_desc_a, d_n_a, frames[0], -1, shape);
  fill_frame(c, c->ws[1], d_img_b, pitch, d_pts_b, d_desc_b, d_n_b, frames[1], -1, shape);
  LaunchPlan pl;
  if ((rc = upload_batch(c, c->pair, frames, &pl)) != 0) return rc;
  MatchArgs a{};
  a.q = d_desc_a;
  a.db = d_desc_b;
  a.nq = c->p.max_pts;
  a.ndb = c->p.max_pts;
  a.d_nq = d_n_a;
  a.d_ndb = d_n_b;
  a.pts = d_pts_a;
  match_bounds(c, a, c->p.max_pts, c->p.max_pts, c->p.max_pts);
  if (c->pair_form == 1 && mode == ORBX_MATCH_POPC) return pair_persistent(c, pl, frames, a);
  // graph key: launch shapes and every pointer baked into the captured launches
  std::vector<uint8_t> key(sizeof(Batch) + sizeof(MatchArgs) + sizeof(LaunchPlan) + sizeof(int));
  {
    uint8_t* k = key.data();
    std::memcpy(k, &pl.b, sizeof(Batch));
    std::memcpy(k + sizeof(Batch), &a, sizeof(MatchArgs));
    LaunchPlan pz = pl;
    std::memset(&pz.b, 0, sizeof(Batch));
    std::memcpy(k + sizeof(Batch) + sizeof(MatchArgs), &pz, sizeof(LaunchPlan));
    std::memcpy(k + sizeof(Batch) + sizeof(MatchArgs) + sizeof(LaunchPlan), &mode, sizeof(int));
  }
  PairGraph& pg = c->pg;
  if (!(pg.valid && pg.key == key)) {
    if (pg.exec) {
      cudaGraphExecDestroy(pg.exec);
      pg.exec = nullptr;
    }
    pg.valid = false;
    if ((rc = mw_ensure(pg.mw, c->p.max_pts)) != 0) return rc;
    cudaGraph_t graph = nullptr;
    ORBX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int lrc = launch_frames(c, pl, true);
    if (lrc == ORBX_OK) lrc = launch_match(c, pg.mw, a, c->p.max_pts, c->p.max_pts, mode);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (lrc != ORBX_OK) {
      if (graph) cudaGraphDestroy(graph);
      return lrc;
    }
    ORBX_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&pg.exec, graph, 0);
    cudaGraphDestroy(graph);
    ORBX_CUDA(ie);
    pg.key.swap(key);
    pg.valid = true;
  }
  ORBX_CUDA(cudaGraphLaunch(pg.exec, c->stream));
  return ORBX_OK;
}

// cuStreamWriteValue32 through the runtime's driver entry point (no link-time
// dependency on the driver library): a copy stream publishes each uploaded band.
typedef CUresult (*WriteValue32Fn)(CUstream, CUdeviceptr, cuuint32_t, unsigned int);
static WriteValue32Fn write_value32() {
  static WriteValue32Fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuStreamWriteValue32", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<WriteValue32Fn>(p);
    (void)cudaGetLastError();
  });
  return fn;
}

// Whether stream write-value operations work on this context's device: one
// write to device memory, checked after a synchronisation.
static bool memops_ok(orbx_ctx* c) {
  if (c->memops >= 0) return c->memops == 1;
  c->memops = 0;
  WriteValue32Fn wv = write_value32();
  if (!wv) return false;
  int* d = nullptr;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  int h = 0;
  if (cudaMemsetAsync(d, 0, sizeof(int), c->stream) == cudaSuccess &&
      wv((CUstream)c->stream, (CUdeviceptr)d, 7u, 0) == CUDA_SUCCESS &&
      cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, c->stream) == cudaSuccess &&
      cudaStreamSynchronize(c->stream) == cudaSuccess && h == 7)
    c->memops = 1;
  (void)cudaGetLastError();
  cudaFree(d);
  return c->memops == 1;
}

// orbx_pair_host with the uploads overlapped: the two images go up in
// `bands` row bands on a copy stream, each followed by a write of its band
// count to a device flag, while one persistent launch (orbx_persist.cu) is
// already running: a pyramid tile starts as soon as the rows it reads have
// arrived, so frame A is processed while frame B is still being copied.  The
// export kernel follows in the same graph.  Returns the mapped result block.
static int pair_host_overlap(orbx_ctx* c, const uint8_t* h_a, const uint8_t* h_b, int w, int h, int pitch,
                             bool with_desc, const uint8_t** res) {
  int rc;
  if ((rc = ws_ensure(c, c->ws[0], w, h)) != 0) return rc;
  if ((rc = ws_ensure(c, c->ws[1], w, h)) != 0) return rc;
  if (!c->copy_stream) ORBX_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  if (!c->ev_reset) ORBX_CUDA(cudaEventCreateWithFlags(&c->ev_reset, cudaEventDisableTiming));
  std::vector<Frame> frames(2);
  fill_frame(c, c->ws[0], c->io_img[0], pitch, c->io_pts[0], c->io_desc[0], c->io_count, frames[0]);
  fill_frame(c, c->ws[1], c->io_img[1], pitch, c->io_pts[1], c->io_desc[1], c->io_count + 1, frames[1]);
  LaunchPlan pl;
  if ((rc = upload_batch(c, c->pair, frames, &pl)) != 0) return rc;
  PairGraph& pg = c->pho;
  if ((rc = mw_ensure(pg.mw, c->p.max_pts)) != 0) return rc;
  std::vector<MatchJob> jobs(1);
  std::memset(jobs.data(), 0, sizeof(MatchJob));
  jobs[0].args.q = c->io_desc[0];
  jobs[0].args.db = c->io_desc[1];
  jobs[0].args.nq = c->p.max_pts;
  jobs[0].args.ndb = c->p.max_pts;
  jobs[0].args.d_nq = c->io_count;
  jobs[0].args.d_ndb = c->io_count + 1;
  jobs[0].args.pts = c->io_pts[0];
  match_bounds(c, jobs[0].args, c->p.max_pts, c->p.max_pts, c->p.max_pts);
  jobs[0].work = pg.mw;
  const int match_items = 2 * 148;
  PersistArgs a;
  int grid = 0;
  if ((rc = persist_prepare(c, c->ppair, pl, frames, jobs, match_items, 0, &a, &grid)) != 0) return rc;
  const int bands = c->upload_bands;
  const int band_rows = div_up(h, bands);
  a.upload_flags = a.done + 4 * 2 + 1;
  a.band_rows = band_rows;
  const uint8_t* map_dev = nullptr;
  if ((rc = hostio_map(c, c->p.max_pts, res, &map_dev)) != 0) return rc;
  std::vector<uint8_t> key(sizeof(PersistArgs) + 4 * sizeof(int) + sizeof(void*));
  std::memcpy(key.data(), &a, sizeof(PersistArgs));
  const int extra[4] = {grid, c->p.max_pts, with_desc ? 1 : 0, (int)c->ppair.done_ints};
  std::memcpy(key.data() + sizeof(PersistArgs), extra, sizeof(extra));
  std::memcpy(key.data() + sizeof(PersistArgs) + sizeof(extra), &map_dev, sizeof(void*));
  if (!(pg.valid && pg.key == key)) {
    if (pg.exec) {
      cudaGraphExecDestroy(pg.exec);
      pg.exec = nullptr;
    }
    pg.valid = false;
    cudaGraph_t graph = nullptr;
    ORBX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int lrc = launch_batch_persistent(a, grid, c->stream) == cudaSuccess ? ORBX_OK : ORBX_ERR_CUDA;
    if (lrc == ORBX_OK)
      lrc = hostio_export_pair(c, c->io_pts[0], c->io_pts[1], c->io_desc[0], c->io_desc[1], c->io_count,
                               c->p.max_pts, with_desc, res);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (lrc != ORBX_OK) {
      if (graph) cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      return lrc;
    }
    ORBX_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&pg.exec, graph, 0);
    cudaGraphDestroy(graph);
    ORBX_CUDA(ie);
    pg.key.swap(key);
    pg.valid = true;
  }
  // reset the counters and flags, start the launch, then feed it the bands
  ORBX_CUDA(cudaMemsetAsync(a.done, 0, sizeof(int) * c->ppair.done_ints, c->stream));
  ORBX_CUDA(cudaEventRecord(c->ev_reset, c->stream));
  ORBX_CUDA(cudaGraphLaunch(pg.exec, c->stream));
  ORBX_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_reset, 0));
  WriteValue32Fn wv = write_value32();
  const uint8_t* src[2] = {h_a, h_b};
  for (int f = 0; f < 2; f++) {
    for (int k = 0; k < bands; k++) {
      const int r0 = k * band_rows, r1 = std::min(h, r0 + band_rows);
      if (r1 > r0)
        ORBX_CUDA(cudaMemcpyAsync(c->io_img[f] + (size_t)r0 * pitch, src[f] + (size_t)r0 * pitch,
                                  (size_t)(r1 - r0) * pitch, cudaMemcpyHostToDevice, c->copy_stream));
      if (wv((CUstream)c->copy_stream, (CUdeviceptr)(a.upload_flags + f), (cuuint32_t)(k + 1), 0) != CUDA_SUCCESS)
        return ORBX_ERR_CUDA;
    }
  }
  return ORBX_OK;
}

static bool host_pinned(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// The work of pair_host_streams from the fork on: the copies, both frames'
// kernels on their streams, the join, matching and the export.  ev_uploaded
// (profiling) is recorded after the copies; under capture as an external
// event node, so that each replay records it.
static int pair_host_streams_enqueue(orbx_ctx* c, const uint8_t* h_a, const uint8_t* h_b, size_t ibytes,
                                     const LaunchPlan& pa, const LaunchPlan& pb, const MatchArgs& m, bool with_desc,
                                     const uint8_t** res, cudaEvent_t ev_uploaded, bool capturing) {
  int rc;
  // fork: the copy stream starts after everything queued before this call
  ORBX_CUDA(cudaEventRecord(c->ev_fork, c->stream));
  ORBX_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_fork, 0));
  ORBX_CUDA(cudaMemcpyAsync(c->io_img[0], h_a, ibytes, cudaMemcpyHostToDevice, c->stream));
  ORBX_CUDA(cudaMemcpyAsync(c->io_img[1], h_b, ibytes, cudaMemcpyHostToDevice, c->copy_stream));
  if (ev_uploaded)
    ORBX_CUDA(capturing ? cudaEventRecordWithFlags(ev_uploaded, c->copy_stream, cudaEventRecordExternal)
                        : cudaEventRecord(ev_uploaded, c->copy_stream));
  if ((rc = launch_frames(c, pa, true, c->stream)) != 0) return rc;
  if ((rc = launch_frames(c, pb, true, c->copy_stream)) != 0) return rc;
  ORBX_CUDA(cudaEventRecord(c->ev_join, c->copy_stream));
  ORBX_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  ORBX_CUDA(launch_match_popc(m, c->hmw, c->stream, c->match_bps));
  return hostio_export_pair(c, c->io_pts[0], c->io_pts[1], c->io_desc[0], c->io_desc[1], c->io_count,
                            c->p.max_pts, with_desc, res);
}

// orbx_pair_host with the two frames on two streams: image A is copied and
// processed on the context's stream while image B is copied, then processed,
// on the copy stream; matching and the export follow on the context's stream
// once both are done.  The same five kernels per frame as orbx_pair.  When
// both images are in pinned memory the sequence is captured once into a CUDA
// graph (keyed on the images' addresses and every launch parameter) and
// replayed, which removes the gaps between ten separately issued launches.
static int pair_host_streams(orbx_ctx* c, const uint8_t* h_a, const uint8_t* h_b, int w, int h, int pitch,
                             bool with_desc, const uint8_t** res, cudaEvent_t ev_uploaded = nullptr) {
  int rc;
  if ((rc = ws_ensure(c, c->ws[0], w, h)) != 0) return rc;
  if ((rc = ws_ensure(c, c->ws[1], w, h)) != 0) return rc;
  if (!c->copy_stream) ORBX_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  if (!c->ev_fork) ORBX_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  if (!c->ev_join) ORBX_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  std::vector<Frame> fa(1), fb(1);
  fill_frame(c, c->ws[0], c->io_img[0], pitch, c->io_pts[0], c->io_desc[0], c->io_count, fa[0], -1, c->pyr_shape);
  fill_frame(c, c->ws[1], c->io_img[1], pitch, c->io_pts[1], c->io_desc[1], c->io_count + 1, fb[0], -1,
             c->pyr_shape);
  LaunchPlan pa, pb;
  if ((rc = upload_batch(c, c->pair, fa, &pa)) != 0) return rc;
  if ((rc = upload_batch(c, c->pair_b, fb, &pb)) != 0) return rc;
  if ((rc = mw_ensure(c->hmw, c->p.max_pts)) != 0) return rc;
  const size_t ibytes = (size_t)h * pitch;
  MatchArgs m{};
  m.q = c->io_desc[0];
  m.db = c->io_desc[1];
  m.nq = c->p.max_pts;
  m.ndb = c->p.max_pts;
  m.d_nq = c->io_count;
  m.d_ndb = c->io_count + 1;
  m.pts = c->io_pts[0];
  match_bounds(c, m, c->p.max_pts, c->p.max_pts, c->p.max_pts);
  if (!host_pinned(h_a) || !host_pinned(h_b))
    return pair_host_streams_enqueue(c, h_a, h_b, ibytes, pa, pb, m, with_desc, res, ev_uploaded, false);
  const uint8_t* map_dev = nullptr;
  if ((rc = hostio_map(c, c->p.max_pts, res, &map_dev)) != 0) return rc;
  PairGraph& g = c->phs;
  const void* ptrs[5] = {h_a, h_b, map_dev, c->hmw.part, ev_uploaded};
  const long long extra[4] = {(long long)ibytes, with_desc ? 1 : 0, c->match_bps, c->describe_bps};
  std::vector<uint8_t> key(2 * sizeof(Batch) + 6 * sizeof(int) + sizeof(MatchArgs) + sizeof(ptrs) + sizeof(extra));
  {
    uint8_t* k = key.data();
    const int shapes[6] = {pa.pyr_tiles, pa.det_tiles, pa.nms_strips, pb.pyr_tiles, pb.det_tiles, pb.nms_strips};
    std::memcpy(k, &pa.b, sizeof(Batch));
    k += sizeof(Batch);
    std::memcpy(k, &pb.b, sizeof(Batch));
    k += sizeof(Batch);
    std::memcpy(k, shapes, sizeof(shapes));
    k += sizeof(shapes);
    std::memcpy(k, &m, sizeof(MatchArgs));
    k += sizeof(MatchArgs);
    std::memcpy(k, ptrs, sizeof(ptrs));
    k += sizeof(ptrs);
    std::memcpy(k, extra, sizeof(extra));
  }
  if (!(g.valid && g.key == key)) {
    if (g.exec) {
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
    g.valid = false;
    cudaGraph_t graph = nullptr;
    ORBX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int lrc = pair_host_streams_enqueue(c, h_a, h_b, ibytes, pa, pb, m, with_desc, res, ev_uploaded, true);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (lrc != ORBX_OK || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      return lrc != ORBX_OK ? lrc : ORBX_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    ORBX_CUDA(ie);
    g.key.swap(key);
    g.valid = true;
  }
  ORBX_CUDA(cudaGraphLaunch(g.exec, c->stream));
  return ORBX_OK;
}

// orbx_pair_host; with `prof`, CUDA events and host clocks between the phases.
struct PairHostProf {
  cudaEvent_t ev[4];  // start, uploads done, kernels done, export done
  double t_enqueued = 0, t_synced = 0;
};

static int pair_host_impl(orbx_ctx* c, const uint8_t* h_img_a, const uint8_t* h_img_b, int w, int h, int pitch,
                          orbx_point* h_pts_a, int* h_n_a, orbx_point* h_pts_b, int* h_n_b, uint8_t* h_desc_a,
                          uint8_t* h_desc_b, int mode, PairHostProf* prof) {
  int rc = check_image(c, h_img_a, w, h, pitch);
  if (rc) return rc;
  if (!h_img_b || !h_pts_a || !h_n_a || !h_pts_b || !h_n_b) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  const size_t ibytes = (size_t)h * pitch;
  if (c->io_img_bytes < ibytes) {
    for (auto& p : c->io_img) {
      cudaFree(p);
      p = nullptr;
    }
    c->io_img_bytes = 0;
    for (auto& p : c->io_img) ORBX_CUDA(cudaMalloc(&p, ibytes));
    c->io_img_bytes = ibytes;
  }
  if (c->io_max_pts < c->p.max_pts) {
    for (int i = 0; i < 2; i++) {
      cudaFree(c->io_pts[i]);
      cudaFree(c->io_desc[i]);
      c->io_pts[i] = nullptr;
      c->io_desc[i] = nullptr;
    }
    c->io_max_pts = 0;
    for (int i = 0; i < 2; i++) {
      ORBX_CUDA(cudaMalloc(&c->io_pts[i], sizeof(orbx_point) * (size_t)c->p.max_pts));
      ORBX_CUDA(cudaMalloc(&c->io_desc[i], (size_t)32 * c->p.max_pts));
    }
    if (!c->io_count) ORBX_CUDA(cudaMalloc(&c->io_count, 2 * sizeof(int)));
    if (!c->io_count_host) ORBX_CUDA(cudaMallocHost(&c->io_count_host, 2 * sizeof(int)));
    c->io_max_pts = c->p.max_pts;
  }
  const uint8_t* res = nullptr;
  const bool with_desc = h_desc_a || h_desc_b;
  if (prof) ORBX_CUDA(cudaEventRecord(prof->ev[0], c->stream));
  if (c->host_overlap == 1 && c->upload_bands == 0 && mode != ORBX_MATCH_IMMA) {
    rc = pair_host_streams(c, h_img_a, h_img_b, w, h, pitch, with_desc, &res, prof ? prof->ev[1] : nullptr);
    if (rc) {
      cudaStreamSynchronize(c->copy_stream);
      cudaStreamSynchronize(c->stream);
      return rc;
    }
    if (prof) {
      ORBX_CUDA(cudaEventRecord(prof->ev[2], c->stream));
      ORBX_CUDA(cudaEventRecord(prof->ev[3], c->stream));
      prof->t_enqueued = host_seconds();
    }
    ORBX_CUDA(cudaStreamSynchronize(c->stream));
  } else if (c->upload_bands > 0 && mode != ORBX_MATCH_IMMA && memops_ok(c)) {
    rc = pair_host_overlap(c, h_img_a, h_img_b, w, h, pitch, with_desc, &res);
    if (rc) {
      cudaStreamSynchronize(c->copy_stream);
      cudaStreamSynchronize(c->stream);
      return rc;
    }
    if (prof) {
      // the uploads end on the copy stream; kernels and export are one graph
      ORBX_CUDA(cudaEventRecord(prof->ev[1], c->copy_stream));
      ORBX_CUDA(cudaEventRecord(prof->ev[2], c->stream));
      ORBX_CUDA(cudaEventRecord(prof->ev[3], c->stream));
      prof->t_enqueued = host_seconds();
    }
    ORBX_CUDA(cudaStreamSynchronize(c->stream));
    ORBX_CUDA(cudaStreamSynchronize(c->copy_stream));
  } else {
    ORBX_CUDA(cudaMemcpyAsync(c->io_img[0], h_img_a, ibytes, cudaMemcpyHostToDevice, c->stream));
    ORBX_CUDA(cudaMemcpyAsync(c->io_img[1], h_img_b, ibytes, cudaMemcpyHostToDevice, c->stream));
    if (prof) ORBX_CUDA(cudaEventRecord(prof->ev[1], c->stream));
    rc = orbx_pair(c, c->io_img[0], c->io_img[1], w, h, pitch, c->io_pts[0], c->io_desc[0], c->io_count,
                   c->io_pts[1], c->io_desc[1], c->io_count + 1, mode);
    if (rc) return rc;
    if (prof) ORBX_CUDA(cudaEventRecord(prof->ev[2], c->stream));
    // one export kernel writes counts, the error word, keypoints (and
    // descriptors) into mapped pinned memory, so the host waits once and
    // copies only what was found
    if ((rc = hostio_export_pair(c, c->io_pts[0], c->io_pts[1], c->io_desc[0], c->io_desc[1], c->io_count,
                                 c->p.max_pts, with_desc, &res)) != 0)
      return rc;
    if (prof) {
      ORBX_CUDA(cudaEventRecord(prof->ev[3], c->stream));
      prof->t_enqueued = host_seconds();
    }
    ORBX_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (prof) prof->t_synced = host_seconds();
  if (reinterpret_cast<const int*>(res)[2]) return ORBX_ERR_TIMEOUT;  // a bounded wait gave up
  const int na = reinterpret_cast<const int*>(res)[0], nb = reinterpret_cast<const int*>(res)[1];
  *h_n_a = na;
  *h_n_b = nb;
  const size_t mp = (size_t)c->p.max_pts;
  const uint8_t* pts = res + 16;
  const uint8_t* desc = pts + 2 * mp * sizeof(orbx_point);
  std::memcpy(h_pts_a, pts, sizeof(orbx_point) * (size_t)na);
  std::memcpy(h_pts_b, pts + mp * sizeof(orbx_point), sizeof(orbx_point) * (size_t)nb);
  if (h_desc_a) std::memcpy(h_desc_a, desc, (size_t)32 * na);
  if (h_desc_b) std::memcpy(h_desc_b, desc + mp * 32, (size_t)32 * nb);
  return ORBX_OK;
}

ORBX_API int orbx_pair_host(orbx_ctx* c, const uint8_t* h_img_a, const uint8_t* h_img_b, int w, int h, int pitch,
                            orbx_point* h_pts_a, int* h_n_a, orbx_point* h_pts_b, int* h_n_b, uint8_t* h_desc_a,
                            uint8_t* h_desc_b, int mode) {
  return pair_host_impl(c, h_img_a, h_img_b, w, h, pitch, h_pts_a, h_n_a, h_pts_b, h_n_b, h_desc_a, h_desc_b, mode,
                        nullptr);
}

ORBX_API int orbx_profile_pair_host(orbx_ctx* c, const uint8_t* h_img_a, const uint8_t* h_img_b, int w, int h,
                                    int pitch, orbx_point* h_pts_a, int* h_n_a, orbx_point* h_pts_b, int* h_n_b,
                                    uint8_t* h_desc_a, uint8_t* h_desc_b, int mode, float* phase_ms) {
  if (!c || !phase_ms) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  PairHostProf prof;
  for (auto& e : prof.ev) ORBX_CUDA(cudaEventCreate(&e));
  const double t0 = host_seconds();
  const int rc = pair_host_impl(c, h_img_a, h_img_b, w, h, pitch, h_pts_a, h_n_a, h_pts_b, h_n_b, h_desc_a, h_desc_b,
                                mode, &prof);
  const double t1 = host_seconds();
  if (rc == ORBX_OK) {
    for (int i = 0; i < 3; i++) cudaEventElapsedTime(&phase_ms[i], prof.ev[0], prof.ev[i + 1]);
    phase_ms[3] = (float)(1e3 * (prof.t_enqueued - t0));
    phase_ms[4] = (float)(1e3 * (prof.t_synced - prof.t_enqueued));
    phase_ms[5] = (float)(1e3 * (t1 - prof.t_synced));
    phase_ms[6] = (float)(1e3 * (t1 - t0));
  }
  for (auto& e : prof.ev) cudaEventDestroy(e);
  return rc;
}

ORBX_API int orbx_profile_pair(orbx_ctx* c, const uint8_t* d_img_a, const uint8_t* d_img_b, int w, int h, int pitch,
                               orbx_point* d_pts_a, uint8_t* d_desc_a, int* d_n_a, orbx_point* d_pts_b,
                               uint8_t* d_desc_b, int* d_n_b, int mode, float* stage_ms) {
  int rc = check_image(c, d_img_a, w, h, pitch);
  if (rc) return rc;
  if (!d_img_b || !d_pts_a || !d_desc_a || !d_n_a || !d_pts_b || !d_desc_b || !d_n_b || !stage_ms)
    return ORBX_ERR_ARG;
  if (mode != ORBX_MATCH_POPC && mode != ORBX_MATCH_AUTO) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  if ((rc = ws_ensure(c, c->ws[0], w, h)) != 0) return rc;
  if ((rc = ws_ensure(c, c->ws[1], w, h)) != 0) return rc;
  std::vector<Frame> frames(2);
  fill_frame(c, c->ws[0], d_img_a, pitch, d_pts_a, d_desc_a, d_n_a, frames[0], -1, c->pyr_shape);
  fill_frame(c, c->ws[1], d_img_b, pitch, d_pts_b, d_desc_b, d_n_b, frames[1], -1, c->pyr_shape);
  LaunchPlan pl;
  if ((rc = upload_batch(c, c->pair, frames, &pl)) != 0) return rc;
  if ((rc = mw_ensure(c->mw, c->p.max_pts)) != 0) return rc;
  for (auto& e : c->prof_ev)
    if (!e) ORBX_CUDA(cudaEventCreate(&e));
  MatchArgs a{};
  a.q = d_desc_a;
  a.db = d_desc_b;
  a.nq = c->p.max_pts;
  a.ndb = c->p.max_pts;
  a.d_nq = d_n_a;
  a.d_ndb = d_n_b;
  a.pts = d_pts_a;
  match_bounds(c, a, c->p.max_pts, c->p.max_pts, c->p.max_pts);
  ORBX_CUDA(cudaEventRecord(c->prof_ev[0], c->stream));
  ORBX_CUDA(launch_pyramid_blur(pl.b, pl.pyr_tiles, c->stream));
  ORBX_CUDA(cudaEventRecord(c->prof_ev[1], c->stream));
  ORBX_CUDA(launch_detect(pl.b, pl.det_tiles, c->stream));
  ORBX_CUDA(cudaEventRecord(c->prof_ev[2], c->stream));
  ORBX_CUDA(launch_nms(pl.b, pl.nms_strips, c->stream));
  ORBX_CUDA(cudaEventRecord(c->prof_ev[3], c->stream));
  ORBX_CUDA(launch_describe(pl.b, pl.total_max_pts, c->stream, c->describe_bps));
  ORBX_CUDA(cudaEventRecord(c->prof_ev[4], c->stream));
  ORBX_CUDA(launch_match_popc(a, c->mw, c->stream, c->match_bps));
  ORBX_CUDA(cudaEventRecord(c->prof_ev[5], c->stream));
  ORBX_CUDA(cudaEventSynchronize(c->prof_ev[5]));
  for (int i = 0; i < 5; i++) ORBX_CUDA(cudaEventElapsedTime(&stage_ms[i], c->prof_ev[i], c->prof_ev[i + 1]));
  return ORBX_OK;
}

ORBX_API int orbx_get_tuning(orbx_ctx* c, orbx_tuning* t) {
  if (!c || !t) return ORBX_ERR_ARG;
  t->nms_rows = c->nms_rows;
  t->describe_blocks_per_sm = c->describe_bps;
  t->match_blocks_per_sm = c->match_bps;
  t->match_blocks_per_pair = c->match_blocks_per_pair;
  t->batch_form = c->batch_form;
  t->persist_group = c->persist_group;
  t->persist_blocks_per_sm = c->persist_bps;
  t->wait_timeout_us = c->wait_us;
  t->upload_bands = c->upload_bands;
  t->pair_form = c->pair_form;
  t->pyr_tile = c->pyr_shape;
  t->persist_row_deps = c->row_deps;
  t->host_overlap = c->host_overlap;
  return ORBX_OK;
}

ORBX_API int orbx_set_tuning(orbx_ctx* c, const orbx_tuning* t) {
  if (!c || !t) return ORBX_ERR_ARG;
  if (t->nms_rows < 1 || t->nms_rows > kNmsMaxRows || t->describe_blocks_per_sm < 1 ||
      t->describe_blocks_per_sm > 64 || t->match_blocks_per_sm < 1 || t->match_blocks_per_sm > 64 ||
      t->match_blocks_per_pair < 0 || t->match_blocks_per_pair > 4096 || t->batch_form < 0 || t->batch_form > 1 ||
      t->persist_group < 0 || t->persist_group > kMaxFramesPerLaunch || t->persist_blocks_per_sm < 0 ||
      t->persist_blocks_per_sm > 32 || t->wait_timeout_us < 1 || t->wait_timeout_us > 10000000 ||
      t->upload_bands < 0 || t->upload_bands > 16 || t->pair_form < 0 || t->pair_form > 1 ||
      t->pyr_tile < 0 || t->pyr_tile >= kPyrShapes || t->persist_row_deps < 0 || t->persist_row_deps > 1 ||
      t->host_overlap < 0 || t->host_overlap > 1)
    return ORBX_ERR_ARG;
  c->nms_rows = t->nms_rows;
  c->describe_bps = t->describe_blocks_per_sm;
  c->match_bps = t->match_blocks_per_sm;
  c->match_blocks_per_pair = t->match_blocks_per_pair;
  c->batch_form = t->batch_form;
  c->persist_group = t->persist_group;
  c->persist_bps = t->persist_blocks_per_sm;
  c->wait_us = t->wait_timeout_us;
  c->upload_bands = t->upload_bands;
  c->pair_form = t->pair_form;
  c->pyr_shape = t->pyr_tile;
  c->row_deps = t->persist_row_deps;
  c->host_overlap = t->host_overlap;
  c->wait_cycles = (long long)c->wait_us * c->clock_khz / 1000;
  if (c->batch_exec) {
    cudaGraphExecDestroy(c->batch_exec);
    c->batch_exec = nullptr;
  }
  c->batch_key.clear();
  // cached graphs baked in the old shapes
  for (PairGraph* g : {&c->pg, &c->ppg, &c->pho, &c->phs}) {
    if (g->exec) {
      cudaGraphExecDestroy(g->exec);
      g->exec = nullptr;
    }
    g->valid = false;
  }
  c->single.last.clear();
  c->pair.last.clear();
  return ORBX_OK;
}

static constexpr int kBatchSplitsCap = 16;

// Builds the run table of a persistent launch over `frames` (orbx_persist.cu),
// uploads the tables to `pb` when their content changed, and fills the launch
// arguments and grid.  Uploads are synchronous (they happen only when a batch
// layout is new).
static int persist_prepare(orbx_ctx* c, PersistBufs& pb, const LaunchPlan& pl, const std::vector<Frame>& frames,
                           const std::vector<MatchJob>& jobs, int blocks_per_pair, int group, PersistArgs* out,
                           int* grid_out) {
  const int nf = (int)frames.size();
  const int n_pairs = (int)jobs.size();
  std::vector<int> pyr_n(nf), det_n(nf), nms_n(nf), desc_n(nf), desc_base(nf + 1, 0);
  for (int f = 0; f < nf; f++) {
    const Frame& F = frames[f];
    pyr_n[f] = F.pyr_tile_base[F.n_oct];
    det_n[f] = F.det_tiles_x * F.det_tiles_y;
    nms_n[f] = F.nms_strips;
    desc_n[f] = std::max(1, std::min(div_up(F.w * F.h, kDescSlicePixels), div_up(F.max_pts, 8)));
    desc_base[f + 1] = desc_base[f] + desc_n[f];
  }
  std::vector<PersistRun> runs;
  std::vector<int> run_base;
  std::vector<PersistRows> rows;
  int n_rows = 0;
  if (c->row_deps)
    n_rows = build_persist_runs_rows(frames, desc_n.data(), blocks_per_pair, &runs, &run_base, &rows);
  else
    build_persist_runs(nf, group > 0 ? group : nf, pyr_n.data(), det_n.data(), nms_n.data(), desc_n.data(),
                       blocks_per_pair, &runs, &run_base);
  // counters: [4 x frames] stage counters, the item counter, [frames] upload flags, row counters
  const size_t done_ints = 5 * (size_t)nf + 1 + (size_t)n_rows;
  // one packed item per ticket: a claim decodes its item with one load
  std::vector<unsigned long long> items((size_t)run_base.back());
  for (size_t r = 0; r < runs.size(); r++)
    for (int t = run_base[r]; t < run_base[r + 1]; t++)
      items[t] = persist_item(runs[r].stage, runs[r].frame, runs[r].first + (t - run_base[r]));
  const int bps_max = persist_blocks_per_sm(c->p.wta_k);
  if (bps_max <= 0) return ORBX_ERR_CUDA;
  const int bps = c->persist_bps > 0 ? std::min(c->persist_bps, bps_max) : bps_max;
  int nsm = 0;
  ORBX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  *grid_out = bps * nsm;
  std::vector<uint8_t> blob(sizeof(unsigned long long) * items.size() + sizeof(int) * (nf + 1) +
                            sizeof(MatchJob) * n_pairs + sizeof(PersistRows) * rows.size() + sizeof(size_t));
  {
    uint8_t* q = blob.data();
    std::memcpy(q, &done_ints, sizeof(size_t));
    q += sizeof(size_t);
    if (!rows.empty()) std::memcpy(q, rows.data(), sizeof(PersistRows) * rows.size());
    q += sizeof(PersistRows) * rows.size();
    std::memcpy(q, items.data(), sizeof(unsigned long long) * items.size());
    q += sizeof(unsigned long long) * items.size();
    std::memcpy(q, desc_base.data(), sizeof(int) * (nf + 1));
    q += sizeof(int) * (nf + 1);
    std::memcpy(q, jobs.data(), sizeof(MatchJob) * n_pairs);
  }
  if (pb.last != blob) {
    ORBX_CUDA(cudaStreamSynchronize(c->stream));
    if (pb.items_cap < items.size()) {
      cudaFree(pb.items);
      pb.items = nullptr;
      pb.items_cap = 0;
      ORBX_CUDA(cudaMalloc(&pb.items, sizeof(unsigned long long) * items.size()));
      pb.items_cap = items.size();
    }
    if (pb.frames_cap < (size_t)nf) {
      cudaFree(pb.desc_base);
      cudaFree(pb.rows);
      pb.desc_base = nullptr;
      pb.rows = nullptr;
      pb.frames_cap = 0;
      ORBX_CUDA(cudaMalloc(&pb.desc_base, sizeof(int) * (nf + 1)));
      ORBX_CUDA(cudaMalloc(&pb.rows, sizeof(PersistRows) * nf));
      pb.frames_cap = nf;
    }
    if (pb.done_cap < done_ints) {
      cudaFree(pb.done);
      pb.done = nullptr;
      pb.done_cap = 0;
      ORBX_CUDA(cudaMalloc(&pb.done, sizeof(int) * done_ints));
      pb.done_cap = done_ints;
    }
    if (!rows.empty())
      ORBX_CUDA(cudaMemcpy(pb.rows, rows.data(), sizeof(PersistRows) * nf, cudaMemcpyHostToDevice));
    if (pb.jobs_cap < (size_t)n_pairs) {
      cudaFree(pb.jobs);
      pb.jobs = nullptr;
      pb.jobs_cap = 0;
      ORBX_CUDA(cudaMalloc(&pb.jobs, sizeof(MatchJob) * n_pairs));
      pb.jobs_cap = n_pairs;
    }
    ORBX_CUDA(cudaMemcpy(pb.items, items.data(), sizeof(unsigned long long) * items.size(),
                         cudaMemcpyHostToDevice));
    ORBX_CUDA(cudaMemcpy(pb.desc_base, desc_base.data(), sizeof(int) * (nf + 1), cudaMemcpyHostToDevice));
    ORBX_CUDA(cudaMemcpy(pb.jobs, jobs.data(), sizeof(MatchJob) * n_pairs, cudaMemcpyHostToDevice));
    pb.last.swap(blob);
  }
  PersistArgs& a = *out;
  a = PersistArgs{};
  a.b = pl.b;
  a.items = pb.items;
  a.run_base_host_total = run_base.back();
  a.desc_base = pb.desc_base;
  a.done = pb.done;
  a.item_counter = reinterpret_cast<unsigned int*>(pb.done + 4 * (size_t)nf);
  a.jobs = pb.jobs;
  a.blocks_per_job = blocks_per_pair;
  if (n_rows > 0) {
    a.rows = pb.rows;
    a.rows_done = pb.done + 5 * (size_t)nf + 1;
  }
  pb.done_ints = done_ints;
  return ORBX_OK;
}

// The persistent form of orbx_batch_pairs: a graph of one counter reset and
// one persistent launch.
static int batch_persistent(orbx_ctx* c, const LaunchPlan& pl, const std::vector<Frame>& frames,
                            const std::vector<MatchJob>& jobs, int blocks_per_pair, std::vector<uint8_t>& key) {
  const int nf = (int)frames.size();
  PersistArgs a;
  int grid = 0;
  int rc = persist_prepare(c, c->pbatch, pl, frames, jobs, blocks_per_pair, c->persist_group, &a, &grid);
  if (rc) return rc;
  {
    const int extra[4] = {1, c->persist_group, grid, (int)c->pbatch.done_ints};
    const size_t k0 = key.size();
    key.resize(k0 + sizeof(extra) + sizeof(void*));
    std::memcpy(key.data() + k0, extra, sizeof(extra));
    std::memcpy(key.data() + k0 + sizeof(extra), &a.done, sizeof(void*));
  }
  if (!(c->batch_exec && c->batch_key == key)) {
    if (c->batch_exec) {
      cudaGraphExecDestroy(c->batch_exec);
      c->batch_exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    ORBX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaMemsetAsync(a.done, 0, sizeof(int) * c->pbatch.done_ints, c->stream);
    if (le == cudaSuccess) le = launch_batch_persistent(a, grid, c->stream);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (le != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      return ORBX_ERR_CUDA;
    }
    ORBX_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&c->batch_exec, graph, 0);
    cudaGraphDestroy(graph);
    ORBX_CUDA(ie);
    c->batch_key.swap(key);
  }
  ORBX_CUDA(cudaGraphLaunch(c->batch_exec, c->stream));
  return ORBX_OK;
}

static int batch_pairs_impl(orbx_ctx* c, int n_pairs, const orbx_image* ia, const orbx_image* ib,
                            const orbx_frame_out* oa, const orbx_frame_out* ob, int mode, float* stage_ms) {
  if (!c || n_pairs < 0 || (n_pairs > 0 && (!ia || !ib || !oa || !ob))) return ORBX_ERR_ARG;
  if (!c->inited) return ORBX_ERR_STATE;
  if (n_pairs == 0) return ORBX_OK;
  if (2 * n_pairs > kMaxFramesPerLaunch) return ORBX_ERR_SIZE;
  if (mode != ORBX_MATCH_POPC && mode != ORBX_MATCH_AUTO) return ORBX_ERR_ARG;
  int rc;
  for (int i = 0; i < n_pairs; i++) {
    for (const orbx_image* im : {&ia[i], &ib[i]}) {
      if ((rc = check_image(c, im->data, im->w, im->h, im->pitch)) != 0) return rc;
    }
    for (const orbx_frame_out* o : {&oa[i], &ob[i]}) {
      if (!o->points || !o->desc || !o->num_pts || o->max_pts < 1 || o->max_pts > (1 << 22) - 1) return ORBX_ERR_ARG;
    }
  }
  DeviceGuard g(c->device);
  if ((int)c->bws.size() < 2 * n_pairs) c->bws.resize(2 * n_pairs);
  std::vector<Frame> frames(2 * n_pairs);
  for (int i = 0; i < n_pairs; i++) {
    for (int s = 0; s < 2; s++) {
      const orbx_image& im = s ? ib[i] : ia[i];
      const orbx_frame_out& o = s ? ob[i] : oa[i];
      Workspace& ws = c->bws[2 * i + s];
      if ((rc = ws_ensure(c, ws, im.w, im.h)) != 0) return rc;
      fill_frame(c, ws, im.data, im.pitch, o.points, o.desc, o.num_pts, frames[2 * i + s], o.max_pts,
                 (c->batch_form == 1 && !stage_ms) ? 0 : c->pyr_shape);
    }
  }
  LaunchPlan pl;
  if ((rc = upload_batch(c, c->batch, frames, &pl)) != 0) return rc;
  // matching jobs, one per pair, with their own slices of the split scratch
  int max_tiles = 1;
  size_t part_words = 0, tile_words = 0;
  std::vector<MatchJob> jobs(n_pairs);
  for (int i = 0; i < n_pairs; i++) {
    const int nq_cap = oa[i].max_pts;
    max_tiles = std::max(max_tiles, div_up(nq_cap, 128));
    part_words += (size_t)2 * kBatchSplitsCap * nq_cap;
    tile_words += (size_t)div_up(nq_cap, 128);
  }
  if (c->batch_part_words < part_words || c->batch_tile_words < tile_words) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->batch_part);
    cudaFree(c->batch_tile_done);
    c->batch_part = nullptr;
    c->batch_tile_done = nullptr;
    c->batch_part_words = c->batch_tile_words = 0;
    ORBX_CUDA(cudaMalloc(&c->batch_part, part_words * sizeof(uint32_t)));
    ORBX_CUDA(cudaMalloc(&c->batch_tile_done, tile_words * sizeof(unsigned int)));
    ORBX_CUDA(cudaMemset(c->batch_tile_done, 0, tile_words * sizeof(unsigned int)));
    c->batch_part_words = part_words;
    c->batch_tile_words = tile_words;
    if (c->batch_exec) {
      cudaGraphExecDestroy(c->batch_exec);
      c->batch_exec = nullptr;
    }
    c->batch_key.clear();
  }
  {
    size_t po = 0, to = 0;
    for (int i = 0; i < n_pairs; i++) {
      MatchJob& J = jobs[i];
      std::memset(&J, 0, sizeof(J));
      J.args.q = oa[i].desc;
      J.args.db = ob[i].desc;
      J.args.nq = oa[i].max_pts;
      J.args.ndb = ob[i].max_pts;
      J.args.d_nq = oa[i].num_pts;
      J.args.d_ndb = ob[i].num_pts;
      J.args.pts = oa[i].points;
      match_bounds(c, J.args, oa[i].max_pts, ob[i].max_pts, oa[i].max_pts);
      J.work.part = c->batch_part + po;
      J.work.tile_done = c->batch_tile_done + to;
      J.work.nq_cap = oa[i].max_pts;
      J.work.splits_cap = kBatchSplitsCap;
      po += (size_t)2 * kBatchSplitsCap * oa[i].max_pts;
      to += (size_t)div_up(oa[i].max_pts, 128);
    }
  }
  int blocks_per_pair = c->match_blocks_per_pair;
  if (blocks_per_pair <= 0) blocks_per_pair = std::max(max_tiles, div_up(8 * 148, n_pairs));
  blocks_per_pair = std::max(blocks_per_pair, max_tiles);  // every query tile needs a block
  // graph key: frames, jobs and launch shapes
  std::vector<uint8_t> key(sizeof(MatchJob) * n_pairs + c->batch.last.size() + 4 * sizeof(int));
  {
    uint8_t* k = key.data();
    std::memcpy(k, jobs.data(), sizeof(MatchJob) * n_pairs);
    k += sizeof(MatchJob) * n_pairs;
    std::memcpy(k, c->batch.last.data(), c->batch.last.size());
    k += c->batch.last.size();
    const int shapes[4] = {c->nms_rows, c->describe_bps, blocks_per_pair, mode};
    std::memcpy(k, shapes, sizeof(shapes));
  }
  if (c->batch_form == 1 && !stage_ms) return batch_persistent(c, pl, frames, jobs, blocks_per_pair, key);
  if (stage_ms) {
    // profiling: the same launches, unrolled, with events between them
    if (c->jobs_cap < n_pairs) {
      cudaStreamSynchronize(c->stream);
      cudaFree(c->d_jobs);
      c->d_jobs = nullptr;
      c->jobs_cap = 0;
      ORBX_CUDA(cudaMalloc(&c->d_jobs, sizeof(MatchJob) * n_pairs));
      c->jobs_cap = n_pairs;
    }
    ORBX_CUDA(cudaMemcpyAsync(c->d_jobs, jobs.data(), sizeof(MatchJob) * n_pairs, cudaMemcpyHostToDevice,
                              c->stream));
    ORBX_CUDA(cudaStreamSynchronize(c->stream));
    c->batch_key.clear();  // the device job table may differ from the captured one now
    for (auto& e : c->prof_ev)
      if (!e) ORBX_CUDA(cudaEventCreate(&e));
    ORBX_CUDA(cudaEventRecord(c->prof_ev[0], c->stream));
    ORBX_CUDA(launch_pyramid_blur(pl.b, pl.pyr_tiles, c->stream));
    ORBX_CUDA(cudaEventRecord(c->prof_ev[1], c->stream));
    ORBX_CUDA(launch_detect(pl.b, pl.det_tiles, c->stream));
    ORBX_CUDA(cudaEventRecord(c->prof_ev[2], c->stream));
    ORBX_CUDA(launch_nms(pl.b, pl.nms_strips, c->stream));
    ORBX_CUDA(cudaEventRecord(c->prof_ev[3], c->stream));
    ORBX_CUDA(launch_describe(pl.b, pl.total_max_pts, c->stream, c->describe_bps));
    ORBX_CUDA(cudaEventRecord(c->prof_ev[4], c->stream));
    ORBX_CUDA(launch_match_popc_batch(c->d_jobs, n_pairs, blocks_per_pair, c->stream));
    ORBX_CUDA(cudaEventRecord(c->prof_ev[5], c->stream));
    ORBX_CUDA(cudaEventSynchronize(c->prof_ev[5]));
    for (int i = 0; i < 5; i++) ORBX_CUDA(cudaEventElapsedTime(&stage_ms[i], c->prof_ev[i], c->prof_ev[i + 1]));
    return ORBX_OK;
  }
  if (!(c->batch_exec && c->batch_key == key)) {
    if (c->batch_exec) {
      cudaGraphExecDestroy(c->batch_exec);
      c->batch_exec = nullptr;
    }
    if (c->jobs_cap < n_pairs) {
      cudaStreamSynchronize(c->stream);
      cudaFree(c->d_jobs);
      c->d_jobs = nullptr;
      c->jobs_cap = 0;
      ORBX_CUDA(cudaMalloc(&c->d_jobs, sizeof(MatchJob) * n_pairs));
      c->jobs_cap = n_pairs;
    }
    ORBX_CUDA(cudaMemcpyAsync(c->d_jobs, jobs.data(), sizeof(MatchJob) * n_pairs, cudaMemcpyHostToDevice,
                              c->stream));
    ORBX_CUDA(cudaStreamSynchronize(c->stream));
    cudaGraph_t graph = nullptr;
    ORBX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int lrc = launch_frames(c, pl, true);
    if (lrc == ORBX_OK)
      lrc = launch_match_popc_batch(c->d_jobs, n_pairs, blocks_per_pair, c->stream) == cudaSuccess ? ORBX_OK
                                                                                                     : ORBX_ERR_CUDA;
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (lrc != ORBX_OK) {
      if (graph) cudaGraphDestroy(graph);
      return lrc;
    }
    ORBX_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&c->batch_exec, graph, 0);
    cudaGraphDestroy(graph);
    ORBX_CUDA(ie);
    c->batch_key.swap(key);
  }
  ORBX_CUDA(cudaGraphLaunch(c->batch_exec, c->stream));
  return ORBX_OK;
}

ORBX_API int orbx_batch_pairs(orbx_ctx* c, int n_pairs, const orbx_image* ia, const orbx_image* ib,
                              const orbx_frame_out* oa, const orbx_frame_out* ob, int mode) {
  return batch_pairs_impl(c, n_pairs, ia, ib, oa, ob, mode, nullptr);
}

ORBX_API int orbx_profile_batch(orbx_ctx* c, int n_pairs, const orbx_image* ia, const orbx_image* ib,
                                const orbx_frame_out* oa, const orbx_frame_out* ob, float* stage_ms) {
  if (!stage_ms) return ORBX_ERR_ARG;
  return batch_pairs_impl(c, n_pairs, ia, ib, oa, ob, ORBX_MATCH_POPC, stage_ms);
}

ORBX_API int orbx_autotune_pairs(orbx_ctx* c, int n_pairs, const orbx_image* ia, const orbx_image* ib,
                                 const orbx_frame_out* oa, const orbx_frame_out* ob, int reps, orbx_tuning* best,
                                 float* best_ms) {
  return orbx_autotune_pairs_forms(c, n_pairs, ia, ib, oa, ob, reps, 3, best, best_ms);
}

ORBX_API int orbx_autotune_pairs_forms(orbx_ctx* c, int n_pairs, const orbx_image* ia, const orbx_image* ib,
                                       const orbx_frame_out* oa, const orbx_frame_out* ob, int reps, int forms,
                                       orbx_tuning* best, float* best_ms) {
  if (!c || reps < 1 || forms < 1 || forms > 3) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  orbx_tuning keep;
  orbx_get_tuning(c, &keep);
  cudaEvent_t e0, e1;
  ORBX_CUDA(cudaEventCreate(&e0));
  ORBX_CUDA(cudaEventCreate(&e1));
  // candidates: the five-launch form over NMS strip height, describe grid and
  // match blocks per pair; the persistent form over NMS strip height, match
  // blocks per pair, frames per wave and resident blocks per SM
  std::vector<orbx_tuning> cands;
  if (forms & 1)
  for (int r : {2, 4, 8, 16})
    for (int d : {3, 4, 8})
      for (int m : {0, 64, 256}) {
        orbx_tuning t = keep;
        t.batch_form = 0;
        t.nms_rows = r;
        t.describe_blocks_per_sm = d;
        t.match_blocks_per_pair = m;
        cands.push_back(t);
      }
  if (forms & 2)
  for (int r : {4, 16})
    for (int m : {0, 64})
      for (int gsz : {0, 4, 16, 48})
        for (int bps : {0, 3}) {
          orbx_tuning t = keep;
          t.batch_form = 1;
          t.nms_rows = r;
          t.match_blocks_per_pair = m;
          t.persist_group = gsz;
          t.persist_blocks_per_sm = bps;
          t.persist_row_deps = 0;
          cands.push_back(t);
          if (gsz == 0) {  // row-level dependencies order items by row, not in waves
            t.persist_row_deps = 1;
            cands.push_back(t);
          }
        }
  orbx_tuning top = keep;
  float top_ms = 1e30f;
  orbx_tuning top5 = keep;  // best of the five-launch form, for the tile-shape pass
  float top5_ms = 1e30f;
  int rc = ORBX_OK;
  // median of `reps` replays of one candidate (the first call captures its graph)
  auto measure = [&](const orbx_tuning& t, float* out) -> int {
    int r;
    if ((r = orbx_set_tuning(c, &t)) != 0) return r;
    if ((r = orbx_batch_pairs(c, n_pairs, ia, ib, oa, ob, ORBX_MATCH_POPC)) != 0) return r;
    std::vector<float> ms;
    for (int k = 0; k < reps; k++) {
      cudaEventRecord(e0, c->stream);
      if ((r = orbx_batch_pairs(c, n_pairs, ia, ib, oa, ob, ORBX_MATCH_POPC)) != 0) return r;
      cudaEventRecord(e1, c->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) return ORBX_ERR_CUDA;
      float v = 0.f;
      cudaEventElapsedTime(&v, e0, e1);
      ms.push_back(v);
    }
    std::sort(ms.begin(), ms.end());
    *out = ms[ms.size() / 2];
    return ORBX_OK;
  };
  for (const orbx_tuning& t : cands) {
    float med = 0.f;
    if ((rc = measure(t, &med)) != 0) goto done;
    if (med < top_ms) {
      top_ms = med;
      top = t;
    }
    if (t.batch_form == 0 && med < top5_ms) {
      top5_ms = med;
      top5 = t;
    }
  }
  // second pass: the pyramid tile shapes on the best five-launch candidate
  if (forms & 1) {
    for (int shape = 0; shape < kPyrShapes; shape++) {
      if (shape == top5.pyr_tile) continue;
      orbx_tuning t = top5;
      t.pyr_tile = shape;
      float med = 0.f;
      if ((rc = measure(t, &med)) != 0) goto done;
      if (med < top_ms) {
        top_ms = med;
        top = t;
      }
    }
  }
done:
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != ORBX_OK) {
    orbx_set_tuning(c, &keep);
    return rc;
  }
  orbx_set_tuning(c, &top);
  if (best) *best = top;
  if (best_ms) *best_ms = top_ms;
  return orbx_sync(c);
}

ORBX_API int orbx_debug_buffers(orbx_ctx* c, uint8_t* h_pyr, uint8_t* h_blur, float* h_vmap, int* h_layer,
                                int* h_total) {
  if (!c) return ORBX_ERR_ARG;
  const Workspace& ws = c->ws[0];
  if (!ws.pyr_alloc) return ORBX_ERR_STATE;
  DeviceGuard g(c->device);
  ORBX_CUDA(cudaStreamSynchronize(c->stream));
  const size_t npx = (size_t)ws.h * ws.oszp[3 * ws.n];
  if (h_pyr) ORBX_CUDA(cudaMemcpy(h_pyr, ws.pyr_alloc + ws.guard, ws.obytes, cudaMemcpyDeviceToHost));
  if (h_blur) ORBX_CUDA(cudaMemcpy(h_blur, ws.blr_alloc + ws.guard, ws.obytes, cudaMemcpyDeviceToHost));
  if (h_vmap || h_layer) {
    // the dense reference-layout maps of the last single-image call
    float* dv = nullptr;
    int* dl = nullptr;
    ORBX_CUDA(cudaMalloc(&dv, npx * sizeof(float)));
    if (cudaMalloc(&dl, npx * sizeof(int)) != cudaSuccess) {
      cudaFree(dv);
      return ORBX_ERR_NOMEM;
    }
    cudaError_t e = launch_expand_score_map(c->single.d_frames, dv, dl, (long long)npx, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess && h_vmap) e = cudaMemcpy(h_vmap, dv, npx * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h_layer) e = cudaMemcpy(h_layer, dl, npx * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dv);
    cudaFree(dl);
    ORBX_CUDA(e);
  }
  if (h_total) ORBX_CUDA(cudaMemcpy(h_total, ws.total, sizeof(int), cudaMemcpyDeviceToHost));
  return ORBX_OK;
}

ORBX_API int orbx_selftest_wait_timeout(orbx_ctx* c, int timeout_us) {
  if (!c || timeout_us < 1 || timeout_us > 10000000) return ORBX_ERR_ARG;
  DeviceGuard g(c->device);
  int* ctr = nullptr;
  ORBX_CUDA(cudaMallocAsync(&ctr, sizeof(int), c->stream));
  cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(int), c->stream);
  if (e == cudaSuccess)
    e = launch_wait_selftest(ctr, 1, c->d_err, (long long)timeout_us * c->clock_khz / 1000, c->stream);
  cudaFreeAsync(ctr, c->stream);
  ORBX_CUDA(e);
  return orbx_sync(c);
}

ORBX_API long long orbx_selftest_pi_minus(uint32_t lo_bits, uint32_t hi_bits) {
  long long bad = 0;
  for (uint64_t b = lo_bits; b < hi_bits; b++) {
    const uint32_t bits = (uint32_t)b;
    float r;
    std::memcpy(&r, &bits, 4);
    if (!(r >= 0.f && r < 2.f)) continue;
    const float want = (float)(3.14159265358979323846 - (double)r);
    const float got = pi_minus_as_double(r);
    uint32_t wb, gb;
    std::memcpy(&wb, &want, 4);
    std::memcpy(&gb, &got, 4);
    bad += (wb != gb);
  }
  return bad;
}

}  // extern "C"

namespace orbx {
int ctx_device(const orbx_ctx* c) { return c->device; }
cudaStream_t ctx_stream(const orbx_ctx* c) { return c->stream; }
int* ctx_err(orbx_ctx* c) { return c->d_err; }
void umax_table(int patch_size, int* umax) { make_umax(patch_size, umax); }
OcvWork*& ctx_ocv(orbx_ctx* c) { return c->ocv; }
HostIO*& ctx_hostio(orbx_ctx* c) { return c->hostio; }
}  // namespace orbx
