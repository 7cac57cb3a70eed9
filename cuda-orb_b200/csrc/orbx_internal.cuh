// Internal structures shared by the sm_100a ORB kernels and the C ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/orbx.h"

namespace orbx {

constexpr int kMaxOctaves = 5;        // MAX_OCTAVE, orbd.cu:18
constexpr int kMaxFramesPerLaunch = 1024;
constexpr int kInlineFrames = 2;  // frames carried in the launch parameters (a pair)
constexpr size_t kGuard = 256 * 1024; // zeroed bytes before/after each pyramid

// Pyramid-and-blur tile (octave pixels): the default shape, which the
// persistent kernel uses; the five-launch kernel also has the other shapes of
// kPyrShapeTW/TH (tuning pyr_tile), one instantiation each
constexpr int kPyrThreads = 256;  // threads of every block that runs pyramid tiles
constexpr int kPyrShapes = 4;
// 128 x 30 keeps a tile's shared memory (44.1 KB) under the 44.6 KB of five
// blocks per SM, and a 1080p pair's 1,460 tiles within two waves of them
constexpr int kPyrShapeTW[kPyrShapes] = {128, 64, 128, 64};
constexpr int kPyrShapeTH[kPyrShapes] = {30, 32, 16, 64};
constexpr int kPyrTW = kPyrShapeTW[0];
constexpr int kPyrTH = kPyrShapeTH[0];
// Detect tile (level-0 pixels); 32 keeps octave 4/5 tiles whole
constexpr int kDetTW = 64;
constexpr int kDetTH = 32;
// NMS strips span the full valid width; default and largest strip height
constexpr int kNmsRows = 4;
constexpr int kNmsMaxRows = 16;
constexpr int kNmsMaxWords = 2048;  // occupancy words per NMS strip (rows x words per row)

// Bounds-checked build (the same sources compiled with -DORBX_BOUNDS_CHECK
// into liborbx_checked.so).  Every global access of the pipeline's stage
// bodies and of the popcount matcher is first tested against the extent of
// the buffer it belongs to (a Span).  An access outside it is skipped, a load
// giving zero, and counted in the launch's BoundsRec with the site, the byte
// offset from the buffer's base and the extent of the first one.  Launches
// without a record (bounds == nullptr) and the normal build test nothing:
// there ORBX_IN is the constant true and the spans compile away.
struct BoundsRec {
  unsigned long long n;     // accesses skipped
  long long site, off, extent;  // the first of them
};
struct Span {
  const void* base;
  long long bytes;
};
enum : int {
  kSitePyrLoad = 1,  // pyramid staging: level-0 image or caller pyramid
  kSitePyrPadLoad,   // pyramid: row padding copied from level 0
  kSitePyrStore,     // pyramid: raw and blurred tile stores (within the octave)
  kSiteFrameState,   // per-frame counters and NMS look-back words
  kSiteDetLoad,      // detect: octave staging with halo (guarded pyramid)
  kSiteDetStore,     // detect: occupancy, score and octave maps
  kSiteNmsOcc,       // NMS: occupancy words
  kSiteNmsScore,     // NMS: scores and octaves
  kSiteNmsPts,       // NMS: keypoint stores
  kSiteDescPts,      // describe: keypoint index (its loads, angle and descriptor stores)
  kSiteDescMoment,   // describe: raw patch rows (guarded pyramid)
  kSiteDescSample,   // describe: blurred sampling points (guarded pyramid)
  kSiteMatchQ,       // popcount matcher: query rows
  kSiteMatchDb,      // popcount matcher: train rows
  kSiteMatchOut,     // matcher outputs (keypoint match fields, k = 2 lists)
};

// Per-frame state, in device memory (one entry per frame of a launch).
struct Frame {
  const uint8_t* img;  // level-0 input, row pitch `pitch_in`
  const uint8_t* pyr_src;  // optional: an existing pyramid (reference layout) to blur instead of img
  int w, h, pitch_in;
  int n_oct;
  int ow[kMaxOctaves], oh[kMaxOctaves], op[kMaxOctaves];
  long long ooff[kMaxOctaves + 1];  // octave offsets in the pyramid (orb.cpp:151-174)
  uint8_t* pyr;  // octave 0 of the raw pyramid (kGuard zeroed bytes on both sides)
  uint8_t* blr;  // octave 0 of the blurred pyramid (same layout and guards)
  float* vmap;    // level-0 keyed scores, h * op[0] floats, valid where the occupancy bit is set
  uint8_t* oct8;  // octave of each score, h * op[0] bytes, valid where the occupancy bit is set
  uint32_t* occ;  // occupancy bits: bit (y * op[0] + x) set where score > 0, h * op[0] / 32 words
  int* layer;     // dense octave map of the reference's vmem layout (debug and orbd.h only)
  orbx_point* pts;
  uint8_t* desc;
  int* count;    // min(survivors, max_pts)
  int* total;    // survivors before the cap (may be null)
  int max_pts;
  int border;    // max(edge_threshold, 3)
  // tiling
  int pyr_shape;  // index into kPyrShapeTW/TH of the pyramid tile tables below
  int pyr_tiles_x[kMaxOctaves], pyr_tiles_y[kMaxOctaves];
  int pyr_tile_base[kMaxOctaves + 1];  // per-octave prefix within the frame
  int det_tiles_x, det_tiles_y;
  int nms_rows;      // level-0 rows per NMS strip (tunable, <= kNmsMaxRows)
  int nms_strips;
  unsigned long long* nms_status;  // look-back words, one per strip
  long long img_bytes;  // extent of img as the bounds-checked build tests it (h * pitch_in)
};

// Per-launch view of a batch of frames.
struct Batch {
  Frame* frames;
  int n_frames;
  const int* pyr_base;   // [n_frames + 1] tile prefix over frames for k_pyramid_blur
  const int* det_base;   // [n_frames + 1] for k_detect
  const int* nms_base;   // [n_frames + 1] for k_nms
  unsigned int* nms_ticket;  // dynamic strip ticket (reset by k_pyramid_blur)
  int* err;              // sticky error word (bounded waits that gave up)
  BoundsRec* bounds;     // bounds-checked build: record of skipped accesses (else null)
  long long wait_cycles; // bound of every device-side wait, in SM clock cycles
  int pyr_shape;         // pyramid tile shape of every frame of the launch
  int describe_mode;     // 0: angle + descriptor, 1: angle only, 2: descriptor only
  // parameters (Orbor::init, orb.h:18-19)
  int fast_thr;
  int harris;            // 1: HARRIS_SCORE, 0: FAST_SCORE
  int wta_k;
  int half_k;            // patch_size / 2
  float gauss[4];        // setGaussianKernel weights (host expf, orbd.cu:413-433)
  float harris_scale4;   // setScaleSqSq (orbd.cu:436-441)
  const int8_t* pattern; // [512][2] sampling points (setPattern)
  const int* umax;       // [half_k + 2] (setUmax)
  // A batch of up to kInlineFrames frames also carries its frame table and
  // tile prefixes in the launch parameters (n_inline = n_frames, else 0), so
  // that the kernels read them from the constant bank instead of global memory.
  int n_inline;
  int inl_pyr_base[kInlineFrames + 1], inl_det_base[kInlineFrames + 1], inl_nms_base[kInlineFrames + 1];
  Frame inl[kInlineFrames];
};

enum : int {
  kErrLookbackTimeout = 1,
  kErrImmaTimeout = 2,
  kErrStageTimeout = 4,  // persistent batch kernel: a stage dependency never completed
};
enum : int { kDescribeBoth = 0, kDescribeAngleOnly = 1, kDescribeDescOnly = 2 };

// host-side helpers implemented in orbx_api.cu
}  // namespace orbx

// kernel launchers (orbx_detect.cu / orbx_describe.cu / orbx_match.cu)
namespace orbx {
cudaError_t launch_pyramid_blur(const Batch& b, int total_tiles, cudaStream_t s);
cudaError_t launch_detect(const Batch& b, int total_tiles, cudaStream_t s);
cudaError_t launch_nms(const Batch& b, int total_strips, cudaStream_t s);
// dense reference-layout score and octave maps from the sparse ones (frame 0 of b)
cudaError_t launch_expand_score_map(const Frame* d_frame, float* vmap_dense, int* layer_dense, long long npx,
                                    cudaStream_t s);
cudaError_t launch_describe(const Batch& b, int total_max_pts, cudaStream_t s, int blocks_per_sm = 8);

struct MatchArgs {
  const uint8_t* q;      // [nq][32]
  const uint8_t* db;     // [ndb][32]
  int nq, ndb;
  const int* d_nq;       // optional device counts (override nq/ndb when non-null)
  const int* d_ndb;
  uint32_t* dist2;       // optional [nq][2]
  int32_t* idx2;         // optional [nq][2]
  orbx_point* pts;         // optional: reference-semantics match/distance (orbd.cu:1545-1557)
  BoundsRec* bounds;       // bounds-checked build: record of skipped accesses (else null)
  int q_cap, db_cap, out_cap;  // rows of q, db and of the outputs (checked with bounds)
  int unused_;                 // no tail padding: whole-struct bytes key the CUDA graphs
};
struct MatchWork {          // scratch for split-train merging
  uint32_t* part;           // [splits_cap][nq_cap][2] partial top-2 keys
  unsigned int* tile_done;  // [ceil(nq_cap / 128)] arrival counters, self-resetting
  int nq_cap;               // query capacity the grid is sized for
  int splits_cap;           // most train splits per query tile
};
int match_popc_blocks(int nq_cap, int splits_cap, int blocks_per_sm = 8);

// int8 tensor-core form (orbx_match_imma.cu)
struct ImmaLaunch {
  MatchArgs args;     // queries, database, counts, outputs
  MatchWork work;     // split merging (splits_cap >= splits)
  int8_t* q_pm1;      // [imma_rows_q(nq_cap)][256] scratch
  int8_t* db_pm1;     // [imma_rows_db(ndb_cap)][256] scratch
  int nq_cap, ndb_cap;
  int splits;         // database splits per query tile
  int* err;
  bool q_ready;       // q_pm1 already holds the expanded queries (rows >= nq zero)
  bool db_ready;      // db_pm1 already holds the expanded database (rows >= ndb zero)
};
// bits -> +-1 int8 rows (rows beyond the count are zero); 4 * 148 blocks of 256
cudaError_t launch_expand_pm1(const uint8_t* bits, int n, const int* d_n, int rows, int8_t* out, cudaStream_t s);
int imma_rows_q(int n);
int imma_rows_db(int n);
int imma_default_splits(int nq_cap);
cudaError_t launch_match_imma(const ImmaLaunch& L, cudaStream_t s);

// Probe rerank of the learned proposal on the int8 tensor cores
// (orbx_match_imma.cu): per (cluster, up to 128 probing slots), the exact top-2
// keys of each slot over the cluster's rows, one pair per 64-column group.
constexpr int kRrGroups = 4;
struct RerankImmaArgs {
  const uint8_t* q_bits;     // [nq][32] queries
  const int* list;           // probing slots grouped by cluster (slot = query * 8 + probe)
  const int* probe_offsets;  // [C + 1] each cluster's first slot in list
  const int* item_offsets;   // [C + 1] exclusive scan of ceil(slots / 128)
  int n_clusters;
  const int* ivf_offsets;    // [C + 1] list offsets: the cluster's row count
  const int* pad_offsets;    // [C + 1] the cluster's first padded row (multiples of 256)
  const int* pad_members;    // [pad_rows] database index of each padded row, -1 in the padding
  const uint8_t* pad_desc;   // [pad_rows][32] packed rows of the padded lists (padding zero), 16-byte aligned
  uint2* partial;            // [slots][kRrGroups] top-2 keys
  int* item_counter;         // zero at launch: the blocks claim items from it
  uint32_t* q_bound;         // [nq] 0xFFFFFFFF at launch: per query the least second-best key any item has found
  int* err;
};
cudaError_t launch_rerank_imma(const RerankImmaArgs& a, int max_items, cudaStream_t s);

// Top-2 keys shared by both matcher forms: key = distance << 22 | index, so
// ordering keys orders by (distance, index); 0xFFFFFFFF means "none".
constexpr int kIdxBitsShared = 22;
constexpr uint32_t kIdxMaskShared = (1u << kIdxBitsShared) - 1u;
constexpr uint32_t kNoKeyShared = 0xFFFFFFFFu;
constexpr int kMaxDistShared = 64;  // MAX_DIST, orbd.cu:26

#ifdef __CUDACC__
#ifdef ORBX_BOUNDS_CHECK
// [off, off + len) within [0, extent), else recorded
__device__ __forceinline__ bool in_range(BoundsRec* rec, int site, long long off, long long len, long long extent) {
  if (!rec) return true;
  if (off >= 0 && off + len <= extent) return true;
  if (atomicAdd(&rec->n, 1ull) == 0ull) {
    rec->site = site;
    rec->off = off;
    rec->extent = extent;
  }
  return false;
}
__device__ __forceinline__ bool in_span(BoundsRec* rec, int site, Span s, const void* p, int bytes) {
  return in_range(rec, site, (long long)(reinterpret_cast<const char*>(p) - reinterpret_cast<const char*>(s.base)),
                  bytes, s.bytes);
}
#define ORBX_IN(rec, site, span, p, bytes) ::orbx::in_span((rec), (site), (span), (p), (bytes))
#define ORBX_IN_ROWS(rec, site, row, rows) ::orbx::in_range((rec), (site), (row), 1, (rows))
#else
#define ORBX_IN(rec, site, span, p, bytes) true
#define ORBX_IN_ROWS(rec, site, row, rows) true
#endif
// Extents of a frame's buffers: the level-0 image (h rows of pitch_in bytes),
// the pyramid with its guard zones, one octave of it, and the level-0 maps.
__host__ __device__ __forceinline__ Span img_span(const Frame& F) { return {F.img, F.img_bytes}; }
__host__ __device__ __forceinline__ Span guarded_span(const uint8_t* pyr, const Frame& F) {
  return {pyr - kGuard, F.ooff[F.n_oct] + 2 * (long long)kGuard};
}
__host__ __device__ __forceinline__ Span octave_span(const uint8_t* pyr, const Frame& F, int o) {
  return {pyr + F.ooff[o], F.ooff[o + 1] - F.ooff[o]};
}
__host__ __device__ __forceinline__ long long map_px(const Frame& F) { return (long long)F.h * F.op[0]; }

__device__ __forceinline__ void top2_push_shared(uint32_t& k1, uint32_t& k2, uint32_t key) {
  k2 = min(k2, max(k1, key));
  k1 = min(k1, key);
}

// Reference semantics of the final step (orbd.cu:1545-1557): both best scores
// start at 256 and only strictly smaller distances replace them, so a match is
// reported when the nearest distance is unique and below MAX_DIST.
__device__ __forceinline__ void finish_query_shared(const MatchArgs& a, int q, uint32_t k1, uint32_t k2) {
  const uint32_t d1 = (k1 == kNoKeyShared) ? kNoKeyShared : (k1 >> kIdxBitsShared);
  const uint32_t d2 = (k2 == kNoKeyShared) ? kNoKeyShared : (k2 >> kIdxBitsShared);
  const int i1 = (k1 == kNoKeyShared) ? -1 : (int)(k1 & kIdxMaskShared);
  const int i2 = (k2 == kNoKeyShared) ? -1 : (int)(k2 & kIdxMaskShared);
  if (!ORBX_IN_ROWS(a.bounds, orbx::kSiteMatchOut, q, a.out_cap)) return;
  if (a.dist2) {
    a.dist2[2 * q] = d1;
    a.dist2[2 * q + 1] = d2;
  }
  if (a.idx2) {
    a.idx2[2 * q] = i1;
    a.idx2[2 * q + 1] = i2;
  }
  if (a.pts) {
    const uint32_t c1 = min(d1, 256u), c2 = min(d2, 256u);
    const bool ok = (c1 < c2) && (c1 < (uint32_t)kMaxDistShared);
    a.pts[q].match = ok ? i1 : -1;
    a.pts[q].distance = ok ? (int)c1 : -1;
  }
}
#endif

// orbd.h lower-level entry points on caller-owned pyramid buffers (orbx_api.cu)
int lower_detect(orbx_ctx* c, const uint8_t* image, uint8_t* octave_images, float* vmem, orbx_point* pts,
                 int* d_count, const int* oszp, int noctaves, int threshold, int border, bool harris);
int lower_angle(orbx_ctx* c, const uint8_t* octave_images, orbx_point* pts, int n_pts, const int* oszp,
                int noctaves, int patch_size, int* d_tmp_count);
int lower_blur(orbx_ctx* c, uint8_t* octave_images, const int* oszp, int noctaves, int* d_tmp_count);
int lower_last_layout(orbx_ctx* c, int* oszp, int noctaves);
int lower_describe(orbx_ctx* c, const uint8_t* octave_images, orbx_point* pts, int n_pts, uint8_t* desc, int wta_k,
                   const int* oszp, int noctaves, int* d_tmp_count);
cudaError_t launch_match_popc(const MatchArgs& a, const MatchWork& w, cudaStream_t s, int blocks_per_sm = 8);

// one matching job of a batch (one frame pair)
struct MatchJob {
  MatchArgs args;
  MatchWork work;
};
cudaError_t launch_match_popc_batch(const MatchJob* d_jobs, int n_jobs, int blocks_per_job, cudaStream_t s);

// context accessors for the entry points outside orbx_api.cu
int ctx_device(const orbx_ctx* c);
cudaStream_t ctx_stream(const orbx_ctx* c);
int* ctx_err(orbx_ctx* c);
struct HostIO;  // orbx_hostio.cu: pinned staging of the host I/O entry points
struct OcvWork;  // orbx_ocv.cu: buffers of the OpenCV-style pipeline
OcvWork*& ctx_ocv(orbx_ctx* c);
void ocv_free(OcvWork* w);
void umax_table(int patch_size, int* umax);  // setUmax (orbd.cu:66-92)
HostIO*& ctx_hostio(orbx_ctx* c);
void hostio_free(HostIO* io);
// The pinned, mapped result block of orbx_pair_host (allocated or grown here).
int hostio_map(orbx_ctx* c, int max_pts, const uint8_t** host, const uint8_t** dev);
int hostio_export_pair(orbx_ctx* c, const orbx_point* pa, const orbx_point* pb, const uint8_t* da, const uint8_t* db,
                       const int* d_count, int max_pts, bool with_desc, const uint8_t** host);
}  // namespace orbx
