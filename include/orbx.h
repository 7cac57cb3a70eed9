/* orbx -- C ABI of the sm_100a ORB detect / describe / match library.
 *
 * Plain pointers and sizes only.  Device pointers are prefixed d_, host
 * pointers h_.  Every call returns an ORBX_* status; nothing exits the process.
 * Work is queued on the context's CUDA stream and does not synchronise the
 * host unless the call says so.
 *
 * Each entry point names the reference interface it replaces (CUDA-ORB,
 * file:line).  The C++ classes of the reference (orb.h, orbd.h) are provided on
 * top of this ABI by include/orb.h and include/orbd.h.
 */
#ifndef ORBX_H
#define ORBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORBX_API __attribute__((visibility("default")))

/* Same 28-byte layout and field order as orb::OrbPoint (orb_structures.h:8-17):
 * x, y are level-0 coordinates; octave is the pyramid level; score is the Harris
 * (or FAST) score; angle is in radians; match/distance are written by matching. */
typedef struct orbx_point {
  int x;
  int y;
  int octave;
  float score;
  float angle;
  int match;
  int distance;
} orbx_point;

/* Orbor::init arguments (orb.h:18-19, orb.cpp:32-54). */
typedef struct orbx_params {
  int noctaves;       /* requested levels; clamped as orb.cpp:148 does */
  int edge_threshold; /* NMS border in level-0 pixels */
  int wta_k;          /* 2, 3 or 4 */
  int score_type;     /* 0 = HARRIS_SCORE, 1 = FAST_SCORE (orb_structures.h:31-35) */
  int patch_size;     /* <= 31 */
  int fast_threshold;
  int retain_topn;    /* accepted and ignored, as in the reference (orb.cpp:41) */
  int max_pts;        /* keypoint cap per image */
} orbx_params;

typedef struct orbx_ctx orbx_ctx;

enum {
  ORBX_OK = 0,
  ORBX_ERR_ARG = 1,     /* bad argument (null pointer, negative size, ...) */
  ORBX_ERR_CUDA = 2,    /* a CUDA runtime call failed */
  ORBX_ERR_SIZE = 3,    /* image or set size outside the supported range */
  ORBX_ERR_STATE = 4,   /* orbx_init not called */
  ORBX_ERR_TIMEOUT = 5, /* a bounded device-side wait gave up */
  ORBX_ERR_NOMEM = 6    /* device allocation failed */
};

enum {
  ORBX_MATCH_POPC = 0, /* XOR + popcount over 32-bit words */
  ORBX_MATCH_IMMA = 1, /* +-1 int8 tcgen05 MMA, Hamming = (256 - dot) / 2 */
  ORBX_MATCH_AUTO = 2
};

ORBX_API const char* orbx_version(void);
ORBX_API const char* orbx_status_string(int status);

/* Context: holds what the reference keeps in process-global __constant__ and
 * __device__ state (orbd.cu:32-41) plus its own stream and workspaces, so that
 * several contexts can coexist.  Replaces orb::Orbor::Orbor/~Orbor (orb.cpp:14-29). */
ORBX_API int orbx_create(orbx_ctx** ctx, int device);
ORBX_API int orbx_destroy(orbx_ctx* ctx);
ORBX_API int orbx_set_stream(orbx_ctx* ctx, void* cuda_stream);
ORBX_API void* orbx_get_stream(orbx_ctx* ctx);
ORBX_API int orbx_sync(orbx_ctx* ctx);

/* Orbor::init (orb.cpp:32-54) with setMaxNumPoints, setFastThresholdLUT,
 * setUmax, setPattern, setGaussianKernel, setScaleSqSq (orbd.cu:45-441). */
ORBX_API int orbx_default_params(orbx_params* p);
ORBX_API int orbx_init(orbx_ctx* ctx, const orbx_params* p);

/* Orbor::updateParam sizes (orb.cpp:145-191): writes
 * [osizes|widths|heights|pitchs|offsets] (5n+1 ints) into oszp; returns n, or a
 * negative ORBX_* status. */
ORBX_API int orbx_layout(int w, int h, int noctaves, int* oszp, int cap);

/* Orbor::detectAndCompute (orb.cpp:57-101) = hFastDectectWithNMS +
 * hComputeAngle + hGassianBlur + hDescribe (orbd.cu:1564-1783), for one image.
 * d_image: w x h bytes with row pitch `pitch` (the reference requires
 * pitch == align_up(w, 128); other pitches are accepted, their padding reads as 0).
 * d_points: max_pts entries; d_desc: max_pts * 32 bytes; d_num_pts: 1 int.
 * Keypoints come out in raster order (y, then x); when more than max_pts survive,
 * the first max_pts in that order are kept and *d_num_pts = max_pts.
 * Asynchronous: *d_num_pts stays on the device. */
ORBX_API int orbx_detect_and_compute(orbx_ctx* ctx, const uint8_t* d_image, int w, int h, int pitch,
                                     orbx_point* d_points, uint8_t* d_desc, int* d_num_pts, int compute_desc);

/* Orbor::match / hMatch / gHammingMatch (orb.cpp:104-113, orbd.cu:1471-1559,
 * 1786-1793): for i < *d_n1 sets d_points1[i].match = index of the nearest
 * descriptor in d_desc2 and .distance = its Hamming distance when that nearest
 * is unique and closer than 64, else -1 / -1.  Counts are read on the device. */
ORBX_API int orbx_match(orbx_ctx* ctx, orbx_point* d_points1, const int* d_n1, const uint8_t* d_desc1,
                        const int* d_n2, const uint8_t* d_desc2, int n1_cap, int n2_cap, int mode);

/* Brute-force k = 2 Hamming search (the gHammingMatch reduction, orbd.cu:1489-1542,
 * exposed as a result): d_dist2[2i], d_dist2[2i+1] and d_idx2[...] are the two
 * nearest database rows of query i ordered by (distance, index); missing entries
 * are (0xFFFFFFFF, -1).  Sizes up to 4,194,303 database rows. */
ORBX_API int orbx_match_knn2(orbx_ctx* ctx, const uint8_t* d_q, int nq, const uint8_t* d_db, int ndb,
                             uint32_t* d_dist2, int32_t* d_idx2, int mode);

/* No counterpart in the reference.  The orbx_match_knn2 popcount search with the
 * same outputs, for callers that may not allocate device memory: it needs no
 * context and allocates nothing.  Its scratch (about 4 MiB) is one fixed
 * device array per device, whose address is looked up on every call with that
 * device current.  The first call on a device loads the library's module
 * there and so commits the 4 MiB (a failure then, e.g. with no device memory
 * left, returns ORBX_ERR_CUDA): make that first call at start-up, before any
 * stream capture.  Later calls only look the address up.
 * Runs on the current device and on cuda_stream (0 = the legacy default stream).
 * nq above ORBX_STATIC_MAX_QUERIES returns ORBX_ERR_SIZE.  Calls on one device
 * share the scratch: calls whose work overlaps on the device race. */
#define ORBX_STATIC_MAX_QUERIES 16384
ORBX_API int orbx_match_knn2_static(const uint8_t* d_q, int nq, const uint8_t* d_db, int ndb,
                                    uint32_t* d_dist2, int32_t* d_idx2, void* cuda_stream);

/* A frame pair end to end: detect + describe A and B in shared launches, then
 * match A -> B (Orbor::detectAndCompute x2 + Orbor::match, main.cpp:233-243).
 * Replayed from a CUDA graph cached per (shape, pointers). */
ORBX_API int orbx_pair(orbx_ctx* ctx, const uint8_t* d_img_a, const uint8_t* d_img_b, int w, int h, int pitch,
                       orbx_point* d_pts_a, uint8_t* d_desc_a, int* d_n_a, orbx_point* d_pts_b,
                       uint8_t* d_desc_b, int* d_n_b, int mode);

/* orbx_pair with host buffers, synchronous: copies both images (h x pitch bytes
 * each; pinned memory makes the copies asynchronous DMA) to the device, runs the
 * pair, and copies back the keypoint counts, the keypoints of both images
 * (h_pts_* need max_pts entries; match/distance of A are filled) and, when the
 * pointers are non-null, the descriptors (max_pts * 32 bytes each).  This is
 * what Orbor::detectAndCompute x2 + Orbor::match hand back to the host
 * (orb.cpp:95-112). */
ORBX_API int orbx_pair_host(orbx_ctx* ctx, const uint8_t* h_img_a, const uint8_t* h_img_b, int w, int h, int pitch,
                            orbx_point* h_pts_a, int* h_n_a, orbx_point* h_pts_b, int* h_n_b, uint8_t* h_desc_a,
                            uint8_t* h_desc_b, int mode);

/* orbx_pair_host with its phases timed (no counterpart in the reference):
 * phase_ms[0..2] = CUDA-event times from the start to the end of the image
 * uploads, of the kernels and of the export kernel (with overlapped uploads
 * the kernels and the export are one launch sequence, so [1] = [2]);
 * phase_ms[3..6] = host times of enqueueing everything, of the wait for the
 * stream, of the copy-out, and of the whole call. */
ORBX_API int orbx_profile_pair_host(orbx_ctx* ctx, const uint8_t* h_img_a, const uint8_t* h_img_b, int w, int h,
                                    int pitch, orbx_point* h_pts_a, int* h_n_a, orbx_point* h_pts_b, int* h_n_b,
                                    uint8_t* h_desc_a, uint8_t* h_desc_b, int mode, float* phase_ms);

/* Host I/O.  orbx_upload_image copies a host image with any row pitch h_pitch
 * >= w (pinned or pageable memory) into a device image with row pitch d_pitch
 * >= w (the reference's layout is d_pitch = align_up(w, 128)), with zero
 * padding.  Asynchronous for pinned sources; for pageable ones it returns once
 * the rows are staged in the context's pinned buffers.  The reference leaves
 * this to its callers (main.cpp). */
ORBX_API int orbx_upload_image(orbx_ctx* ctx, const uint8_t* h_img, int w, int h, int h_pitch, uint8_t* d_img,
                               int d_pitch);
/* Copies fields of the first n device keypoints into the host OrbPoint array,
 * leaving the other fields of each host entry as they were: ORBX_FIELDS_KEYPOINT
 * (x, y, octave, score, angle: the copy at orb.cpp:95-100), ORBX_FIELDS_MATCH
 * (match, distance: orb.cpp:108-111), or both.  One packing kernel and one
 * contiguous DMA instead of the reference's strided cudaMemcpy2D.  Synchronous. */
#define ORBX_FIELDS_KEYPOINT 1
#define ORBX_FIELDS_MATCH 2
ORBX_API int orbx_download_points(orbx_ctx* ctx, const orbx_point* d_points, int n, orbx_point* h_points, int fields);

/* OpenCV-compatible mode.  cv::ORB's algorithm rather than the reference's:
 * a pyramid of `nlevels` levels, each resized from the previous one by
 * 1 / scale_factor (bilinear); FAST-9 with 3x3 non-maximum suppression on each
 * level, outside `edge_threshold`; a per-level feature budget (geometric in
 * 1 / scale_factor) filled by FAST score (2x budget) then Harris score (budget),
 * as orb.cpp's unused retain_topn hints at (orb.cpp:41); intensity-centroid
 * angle; rBRIEF with the rotated pattern on each level blurred by a 7x7 sigma 2
 * Gaussian.  Comparable with cv2.ORB statistically, not bit for bit.  Keypoints
 * are sorted by level, then by decreasing score. */
typedef struct orbx_ocv_params {
  int nfeatures;       /* total budget, <= 16000 */
  float scale_factor;  /* (1, 2] */
  int nlevels;         /* 1..16 */
  int edge_threshold;  /* >= 19: the angle disc and rotated pattern stay in the level */
  int score_type;      /* 0 = HARRIS_SCORE, 1 = FAST_SCORE */
  int patch_size;      /* 31 */
  int fast_threshold;  /* 0..255 */
} orbx_ocv_params;

/* cv::KeyPoint fields: level-0 position, diameter, angle in degrees [0, 360),
 * response (Harris or FAST score) and pyramid level. */
typedef struct orbx_ocv_keypoint {
  float x, y, size, angle, response;
  int octave;
} orbx_ocv_keypoint;

ORBX_API int orbx_ocv_default_params(orbx_ocv_params* p);
/* d_keypoints: cap entries; d_desc: cap * 32 bytes; *d_n (device) = keypoints
 * written (min(found, cap)).  Asynchronous. */
ORBX_API int orbx_ocv_detect_and_compute(orbx_ctx* ctx, const orbx_ocv_params* p, const uint8_t* d_image, int w, int h,
                                         int pitch, orbx_ocv_keypoint* d_keypoints, uint8_t* d_desc, int* d_n,
                                         int cap);

/* Profiling variant of orbx_pair: the same launches without the graph, with a
 * CUDA event between consecutive kernels; writes the milliseconds of the
 * pyramid/blur, detect, NMS, describe and match kernels to stage_ms[0..4].
 * Synchronises the stream. */
ORBX_API int orbx_profile_pair(orbx_ctx* ctx, const uint8_t* d_img_a, const uint8_t* d_img_b, int w, int h, int pitch,
                               orbx_point* d_pts_a, uint8_t* d_desc_a, int* d_n_a, orbx_point* d_pts_b,
                               uint8_t* d_desc_b, int* d_n_b, int mode, float* stage_ms);

/* One image of a batch: device pointer, size and row pitch (>= w). */
typedef struct orbx_image {
  const uint8_t* data;
  int w, h, pitch;
} orbx_image;

/* Device outputs of one image of a batch: max_pts keypoints, max_pts*32
 * descriptor bytes, one int count; max_pts is this image's keypoint cap. */
typedef struct orbx_frame_out {
  orbx_point* points;
  uint8_t* desc;
  int* num_pts;
  int max_pts;
} orbx_frame_out;

/* Launch shapes the autotuner chooses among, and the bound of device-side waits. */
typedef struct orbx_tuning {
  int nms_rows;              /* level-0 rows per NMS strip, 1..16 */
  int describe_blocks_per_sm; /* grid of the orientation + descriptor kernel */
  int match_blocks_per_sm;    /* grid of the popcount matcher (single pairs) */
  int match_blocks_per_pair;  /* grid per pair of the batched matcher, 0 = automatic */
  int batch_form;             /* orbx_batch_pairs: 0 = five graph-replayed launches, 1 = one persistent launch */
  int persist_group;          /* persistent form: frames per wave of the work order (even), 0 = all frames */
  int persist_blocks_per_sm;  /* persistent form: resident blocks per SM, 0 = the occupancy limit */
  int wait_timeout_us;        /* bound of every device-side wait, 1 .. 10,000,000 us (default 1,000,000) */
  int upload_bands;           /* orbx_pair_host: 0 = copy both images, then run the pair; 1..16 = copy them in
                                 this many row bands per image on a second stream while one persistent launch
                                 already processes the bands that have arrived (popcount matching) */
  int pair_form;              /* orbx_pair: 0 = five graph-replayed launches, 1 = one persistent launch
                                 (popcount matching) */
  int pyr_tile;               /* pyramid + blur tile of the five-launch forms: 0 = 128 x 30, 1 = 64 x 32,
                                 2 = 128 x 16, 3 = 64 x 64 octave pixels (the persistent forms use 128 x 30) */
  int persist_row_deps;       /* persistent launches: 1 = a detect tile row waits only for the pyramid tile rows
                                 it reads (a frame's stages overlap row by row), 0 = for the whole frame */
  int host_overlap;           /* orbx_pair_host with upload_bands = 0: 1 (default) = image B is copied while
                                 frame A's kernels run (the frames on two streams, popcount matching), 0 = copy
                                 both, then run the pair */
} orbx_tuning;

ORBX_API int orbx_get_tuning(orbx_ctx* ctx, orbx_tuning* t);
ORBX_API int orbx_set_tuning(orbx_ctx* ctx, const orbx_tuning* t);

/* No counterpart in the reference (its CUDA errors exit the process,
 * cuda_utils.h:18-38).  Runs the device-side bounded wait of the persistent
 * batch kernel on a counter that nothing increments, bounded by timeout_us:
 * the wait gives up, the call returns ORBX_ERR_TIMEOUT through the context's
 * error word (as any call that timed out does at orbx_sync), and the context
 * stays usable.  For tests of the failure path. */
ORBX_API int orbx_selftest_wait_timeout(orbx_ctx* ctx, int timeout_us);

/* No counterpart in the reference (it has no checked build; its CHECK macros,
 * cuda_utils.h:18-38, catch only failed API calls, and its kernels read past
 * their buffers by design, orbd.cu:1001-1036 and 1437-1468).
 * 1 in the bounds-checked build of this library (liborbx_checked.so: the same
 * sources compiled with -DORBX_BOUNDS_CHECK), 0 in the normal build. */
ORBX_API int orbx_bounds_checked(void);

/* Bounds-checked build only.  There every global access of the pyramid,
 * detect, NMS and describe stages (five-launch, persistent and batched forms)
 * and of the popcount matcher is tested against the extent of its buffer
 * (the h x pitch image, the pyramid with its guard zones, one octave for the
 * pyramid's stores, the h x pitch0 maps, max_pts keypoints and descriptors,
 * the match capacities).  An access outside it is skipped (a load reads zero)
 * and counted.  This waits for the context's streams, then writes
 * out[0] = accesses skipped since the last report, out[1] = the site of the
 * first (kSite* in csrc/orbx_internal.cuh), out[2] = its byte (or row)
 * offset from the buffer's base, out[3] = the buffer's extent, and clears
 * the record.  The normal build returns ORBX_ERR_STATE. */
ORBX_API int orbx_bounds_report(orbx_ctx* ctx, long long* out);

/* Bounds-checked build only; no counterpart in the reference.  Frames set up
 * by later calls on this context have their image's checked extent reduced by
 * `bytes` (h x pitch - bytes), so the kernels' reads of the image's last bytes,
 * which lie in memory the caller owns, are skipped and reported.  A test of
 * the checker itself: it shows that a read outside a buffer's extent is caught
 * without making any access outside an allocation.  0 restores the extent.
 * The normal build returns ORBX_ERR_STATE. */
ORBX_API int orbx_bounds_set_slack(orbx_ctx* ctx, long long bytes);

/* Many frame pairs of any sizes and keypoint caps: every stage of every image
 * runs in shared launches (one per stage for the whole batch), then every pair
 * is matched A -> B in one launch; or, with tuning batch_form = 1, all of it
 * runs in one persistent launch whose blocks claim (stage, frame, tile) work
 * items from a device queue, waiting per frame on the stage before.  Replayed
 * from a CUDA graph cached per (shapes, pointers, tuning).  Per pair the results are identical to
 * orbx_pair on that pair with the same cap.  This batches what the reference
 * does one Orbor::detectAndCompute / Orbor::match call at a time
 * (orb.cpp:57-113).  Asynchronous. */
ORBX_API int orbx_batch_pairs(orbx_ctx* ctx, int n_pairs, const orbx_image* imgs_a, const orbx_image* imgs_b,
                              const orbx_frame_out* out_a, const orbx_frame_out* out_b, int mode);

/* Project-written autotuner: times orbx_batch_pairs on these inputs for every
 * candidate tuning (CUDA events, median of `reps` replays), keeps the fastest
 * in the context and returns it with its time.  Synchronises. */
ORBX_API int orbx_autotune_pairs(orbx_ctx* ctx, int n_pairs, const orbx_image* imgs_a, const orbx_image* imgs_b,
                                 const orbx_frame_out* out_a, const orbx_frame_out* out_b, int reps,
                                 orbx_tuning* best, float* best_ms);

/* orbx_autotune_pairs over the batch forms in `forms`: bit 0 the five-launch
 * form, bit 1 the persistent form (3 = both, as orbx_autotune_pairs). */
ORBX_API int orbx_autotune_pairs_forms(orbx_ctx* ctx, int n_pairs, const orbx_image* imgs_a,
                                       const orbx_image* imgs_b, const orbx_frame_out* out_a,
                                       const orbx_frame_out* out_b, int reps, int forms, orbx_tuning* best,
                                       float* best_ms);

/* Profiling variant of orbx_batch_pairs: the same launches without the graph,
 * with a CUDA event between consecutive kernels; stage_ms[0..4] as for
 * orbx_profile_pair.  Synchronises. */
ORBX_API int orbx_profile_batch(orbx_ctx* ctx, int n_pairs, const orbx_image* imgs_a, const orbx_image* imgs_b,
                                const orbx_frame_out* out_a, const orbx_frame_out* out_b, float* stage_ms);

/* Debug: copy the internal buffers of the last single-image call to the host:
 * raw pyramid, blurred pyramid (offsets[n] bytes each, reference layout),
 * score map and octave map (h * pitch0 each).  Synchronises the stream. */
ORBX_API int orbx_debug_buffers(orbx_ctx* ctx, uint8_t* h_pyr, uint8_t* h_blur, float* h_vmap, int* h_layer,
                                int* h_total);

/* ---- Learned matching proposal.  No counterpart in the reference, whose only
 * matcher is exact brute force (orbd.cu:1471-1559).
 *
 * An index over a database of descriptors for k = 2 search.  An MLP (256 +-1
 * inputs -> hidden ReLU -> n_clusters logits, BF16 weights, FP32 accumulate,
 * trained on the GPU by this library's own forward and backward kernels on the
 * exact nearest neighbours of training descriptors) picks the n_probe most
 * likely clusters of a Hamming k-majority clustering of the database; those
 * clusters are searched exactly; a query whose top-2 logit margin is below
 * `margin` is answered by exact brute force over the whole database instead.
 * Outputs have the layout of orbx_match_knn2.  ORBX_PROPOSAL_LSH swaps the
 * MLP and the clustering for random-projection buckets (for comparison). */
enum { ORBX_PROPOSAL_MLP = 0, ORBX_PROPOSAL_LSH = 1 };

typedef struct orbx_learned_params {
  int proposal;     /* ORBX_PROPOSAL_* */
  int n_clusters;   /* multiple of 256, <= 4096; LSH: 2^lsh_bits */
  int hidden;       /* multiple of 256 */
  int n_probe;      /* clusters searched per query, 1..8 */
  int kmeans_iters; /* upper bound; stops when fewer than 0.1% of rows move */
  int epochs;
  int batch;        /* training rows per step, multiple of 128 */
  float lr;         /* Adam step size, cosine-decayed over the run */
  float margin;     /* exact fallback below this top-1 minus top-2 logit */
  int lsh_bits;     /* LSH: log2 of the bucket count, 8..12 */
  unsigned long long seed;
  int max_distance; /* exact fallback also when the best reranked distance exceeds this (>= 256: off) */
  int spill;        /* MLP: each database row is listed in its `spill` nearest clusters, 1..16
                       (1, 2: by the int8 matcher; 3..16: by the BF16 GEMM's per-128-centroid
                       top 8, exactly the nearest up to 8) */
  int init;         /* ORBX_INIT_CENTROIDS or ORBX_INIT_RANDOM */
  int synth_train;  /* extra training rows: database rows with random bit flips, exactly labelled */
  float flip_lo;    /* per-row bit-flip probability of those rows, uniform in [flip_lo, flip_hi] */
  float flip_hi;
  int rerank;       /* ORBX_RERANK_TENSOR (int8 tensor cores) or ORBX_RERANK_POPC (XOR-popc) */
  int label_mode;   /* training target: ORBX_LABEL_NEAREST or ORBX_LABEL_LISTED */
} orbx_learned_params;
/* ORBX_LABEL_NEAREST trains on the cluster of each training row's exact nearest
 * database row (cross-entropy); ORBX_LABEL_LISTED on all `spill` clusters that
 * row is listed in, maximising the softmax mass on that set, which is what a
 * probe needs to find it. */
enum { ORBX_LABEL_NEAREST = 0, ORBX_LABEL_LISTED = 1 };
/* Exact rerank of the probed clusters: both forms give the same results. */
enum { ORBX_RERANK_TENSOR = 0, ORBX_RERANK_POPC = 1 };
/* ORBX_INIT_CENTROIDS starts the MLP as nearest-centroid scoring (hidden units
 * relu(x_k) and relu(-x_k), output c = scaled dot product with centroid c), so
 * training refines the clustering's own proposal; needs hidden >= 512. */
enum { ORBX_INIT_CENTROIDS = 0, ORBX_INIT_RANDOM = 1 };

typedef struct orbx_learned_stats {
  int kmeans_iters_run;
  int kmeans_last_moved; /* rows that changed cluster in the last iteration */
  int largest_cluster;
  int epochs_run;
  float loss[64];        /* mean training cross-entropy per epoch */
  float accuracy[64];    /* training top-1 cluster accuracy per epoch */
  float build_ms[4];     /* clustering, labels, training, total */
} orbx_learned_stats;

typedef struct orbx_learned orbx_learned;

ORBX_API int orbx_learned_default_params(orbx_learned_params* p);
/* Clusters d_db (ndb rows of 32 bytes, kept as a copy), labels the d_train rows
 * with the clusters their exact nearest database row is listed in (or only its
 * nearest cluster, per label_mode) and trains the MLP.  Runs on the context's
 * stream and synchronises it. */
ORBX_API int orbx_learned_build(orbx_ctx* ctx, const orbx_learned_params* p, const uint8_t* d_db, int ndb,
                                const uint8_t* d_train, int ntrain, orbx_learned** out);
/* k = 2 search of nq queries; optional d_margin [nq] (top-1 minus top-2 logit)
 * and d_fallback_count (queries sent to exact search: margin below `margin`, or
 * best distance in the probed clusters above `max_distance`).  Asynchronous. */
ORBX_API int orbx_learned_search(orbx_ctx* ctx, orbx_learned* index, const uint8_t* d_q, int nq,
                                 uint32_t* d_dist2, int32_t* d_idx2, float* d_margin, int* d_fallback_count);
/* orbx_learned_search with per-phase device times in h_ms[5]: proposal (MLP or
 * buckets), probe lists, exact rerank, merge, exact fallback.  Synchronises. */
ORBX_API int orbx_learned_profile_search(orbx_ctx* ctx, orbx_learned* index, const uint8_t* d_q, int nq,
                                         uint32_t* d_dist2, int32_t* d_idx2, float* h_ms);
ORBX_API int orbx_learned_set_margin(orbx_learned* index, float margin);
ORBX_API int orbx_learned_set_max_distance(orbx_learned* index, int max_distance);
ORBX_API int orbx_learned_set_rerank(orbx_learned* index, int form); /* ORBX_RERANK_* */
/* (query, database row) pairs the last search's rerank scanned (its probing
 * slots times the rows of their clusters).  Synchronises. */
ORBX_API int orbx_learned_probe_pairs(orbx_ctx* ctx, const orbx_learned* index, unsigned long long* h_pairs);
ORBX_API int orbx_learned_get_stats(const orbx_learned* index, orbx_learned_stats* s);
/* Host copies for checks: cluster of every database row, cluster offsets
 * [n_clusters + 1] and the bf16 weights widened to float (any may be NULL). */
ORBX_API int orbx_learned_export(orbx_ctx* ctx, const orbx_learned* index, int* h_assign, int* h_offsets,
                                 float* h_w1, float* h_b1, float* h_w2, float* h_b2);
/* Training loss and gradients of the current weights on n rows with labels
 * (dW1 [hidden][256], db1, dW2 [n_clusters][hidden], db2), as one training
 * step computes them, copied to the host.  n is a multiple of 128. */
ORBX_API int orbx_learned_gradients(orbx_ctx* ctx, orbx_learned* index, const uint8_t* d_x, const int* d_labels, int n,
                                    float* h_loss, float* h_dw1, float* h_db1, float* h_dw2, float* h_db2);
/* Checkpoint of a built index: parameters, statistics, cluster centroids and
 * the MLP's search weights (bf16 W1, W2; fp32 b1, b2), or the LSH projections,
 * with a hash of the bytes.  Not the database and not the cluster lists.
 * h_buf NULL: only *h_need is set.  cap < *h_need: ORBX_ERR_SIZE.
 * Synchronises the context's stream. */
ORBX_API int orbx_learned_save(orbx_ctx* ctx, const orbx_learned* index, void* h_buf, size_t cap, size_t* h_need);
/* An index from a checkpoint over d_db (the database it was built on, or
 * another one), without clustering or training: each row is listed under its
 * `spill` nearest saved centroids (chosen as orbx_learned_build chooses them),
 * or under its LSH bucket.  Over the same database the loaded index searches
 * exactly like the saved one.  A checkpoint with a wrong magic, version, size
 * or hash, or invalid parameters, returns ORBX_ERR_ARG before any device work.
 * The fp32 master weights stay behind, so orbx_learned_gradients works on a
 * loaded index but no training continues from it.  Synchronises. */
ORBX_API int orbx_learned_load(orbx_ctx* ctx, const void* h_buf, size_t bytes, const uint8_t* d_db, int ndb,
                               orbx_learned** out);
ORBX_API int orbx_learned_get_params(const orbx_learned* index, orbx_learned_params* p);
ORBX_API int orbx_learned_destroy(orbx_learned* index);

/* The BF16 tensor-core GEMM used by the MLP: C = A * B^T with A [M][K] and
 * B [N][K] row-major bf16; M % 128 == 0, N % 256 == 0, K % (64 * splits) == 0.
 * mode 0: fp32 C (+ bias; with splits > 1, splits partial sums [splits][M][N]
 * and no bias); 1: bf16 relu(C + bias); 2: bf16 C where aux [M][N] > 0;
 * 3: bf16 C + bias; 4: per row and 128 columns the 8 largest C + bias as
 * packed keys, uint32 [M][N / 128][8]; 5: per row the 8 largest C + bias of
 * each of L column sets, uint32 [M][L][8] with L = 4 when N / 256 is even, else
 * 2 (set 2p + h: columns 256 t + 128 h + c, c < 128, for the tiles t of the
 * p-th half of the N / 256 tiles, or of all of them when L = 2).  Keys are the
 * logit's order-preserving bits with the low 12 replaced by 4095 - column, in
 * descending order; N <= 4096 for modes 4 and 5.  Asynchronous. */
ORBX_API int orbx_gemm_bf16(orbx_ctx* ctx, const void* d_a, const void* d_b, int M, int N, int K, const float* d_bias,
                            int mode, int splits, void* d_c, const void* d_aux);

/* Host self-check of the float rounding of (double)pi - r used by the angle
 * kernel (orbd.cu:995), over every float r with bits in [lo_bits, hi_bits).
 * Returns the number of mismatches. */
ORBX_API long long orbx_selftest_pi_minus(uint32_t lo_bits, uint32_t hi_bits);

#ifdef __cplusplus
}
#endif
#endif /* ORBX_H */
