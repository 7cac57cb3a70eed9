// orb::Orbor and the orbd.h free functions (the reference's C++ API,
// orb.h:9-78 and orbd.h:10-48) implemented on the orbx C ABI.  Behaviour kept
// from the reference: Orbor::detectAndCompute returns num_pts on the host and
// (re)allocates the caller's descriptor buffer with num_pts * 32 bytes
// (orb.cpp:84-90); host copies fill the first five OrbPoint fields after
// detection (orb.cpp:95-100) and match/distance after matching
// (orb.cpp:107-112); any failure prints and exits (cuda_utils.h:18-38).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "../../include/orb.h"
#include "../../include/orbd.h"
#include "../../include/orbx.h"
#include "orbx_internal.cuh"

static_assert(sizeof(orb::OrbPoint) == sizeof(orbx_point), "OrbPoint layout");

static void orbx_check(int status, const char* what) {
  if (status != ORBX_OK) {
    std::fprintf(stderr, "orbx error in %s: %s\n", what, orbx_status_string(status));
    std::exit(-1);
  }
}

namespace orb {

Orbor::Orbor() {}

Orbor::~Orbor() {
  if (ctx_) orbx_destroy(ctx_);
  if (d_counts_) cudaFree(d_counts_);
  if (d_desc_work_) cudaFree(d_desc_work_);
}

void Orbor::init(int _noctaves, int _edge_threshold, int _wta_k, ScoreType _score_type, int _patch_size,
                 int _fast_threshold, int _retain_topn, int _max_pts) {
  if (!ctx_) {
    int dev = 0;
    CHECK(cudaGetDevice(&dev));
    orbx_check(orbx_create(&ctx_, dev), "Orbor::init");
    CHECK(cudaMalloc((void**)&d_counts_, 4 * sizeof(int)));
  }
  orbx_params p;
  p.noctaves = _noctaves;
  p.edge_threshold = _edge_threshold;
  p.wta_k = _wta_k;
  p.score_type = (int)_score_type;
  p.patch_size = _patch_size;
  p.fast_threshold = _fast_threshold;
  p.retain_topn = _retain_topn;
  p.max_pts = _max_pts;
  orbx_check(orbx_init(ctx_, &p), "Orbor::init");
  max_pts_ = _max_pts;
  if (desc_work_cap_ < _max_pts) {
    if (d_desc_work_) CHECK(cudaFree(d_desc_work_));
    CHECK(cudaMalloc((void**)&d_desc_work_, (size_t)_max_pts * 32));
    desc_work_cap_ = _max_pts;
  }
}

void Orbor::detectAndCompute(unsigned char* image, OrbData& result, int3 whp0, void** desc_addr,
                             const bool compute_desc) {
  if (!ctx_) orbx_check(ORBX_ERR_STATE, "Orbor::detectAndCompute");
  orbx_check(orbx_detect_and_compute(ctx_, image, whp0.x, whp0.y, whp0.z, (orbx_point*)result.d_data,
                                     d_desc_work_, d_counts_, compute_desc ? 1 : 0),
             "Orbor::detectAndCompute");
  cudaStream_t s = (cudaStream_t)orbx_get_stream(ctx_);
  int n = 0;
  CHECK(cudaMemcpyAsync(&n, d_counts_, sizeof(int), cudaMemcpyDeviceToHost, s));
  orbx_check(orbx_sync(ctx_), "Orbor::detectAndCompute");
  result.num_pts = n;
  if (compute_desc && n > 0 && desc_addr) {
    if (*desc_addr) CHECK(cudaFree(*desc_addr));
    CHECK(cudaMalloc(desc_addr, (size_t)n * 32));
    CHECK(cudaMemcpy(*desc_addr, d_desc_work_, (size_t)n * 32, cudaMemcpyDeviceToDevice));
  }
  // x, y, octave, score, angle of each host entry (orb.cpp:95-100), as one packed copy
  if (result.h_data && n > 0)
    orbx_check(orbx_download_points(ctx_, (const orbx_point*)result.d_data, n, (orbx_point*)result.h_data,
                                    ORBX_FIELDS_KEYPOINT),
               "Orbor::detectAndCompute");
}

// hMatch on a given context: the counts are host values (orbd.cu:1788-1790),
// staged into two device ints for the device-count ABI.
static void match_on(orbx_ctx* c, int* d_cnt, OrbData& result1, OrbData& result2, unsigned char* desc1,
                     unsigned char* desc2, const char* what) {
  const int n[2] = {result1.num_pts, result2.num_pts};
  CHECK(cudaMemcpy(d_cnt, n, sizeof(n), cudaMemcpyHostToDevice));
  orbx_check(orbx_match(c, (orbx_point*)result1.d_data, d_cnt, desc1, d_cnt + 1, desc2, n[0], n[1],
                        ORBX_MATCH_POPC),
             what);
  orbx_check(orbx_sync(c), what);
}

void Orbor::match(OrbData& result1, OrbData& result2, unsigned char* desc1, unsigned char* desc2) {
  if (!ctx_) orbx_check(ORBX_ERR_STATE, "Orbor::match");
  match_on(ctx_, d_counts_ + 1, result1, result2, desc1, desc2, "Orbor::match");
  // match, distance of each host entry (orb.cpp:108-111), as one packed copy
  if (result1.h_data && result1.num_pts > 0)
    orbx_check(orbx_download_points(ctx_, (const orbx_point*)result1.d_data, result1.num_pts,
                                    (orbx_point*)result1.h_data, ORBX_FIELDS_MATCH),
               "Orbor::match");
}

void Orbor::initOrbData(OrbData& data, const int max_pts, const bool host, const bool dev) {
  data.num_pts = 0;
  const size_t size = sizeof(OrbPoint) * (size_t)max_pts;
  data.h_data = host ? (OrbPoint*)std::malloc(size) : NULL;
  data.d_data = NULL;
  if (dev) CHECK(cudaMalloc((void**)&data.d_data, size));
}

void Orbor::freeOrbData(OrbData& data) {
  if (data.d_data) CHECK(cudaFree(data.d_data));
  if (data.h_data) std::free(data.h_data);
  data.d_data = NULL;
  data.h_data = NULL;
  data.num_pts = 0;
}

// ---------------------------------------------------------------------------
// orbd.h: one process-wide context, as the reference's tables are process-wide
// (orbd.cu:32-41).
// ---------------------------------------------------------------------------
namespace {
std::mutex g_mu;
orbx_ctx* g_ctx = nullptr;
orbx_params g_params;
int* g_counter = nullptr;  // [0] point counter (getPointCounter), [1..3] scratch counts

orbx_ctx* lower_ctx() {
  if (!g_ctx) {
    int dev = 0;
    CHECK(cudaGetDevice(&dev));
    orbx_check(orbx_create(&g_ctx, dev), "orbd");
    orbx_default_params(&g_params);
    CHECK(cudaMalloc((void**)&g_counter, 4 * sizeof(int)));
    CHECK(cudaMemset(g_counter, 0, 4 * sizeof(int)));
    orbx_check(orbx_init(g_ctx, &g_params), "orbd");
  }
  return g_ctx;
}

void reinit() { orbx_check(orbx_init(lower_ctx(), &g_params), "orbd"); }
}  // namespace

void setMaxNumPoints(const int num) {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
  g_params.max_pts = num;
  reinit();
}

void getPointCounter(void** addr) {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
  *addr = (void*)g_counter;
}

void setFastThresholdLUT(int fast_threshold) {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
  g_params.fast_threshold = fast_threshold;
  reinit();
}

void setUmax(const int patch_size) {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
  g_params.patch_size = patch_size;
  reinit();
}

void setPattern(const int patch_size, const int wta_k) {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
  g_params.patch_size = patch_size;
  g_params.wta_k = wta_k;
  reinit();
}

// The Gaussian weights and the Harris scale are fixed values computed at init.
void setGaussianKernel() {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
}

void setScaleSqSq() {
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
}

// The FAST ring offsets follow from each call's pyramid pitches.
void makeOffsets(int* pitchs, int noctaves) {
  (void)pitchs;
  (void)noctaves;
  std::lock_guard<std::mutex> lk(g_mu);
  lower_ctx();
}

void hFastDectectWithNMS(unsigned char* image, unsigned char* octave_images, float* vmem, OrbData& result, int* oszp,
                         int noctaves, int threshold, int border, bool harris_score) {
  std::lock_guard<std::mutex> lk(g_mu);
  orbx_ctx* c = lower_ctx();
  orbx_check(orbx::lower_detect(c, image, octave_images, vmem, (orbx_point*)result.d_data, g_counter, oszp,
                                noctaves, threshold, border, harris_score),
             "hFastDectectWithNMS");
  orbx_check(orbx_sync(c), "hFastDectectWithNMS");
}

void hComputeAngle(unsigned char* octave_images, OrbData& result, int* oszp, int noctaves, int patch_size) {
  std::lock_guard<std::mutex> lk(g_mu);
  orbx_ctx* c = lower_ctx();
  orbx_check(orbx::lower_angle(c, octave_images, (orbx_point*)result.d_data, result.num_pts, oszp, noctaves,
                               patch_size, g_counter + 1),
             "hComputeAngle");
  orbx_check(orbx_sync(c), "hComputeAngle");
}

void hGassianBlur(unsigned char* octave_images, int* oszp, int noctaves) {
  std::lock_guard<std::mutex> lk(g_mu);
  orbx_ctx* c = lower_ctx();
  orbx_check(orbx::lower_blur(c, octave_images, oszp, noctaves, g_counter + 1), "hGassianBlur");
  orbx_check(orbx_sync(c), "hGassianBlur");
}

void hDescribe(unsigned char* octave_images, OrbData& result, unsigned char* desc, int wta_k, int noctaves) {
  // The reference reads the octave layout set by hComputeAngle (angle_param,
  // orbd.cu:1719); here the layout is the one of the last pyramid call.
  std::lock_guard<std::mutex> lk(g_mu);
  orbx_ctx* c = lower_ctx();
  int oszp[5 * 5 + 1];
  orbx_check(orbx::lower_last_layout(c, oszp, noctaves), "hDescribe");
  orbx_check(orbx::lower_describe(c, octave_images, (orbx_point*)result.d_data, result.num_pts, desc, wta_k, oszp,
                                  noctaves, g_counter + 1),
             "hDescribe");
  orbx_check(orbx_sync(c), "hDescribe");
}

void hMatch(OrbData& result1, OrbData& result2, unsigned char* desc1, unsigned char* desc2) {
  std::lock_guard<std::mutex> lk(g_mu);
  orbx_ctx* c = lower_ctx();
  match_on(c, g_counter + 2, result1, result2, desc1, desc2, "hMatch");
}

}  // namespace orb
