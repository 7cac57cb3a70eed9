// orb::Orbor -- the CUDA-ORB host class (orb.h:9-78 of the reference), same
// public interface and defaults, implemented on the sm_100a orbx library
// (orbx.h).  Errors print and exit(-1), as in the reference.
#pragma once
#include <cuda_runtime.h>

#include "cuda_utils.h"
#include "orb_structures.h"

struct orbx_ctx;

namespace orb {

class Orbor {
 public:
  Orbor();
  ~Orbor();

  /* Initialization (orb.h:18-19) */
  void init(int _noctaves = 5, int _edge_threshold = 31, int _wta_k = 2, ScoreType _score_type = HARRIS_SCORE,
            int _patch_size = 31, int _fast_threshold = 20, int _retain_topn = -1, int _max_pts = 1000);

  /* Detect keypoints and compute descriptors.  image: device buffer, row pitch
   * whp0.z.  *desc_addr is freed and re-allocated with num_pts * 32 bytes, as the
   * reference does (orb.cpp:84-90). */
  void detectAndCompute(unsigned char* image, OrbData& result, int3 whp0, void** desc_addr = NULL,
                        const bool compute_desc = true);

  /* Match result1 against result2: writes result1 match / distance. */
  void match(OrbData& result1, OrbData& result2, unsigned char* desc1, unsigned char* desc2);

  /* Allocate / free keypoint arrays. */
  void initOrbData(OrbData& data, const int max_pts, const bool host, const bool dev);
  void freeOrbData(OrbData& data);

 private:
  orbx_ctx* ctx_ = nullptr;
  int max_pts_ = 1000;
  int* d_counts_ = nullptr;          // [0]: detect count, [1], [2]: match counts
  unsigned char* d_desc_work_ = nullptr;  // max_pts * 32 descriptor staging
  int desc_work_cap_ = 0;
};

}  // namespace orb
