// Data types of the CUDA-ORB C++ API (orb_structures.h:1-36 of the reference),
// binary-identical so that existing callers and their cudaMemcpy2D field copies
// keep working.  orb::OrbPoint has the layout of orbx_point (orbx.h).
#pragma once

namespace orb {

// One keypoint: level-0 coordinates, pyramid level, score, angle (radians),
// and the match index / Hamming distance written by Orbor::match.
struct OrbPoint {
  int x;
  int y;
  int octave;
  float score;
  float angle;
  int match;
  int distance;
};

// Keypoints of one image: count, optional host copy, device array.
struct OrbData {
  int num_pts;
  OrbPoint* h_data;
  OrbPoint* d_data;
};

// Keypoint ranking score.
enum ScoreType { HARRIS_SCORE = 0, FAST_SCORE = 1 };

}  // namespace orb
