// Persistent batch kernel (orbx_persist.cu): work-item run table and launch arguments.
#pragma once
#include <vector>

#include "orbx_internal.cuh"

namespace orbx {

enum : int { kStagePyr = 0, kStageDet = 1, kStageNms = 2, kStageDesc = 3, kStageMatch = 4, kNumStages = 5 };

// A run of consecutive tickets: every item of one stage of one frame (for the
// match stage, frame = frame A of the pair).
struct PersistRun {
  int stage;
  int frame;
  int first;  // local index (within the stage and frame) of the run's first ticket
};

// Row-level dependencies (optional): per frame, the offsets in rows_done of
// its counters of finished pyramid tiles per (octave, tile row) and of
// finished detect tiles per tile row.
struct PersistRows {
  int pyr[kMaxOctaves];
  int det;
};

// One work item, packed: stage << 56 | frame << 32 | index within the stage and frame.
__host__ __device__ inline unsigned long long persist_item(int stage, int frame, int local) {
  return ((unsigned long long)stage << 56) | ((unsigned long long)frame << 32) | (unsigned)local;
}

struct PersistArgs {
  Batch b;
  const unsigned long long* items;  // [total tickets] packed items in claim order
  int run_base_host_total;   // total tickets
  const int* desc_base;      // [n_frames + 1] prefix of describe slices per frame
  int* done;                 // [4][n_frames] completed items per (stage, frame); zero at launch
  unsigned int* item_counter;  // zero at launch
  const MatchJob* jobs;      // one per pair
  int blocks_per_job;        // match items per pair
  // optional: level-0 images arrive during the launch in bands of band_rows
  // rows; upload_flags[f] = bands of frame f already copied (written by the
  // copy stream after each band), and pyramid tiles wait for the rows they read
  const int* upload_flags;
  int band_rows;
  // optional: row-level dependencies.  A detect tile row then waits only for
  // the pyramid tile rows it reads, so a frame's detection overlaps its
  // pyramid row by row (NMS strips still wait for the whole frame).
  const PersistRows* rows;  // [n_frames], null: per-frame dependencies only
  int* rows_done;           // counters, zero at launch
};

// Level-0 pixels per describe slice: a frame's keypoints are split into
// ceil(w * h / kDescSlicePixels) slices (at most one per 8 keypoints of its
// cap), about one keypoint per warp at the synthetic images' density.
constexpr int kDescSlicePixels = 8192;

int persist_blocks_per_sm(int wta_k);
cudaError_t launch_batch_persistent(const PersistArgs& p, int blocks, cudaStream_t s);
cudaError_t launch_wait_selftest(const int* ctr, int need, int* err, long long wait_cycles, cudaStream_t s);
void build_persist_runs(int nf, int group, const int* pyr_n, const int* det_n, const int* nms_n, const int* desc_n,
                        int match_per_pair, std::vector<PersistRun>* runs, std::vector<int>* run_base);
// The run table with row-level dependencies: items ordered by the level-0 row
// from which they can run, stage and frame.  Fills the per-frame counter
// offsets and returns the number of row counters.
int build_persist_runs_rows(const std::vector<Frame>& frames, const int* desc_n, int match_per_pair,
                            std::vector<PersistRun>* runs, std::vector<int>* run_base,
                            std::vector<PersistRows>* rows);

}  // namespace orbx
