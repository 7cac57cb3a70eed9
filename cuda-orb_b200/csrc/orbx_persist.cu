// Batched frame pairs in one persistent launch with a device work queue.
//
// The reference runs one Orbor::detectAndCompute / Orbor::match call at a time
// (orb.cpp:57-113).  Here every stage of every frame of a batch is a list of
// work items: pyramid + blur tiles, detect tiles, NMS strips, describe slices
// (a share of one frame's keypoints) and match blocks (a share of one pair's
// k = 2 search).  A host-built run table orders the items; resident blocks
// claim items from a global counter in that order and run the same stage
// bodies as the five-launch form (orbx_stages.cuh), so results are identical.
//
// Dependencies are per frame: an item of stage k for frame f waits until every
// item of stage k - 1 for f has finished (a completion counter per stage and
// frame, released with a fence and read with an acquire).  The run table puts
// every item after all items it depends on, so the item with the smallest
// unfinished ticket never waits: progress needs only one resident block, and
// blocks that are not resident hold no ticket.  Each wait is bounded by
// wait_cycles of clock64(); on expiry it sets kErrStageTimeout, later waits
// stop waiting, and the kernel finishes (the host reports ORBX_ERR_TIMEOUT).
//
// The run table is built in "waves" of G frames: wave w holds the pyramid
// tiles of frame group w, the detect tiles of group w - 1, the NMS strips of
// group w - 2, the describe slices of group w - 3 and the match blocks of the
// pairs of group w - 4.  G = all frames gives stage-major order; smaller G
// overlaps the memory-bound pyramid of later frames with the ALU-bound detect
// of earlier ones.  G and the grid are chosen by the autotuner.
#include <algorithm>

#include "orbx_stages.cuh"
#include "orbx_persist.cuh"

namespace orbx {

union PersistSmem {
  PyrSmem<kPyrTW, kPyrTH> pyr;
  DetSmem det;
  NmsSmem nms;
  struct {
    int umax[32];
  } desc;
  struct {
    uint4 db[kMChunk * 2];
    unsigned int last;
  } match;
};

constexpr int kPersistThreads = 256;
static_assert(kPersistThreads == kPyrThreads, "pyramid tiles assume kPyrThreads threads per block");

// One thread waits until *ctr >= need (acquire), bounded by wait_cycles.
// After one wait has given up, later waits return at once so the launch drains.
__device__ __forceinline__ void wait_counter(const int* ctr, int need, int* err, long long wait_cycles) {
  const long long t0 = clock64();
  for (;;) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
    if (v >= need) break;
    if (*(volatile int*)err & kErrStageTimeout) break;
    if (clock64() - t0 > wait_cycles) {
      atomicOr(err, kErrStageTimeout);
      break;
    }
    __nanosleep(64);
  }
}

// Thread 0 waits; the block then proceeds together.
__device__ __forceinline__ void stage_wait(const int* ctr, int need, int* err, long long wait_cycles) {
  if (threadIdx.x == 0) wait_counter(ctr, need, err, wait_cycles);
  __syncthreads();
}

__device__ __forceinline__ void stage_done(int* ctr, int* ctr2 = nullptr) {
  __syncthreads();  // every thread's stores of this item precede the release
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1);
    if (ctr2) atomicAdd(ctr2, 1);
  }
}

// Octave and tile row of pyramid tile `local` of frame F.
__device__ __forceinline__ void pyr_tile_pos(const Frame& F, int local, int* o_out, int* row_out) {
  int o = 0;
  while (o + 1 < F.n_oct && local >= F.pyr_tile_base[o + 1]) o++;
  *o_out = o;
  *row_out = (local - F.pyr_tile_base[o]) / F.pyr_tiles_x[o];
}

// Thread 0: waits for every pyramid tile row that detect tile row `ty` reads.
// At octave o the tile stages rows (32 ty >> o) - 4 .. ((32 ty + 31) >> o) + 4
// with the linear addressing of the pyramid, so one more row on each side (a
// column past the edge is the neighbouring row), and rows outside the octave
// are the last rows of octave o - 1 or the first rows of octave o + 1 (the
// guard before octave 0 and after the last octave needs nothing).
__device__ __forceinline__ void wait_detect_row_deps(const Frame& F, const PersistRows& R, const int* rows_done,
                                                     int ty, int* err, long long wait_cycles) {
  for (int o = 0; o < F.n_oct; o++) {
    const int r_lo = ((kDetTH * ty) >> o) - 4 - 1;
    const int r_hi = ((kDetTH * ty + kDetTH - 1) >> o) + 4 + 1;
    const int lo = max(r_lo, 0), hi = min(r_hi, F.oh[o] - 1);
    for (int t = lo / kPyrTH; lo <= hi && t <= hi / kPyrTH; t++)
      wait_counter(rows_done + R.pyr[o] + t, F.pyr_tiles_x[o], err, wait_cycles);
    if (r_lo < 0 && o > 0)
      for (int t = max(0, F.pyr_tiles_y[o - 1] - 2); t < F.pyr_tiles_y[o - 1]; t++)
        wait_counter(rows_done + R.pyr[o - 1] + t, F.pyr_tiles_x[o - 1], err, wait_cycles);
    if (r_hi >= F.oh[o] && o + 1 < F.n_oct)
      for (int t = 0; t < min(2, F.pyr_tiles_y[o + 1]); t++)
        wait_counter(rows_done + R.pyr[o + 1] + t, F.pyr_tiles_x[o + 1], err, wait_cycles);
  }
}

// Level-0 rows [0, n) that pyramid tile `local` of frame F reads: octave o
// samples row y << o for the tile's rows and its 3-row reflected halo.
__device__ __forceinline__ int pyr_tile_rows(const Frame& F, int local) {
  int o = 0;
  while (o + 1 < F.n_oct && local >= F.pyr_tile_base[o + 1]) o++;
  const int lt = local - F.pyr_tile_base[o];
  const int y0 = (lt / F.pyr_tiles_x[o]) * kPyrTH;
  const int ylast = min(y0 + kPyrTH - 1 + 3, F.oh[o] - 1);
  return (ylast << o) + 1;
}


template <int WTA>
__global__ void __launch_bounds__(kPersistThreads, 4) k_batch_persistent(PersistArgs p) {
  __shared__ PersistSmem sm;
  __shared__ int s_item;
  const Batch& b = p.b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int total = p.run_base_host_total;
  // Thread 0 claims the next ticket while the block works on the current one
  // (its result is only stored at the end of the item), so the claim's
  // latency overlaps the work.  A claimed ticket waits only for its own
  // block's current item, which has a smaller ticket, so the smallest
  // unfinished ticket still always runs.
  if (threadIdx.x == 0) s_item = (int)atomicAdd(p.item_counter, 1u);
  for (;;) {
    __syncthreads();  // the previous item is done with shared memory; s_item holds the ticket
    const int t = s_item;
    __syncthreads();  // every thread has read it before thread 0 may overwrite it
    if (t >= total) break;
    int next = 0;
    if (threadIdx.x == 0) next = (int)atomicAdd(p.item_counter, 1u);
    const unsigned long long it = __ldg(p.items + t);
    const int stage = (int)(it >> 56);
    const int f = (int)((it >> 32) & 0xFFFFFFu);
    const int local = (int)(unsigned)it;
    int* done = p.done;
    const int nf = b.n_frames;
    switch (stage) {
      case kStagePyr: {
        if (p.upload_flags) {
          const int rows = pyr_tile_rows(b.frames[f], local);
          stage_wait(p.upload_flags + f, (rows + p.band_rows - 1) / p.band_rows, b.err, b.wait_cycles);
          pyr_tile<true>(b, __ldg(b.pyr_base + f) + local, sm.pyr);
        } else {
          pyr_tile<false>(b, __ldg(b.pyr_base + f) + local, sm.pyr);
        }
        int* row_ctr = nullptr;
        if (p.rows) {
          int o, tr;
          pyr_tile_pos(b.frames[f], local, &o, &tr);
          row_ctr = p.rows_done + p.rows[f].pyr[o] + tr;
        }
        stage_done(done + 0 * nf + f, row_ctr);
        break;
      }
      case kStageDet: {
        const Frame& F = b.frames[f];
        const int ty = local / F.det_tiles_x;
        if (p.rows) {
          if (threadIdx.x == 0) wait_detect_row_deps(F, p.rows[f], p.rows_done, ty, b.err, b.wait_cycles);
          __syncthreads();
        } else {
          stage_wait(done + 0 * nf + f, __ldg(b.pyr_base + f + 1) - __ldg(b.pyr_base + f), b.err, b.wait_cycles);
        }
        det_tile<true>(b, __ldg(b.det_base + f) + local, sm.det);
        stage_done(done + 1 * nf + f, p.rows ? p.rows_done + p.rows[f].det + ty : nullptr);
        break;
      }
      case kStageNms:
        // per frame in both modes: the strips' look-back needs them to start in
        // order, and the top strips read detect rows that wait for the bottom
        // of the octave before (the window's row -1 is that octave's last row)
        stage_wait(done + 1 * nf + f, __ldg(b.det_base + f + 1) - __ldg(b.det_base + f), b.err, b.wait_cycles);
        nms_strip<true>(b, __ldg(b.nms_base + f) + local, sm.nms);
        stage_done(done + 2 * nf + f);
        break;
      case kStageDesc: {
        // with row-level dependencies, NMS completion does not imply every
        // pyramid tile: the patches may read rows no NMS strip waited for
        if (p.rows && threadIdx.x == 0)
          wait_counter(done + 0 * nf + f, __ldg(b.pyr_base + f + 1) - __ldg(b.pyr_base + f), b.err, b.wait_cycles);
        stage_wait(done + 2 * nf + f, __ldg(b.nms_base + f + 1) - __ldg(b.nms_base + f), b.err, b.wait_cycles);
        if (threadIdx.x < b.half_k + 1) sm.desc.umax[threadIdx.x] = __ldg(b.umax + threadIdx.x);
        __syncthreads();
        const Frame& F = b.frames[f];
        const int n = __ldcg(F.count);
        const int slices = __ldg(p.desc_base + f + 1) - __ldg(p.desc_base + f);
        const int k0 = (int)((long long)n * local / slices);
        const int k1 = (int)((long long)n * (local + 1) / slices);
        constexpr int PSTEP = (WTA == 3) ? 12 : 16;
        float px[PSTEP], py[PSTEP];
        load_pattern<WTA>(b, lane, px, py);
        for (int k = k0 + warp; k < k1; k += kPersistThreads / 32)
          describe_keypoint<WTA, true>(b, F, k, px, py, sm.desc.umax, lane);
        stage_done(done + 3 * nf + f);
        break;
      }
      default: {  // kStageMatch: run.frame is frame A of pair f / 2
        const int fa = f, fb = f + 1;
        stage_wait(done + 3 * nf + fa, __ldg(p.desc_base + fa + 1) - __ldg(p.desc_base + fa), b.err,
                   b.wait_cycles);
        stage_wait(done + 3 * nf + fb, __ldg(p.desc_base + fb + 1) - __ldg(p.desc_base + fb), b.err,
                   b.wait_cycles);
        const MatchJob& J = p.jobs[f >> 1];
        match_popc_block<kPersistThreads, true>(J.args, J.work, local, p.blocks_per_job, sm.match.db,
                                                sm.match.last);
        break;
      }
    }
    if (threadIdx.x == 0) s_item = next;  // published to the block by the barrier at the loop's top
  }
}

int persist_blocks_per_sm(int wta_k) {
  int n = 0;
  cudaError_t e;
  if (wta_k == 3)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_persistent<3>, kPersistThreads, 0);
  else if (wta_k == 4)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_persistent<4>, kPersistThreads, 0);
  else
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_persistent<2>, kPersistThreads, 0);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

cudaError_t launch_batch_persistent(const PersistArgs& p, int blocks, cudaStream_t s) {
  if (blocks <= 0 || p.run_base_host_total <= 0) return cudaSuccess;
  if (p.b.wta_k == 3)
    k_batch_persistent<3><<<blocks, kPersistThreads, 0, s>>>(p);
  else if (p.b.wta_k == 4)
    k_batch_persistent<4><<<blocks, kPersistThreads, 0, s>>>(p);
  else
    k_batch_persistent<2><<<blocks, kPersistThreads, 0, s>>>(p);
  return cudaGetLastError();
}

// A wait on a counter that nothing increments: the bounded-wait path of the
// persistent kernel, run on its own so that a test can make it expire.
__global__ void k_wait_selftest(const int* ctr, int need, int* err, long long wait_cycles) {
  stage_wait(ctr, need, err, wait_cycles);
}

cudaError_t launch_wait_selftest(const int* ctr, int need, int* err, long long wait_cycles, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(ctr, need, err, wait_cycles);
  return cudaGetLastError();
}

// Host side: the run table in waves of `group` frames (pairs kept whole).
void build_persist_runs(int nf, int group, const int* pyr_n, const int* det_n, const int* nms_n,
                        const int* desc_n, int match_per_pair, std::vector<PersistRun>* runs,
                        std::vector<int>* run_base) {
  runs->clear();
  run_base->clear();
  if (group < 2) group = 2;
  group += group & 1;
  const int groups = (nf + group - 1) / group;
  int acc = 0;
  auto add = [&](int stage, int frame, int count) {
    if (count <= 0) return;
    runs->push_back(PersistRun{stage, frame, 0});
    run_base->push_back(acc);
    acc += count;
  };
  for (int w = 0; w < groups + kNumStages - 1; w++) {
    for (int k = 0; k < kNumStages; k++) {
      const int g = w - k;
      if (g < 0 || g >= groups) continue;
      const int f0 = g * group, f1 = std::min(nf, f0 + group);
      for (int f = f0; f < f1; f++) {
        switch (k) {
          case kStagePyr: add(k, f, pyr_n[f]); break;
          case kStageDet: add(k, f, det_n[f]); break;
          case kStageNms: add(k, f, nms_n[f]); break;
          case kStageDesc: add(k, f, desc_n[f]); break;
          default:
            if ((f & 1) == 0) add(k, f, match_per_pair);
        }
      }
    }
  }
  run_base->push_back(acc);
}

// Host side: the run table with row-level dependencies.  Each item gets the
// level-0 row from which it can run (a pyramid tile row its start row, a
// detect tile row the largest of its pyramid dependencies' keys, the NMS
// strips of a frame the largest key of its detect rows); items sort by (key,
// stage, frame, index), which puts every item after its dependencies and the
// NMS strips of a frame in order.  Consecutive items of one stage and frame
// form a run.
int build_persist_runs_rows(const std::vector<Frame>& frames, const int* desc_n, int match_per_pair,
                            std::vector<PersistRun>* runs, std::vector<int>* run_base,
                            std::vector<PersistRows>* rows) {
  struct Item {
    long long key;
    int stage, frame, local;
  };
  const int nf = (int)frames.size();
  std::vector<Item> items;
  rows->assign(nf, PersistRows{});
  int n_rows = 0;
  const long long kEnd = 1ll << 40;
  for (int f = 0; f < nf; f++) {
    const Frame& F = frames[f];
    PersistRows& R = (*rows)[f];
    std::vector<std::vector<long long>> pkey(F.n_oct);
    for (int o = 0; o < F.n_oct; o++) {
      R.pyr[o] = n_rows;
      n_rows += F.pyr_tiles_y[o];
      pkey[o].resize(F.pyr_tiles_y[o]);
      for (int t = 0; t < F.pyr_tiles_y[o]; t++) {
        pkey[o][t] = (long long)(kPyrTH * t) << o;
        for (int x = 0; x < F.pyr_tiles_x[o]; x++)
          items.push_back({pkey[o][t], kStagePyr, f, F.pyr_tile_base[o] + t * F.pyr_tiles_x[o] + x});
      }
    }
    R.det = n_rows;
    n_rows += F.det_tiles_y;
    std::vector<long long> dkey(F.det_tiles_y, 0);
    for (int ty = 0; ty < F.det_tiles_y; ty++) {
      long long k = 0;
      for (int o = 0; o < F.n_oct; o++) {  // the same rows as wait_detect_row_deps
        const int r_lo = ((kDetTH * ty) >> o) - 4 - 1;
        const int r_hi = ((kDetTH * ty + kDetTH - 1) >> o) + 4 + 1;
        const int lo = std::max(r_lo, 0), hi = std::min(r_hi, F.oh[o] - 1);
        for (int t = lo / kPyrTH; lo <= hi && t <= hi / kPyrTH; t++) k = std::max(k, pkey[o][t]);
        if (r_lo < 0 && o > 0) k = std::max(k, pkey[o - 1][F.pyr_tiles_y[o - 1] - 1]);
        if (r_hi >= F.oh[o] && o + 1 < F.n_oct) k = std::max(k, pkey[o + 1][std::min(1, F.pyr_tiles_y[o + 1] - 1)]);
      }
      dkey[ty] = k;
      for (int x = 0; x < F.det_tiles_x; x++) items.push_back({k, kStageDet, f, ty * F.det_tiles_x + x});
    }
    long long nkey = 0;  // NMS strips wait for every detect tile of the frame
    for (long long k : dkey) nkey = std::max(nkey, k);
    for (int st = 0; st < F.nms_strips; st++) items.push_back({nkey, kStageNms, f, st});
    for (int d = 0; d < desc_n[f]; d++) items.push_back({kEnd, kStageDesc, f, d});
    if ((f & 1) == 0)
      for (int m = 0; m < match_per_pair; m++) items.push_back({kEnd, kStageMatch, f, m});
  }
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
    if (a.key != b.key) return a.key < b.key;
    if (a.stage != b.stage) return a.stage < b.stage;
    if (a.frame != b.frame) return a.frame < b.frame;
    return a.local < b.local;
  });
  runs->clear();
  run_base->clear();
  for (size_t i = 0; i < items.size(); i++) {
    const Item& it = items[i];
    const bool extend = !runs->empty() && runs->back().stage == it.stage && runs->back().frame == it.frame &&
                        runs->back().first + (int)(i - (size_t)run_base->back()) == it.local;
    if (!extend) {
      runs->push_back(PersistRun{it.stage, it.frame, it.local});
      run_base->push_back((int)i);
    }
  }
  run_base->push_back((int)items.size());
  return n_rows;
}

}  // namespace orbx
