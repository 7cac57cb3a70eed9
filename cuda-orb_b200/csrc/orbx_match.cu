// Brute-force k = 2 Hamming matching, XOR + popcount form, for sm_100a.
//
// gHammingMatch (orbd.cu:1471-1559) gives each query a 32-thread block that
// re-reads the whole train set.  Here a 128-thread block owns 128 queries (one
// per thread, held in registers) and streams a slice of the train set through
// shared memory, so each train row is read once per 128 queries.  When there
// are few queries the train set is split across blocks; the last block to
// finish a query tile merges the partial results.  The running top-2 is kept
// as two 32-bit keys (distance << 22 | index), which orders by distance, then
// index, and needs three integer min/max per pair.
#include "orbx_device.cuh"
#include "orbx_internal.cuh"

namespace orbx {

constexpr int kMQ = 128;      // queries per block
constexpr int kMChunk = 512;  // train rows per shared-memory chunk (16 KB)
constexpr int kIdxBits = kIdxBitsShared;
constexpr uint32_t kNoKey = kNoKeyShared;

__device__ __forceinline__ void top2_push(uint32_t& k1, uint32_t& k2, uint32_t key) { top2_push_shared(k1, k2, key); }
__device__ __forceinline__ void finish_query(const MatchArgs& a, int q, uint32_t k1, uint32_t k2) {
  finish_query_shared(a, q, k1, k2);
}

// One block's share of a k = 2 search; bid / nblk replace blockIdx.x / gridDim.x
// so that a batch launch can run one search per blockIdx.y.
__device__ __forceinline__ void match_popc_block(const MatchArgs& a, const MatchWork& w, int bid, int nblk,
                                                 uint4* s_db, unsigned int& s_last) {

  const int nq = min(a.d_nq ? *a.d_nq : a.nq, w.nq_cap);
  const int ndb = a.d_ndb ? *a.d_ndb : a.ndb;
  // Spread (query tile, train split) pairs over the launched blocks using the
  // actual counts, which may be far below the capacities the grid was sized for.
  const int tiles = (nq + kMQ - 1) / kMQ;
  if (tiles == 0) return;
  int splits = nblk / tiles;
  splits = min(splits, w.splits_cap);
  splits = min(splits, max(1, (ndb + 63) / 64));
  splits = max(splits, 1);
  const int tile = bid / splits;
  const int split = bid - tile * splits;
  if (tile >= tiles) return;
  const int q = tile * kMQ + threadIdx.x;
  const bool active = q < nq;

  uint32_t qw[8];
  {
    const uint4* qp = reinterpret_cast<const uint4*>(a.q) + 2 * (size_t)(active ? q : 0);
    const uint4 v0 = __ldg(qp), v1 = __ldg(qp + 1);
    qw[0] = v0.x; qw[1] = v0.y; qw[2] = v0.z; qw[3] = v0.w;
    qw[4] = v1.x; qw[5] = v1.y; qw[6] = v1.z; qw[7] = v1.w;
  }

  const int r_beg = (int)((long long)ndb * split / splits);
  const int r_end = (int)((long long)ndb * (split + 1) / splits);
  uint32_t k1 = kNoKey, k2 = kNoKey;
  const uint4* db4 = reinterpret_cast<const uint4*>(a.db);
  for (int r0 = r_beg; r0 < r_end; r0 += kMChunk) {
    const int rows = min(kMChunk, r_end - r0);
    __syncthreads();
    for (int i = threadIdx.x; i < rows * 2; i += kMQ) s_db[i] = __ldg(db4 + 2 * (size_t)r0 + i);
    __syncthreads();
    for (int j = 0; j < rows; j++) {
      const uint4 t0 = s_db[2 * j], t1 = s_db[2 * j + 1];
      const uint32_t d = __popc(qw[0] ^ t0.x) + __popc(qw[1] ^ t0.y) + __popc(qw[2] ^ t0.z) +
                         __popc(qw[3] ^ t0.w) + __popc(qw[4] ^ t1.x) + __popc(qw[5] ^ t1.y) +
                         __popc(qw[6] ^ t1.z) + __popc(qw[7] ^ t1.w);
      top2_push(k1, k2, (d << kIdxBits) | (uint32_t)(r0 + j));
    }
  }

  if (splits == 1) {
    if (active) finish_query(a, q, k1, k2);
    return;
  }
  // publish this split's partial top-2; the last split to finish the tile merges
  if (active) {
    uint2* part = reinterpret_cast<uint2*>(w.part);
    part[(size_t)split * w.nq_cap + q] = make_uint2(k1, k2);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&w.tile_done[tile], 1u) == (unsigned)(splits - 1)) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) w.tile_done[tile] = 0u;  // ready for the next launch
  if (!active) return;
  const uint2* part = reinterpret_cast<const uint2*>(w.part);
  uint32_t m1 = kNoKey, m2 = kNoKey;
  for (int sp = 0; sp < splits; sp++) {
    const uint2 pk = __ldcg(part + (size_t)sp * w.nq_cap + q);
    top2_push(m1, m2, pk.x);
    top2_push(m1, m2, pk.y);
  }
  finish_query(a, q, m1, m2);
}

__global__ void __launch_bounds__(kMQ) k_match_popc(MatchArgs a, MatchWork w) {
  __shared__ uint4 s_db[kMChunk * 2];
  __shared__ unsigned int s_last;
  match_popc_block(a, w, blockIdx.x, gridDim.x, s_db, s_last);
}

__global__ void __launch_bounds__(kMQ) k_match_popc_batch(const MatchJob* __restrict__ jobs) {
  __shared__ uint4 s_db[kMChunk * 2];
  __shared__ unsigned int s_last;
  const MatchJob& J = jobs[blockIdx.y];
  match_popc_block(J.args, J.work, blockIdx.x, gridDim.x, s_db, s_last);
}

int match_popc_blocks(int nq_cap, int splits_cap, int blocks_per_sm) {
  const int tiles = (nq_cap + kMQ - 1) / kMQ;
  const long long target = (long long)(blocks_per_sm > 0 ? blocks_per_sm : 8) * 148;
  long long blocks = (long long)tiles * splits_cap;
  if (blocks > target) blocks = target;
  if (blocks < tiles) blocks = tiles;
  return (int)blocks;
}

cudaError_t launch_match_popc(const MatchArgs& a, const MatchWork& w, cudaStream_t s, int blocks_per_sm) {
  if (w.nq_cap <= 0) return cudaSuccess;
  k_match_popc<<<match_popc_blocks(w.nq_cap, w.splits_cap, blocks_per_sm), kMQ, 0, s>>>(a, w);
  return cudaGetLastError();
}

cudaError_t launch_match_popc_batch(const MatchJob* d_jobs, int n_jobs, int blocks_per_job, cudaStream_t s) {
  if (n_jobs <= 0 || blocks_per_job <= 0) return cudaSuccess;
  k_match_popc_batch<<<dim3(blocks_per_job, n_jobs), kMQ, 0, s>>>(d_jobs);
  return cudaGetLastError();
}

}  // namespace orbx
