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
#include "orbx_stages.cuh"

namespace orbx {

__global__ void __launch_bounds__(kMQ) k_match_popc(MatchArgs a, MatchWork w) {
  __shared__ uint4 s_db[kMChunk * 2];
  __shared__ unsigned int s_last;
  match_popc_block<kMQ, false>(a, w, blockIdx.x, gridDim.x, s_db, s_last);
}

__global__ void __launch_bounds__(kMQ) k_match_popc_batch(const MatchJob* __restrict__ jobs) {
  __shared__ uint4 s_db[kMChunk * 2];
  __shared__ unsigned int s_last;
  const MatchJob& J = jobs[blockIdx.y];
  match_popc_block<kMQ, false>(J.args, J.work, blockIdx.x, gridDim.x, s_db, s_last);
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
