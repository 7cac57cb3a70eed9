// orbx_match_knn2_static: the k = 2 popcount matcher of orbx_match_knn2 with
// its split-merging scratch in a fixed file-scope device array instead of
// memory from cudaMalloc.  Nothing here allocates device or pinned memory.
//
// The scratch holds, for at most kStaticMaxQueries queries and kStaticSplits
// train splits, the partial top-2 keys of every split (8 bytes per query and
// split) and one arrival counter per 128-query tile.  Its device address is
// looked up with cudaGetSymbolAddress on every call, with the caller's device
// current.  The first call on a device loads this module there, which commits
// the array; later calls only look the address up, and a cudaDeviceReset (which
// unloads the module) between calls cannot leave a stale address behind.  The
// counters are cleared on the caller's stream before every search.  All calls
// on one device share the array, so two calls whose work overlaps on the
// device (different streams, or different host threads) race.

#include "../../include/orbx.h"
#include "orbx_internal.cuh"

namespace orbx {

constexpr int kStaticMaxQueries = ORBX_STATIC_MAX_QUERIES;
constexpr int kStaticSplits = 32;
constexpr int kStaticTiles = (kStaticMaxQueries + 127) / 128;
constexpr size_t kStaticPartWords = 2ull * kStaticSplits * kStaticMaxQueries;

struct StaticScratch {
  uint32_t part[kStaticPartWords];    // [splits][max queries][2] partial top-2 keys
  unsigned int tile_done[kStaticTiles];  // per query tile arrival counters
};
static_assert(sizeof(StaticScratch) <= (5u << 20), "static matcher scratch should stay near 4 MiB");

static __device__ __align__(256) StaticScratch g_static_scratch;

// Address of g_static_scratch on the current device.  In host code the symbol
// is a host-side stand-in, never a device address, so kernels get this value.
static int static_scratch(StaticScratch** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess || !p) {
    (void)cudaGetLastError();
    return ORBX_ERR_CUDA;
  }
  *out = static_cast<StaticScratch*>(p);
  return ORBX_OK;
}

}  // namespace orbx

using namespace orbx;

ORBX_API int orbx_match_knn2_static(const uint8_t* d_q, int nq, const uint8_t* d_db, int ndb, uint32_t* d_dist2,
                                    int32_t* d_idx2, void* cuda_stream) {
  if (nq < 0 || ndb < 0 || (nq > 0 && (!d_q || !d_dist2 || !d_idx2)) || (ndb > 0 && !d_db)) return ORBX_ERR_ARG;
  if (nq > kStaticMaxQueries || ndb > (1 << 22) - 1) return ORBX_ERR_SIZE;
  if (nq == 0) return ORBX_OK;
  StaticScratch* s = nullptr;
  int rc = static_scratch(&s);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  const int tiles = (nq + 127) / 128;
  cudaError_t e = cudaMemsetAsync(s->tile_done, 0, sizeof(unsigned int) * (size_t)tiles, stream);
  if (e == cudaSuccess) {
    MatchArgs a{};
    a.q = d_q;
    a.db = d_db;
    a.nq = nq;
    a.ndb = ndb;
    a.dist2 = d_dist2;
    a.idx2 = d_idx2;
    MatchWork w{};
    w.part = s->part;
    w.tile_done = s->tile_done;
    w.nq_cap = nq;  // partials indexed [split][query] with this row stride; nq <= kStaticMaxQueries
    w.splits_cap = kStaticSplits;
    e = launch_match_popc(a, w, stream);
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return ORBX_ERR_CUDA;
  }
  return ORBX_OK;
}
