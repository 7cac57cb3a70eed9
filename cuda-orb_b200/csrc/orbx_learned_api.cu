// Host side of the learned matching proposal (include/orbx.h, orbx_learned_*).
// No counterpart in the reference: its matcher is exact brute force only
// (orbd.cu:1471-1559, orb.cpp:104-113).
//
// Build:  copy + expand the database; Hamming k-majority clustering whose
//         assignment step is the exact int8 tensor-core k = 2 matcher against
//         the centroids; labels = cluster of each training row's exact nearest
//         database row; MLP training with the BF16 tcgen05 GEMM (forward and
//         backward), softmax cross-entropy and Adam, all on the context stream.
// Search: MLP forward with a fused top-8 epilogue, probe selection, per-cluster
//         probe lists, exact rerank of the probed clusters, merge, and exact
//         brute force for the low-margin queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "orbx_internal.cuh"
#include "orbx_learned.cuh"

using namespace orbx;
typedef __nv_bfloat16 bf16;
static_assert(kRerankQ == 128, "the tensor-core rerank takes 128 probing slots per item");

namespace {

struct Guard {
  int prev = -1;
  explicit Guard(int d) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != d)
      cudaSetDevice(d);
    else
      prev = -1;
  }
  ~Guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

#define LCHK(x)                                                             \
  do {                                                                      \
    cudaError_t _e = (x);                                                   \
    if (_e != cudaSuccess) {                                                \
      (void)cudaGetLastError();                                             \
      return _e == cudaErrorMemoryAllocation ? ORBX_ERR_NOMEM : ORBX_ERR_CUDA; \
    }                                                                       \
  } while (0)
#define LRC(x)              \
  do {                      \
    int _r = (x);           \
    if (_r) return _r;      \
  } while (0)

struct Arena {
  std::vector<void*> ptrs;
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
      *p = nullptr;
      return e;
    }
    ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return cudaSuccess;
  }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
  ~Arena() { release(); }
};

int round_up(int a, int b) { return (a + b - 1) / b * b; }
unsigned grid1(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

cudaError_t gemm(cudaStream_t s, int* err, const bf16* a, const bf16* b, int M, int N, int K, const float* bias,
                 int mode, int splits, float* cf, bf16* cb, const bf16* aux, uint32_t* keys) {
  GemmArgs g{};
  g.a = a;
  g.b = b;
  g.M = M;
  g.N = N;
  g.K = K;
  g.splits = splits;
  g.mode = mode;
  g.bias = bias;
  g.c_f32 = cf;
  g.c_bf16 = cb;
  g.aux = aux;
  g.top_keys = keys;
  g.err = err;
  return launch_gemm_bf16(g, s);
}

// K splits for a weight-gradient GEMM: fill about one wave of 148 SMs.
int pick_splits(int tiles, int kblocks) {
  int s = 1;
  while (tiles * s * 2 <= 148 && kblocks % (s * 2) == 0) s *= 2;
  return s;
}

// Split-merge scratch of the int8 tensor-core matcher for nq_cap queries,
// with the database splits chosen for splits_for queries.
struct ImmaWork {
  MatchWork w{};
  int splits = 1;
};
int imma_work_alloc(Arena& a, ImmaWork& iw, int nq_cap, int splits_for, cudaStream_t s, int splits_cap = 0) {
  iw.splits = imma_default_splits(std::max(1, splits_for));
  iw.w.nq_cap = nq_cap;
  iw.w.splits_cap = std::max(iw.splits, splits_cap);
  if (iw.w.splits_cap > 1) {
    const int tiles = (nq_cap + 127) / 128;
    LCHK(a.alloc(&iw.w.part, (size_t)2 * iw.w.splits_cap * nq_cap));
    LCHK(a.alloc(&iw.w.tile_done, (size_t)tiles));
    LCHK(cudaMemsetAsync(iw.w.tile_done, 0, sizeof(unsigned) * (size_t)tiles, s));
  }
  return ORBX_OK;
}

// Exact k = 2 search with the int8 tensor-core matcher.
int imma_knn(cudaStream_t s, int* err, const ImmaWork& iw, const uint8_t* q, int nq_cap, const int* d_nq,
             int8_t* q_pm1, bool q_ready, const uint8_t* db, int ndb, int8_t* db_pm1, bool db_ready, uint32_t* dist2,
             int32_t* idx2) {
  ImmaLaunch L{};
  L.args.q = q;
  L.args.db = db;
  L.args.nq = nq_cap;
  L.args.ndb = ndb;
  L.args.d_nq = d_nq;
  L.args.dist2 = dist2;
  L.args.idx2 = idx2;
  L.work = iw.w;
  L.splits = iw.splits;
  L.q_pm1 = q_pm1;
  L.db_pm1 = db_pm1;
  L.nq_cap = nq_cap;
  L.ndb_cap = ndb;
  L.err = err;
  L.q_ready = q_ready;
  L.db_ready = db_ready;
  LCHK(launch_match_imma(L, s));
  return ORBX_OK;
}

// Buffers of one forward + backward pass over B rows.
struct TrainBufs {
  Arena a;
  int B = 0, s1 = 1, s2 = 1, chunks = 1;
  uint8_t* xbits = nullptr;
  int* lbl = nullptr;
  bf16 *X = nullptr, *XT = nullptr, *H = nullptr, *HT = nullptr, *dL = nullptr, *dLT = nullptr, *dH = nullptr,
       *dHT = nullptr;
  float *logits = nullptr, *P1 = nullptr, *P2 = nullptr, *Pb1 = nullptr, *Pb2 = nullptr, *loss = nullptr;
  int* correct = nullptr;
};

}  // namespace

struct orbx_learned {
  int device = 0;
  orbx_learned_params p{};
  int ndb = 0, C = 0, Hd = 0;
  int n_entries = 0;  // cluster list entries (ndb, or up to spill * ndb)
  // during a build only: each database row's listed clusters, nearest first
  int* row_sets = nullptr;
  int set_width = 1;
  Arena keep;
  uint8_t* db = nullptr;
  int8_t* db_pm1 = nullptr;
  uint8_t* centroids = nullptr;
  int* assign = nullptr;
  int* ivf_offsets = nullptr;
  int* ivf_members = nullptr;
  uint8_t* ivf_desc = nullptr;
  // the lists padded per cluster to 256-row tiles (packed rows), for the tensor-core rerank
  int pad_rows = 0;
  int* pad_offsets = nullptr;
  int* pad_members = nullptr;
  uint8_t* pad_desc = nullptr;
  float *w1 = nullptr, *b1 = nullptr, *w2 = nullptr, *b2 = nullptr;
  bf16 *w1b = nullptr, *w2b = nullptr, *w2tb = nullptr;
  bf16* lsh = nullptr;  // [256][256] projections, rows >= lsh_bits unused
  // search scratch, sized for nq_cap queries
  Arena scratch;
  int nq_cap = 0;
  bf16 *xq = nullptr, *hq = nullptr;
  uint32_t* keys = nullptr;
  float* proj = nullptr;
  int *probes = nullptr, *counts = nullptr, *offsets = nullptr, *cursor = nullptr, *items = nullptr, *list = nullptr;
  float* margin = nullptr;
  uint2* partial = nullptr;
  int *fb_list = nullptr, *fb_count = nullptr;
  int* rr_counter = nullptr;
  uint32_t* rr_bound = nullptr;
  uint8_t* fb_q = nullptr;
  uint32_t* fb_d = nullptr;
  int32_t* fb_i = nullptr;
  int8_t* fb_pm1 = nullptr;
  ImmaWork fb_work;
  orbx_learned_stats stats{};
};

namespace {

int train_alloc(orbx_learned* L, TrainBufs& T, int B, int S = 1) {
  const int C = L->C, Hd = L->Hd;
  T.B = B;
  T.s2 = pick_splits((C / 128) * (Hd / 256), B / 64);
  T.s1 = pick_splits((Hd / 128) * (256 / 256), B / 64);
  T.chunks = B / 128;
  LCHK(T.a.alloc(&T.xbits, (size_t)B * 32));
  LCHK(T.a.alloc(&T.lbl, (size_t)B * S));
  LCHK(T.a.alloc(&T.X, (size_t)B * 256));
  LCHK(T.a.alloc(&T.XT, (size_t)B * 256));
  LCHK(T.a.alloc(&T.H, (size_t)B * Hd));
  LCHK(T.a.alloc(&T.HT, (size_t)B * Hd));
  LCHK(T.a.alloc(&T.logits, (size_t)B * C));
  LCHK(T.a.alloc(&T.dL, (size_t)B * C));
  LCHK(T.a.alloc(&T.dLT, (size_t)B * C));
  LCHK(T.a.alloc(&T.dH, (size_t)B * Hd));
  LCHK(T.a.alloc(&T.dHT, (size_t)B * Hd));
  LCHK(T.a.alloc(&T.P2, (size_t)T.s2 * C * Hd));
  LCHK(T.a.alloc(&T.P1, (size_t)T.s1 * Hd * 256));
  LCHK(T.a.alloc(&T.Pb2, (size_t)T.chunks * C));
  LCHK(T.a.alloc(&T.Pb1, (size_t)T.chunks * Hd));
  LCHK(T.a.alloc(&T.loss, (size_t)B));
  LCHK(T.a.alloc(&T.correct, (size_t)B));
  return ORBX_OK;
}

// Forward and backward over the B rows of xbits / lbl: leaves the loss per row
// and the gradients as split partial sums (P1 [s1][Hd][256], Pb1 [chunks][Hd],
// P2 [s2][C][Hd], Pb2 [chunks][C]).
int forward_backward(orbx_learned* L, TrainBufs& T, const uint8_t* xbits, const int* lbl, int S, cudaStream_t s,
                     int* err) {
  const int B = T.B, C = L->C, Hd = L->Hd;
  k_bits_pm1_bf16<<<grid1((long long)B * 32, 256), 256, 0, s>>>(xbits, B, nullptr, B, T.X);
  k_bits_pm1_bf16_t<<<B / 64, 256, 0, s>>>(xbits, B, B, T.XT);
  LCHK(gemm(s, err, T.X, L->w1b, B, Hd, 256, L->b1, kBiasReluBF16, 1, nullptr, T.H, nullptr, nullptr));
  LCHK(gemm(s, err, T.H, L->w2b, B, C, Hd, L->b2, kStoreF32, 1, T.logits, nullptr, nullptr, nullptr));
  k_softmax_xent<<<grid1((long long)B * 32, 256), 256, 0, s>>>(T.logits, lbl, S, B, B, C, 1.0f / (float)B, T.dL, T.loss,
                                                                T.correct);
  k_transpose_bf16<<<dim3(C / 32, B / 32), dim3(32, 8), 0, s>>>(T.dL, B, C, T.dLT);
  k_transpose_bf16<<<dim3(Hd / 32, B / 32), dim3(32, 8), 0, s>>>(T.H, B, Hd, T.HT);
  // dW2 = dL^T H
  LCHK(gemm(s, err, T.dLT, T.HT, C, Hd, B, nullptr, kStoreF32, T.s2, T.P2, nullptr, nullptr, nullptr));
  // dH = (dL W2) * (H > 0)
  LCHK(gemm(s, err, T.dL, L->w2tb, B, Hd, C, nullptr, kMaskBF16, 1, nullptr, T.dH, T.H, nullptr));
  k_transpose_bf16<<<dim3(Hd / 32, B / 32), dim3(32, 8), 0, s>>>(T.dH, B, Hd, T.dHT);
  // dW1 = dH^T X
  LCHK(gemm(s, err, T.dHT, T.XT, Hd, 256, B, nullptr, kStoreF32, T.s1, T.P1, nullptr, nullptr, nullptr));
  k_colsum_bf16<<<dim3(C / 64, T.chunks), 256, 0, s>>>(T.dL, B, C, 128, T.Pb2);
  k_colsum_bf16<<<dim3(Hd / 64, T.chunks), 256, 0, s>>>(T.dH, B, Hd, 128, T.Pb1);
  LCHK(cudaGetLastError());
  return ORBX_OK;
}

int check_params(const orbx_learned_params* p) {
  if (!p) return ORBX_ERR_ARG;
  if (p->proposal != ORBX_PROPOSAL_MLP && p->proposal != ORBX_PROPOSAL_LSH) return ORBX_ERR_ARG;
  if (p->n_probe < 1 || p->n_probe > kTopK) return ORBX_ERR_ARG;
  if (p->rerank != ORBX_RERANK_TENSOR && p->rerank != ORBX_RERANK_POPC) return ORBX_ERR_ARG;
  if (p->label_mode != ORBX_LABEL_NEAREST && p->label_mode != ORBX_LABEL_LISTED) return ORBX_ERR_ARG;
  if (p->proposal == ORBX_PROPOSAL_LSH) {
    if (p->lsh_bits < 8 || p->lsh_bits > 12 || p->n_clusters != (1 << p->lsh_bits)) return ORBX_ERR_ARG;
  } else {
    if (p->n_clusters < 256 || p->n_clusters > 4096 || p->n_clusters % 256) return ORBX_ERR_ARG;
    if (p->hidden < 256 || p->hidden > 4096 || p->hidden % 256) return ORBX_ERR_ARG;
    if (p->batch < 128 || p->batch % 128 || p->epochs < 0 || p->epochs > 64 || p->kmeans_iters < 1) return ORBX_ERR_ARG;
    if (p->spill < 1 || p->spill > 16 || (p->init != ORBX_INIT_CENTROIDS && p->init != ORBX_INIT_RANDOM)) return ORBX_ERR_ARG;
    if (p->init == ORBX_INIT_CENTROIDS && p->hidden < 512) return ORBX_ERR_ARG;
    if (p->synth_train < 0 || !(p->flip_lo >= 0.f && p->flip_lo <= p->flip_hi && p->flip_hi <= 0.5f)) return ORBX_ERR_ARG;
  }
  return ORBX_OK;
}

// Largest list and the number of list entries, once the lists are built from
// counts; synchronises the stream.
int read_list_stats(orbx_learned* L, const int* counts, cudaStream_t s) {
  const int C = L->C;
  std::vector<int> h_counts(C);
  int total = 0;
  LCHK(cudaGetLastError());
  LCHK(cudaMemcpyAsync(h_counts.data(), counts, sizeof(int) * C, cudaMemcpyDeviceToHost, s));
  LCHK(cudaMemcpyAsync(&total, L->ivf_offsets + C, sizeof(int), cudaMemcpyDeviceToHost, s));
  LCHK(cudaStreamSynchronize(s));
  L->stats.largest_cluster = *std::max_element(h_counts.begin(), h_counts.end());
  L->n_entries = total;
  return ORBX_OK;
}

// Spill 2: every row listed in its nearest and second-nearest cluster, from the
// matcher's top-2 against the centroids.
// The final lists from per-row cluster choices idx[row * per_row + j]: each
// cluster's list holds its rows in increasing index order, the same on every
// run (the tensor-core rerank relies on that order to resolve equal distances).
int spill_lists(orbx_learned* L, const int32_t* idx, int per_row, int* counts, int* cursor, cudaStream_t s) {
  const int n = L->ndb, C = L->C;
  const long long total = (long long)per_row * n;
  const int nb = (int)((total + kStableEntries - 1) / kStableEntries);
  Arena t;
  int* hist;
  LCHK(t.alloc(&hist, (size_t)nb * C));
  LCHK(cudaMemsetAsync(counts, 0, sizeof(int) * C, s));
  k_count_spill<<<grid1(total, 256), 256, 0, s>>>(idx, n, per_row, counts);
  k_scan_counts<<<1, 1024, 0, s>>>(counts, C, L->ivf_offsets, cursor, 0, nullptr);
  k_stable_hist<<<nb, 256, sizeof(int) * C, s>>>(idx, total, C, hist);
  k_stable_scan<<<grid1(C, 256), 256, 0, s>>>(hist, nb, C, L->ivf_offsets);
  k_stable_scatter<<<nb, 32, sizeof(int) * C, s>>>(idx, total, per_row, C, hist, L->ivf_members);
  if (L->row_sets) {
    // a build keeps each row's clusters for the training labels
    LCHK(cudaMemcpyAsync(L->row_sets, idx, sizeof(int) * (size_t)total, cudaMemcpyDeviceToDevice, s));
    L->set_width = per_row;
  }
  return read_list_stats(L, counts, s);
}

// Spill 3 and up: every row listed in its `spill` nearest centroids.  The
// Hamming distances to all centroids come from the BF16 tensor-core GEMM on +-1
// rows (dot = 256 - 2 * Hamming, exact in fp32), whose epilogue keeps the 8
// nearest of each 128 centroids by (distance, centroid index); the row's
// clusters are the best `spill` of those (exactly the nearest for spill <= 8).
int spill_lists_gemm(orbx_learned* L, int* counts, int* cursor, cudaStream_t s, int* err) {
  const int n = L->ndb, C = L->C, S = L->p.spill;
  const int chunk = 65536;
  Arena t;
  bf16 *cent, *x;
  uint32_t* keys;
  int* sel;
  LCHK(t.alloc(&cent, (size_t)C * 256));
  LCHK(t.alloc(&x, (size_t)chunk * 256));
  LCHK(t.alloc(&keys, (size_t)chunk * (C / 128) * kTopK));
  LCHK(t.alloc(&sel, (size_t)n * S));
  k_bits_pm1_bf16<<<grid1((long long)C * 32, 256), 256, 0, s>>>(L->centroids, C, nullptr, C, cent);
  for (int off = 0; off < n; off += chunk) {
    const int m = std::min(chunk, n - off);
    const int rows = round_up(m, 128);
    k_bits_pm1_bf16<<<grid1((long long)rows * 32, 256), 256, 0, s>>>(L->db + (size_t)off * 32, m, nullptr, rows, x);
    LCHK(gemm(s, err, x, cent, rows, C, 256, nullptr, kTop8, 1, nullptr, nullptr, nullptr, keys));
    k_select_topk<<<grid1((long long)m * 32, 256), 256, 0, s>>>(keys, m, C / 128, S, sel + (size_t)off * S);
  }
  return spill_lists(L, sel, S, counts, cursor, s);
}

// Device buffers every index holds: the database (bits and the matcher's +-1
// layout), centroids, assignment, the cluster lists and their rows; the LSH
// projections.
int alloc_core(orbx_learned* L) {
  const int ndb = L->ndb;
  const size_t per = L->p.proposal == ORBX_PROPOSAL_MLP ? (size_t)std::max(1, L->p.spill) : 1;  // list entries per row
  if (L->keep.alloc(&L->db, (size_t)ndb * 32) || L->keep.alloc(&L->db_pm1, (size_t)imma_rows_db(ndb) * 256) ||
      L->keep.alloc(&L->centroids, (size_t)L->C * 32) || L->keep.alloc(&L->assign, (size_t)ndb) ||
      L->keep.alloc(&L->ivf_offsets, (size_t)L->C + 1) || L->keep.alloc(&L->ivf_members, (size_t)ndb * per) ||
      L->keep.alloc(&L->ivf_desc, (size_t)ndb * per * 32) ||
      (L->p.proposal == ORBX_PROPOSAL_LSH && L->keep.alloc(&L->lsh, 256 * 256)))
    return ORBX_ERR_NOMEM;
  return ORBX_OK;
}

// The index's copy of the database and its +-1 layout for the int8 matcher.
int upload_db(orbx_learned* L, const uint8_t* d_db, cudaStream_t s) {
  LCHK(cudaMemcpyAsync(L->db, d_db, (size_t)L->ndb * 32, cudaMemcpyDeviceToDevice, s));
  LCHK(launch_expand_pm1(L->db, L->ndb, nullptr, imma_rows_db(L->ndb), L->db_pm1, s));
  return ORBX_OK;
}

// The padded lists of the tensor-core rerank, once the lists are built:
// offsets, database indices and packed rows.  Synchronises the stream.
int build_padded(orbx_learned* L, cudaStream_t s) {
  const int C = L->C;
  Arena t;
  int *counts, *cursor;
  LCHK(t.alloc(&counts, C));
  LCHK(t.alloc(&cursor, C));
  if (!L->pad_offsets) LCHK(L->keep.alloc(&L->pad_offsets, (size_t)C + 1));
  k_pad_counts<<<grid1(C, 256), 256, 0, s>>>(L->ivf_offsets, C, counts);
  k_scan_counts<<<1, 1024, 0, s>>>(counts, C, L->pad_offsets, cursor, 0, nullptr);
  int rows = 0;
  LCHK(cudaMemcpyAsync(&rows, L->pad_offsets + C, sizeof(int), cudaMemcpyDeviceToHost, s));
  LCHK(cudaStreamSynchronize(s));
  L->pad_rows = rows;
  LCHK(L->keep.alloc(&L->pad_members, (size_t)std::max(rows, 1)));
  LCHK(L->keep.alloc(&L->pad_desc, (size_t)std::max(rows, 1) * 32));
  k_fill_pad<<<C, 256, 0, s>>>(L->db, L->ivf_members, L->ivf_offsets, L->pad_offsets, L->pad_desc, L->pad_members);
  LCHK(cudaGetLastError());
  return ORBX_OK;
}

int cluster_kmeans(orbx_learned* L, cudaStream_t s, int* err) {
  const int n = L->ndb, C = L->C;
  Arena t;
  // initial centroids: C distinct rows from a seeded shuffle
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 rng(L->p.seed ^ 0x6b6d65616e73ull);
  for (int i = 0; i < C && i < n - 1; i++) {
    std::uniform_int_distribution<int> d(i, n - 1);
    std::swap(perm[i], perm[d(rng)]);
  }
  std::vector<int> init(C);
  for (int c = 0; c < C; c++) init[c] = perm[c % n];
  int *d_init, *idx2, *counts, *changed, *cursor;
  uint32_t* dist2;
  int8_t* cent_pm1;
  LCHK(t.alloc(&d_init, C));
  LCHK(t.alloc(&idx2, (size_t)2 * n));
  LCHK(t.alloc(&dist2, (size_t)2 * n));
  LCHK(t.alloc(&counts, C));
  LCHK(t.alloc(&cursor, C));
  LCHK(t.alloc(&changed, 1));
  LCHK(t.alloc(&cent_pm1, (size_t)imma_rows_db(C) * 256));
  LCHK(cudaMemcpyAsync(d_init, init.data(), sizeof(int) * C, cudaMemcpyHostToDevice, s));
  k_gather_rows<<<grid1(2ll * C, 256), 256, 0, s>>>(L->db, d_init, C, L->centroids);
  LCHK(cudaMemsetAsync(L->assign, 0xFF, sizeof(int) * (size_t)n, s));
  ImmaWork iw;
  LRC(imma_work_alloc(t, iw, n, n, s));
  const int iters = L->p.kmeans_iters;
  for (int it = 0; it < iters; it++) {
    LRC(imma_knn(s, err, iw, L->db, n, nullptr, L->db_pm1, true, L->centroids, C, cent_pm1, false, dist2, idx2));
    LCHK(cudaMemsetAsync(counts, 0, sizeof(int) * C, s));
    LCHK(cudaMemsetAsync(changed, 0, sizeof(int), s));
    k_assign<<<grid1(n, 256), 256, 0, s>>>(idx2, n, L->assign, counts, changed);
    k_scan_counts<<<1, 1024, 0, s>>>(counts, C, L->ivf_offsets, cursor, 0, nullptr);
    int moved = 0;
    LCHK(cudaMemcpyAsync(&moved, changed, sizeof(int), cudaMemcpyDeviceToHost, s));
    LCHK(cudaStreamSynchronize(s));
    L->stats.kmeans_iters_run = it + 1;
    L->stats.kmeans_last_moved = moved;
    k_scatter_members<<<grid1(n, 256), 256, 0, s>>>(L->assign, n, cursor, L->ivf_members);
    const bool done = it == iters - 1 || (it > 0 && (long long)moved * 1000 < (long long)n);
    if (done) break;
    k_majority<<<C, 256, 0, s>>>(L->db, n, L->ivf_members, L->ivf_offsets, L->centroids, L->p.seed, it);
    LCHK(cudaGetLastError());
  }
  // spill 2: the last assignment's top-2
  if (L->p.spill == 2) return spill_lists(L, idx2, 2, counts, cursor, s);
  if (L->p.spill > 2) return spill_lists_gemm(L, counts, cursor, s, err);
  return spill_lists(L, L->assign, 1, counts, cursor, s);
}

// Lists over fixed centroids (a loaded index): every row's exact top-2
// centroids by the int8 matcher give its cluster and, for spill 1 and 2, its
// lists; spill 3 and up go through the GEMM as in clustering.  The same
// assignment the last clustering iteration makes.
int lists_from_centroids(orbx_learned* L, cudaStream_t s, int* err) {
  const int n = L->ndb, C = L->C;
  Arena t;
  int *idx2, *counts, *cursor, *changed;
  uint32_t* dist2;
  int8_t* cent_pm1;
  LCHK(t.alloc(&idx2, (size_t)2 * n));
  LCHK(t.alloc(&dist2, (size_t)2 * n));
  LCHK(t.alloc(&counts, C));
  LCHK(t.alloc(&cursor, C));
  LCHK(t.alloc(&changed, 1));
  LCHK(t.alloc(&cent_pm1, (size_t)imma_rows_db(C) * 256));
  ImmaWork iw;
  LRC(imma_work_alloc(t, iw, n, n, s));
  LRC(imma_knn(s, err, iw, L->db, n, nullptr, L->db_pm1, true, L->centroids, C, cent_pm1, false, dist2, idx2));
  LCHK(cudaMemsetAsync(L->assign, 0xFF, sizeof(int) * (size_t)n, s));
  LCHK(cudaMemsetAsync(counts, 0, sizeof(int) * C, s));
  LCHK(cudaMemsetAsync(changed, 0, sizeof(int), s));
  k_assign<<<grid1(n, 256), 256, 0, s>>>(idx2, n, L->assign, counts, changed);
  if (L->p.spill == 2) return spill_lists(L, idx2, 2, counts, cursor, s);
  if (L->p.spill > 2) return spill_lists_gemm(L, counts, cursor, s, err);
  return spill_lists(L, L->assign, 1, counts, cursor, s);
}

// Buckets of the database rows; make_proj draws the projections from the seed
// (a loaded index brings its own).
int cluster_lsh(orbx_learned* L, cudaStream_t s, int* err, bool make_proj) {
  const int n = L->ndb, C = L->C;
  Arena t;
  if (make_proj) {
    float* wtmp;
    LCHK(t.alloc(&wtmp, 256 * 256));
    k_init_normal<<<grid1(256 * 256, 256), 256, 0, s>>>(wtmp, 256 * 256, 1.0f, L->p.seed ^ 0x6c7368ull, L->lsh);
  }
  const int chunk = 65536;
  bf16* x;
  float* proj;
  int* counts;
  int* cursor;
  LCHK(t.alloc(&x, (size_t)chunk * 256));
  LCHK(t.alloc(&proj, (size_t)chunk * 256));
  LCHK(t.alloc(&counts, C));
  LCHK(t.alloc(&cursor, C));
  for (int off = 0; off < n; off += chunk) {
    const int m = std::min(chunk, n - off);
    const int rows = round_up(m, 128);
    k_bits_pm1_bf16<<<grid1((long long)rows * 32, 256), 256, 0, s>>>(L->db + (size_t)off * 32, m, nullptr, rows, x);
    LCHK(gemm(s, err, x, L->lsh, rows, 256, 256, nullptr, kStoreF32, 1, proj, nullptr, nullptr, nullptr));
    k_lsh_probes<<<grid1(m, 128), 128, 0, s>>>(proj, 256, m, L->p.lsh_bits, 0, nullptr, nullptr, nullptr,
                                               L->assign + off, nullptr, nullptr, 1);
  }
  return spill_lists(L, L->assign, 1, counts, cursor, s);
}

int alloc_weights(orbx_learned* L, Arena& a, float** m, float** v) {
  const size_t n1 = (size_t)L->Hd * 256, n2 = (size_t)L->C * L->Hd;
  LCHK(L->keep.alloc(&L->w1, n1));
  LCHK(L->keep.alloc(&L->b1, L->Hd));
  LCHK(L->keep.alloc(&L->w2, n2));
  LCHK(L->keep.alloc(&L->b2, L->C));
  LCHK(L->keep.alloc(&L->w1b, n1));
  LCHK(L->keep.alloc(&L->w2b, n2));
  LCHK(L->keep.alloc(&L->w2tb, n2));
  // Adam moments, in the order w1, b1, w2, b2
  const size_t total = n1 + L->Hd + n2 + L->C;
  LCHK(a.alloc(m, total));
  LCHK(a.alloc(v, total));
  return ORBX_OK;
}

int train_mlp(orbx_learned* L, const uint8_t* d_train, int ntrain, const int* labels, int S, cudaStream_t s,
              int* err) {
  const int Hd = L->Hd, C = L->C, B = L->p.batch;
  Arena a;
  float *m, *v;
  LRC(alloc_weights(L, a, &m, &v));
  const size_t n1 = (size_t)Hd * 256, n2 = (size_t)C * Hd;
  if (L->p.init == ORBX_INIT_CENTROIDS) {
    // logit gap of 0.5 per Hamming bit between centroids
    k_init_centroid_mlp<<<grid1((long long)std::max(n1, n2), 256), 256, 0, s>>>(L->centroids, C, Hd, 0.25f, L->w1,
                                                                                L->b1, L->w2, L->b2, L->w1b, L->w2b);
  } else {
    k_init_normal<<<grid1((long long)n1, 256), 256, 0, s>>>(L->w1, (long long)n1, sqrtf(2.0f / 256.0f),
                                                            L->p.seed ^ 0x77310000ull, L->w1b);
    k_init_normal<<<grid1((long long)n2, 256), 256, 0, s>>>(L->w2, (long long)n2, sqrtf(1.0f / (float)Hd),
                                                            L->p.seed ^ 0x77320000ull, L->w2b);
    LCHK(cudaMemsetAsync(L->b1, 0, sizeof(float) * Hd, s));
    LCHK(cudaMemsetAsync(L->b2, 0, sizeof(float) * C, s));
  }
  LCHK(cudaMemsetAsync(m, 0, sizeof(float) * (n1 + Hd + n2 + C), s));
  LCHK(cudaMemsetAsync(v, 0, sizeof(float) * (n1 + Hd + n2 + C), s));
  k_transpose_bf16<<<dim3(Hd / 32, C / 32), dim3(32, 8), 0, s>>>(L->w2b, C, Hd, L->w2tb);
  LCHK(cudaGetLastError());
  const int steps = ntrain / B;
  const int epochs = steps > 0 ? L->p.epochs : 0;
  if (epochs == 0) return ORBX_OK;
  TrainBufs T;
  LRC(train_alloc(L, T, B, S));
  int* d_perm;
  float* acc;
  LCHK(a.alloc(&d_perm, ntrain));
  LCHK(a.alloc(&acc, 2 * (size_t)epochs));
  LCHK(cudaMemsetAsync(acc, 0, sizeof(float) * 2 * epochs, s));
  std::vector<int> perm(ntrain);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 rng(L->p.seed ^ 0x747261696eull);
  const long long total = (long long)epochs * steps;
  long long t = 0;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int e = 0; e < epochs; e++) {
    std::shuffle(perm.begin(), perm.end(), rng);
    LCHK(cudaStreamSynchronize(s));  // the previous epoch's reads of d_perm are done
    LCHK(cudaMemcpyAsync(d_perm, perm.data(), sizeof(int) * (size_t)ntrain, cudaMemcpyHostToDevice, s));
    LCHK(cudaStreamSynchronize(s));
    for (int st = 0; st < steps; st++) {
      const int* idx = d_perm + (size_t)st * B;
      k_gather_rows<<<grid1(2ll * B, 256), 256, 0, s>>>(d_train, idx, B, T.xbits);
      k_gather_i32<<<grid1((long long)B * S, 256), 256, 0, s>>>(labels, idx, B, S, T.lbl);
      LRC(forward_backward(L, T, T.xbits, T.lbl, S, s, err));
      t++;
      AdamStep as{};
      as.lr = (float)(L->p.lr * 0.5 * (1.0 + cos(M_PI * (double)(t - 1) / (double)total)));
      as.b1 = b1;
      as.b2 = b2;
      as.eps = 1e-8f;
      as.c1 = (float)(1.0 / (1.0 - pow((double)b1, (double)t)));
      as.c2 = (float)(1.0 / (1.0 - pow((double)b2, (double)t)));
      float* mw1 = m;
      float* mb1 = mw1 + n1;
      float* mw2 = mb1 + Hd;
      float* mb2 = mw2 + n2;
      float* vw1 = v;
      float* vb1 = vw1 + n1;
      float* vw2 = vb1 + Hd;
      float* vb2 = vw2 + n2;
      k_adam<<<grid1((long long)n1, 256), 256, 0, s>>>(L->w1, mw1, vw1, T.P1, T.s1, (long long)n1, L->w1b, as);
      k_adam<<<grid1(Hd, 256), 256, 0, s>>>(L->b1, mb1, vb1, T.Pb1, T.chunks, Hd, nullptr, as);
      k_adam<<<grid1((long long)n2, 256), 256, 0, s>>>(L->w2, mw2, vw2, T.P2, T.s2, (long long)n2, L->w2b, as);
      k_adam<<<grid1(C, 256), 256, 0, s>>>(L->b2, mb2, vb2, T.Pb2, T.chunks, C, nullptr, as);
      k_transpose_bf16<<<dim3(Hd / 32, C / 32), dim3(32, 8), 0, s>>>(L->w2b, C, Hd, L->w2tb);
      k_accum_stats<<<grid1(B, 256 * 8), 256, 0, s>>>(T.loss, T.correct, B, acc + 2 * e);
      LCHK(cudaGetLastError());
    }
  }
  std::vector<float> h(2 * (size_t)epochs);
  LCHK(cudaMemcpyAsync(h.data(), acc, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, s));
  LCHK(cudaStreamSynchronize(s));
  L->stats.epochs_run = epochs;
  for (int e = 0; e < epochs && e < 64; e++) {
    L->stats.loss[e] = h[2 * e] / (float)((long long)steps * B);
    L->stats.accuracy[e] = h[2 * e + 1] / (float)((long long)steps * B);
  }
  return ORBX_OK;
}

int ensure_search(orbx_learned* L, int nq) {
  if (L->nq_cap >= nq) return ORBX_OK;
  L->scratch.release();
  L->nq_cap = 0;
  const int rows = round_up(nq, 128), C = L->C;
  Arena& a = L->scratch;
  LCHK(a.alloc(&L->xq, (size_t)rows * 256));
  if (L->p.proposal == ORBX_PROPOSAL_MLP) {
    LCHK(a.alloc(&L->hq, (size_t)rows * L->Hd));
    LCHK(a.alloc(&L->keys, (size_t)rows * (C / 128) * kTopK));
  } else {
    LCHK(a.alloc(&L->proj, (size_t)rows * 256));
  }
  LCHK(a.alloc(&L->probes, (size_t)nq * kTopK));
  LCHK(a.alloc(&L->margin, (size_t)nq));
  LCHK(a.alloc(&L->counts, (size_t)C));
  LCHK(a.alloc(&L->offsets, (size_t)C + 1));
  LCHK(a.alloc(&L->cursor, (size_t)C));
  LCHK(a.alloc(&L->items, (size_t)C + 1));
  LCHK(a.alloc(&L->list, (size_t)nq * kTopK));
  LCHK(a.alloc(&L->partial, (size_t)nq * kTopK * kRrGroups));
  LCHK(a.alloc(&L->fb_list, (size_t)nq));
  LCHK(a.alloc(&L->fb_count, 1));
  LCHK(a.alloc(&L->rr_counter, 1));
  LCHK(a.alloc(&L->rr_bound, (size_t)nq));
  LCHK(a.alloc(&L->fb_q, (size_t)nq * 32));
  LCHK(a.alloc(&L->fb_d, (size_t)nq * 2));
  LCHK(a.alloc(&L->fb_i, (size_t)nq * 2));
  LCHK(a.alloc(&L->fb_pm1, (size_t)imma_rows_q(nq) * 256));
  // fallback splits sized for about one query in eight; fewer fallback queries
  // split the database scan further, up to 32 ways
  L->fb_work = ImmaWork();
  LRC(imma_work_alloc(a, L->fb_work, nq, std::max(128, nq / 8), 0, 32));
  LCHK(cudaDeviceSynchronize());
  L->nq_cap = nq;
  return ORBX_OK;
}

}  // namespace

ORBX_API int orbx_learned_default_params(orbx_learned_params* p) {
  if (!p) return ORBX_ERR_ARG;
  p->proposal = ORBX_PROPOSAL_MLP;
  p->n_clusters = 4096;
  p->hidden = 512;
  p->n_probe = 8;
  p->kmeans_iters = 20;
  p->epochs = 12;
  p->batch = 4096;
  p->lr = 2e-3f;
  p->margin = 0.0f;
  p->lsh_bits = 12;
  p->seed = 0x0C4000ull;
  p->max_distance = 256;
  p->spill = 2;
  p->init = ORBX_INIT_CENTROIDS;
  p->synth_train = 0;
  p->flip_lo = 0.05f;
  p->flip_hi = 0.2f;
  p->rerank = ORBX_RERANK_TENSOR;
  p->label_mode = ORBX_LABEL_LISTED;
  return ORBX_OK;
}

ORBX_API int orbx_learned_build(orbx_ctx* ctx, const orbx_learned_params* p, const uint8_t* d_db, int ndb,
                                const uint8_t* d_train, int ntrain, orbx_learned** out) {
  if (!ctx || !out || !d_db || ndb < 1 || ntrain < 0 || (ntrain > 0 && !d_train)) return ORBX_ERR_ARG;
  *out = nullptr;
  LRC(check_params(p));
  if (ndb > (1 << 22) - 1) return ORBX_ERR_SIZE;
  if (p->proposal == ORBX_PROPOSAL_MLP && (ndb < p->n_clusters || ntrain < p->batch)) return ORBX_ERR_SIZE;
  Guard g(ctx_device(ctx));
  cudaStream_t s = ctx_stream(ctx);
  int* err = ctx_err(ctx);
  orbx_learned* L = new orbx_learned();
  L->device = ctx_device(ctx);
  L->p = *p;
  L->ndb = ndb;
  L->C = p->n_clusters;
  L->Hd = p->hidden;
  auto fail = [&](int rc) {
    cudaStreamSynchronize(s);
    delete L;
    return rc;
  };
  cudaEvent_t ev[4];
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(ORBX_ERR_CUDA);
  auto events_free = [&]() {
    for (auto& e : ev) cudaEventDestroy(e);
  };
  Arena build_tmp;  // buffers that live for the build only
  int rc = ORBX_OK;
  do {
    rc = alloc_core(L);
    if (rc) break;
    cudaEventRecord(ev[0], s);
    rc = upload_db(L, d_db, s);
    if (rc) break;
    if (build_tmp.alloc(&L->row_sets, (size_t)ndb * (p->proposal == ORBX_PROPOSAL_MLP ? std::max(1, p->spill) : 1))) {
      rc = ORBX_ERR_NOMEM;
      break;
    }
    rc = p->proposal == ORBX_PROPOSAL_MLP ? cluster_kmeans(L, s, err) : cluster_lsh(L, s, err, true);
    if (rc) break;
    k_gather_rows<<<grid1(2ll * L->n_entries, 256), 256, 0, s>>>(L->db, L->ivf_members, L->n_entries, L->ivf_desc);
    rc = build_padded(L, s);
    if (rc) break;
    cudaEventRecord(ev[1], s);
    if (p->proposal == ORBX_PROPOSAL_MLP) {
      Arena t;
      int* labels;
      int32_t* idx2;
      uint32_t* dist2;
      int8_t* tq;
      uint8_t* rows;
      const int nt = ntrain + p->synth_train;
      const int S = p->label_mode == ORBX_LABEL_LISTED ? L->set_width : 1;
      if (t.alloc(&labels, (size_t)nt * S) || t.alloc(&idx2, 2 * (size_t)nt) || t.alloc(&dist2, 2 * (size_t)nt) ||
          t.alloc(&tq, (size_t)imma_rows_q(nt) * 256) || t.alloc(&rows, (size_t)nt * 32)) {
        rc = ORBX_ERR_NOMEM;
        break;
      }
      // training rows: the caller's, then database rows with random bit flips
      if (cudaMemcpyAsync(rows, d_train, (size_t)ntrain * 32, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        rc = ORBX_ERR_CUDA;
        break;
      }
      if (p->synth_train > 0)
        k_perturb_rows<<<grid1(8ll * p->synth_train, 256), 256, 0, s>>>(L->db, ndb, p->synth_train,
                                                                         p->seed ^ 0x73796e74ull, p->flip_lo,
                                                                         p->flip_hi, rows + (size_t)ntrain * 32);
      ImmaWork iw;
      rc = imma_work_alloc(t, iw, nt, nt, s);
      if (rc) break;
      rc = imma_knn(s, err, iw, rows, nt, nullptr, tq, false, L->db, ndb, L->db_pm1, true, dist2, idx2);
      if (rc) break;
      k_labels<<<grid1((long long)nt * S, 256), 256, 0, s>>>(idx2, nt, L->row_sets, L->set_width, S, labels);
      cudaEventRecord(ev[2], s);
      rc = train_mlp(L, rows, nt, labels, S, s, err);
      if (rc) break;
    } else {
      cudaEventRecord(ev[2], s);
    }
    cudaEventRecord(ev[3], s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      rc = ORBX_ERR_CUDA;
      break;
    }
    int h_err = 0;
    cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (h_err) {
      cudaMemset(err, 0, sizeof(int));
      rc = ORBX_ERR_TIMEOUT;
      break;
    }
    cudaEventElapsedTime(&L->stats.build_ms[0], ev[0], ev[1]);
    cudaEventElapsedTime(&L->stats.build_ms[1], ev[1], ev[2]);
    cudaEventElapsedTime(&L->stats.build_ms[2], ev[2], ev[3]);
    cudaEventElapsedTime(&L->stats.build_ms[3], ev[0], ev[3]);
  } while (0);
  cudaStreamSynchronize(s);
  L->row_sets = nullptr;
  events_free();
  if (rc) {
    (void)cudaGetLastError();
    return fail(rc);
  }
  *out = L;
  return ORBX_OK;
}

// The search; with ev non-null, events 0..5 bracket the phases proposal,
// probe lists, rerank, merge and exact fallback.
static int search_impl(orbx_ctx* ctx, orbx_learned* L, const uint8_t* d_q, int nq, uint32_t* d_dist2, int32_t* d_idx2,
                       float* d_margin, int* d_fallback_count, cudaEvent_t* ev) {
  if (!ctx || !L || nq < 0 || (nq > 0 && (!d_q || !d_dist2 || !d_idx2))) return ORBX_ERR_ARG;
  if (ctx_device(ctx) != L->device) return ORBX_ERR_ARG;
  if (nq > (1 << 24)) return ORBX_ERR_SIZE;
  if (nq == 0) return ORBX_OK;
  Guard g(L->device);
  cudaStream_t s = ctx_stream(ctx);
  int* err = ctx_err(ctx);
  LRC(ensure_search(L, nq));
  const int rows = round_up(nq, 128), C = L->C;
  const bool mlp = L->p.proposal == ORBX_PROPOSAL_MLP;
  const float thr = mlp ? L->p.margin : -3.0e38f;
  const bool tensor = L->p.rerank == ORBX_RERANK_TENSOR && L->pad_rows > 0;
  const int per_slot = tensor ? kRrGroups : 1;
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], s);
  };
  mark(0);
  LCHK(cudaMemsetAsync(L->counts, 0, sizeof(int) * C, s));
  LCHK(cudaMemsetAsync(L->fb_count, 0, sizeof(int), s));
  k_bits_pm1_bf16<<<grid1((long long)rows * 32, 256), 256, 0, s>>>(d_q, nq, nullptr, rows, L->xq);
  if (mlp) {
    LCHK(gemm(s, err, L->xq, L->w1b, rows, L->Hd, 256, L->b1, kBiasReluBF16, 1, nullptr, L->hq, nullptr, nullptr));
    LCHK(gemm(s, err, L->hq, L->w2b, rows, C, L->Hd, L->b2, kTop8Row, 1, nullptr, nullptr, nullptr, L->keys));
    k_select_probes<<<grid1((long long)nq * 32, 256), 256, 0, s>>>(L->keys, nq, gemm_top_lists(C), L->p.n_probe, thr,
                                                                    L->ivf_offsets, L->probes, L->margin, L->counts,
                                                                    L->partial, per_slot);
  } else {
    LCHK(gemm(s, err, L->xq, L->lsh, rows, 256, 256, nullptr, kStoreF32, 1, L->proj, nullptr, nullptr, nullptr));
    k_lsh_probes<<<grid1(nq, 128), 128, 0, s>>>(L->proj, 256, nq, L->p.lsh_bits, L->p.n_probe, L->ivf_offsets,
                                                L->probes, L->counts, nullptr, L->margin, L->partial, per_slot);
  }
  mark(1);
  k_scan_counts<<<1, 1024, 0, s>>>(L->counts, C, L->offsets, L->cursor, kRerankQ, L->items);
  k_fill_probe_lists<<<grid1((long long)nq * kTopK, 256), 256, 0, s>>>(L->probes, nq, L->cursor, L->list);
  mark(2);
  const unsigned items_max = grid1((long long)nq * kTopK, kRerankQ) + (unsigned)C;
  if (tensor) {
    RerankImmaArgs ra{};
    ra.q_bits = d_q;
    ra.list = L->list;
    ra.probe_offsets = L->offsets;
    ra.item_offsets = L->items;
    ra.n_clusters = C;
    ra.ivf_offsets = L->ivf_offsets;
    ra.pad_offsets = L->pad_offsets;
    ra.pad_members = L->pad_members;
    ra.pad_desc = L->pad_desc;
    ra.partial = L->partial;
    ra.item_counter = L->rr_counter;
    ra.q_bound = L->rr_bound;
    ra.err = err;
    LCHK(cudaMemsetAsync(L->rr_counter, 0, sizeof(int), s));
    LCHK(cudaMemsetAsync(L->rr_bound, 0xFF, sizeof(uint32_t) * (size_t)nq, s));
    LCHK(launch_rerank_imma(ra, (int)items_max, s));
  } else {
    k_rerank<<<items_max, kRerankQ, 0, s>>>(d_q, L->list, L->offsets, L->items, C, L->ivf_desc, L->ivf_members,
                                            L->ivf_offsets, L->partial);
  }
  mark(3);
  k_merge_probes<<<grid1(nq, 256), 256, 0, s>>>(L->partial, per_slot, nq, L->margin, thr, mlp ? L->p.max_distance : 1 << 20,
                                                 d_dist2, d_idx2, mlp ? L->fb_list : nullptr, L->fb_count);
  mark(4);
  LCHK(cudaGetLastError());
  if (mlp) {
    k_gather_fallback<<<grid1(2ll * nq, 256), 256, 0, s>>>(d_q, L->fb_list, L->fb_count, L->fb_q);
    LRC(imma_knn(s, err, L->fb_work, L->fb_q, nq, L->fb_count, L->fb_pm1, false, L->db, L->ndb, L->db_pm1, true,
                 L->fb_d, L->fb_i));
    k_scatter_fallback<<<grid1(nq, 256), 256, 0, s>>>(L->fb_list, L->fb_count, L->fb_d, L->fb_i, d_dist2, d_idx2);
  }
  mark(5);
  if (d_margin) LCHK(cudaMemcpyAsync(d_margin, L->margin, sizeof(float) * nq, cudaMemcpyDeviceToDevice, s));
  if (d_fallback_count) LCHK(cudaMemcpyAsync(d_fallback_count, L->fb_count, sizeof(int), cudaMemcpyDeviceToDevice, s));
  LCHK(cudaGetLastError());
  return ORBX_OK;
}

ORBX_API int orbx_learned_search(orbx_ctx* ctx, orbx_learned* L, const uint8_t* d_q, int nq, uint32_t* d_dist2,
                                 int32_t* d_idx2, float* d_margin, int* d_fallback_count) {
  return search_impl(ctx, L, d_q, nq, d_dist2, d_idx2, d_margin, d_fallback_count, nullptr);
}

ORBX_API int orbx_learned_profile_search(orbx_ctx* ctx, orbx_learned* L, const uint8_t* d_q, int nq,
                                         uint32_t* d_dist2, int32_t* d_idx2, float* h_ms) {
  if (!ctx || !L || !h_ms) return ORBX_ERR_ARG;
  Guard g(L->device);
  cudaEvent_t ev[6];
  int made = 0;
  int rc = ORBX_OK;
  for (; made < 6; made++)
    if (cudaEventCreate(&ev[made]) != cudaSuccess) {
      rc = ORBX_ERR_CUDA;
      break;
    }
  if (!rc) rc = search_impl(ctx, L, d_q, nq, d_dist2, d_idx2, nullptr, nullptr, ev);
  if (!rc && cudaStreamSynchronize(ctx_stream(ctx)) != cudaSuccess) rc = ORBX_ERR_CUDA;
  if (!rc)
    for (int i = 0; i < 5; i++) cudaEventElapsedTime(&h_ms[i], ev[i], ev[i + 1]);
  for (int i = 0; i < made; i++) cudaEventDestroy(ev[i]);
  (void)cudaGetLastError();
  return rc;
}

ORBX_API int orbx_learned_set_margin(orbx_learned* L, float margin) {
  if (!L) return ORBX_ERR_ARG;
  L->p.margin = margin;
  return ORBX_OK;
}

ORBX_API int orbx_learned_probe_pairs(orbx_ctx* ctx, const orbx_learned* L, unsigned long long* h_pairs) {
  if (!ctx || !L || !h_pairs) return ORBX_ERR_ARG;
  if (L->nq_cap == 0) return ORBX_ERR_STATE;
  Guard g(L->device);
  cudaStream_t s = ctx_stream(ctx);
  Arena t;
  unsigned long long* d;
  LCHK(t.alloc(&d, 1));
  k_probe_pairs<<<1, 1024, 0, s>>>(L->offsets, L->ivf_offsets, L->C, d);
  LCHK(cudaGetLastError());
  LCHK(cudaMemcpyAsync(h_pairs, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  LCHK(cudaStreamSynchronize(s));
  return ORBX_OK;
}

ORBX_API int orbx_learned_set_rerank(orbx_learned* L, int form) {
  if (!L || (form != ORBX_RERANK_TENSOR && form != ORBX_RERANK_POPC)) return ORBX_ERR_ARG;
  L->p.rerank = form;
  return ORBX_OK;
}

ORBX_API int orbx_learned_set_max_distance(orbx_learned* L, int max_distance) {
  if (!L) return ORBX_ERR_ARG;
  L->p.max_distance = max_distance;
  return ORBX_OK;
}

ORBX_API int orbx_learned_get_stats(const orbx_learned* L, orbx_learned_stats* s) {
  if (!L || !s) return ORBX_ERR_ARG;
  *s = L->stats;
  return ORBX_OK;
}

ORBX_API int orbx_learned_export(orbx_ctx* ctx, const orbx_learned* L, int* h_assign, int* h_offsets, float* h_w1,
                                 float* h_b1, float* h_w2, float* h_b2) {
  if (!ctx || !L) return ORBX_ERR_ARG;
  Guard g(L->device);
  cudaStream_t s = ctx_stream(ctx);
  LCHK(cudaStreamSynchronize(s));
  if (h_assign) LCHK(cudaMemcpy(h_assign, L->assign, sizeof(int) * (size_t)L->ndb, cudaMemcpyDeviceToHost));
  if (h_offsets) LCHK(cudaMemcpy(h_offsets, L->ivf_offsets, sizeof(int) * ((size_t)L->C + 1), cudaMemcpyDeviceToHost));
  const bool mlp = L->w1b != nullptr;
  if ((h_w1 || h_b1 || h_w2 || h_b2) && !mlp) return ORBX_ERR_STATE;
  auto widen = [](const std::vector<uint16_t>& in, float* out) {
    for (size_t i = 0; i < in.size(); i++) {
      const uint32_t u = (uint32_t)in[i] << 16;
      std::memcpy(out + i, &u, 4);
    }
  };
  if (h_w1) {
    std::vector<uint16_t> t((size_t)L->Hd * 256);
    LCHK(cudaMemcpy(t.data(), L->w1b, t.size() * 2, cudaMemcpyDeviceToHost));
    widen(t, h_w1);
  }
  if (h_w2) {
    std::vector<uint16_t> t((size_t)L->C * L->Hd);
    LCHK(cudaMemcpy(t.data(), L->w2b, t.size() * 2, cudaMemcpyDeviceToHost));
    widen(t, h_w2);
  }
  if (h_b1) LCHK(cudaMemcpy(h_b1, L->b1, sizeof(float) * L->Hd, cudaMemcpyDeviceToHost));
  if (h_b2) LCHK(cudaMemcpy(h_b2, L->b2, sizeof(float) * L->C, cudaMemcpyDeviceToHost));
  return ORBX_OK;
}

// ---------------------------------------------------------------- save / load
// A saved proposal, little-endian, every field 4-byte aligned:
//   "ORBXLRN1", u32 version, u32 total bytes
//   the orbx_learned_params fields in declaration order (seed as two u32, low
//   word first, then rerank and label_mode), then the orbx_learned_stats words
//   MLP: centroids [C][32] u8, W1 [Hd][256] bf16, b1 [Hd] f32, W2 [C][Hd] bf16,
//        b2 [C] f32 (the weights search uses)
//   LSH: projections [256][256] bf16
//   u64 FNV-1a hash of every byte before it
// The database and the cluster lists are not saved: loading lists a database
// under the saved centroids (or buckets) again.
namespace {

constexpr char kSaveMagic[8] = {'O', 'R', 'B', 'X', 'L', 'R', 'N', '1'};
constexpr uint32_t kSaveVersion = 3;
constexpr size_t kSaveParamWords = 20;
constexpr size_t kSaveStatsWords = sizeof(orbx_learned_stats) / 4;
static_assert(sizeof(orbx_learned_stats) == 4 * (4 + 64 + 64 + 4), "stats are whole 4-byte words");

size_t save_payload_bytes(const orbx_learned_params& p) {
  const size_t C = (size_t)p.n_clusters, Hd = (size_t)p.hidden;
  if (p.proposal == ORBX_PROPOSAL_LSH) return 256 * 256 * 2;
  return C * 32 + Hd * 256 * 2 + Hd * 4 + C * Hd * 2 + C * 4;
}

size_t save_bytes(const orbx_learned_params& p) {
  return 16 + 4 * (kSaveParamWords + kSaveStatsWords) + save_payload_bytes(p) + 8;
}

uint64_t fnv1a(const uint8_t* b, size_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

void put32(uint8_t*& w, uint32_t v) {
  for (int i = 0; i < 4; i++) *w++ = (uint8_t)(v >> (8 * i));
}
uint32_t get32(const uint8_t*& r) {
  uint32_t v = 0;
  for (int i = 0; i < 4; i++) v |= (uint32_t)*r++ << (8 * i);
  return v;
}
uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
float bitsf(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

void put_params(uint8_t*& w, const orbx_learned_params& p) {
  const uint32_t v[kSaveParamWords] = {(uint32_t)p.proposal, (uint32_t)p.n_clusters, (uint32_t)p.hidden,
                                       (uint32_t)p.n_probe, (uint32_t)p.kmeans_iters, (uint32_t)p.epochs,
                                       (uint32_t)p.batch, fbits(p.lr), fbits(p.margin), (uint32_t)p.lsh_bits,
                                       (uint32_t)p.seed, (uint32_t)(p.seed >> 32), (uint32_t)p.max_distance,
                                       (uint32_t)p.spill, (uint32_t)p.init, (uint32_t)p.synth_train,
                                       fbits(p.flip_lo), fbits(p.flip_hi), (uint32_t)p.rerank,
                                       (uint32_t)p.label_mode};
  for (uint32_t x : v) put32(w, x);
}
orbx_learned_params get_params(const uint8_t*& r) {
  uint32_t v[kSaveParamWords];
  for (auto& x : v) x = get32(r);
  orbx_learned_params p{};
  p.proposal = (int)v[0];
  p.n_clusters = (int)v[1];
  p.hidden = (int)v[2];
  p.n_probe = (int)v[3];
  p.kmeans_iters = (int)v[4];
  p.epochs = (int)v[5];
  p.batch = (int)v[6];
  p.lr = bitsf(v[7]);
  p.margin = bitsf(v[8]);
  p.lsh_bits = (int)v[9];
  p.seed = (unsigned long long)v[10] | ((unsigned long long)v[11] << 32);
  p.max_distance = (int)v[12];
  p.spill = (int)v[13];
  p.init = (int)v[14];
  p.synth_train = (int)v[15];
  p.flip_lo = bitsf(v[16]);
  p.flip_hi = bitsf(v[17]);
  p.rerank = (int)v[18];
  p.label_mode = (int)v[19];
  return p;
}

// Device -> host copy of n bytes; the stream is already synchronised.
int fetch(uint8_t*& w, const void* d, size_t n) {
  LCHK(cudaMemcpy(w, d, n, cudaMemcpyDeviceToHost));
  w += n;
  return ORBX_OK;
}
// Host -> device copy of n bytes on the stream; the caller synchronises.
int send(const uint8_t*& r, void* d, size_t n, cudaStream_t s) {
  LCHK(cudaMemcpyAsync(d, r, n, cudaMemcpyHostToDevice, s));
  r += n;
  return ORBX_OK;
}

}  // namespace

ORBX_API int orbx_learned_save(orbx_ctx* ctx, const orbx_learned* L, void* h_buf, size_t cap, size_t* h_need) {
  if (!ctx || !L || !h_need) return ORBX_ERR_ARG;
  const size_t need = save_bytes(L->p);
  *h_need = need;
  if (!h_buf) return ORBX_OK;
  if (cap < need) return ORBX_ERR_SIZE;
  if (need > 0xFFFFFFFFull) return ORBX_ERR_SIZE;
  Guard g(L->device);
  LCHK(cudaStreamSynchronize(ctx_stream(ctx)));
  uint8_t* const b = static_cast<uint8_t*>(h_buf);
  uint8_t* w = b;
  std::memcpy(w, kSaveMagic, 8);
  w += 8;
  put32(w, kSaveVersion);
  put32(w, (uint32_t)need);
  put_params(w, L->p);
  uint32_t st[kSaveStatsWords];
  std::memcpy(st, &L->stats, sizeof(st));
  for (uint32_t x : st) put32(w, x);
  const size_t C = (size_t)L->C, Hd = (size_t)L->Hd;
  if (L->p.proposal == ORBX_PROPOSAL_MLP) {
    LRC(fetch(w, L->centroids, C * 32));
    LRC(fetch(w, L->w1b, Hd * 256 * 2));
    LRC(fetch(w, L->b1, Hd * 4));
    LRC(fetch(w, L->w2b, C * Hd * 2));
    LRC(fetch(w, L->b2, C * 4));
  } else {
    LRC(fetch(w, L->lsh, 256 * 256 * 2));
  }
  const uint64_t h = fnv1a(b, (size_t)(w - b));
  put32(w, (uint32_t)h);
  put32(w, (uint32_t)(h >> 32));
  return (size_t)(w - b) == need ? ORBX_OK : ORBX_ERR_STATE;
}

ORBX_API int orbx_learned_load(orbx_ctx* ctx, const void* h_buf, size_t bytes, const uint8_t* d_db, int ndb,
                               orbx_learned** out) {
  if (!ctx || !h_buf || !out || !d_db || ndb < 1) return ORBX_ERR_ARG;
  *out = nullptr;
  if (ndb > (1 << 22) - 1) return ORBX_ERR_SIZE;
  // header, parameters, size and hash before anything touches the device
  const uint8_t* const b = static_cast<const uint8_t*>(h_buf);
  if (bytes < 16 + 4 * kSaveParamWords + 8 || std::memcmp(b, kSaveMagic, 8) != 0) return ORBX_ERR_ARG;
  const uint8_t* r = b + 8;
  if (get32(r) != kSaveVersion || get32(r) != bytes) return ORBX_ERR_ARG;
  const orbx_learned_params p = get_params(r);
  LRC(check_params(&p));
  if (save_bytes(p) != bytes) return ORBX_ERR_ARG;
  {
    const uint8_t* t = b + bytes - 8;
    const uint64_t lo = get32(t), hi = get32(t);
    if (fnv1a(b, bytes - 8) != (lo | (hi << 32))) return ORBX_ERR_ARG;
  }
  Guard g(ctx_device(ctx));
  cudaStream_t s = ctx_stream(ctx);
  int* err = ctx_err(ctx);
  orbx_learned* L = new orbx_learned();
  L->device = ctx_device(ctx);
  L->p = p;
  L->ndb = ndb;
  L->C = p.n_clusters;
  L->Hd = p.hidden;
  uint32_t st[kSaveStatsWords];
  for (auto& x : st) x = get32(r);
  std::memcpy(&L->stats, st, sizeof(st));
  cudaEvent_t ev[2];
  int made = 0;
  int rc = ORBX_OK;
  for (; made < 2; made++)
    if (cudaEventCreate(&ev[made]) != cudaSuccess) {
      rc = ORBX_ERR_CUDA;
      break;
    }
  const size_t C = (size_t)L->C, Hd = (size_t)L->Hd;
  const bool mlp = p.proposal == ORBX_PROPOSAL_MLP;
  do {
    if (rc) break;
    rc = alloc_core(L);
    if (rc) break;
    if (mlp && (L->keep.alloc(&L->w1b, Hd * 256) || L->keep.alloc(&L->b1, Hd) || L->keep.alloc(&L->w2b, C * Hd) ||
                L->keep.alloc(&L->b2, C) || L->keep.alloc(&L->w2tb, C * Hd))) {
      rc = ORBX_ERR_NOMEM;
      break;
    }
    cudaEventRecord(ev[0], s);
    rc = upload_db(L, d_db, s);
    if (rc) break;
    if (mlp) {
      if ((rc = send(r, L->centroids, C * 32, s)) || (rc = send(r, L->w1b, Hd * 256 * 2, s)) ||
          (rc = send(r, L->b1, Hd * 4, s)) || (rc = send(r, L->w2b, C * Hd * 2, s)) || (rc = send(r, L->b2, C * 4, s)))
        break;
      k_transpose_bf16<<<dim3(L->Hd / 32, L->C / 32), dim3(32, 8), 0, s>>>(L->w2b, L->C, L->Hd, L->w2tb);
      rc = lists_from_centroids(L, s, err);
    } else {
      if ((rc = send(r, L->lsh, 256 * 256 * 2, s))) break;
      rc = cluster_lsh(L, s, err, false);
    }
    if (rc) break;
    k_gather_rows<<<grid1(2ll * L->n_entries, 256), 256, 0, s>>>(L->db, L->ivf_members, L->n_entries, L->ivf_desc);
    rc = build_padded(L, s);
    if (rc) break;
    cudaEventRecord(ev[1], s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      rc = ORBX_ERR_CUDA;
      break;
    }
    int h_err = 0;
    cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (h_err) {
      cudaMemset(err, 0, sizeof(int));
      rc = ORBX_ERR_TIMEOUT;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    L->stats.build_ms[0] = ms;
    L->stats.build_ms[1] = 0.f;
    L->stats.build_ms[2] = 0.f;
    L->stats.build_ms[3] = ms;
  } while (0);
  for (int i = 0; i < made; i++) cudaEventDestroy(ev[i]);
  if (rc) {
    cudaStreamSynchronize(s);
    (void)cudaGetLastError();
    delete L;
    return rc;
  }
  *out = L;
  return ORBX_OK;
}

ORBX_API int orbx_learned_get_params(const orbx_learned* L, orbx_learned_params* p) {
  if (!L || !p) return ORBX_ERR_ARG;
  *p = L->p;
  return ORBX_OK;
}

ORBX_API int orbx_learned_gradients(orbx_ctx* ctx, orbx_learned* L, const uint8_t* d_x, const int* d_labels, int n,
                                    float* h_loss, float* h_dw1, float* h_db1, float* h_dw2, float* h_db2) {
  if (!ctx || !L || !d_x || !d_labels || n < 128 || n % 128) return ORBX_ERR_ARG;
  if (!L->w1b) return ORBX_ERR_STATE;
  Guard g(L->device);
  cudaStream_t s = ctx_stream(ctx);
  int* err = ctx_err(ctx);
  TrainBufs T;
  LRC(train_alloc(L, T, n));
  LRC(forward_backward(L, T, d_x, d_labels, 1, s, err));
  LCHK(cudaStreamSynchronize(s));
  const int Hd = L->Hd, C = L->C;
  auto reduce = [&](const float* d, int splits, size_t count, float* out) -> int {
    if (!out) return ORBX_OK;
    std::vector<float> t((size_t)splits * count);
    LCHK(cudaMemcpy(t.data(), d, sizeof(float) * t.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < count; i++) {
      double acc = 0.0;
      for (int k = 0; k < splits; k++) acc += t[(size_t)k * count + i];
      out[i] = (float)acc;
    }
    return ORBX_OK;
  };
  LRC(reduce(T.P1, T.s1, (size_t)Hd * 256, h_dw1));
  LRC(reduce(T.Pb1, T.chunks, (size_t)Hd, h_db1));
  LRC(reduce(T.P2, T.s2, (size_t)C * Hd, h_dw2));
  LRC(reduce(T.Pb2, T.chunks, (size_t)C, h_db2));
  if (h_loss) {
    std::vector<float> t(n);
    LCHK(cudaMemcpy(t.data(), T.loss, sizeof(float) * n, cudaMemcpyDeviceToHost));
    double acc = 0.0;
    for (float v : t) acc += v;
    *h_loss = (float)(acc / n);
  }
  int h_err = 0;
  LCHK(cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h_err) {
    cudaMemset(err, 0, sizeof(int));
    return ORBX_ERR_TIMEOUT;
  }
  return ORBX_OK;
}

ORBX_API int orbx_learned_destroy(orbx_learned* L) {
  if (!L) return ORBX_ERR_ARG;
  Guard g(L->device);
  cudaDeviceSynchronize();
  delete L;
  return ORBX_OK;
}

ORBX_API int orbx_gemm_bf16(orbx_ctx* ctx, const void* d_a, const void* d_b, int M, int N, int K, const float* d_bias,
                            int mode, int splits, void* d_c, const void* d_aux) {
  if (!ctx || !d_a || !d_b || !d_c || M < 0 || N < 0 || K < 0 || mode < kStoreF32 || mode > kTop8Row || splits < 1)
    return ORBX_ERR_ARG;
  if (mode == kMaskBF16 && !d_aux) return ORBX_ERR_ARG;
  if (M % 128 || N % 256 || (K % (64 * splits)) || (splits > 1 && mode != kStoreF32) ||
      ((mode == kTop8 || mode == kTop8Row) && N > 4096))
    return ORBX_ERR_SIZE;
  Guard g(ctx_device(ctx));
  LCHK(gemm(ctx_stream(ctx), ctx_err(ctx), static_cast<const bf16*>(d_a), static_cast<const bf16*>(d_b), M, N, K,
            d_bias, mode, splits, static_cast<float*>(d_c), static_cast<bf16*>(d_c), static_cast<const bf16*>(d_aux),
            static_cast<uint32_t*>(d_c)));
  return ORBX_OK;
}
