// Learned matching proposal: declarations shared by the BF16 tensor-core GEMM
// (orbx_gemm.cu), the MLP / k-means / search kernels (orbx_learned.cu) and the
// host driver (orbx_learned_api.cu).  There is no counterpart in the
// reference: it only has exact brute-force matching (orbd.cu:1471-1559).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace orbx {

// GEMM epilogue modes: C[m][n] = sum_k A[m][k] * B[n][k]
enum GemmMode {
  kStoreF32 = 0,      // fp32 (+ bias[n]); with splits > 1, partial sums at c_f32 + split * M * N
  kBiasReluBF16 = 1,  // bf16 max(acc + bias[n], 0)
  kMaskBF16 = 2,      // bf16 acc where aux[m][n] > 0 else 0 (ReLU backward)
  kStoreBF16 = 3,     // bf16 acc (+ bias[n])
  kTop8 = 4,          // per row and 128 columns: the 8 largest (acc + bias[n]) as packed keys
  kTop8Row = 5,       // per row, the 8 largest over each of gemm_top_lists(N) column sets (see below)
};

// kTop8Row: a block takes an M tile with half of the 256-column N tiles (all
// of them when N / 256 is odd) and each row keeps one running top-8 per
// 128-column half of those tiles, so list l = 2 * part + half covers columns
// {256 t + 128 half + c : t in part's tiles, c < 128}.  Lists per row:
__host__ __device__ __forceinline__ int gemm_top_parts(int n_tiles) { return (n_tiles % 2 == 0) ? 2 : 1; }
__host__ __device__ __forceinline__ int gemm_top_lists(int N) { return 2 * gemm_top_parts(N / 256); }

struct GemmArgs {
  const __nv_bfloat16* a;  // [M][K]
  const __nv_bfloat16* b;  // [N][K]
  int M, N, K;             // M % 128 == 0, N % 256 == 0, K % 64 == 0 (K % (64 * splits) == 0)
  int splits;              // K splits (kStoreF32 only); 1 otherwise
  int mode;
  const float* bias;       // optional [N]
  float* c_f32;            // kStoreF32
  __nv_bfloat16* c_bf16;   // kBiasReluBF16, kMaskBF16, kStoreBF16
  const __nv_bfloat16* aux;  // kMaskBF16: [M][N]
  uint32_t* top_keys;      // kTop8: [M][N / 128][8]; kTop8Row: [M][gemm_top_lists(N)][8]; descending
  int* err;                // device error word
};

cudaError_t launch_gemm_bf16(const GemmArgs& g, cudaStream_t s);

// Top-8 keys: the logit's order-preserving 32-bit image with its low 12 bits
// replaced by 4095 - column, so a larger key is a larger logit (to about
// 2^-11 relative) and, among equal logits, the smaller column.  N <= 4096.
constexpr int kTopK = 8;
constexpr int kTopColBits = 12;
__host__ __device__ __forceinline__ uint32_t float_order_bits(float f) {
#ifdef __CUDA_ARCH__
  const uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  __builtin_memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float order_bits_float(uint32_t o) {
  const uint32_t u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ __forceinline__ uint32_t top_key(float logit, int col) {
  return (float_order_bits(logit) & ~((1u << kTopColBits) - 1u)) | (uint32_t)((1 << kTopColBits) - 1 - col);
}
__host__ __device__ __forceinline__ int top_key_col(uint32_t key) {
  return (1 << kTopColBits) - 1 - (int)(key & ((1u << kTopColBits) - 1u));
}

struct AdamStep {
  float lr, b1, b2, eps;
  float c1, c2;  // 1 / (1 - b1^t), 1 / (1 - b2^t)
};

// orbx_learned.cu
__global__ void k_bits_pm1_bf16(const uint8_t* bits, int n, const int* d_n, int rows, __nv_bfloat16* out);
__global__ void k_bits_pm1_bf16_t(const uint8_t* bits, int n, int rows, __nv_bfloat16* out);
__global__ void k_softmax_xent(const float* logits, const int* labels, int S, int n, int rows, int C,
                               float grad_scale, __nv_bfloat16* dL, float* loss, int* correct);
__global__ void k_transpose_bf16(const __nv_bfloat16* in, int R, int C, __nv_bfloat16* out);
__global__ void k_colsum_bf16(const __nv_bfloat16* in, int R, int C, int rows_per_chunk, float* partial);
__global__ void k_adam(float* w, float* m, float* v, const float* partial, int nsplit, long long n,
                       __nv_bfloat16* w_bf16, AdamStep a);
__global__ void k_init_normal(float* w, long long n, float stddev, unsigned long long seed, __nv_bfloat16* w_bf16);
__global__ void k_assign(const int32_t* idx2, int n, int* assign, int* counts, int* changed);
__global__ void k_scan_counts(const int* counts, int k, int* offsets, int* cursor, int per_item, int* items);
__global__ void k_scatter_members(const int* assign, int n, int* cursor, int* members);
__global__ void k_majority(const uint8_t* db, int n, const int* members, const int* offsets, uint8_t* centroids,
                           unsigned long long seed, int iter);
__global__ void k_gather_rows(const uint8_t* db, const int* members, int n, uint8_t* out);
__global__ void k_gather_i32(const int* in, const int* idx, int n, int width, int* out);
__global__ void k_count(const int* assign, int n, int* counts);
__global__ void k_accum_stats(const float* loss, const int* correct, int n, float* acc);
__global__ void k_labels(const int32_t* idx2, int n, const int* row_sets, int set_width, int S, int* labels);
__global__ void k_select_probes(const uint32_t* keys, int nq, int lists, int n_probe, float margin_thr,
                                const int* ivf_offsets, int* probes, float* margin, int* probe_counts,
                                uint2* partial, int per_slot);
__global__ void k_fill_probe_lists(const int* probes, int nq, int* cursor, int* list);
__global__ void k_rerank(const uint8_t* q_desc, const int* list, const int* probe_offsets, const int* item_offsets,
                         int n_clusters, const uint8_t* ivf_desc, const int* ivf_members, const int* ivf_offsets,
                         uint2* partial);
__global__ void k_merge_probes(const uint2* partial, int per_slot, int nq, const float* margin, float margin_thr,
                               int max_dist, uint32_t* dist2, int32_t* idx2, int* fb_list, int* fb_count);
__global__ void k_pad_counts(const int* ivf_offsets, int C, int* pad_counts);
__global__ void k_probe_pairs(const int* probe_offsets, const int* ivf_offsets, int C, unsigned long long* out);
__global__ void k_fill_pad(const uint8_t* db, const int* ivf_members, const int* ivf_offsets, const int* pad_offsets,
                           uint8_t* pad_desc, int* pad_members);
__global__ void k_init_centroid_mlp(const uint8_t* centroids, int C, int Hd, float scale, float* w1, float* b1,
                                    float* w2, float* b2, __nv_bfloat16* w1b, __nv_bfloat16* w2b);
__global__ void k_perturb_rows(const uint8_t* db, int ndb, int n, unsigned long long seed, float flip_lo,
                               float flip_hi, uint8_t* out);
__global__ void k_count_spill(const int32_t* idx, int n, int per_row, int* counts);
__global__ void k_scatter_spill(const int32_t* idx, int n, int per_row, int* cursor, int* members);
__global__ void k_select_topk(const uint32_t* keys, int n, int lists, int s, int* out);
constexpr int kStableEntries = 4096;  // list entries per block of the stable list construction
__global__ void k_stable_hist(const int32_t* idx, long long total, int C, int* hist);
__global__ void k_stable_scan(int* hist, int nb, int C, const int* offsets);
__global__ void k_stable_scatter(const int32_t* idx, long long total, int per_row, int C, const int* hist,
                                 int* members);
__global__ void k_gather_fallback(const uint8_t* q_desc, const int* fb_list, const int* fb_count, uint8_t* out);
__global__ void k_scatter_fallback(const int* fb_list, const int* fb_count, const uint32_t* fd, const int32_t* fi,
                                   uint32_t* dist2, int32_t* idx2);
__global__ void k_lsh_probes(const float* proj, int rows_stride, int n, int nbits, int n_probe, const int* ivf_offsets,
                             int* probes, int* probe_counts, int* bucket_out, float* margin, uint2* partial,
                             int per_slot);
constexpr int kRerankQ = 128;

}  // namespace orbx
