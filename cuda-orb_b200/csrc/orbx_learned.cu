// Kernels of the learned matching proposal (no counterpart in the reference,
// whose only matcher is exact brute force, orbd.cu:1471-1559):
//  - bit rows -> +-1 bf16 rows (row-major and transposed) for the MLP GEMMs;
//  - softmax cross-entropy forward + gradient, bf16 transposes, column sums
//    and a fused split-sum + Adam update for training;
//  - Hamming k-majority clustering of the database (assignment comes from the
//    exact k = 2 matcher against the centroids);
//  - search: top-8 cluster probes per query from the GEMM's top-8 keys, probe
//    lists per cluster, exact Hamming rerank of each probed cluster, merge,
//    and the plumbing that sends low-margin queries to exact brute force.
#include "orbx_device.cuh"
#include "orbx_internal.cuh"
#include "orbx_learned.cuh"

namespace orbx {

namespace {
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ float u01(uint64_t h) {  // (0, 1]
  return ((float)(h >> 40) + 1.0f) * (1.0f / 16777216.0f);
}
constexpr uint16_t kBfPlus1 = 0x3F80u, kBfMinus1 = 0xBF80u;
}  // namespace

// ---------------------------------------------------------------- expansion
// out[r][k] = bit k of row r ? +1 : -1 (bit k = byte k / 8, bit k % 8), rows
// n..rows-1 are zero.  One thread per (row, byte): one 16-byte store.
__global__ void k_bits_pm1_bf16(const uint8_t* __restrict__ bits, int n, const int* d_n, int rows,
                                __nv_bfloat16* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)rows * 32) return;
  const int r = (int)(t >> 5), j = (int)(t & 31);
  const int nv = d_n ? min(*d_n, n) : n;
  uint4 v = make_uint4(0, 0, 0, 0);
  if (r < nv) {
    const uint32_t b = bits[(size_t)r * 32 + j];
    uint32_t w[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const uint32_t lo = (b >> (2 * e)) & 1u ? kBfPlus1 : kBfMinus1;
      const uint32_t hi = (b >> (2 * e + 1)) & 1u ? kBfPlus1 : kBfMinus1;
      w[e] = lo | (hi << 16);
    }
    v = make_uint4(w[0], w[1], w[2], w[3]);
  }
  reinterpret_cast<uint4*>(out)[t] = v;
}

// Transposed: out[k][r] for r < rows (rows % 64 == 0).  A block takes 64 rows:
// their bits go to shared memory, then thread k writes 64 values of row k.
__global__ void __launch_bounds__(256) k_bits_pm1_bf16_t(const uint8_t* __restrict__ bits, int n, int rows,
                                                         __nv_bfloat16* __restrict__ out) {
  __shared__ uint8_t s[64 * 32];
  const int r0 = blockIdx.x * 64;
  for (int i = threadIdx.x; i < 64 * 32; i += 256) {
    const int r = r0 + i / 32;
    s[i] = r < n ? bits[(size_t)r * 32 + (i & 31)] : 0;
  }
  __syncthreads();
  const int k = threadIdx.x;
  uint4* dst = reinterpret_cast<uint4*>(out + (size_t)k * rows + r0);
#pragma unroll
  for (int q = 0; q < 8; q++) {
    uint32_t w[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int ra = 8 * q + 2 * e, rb = ra + 1;
      const uint32_t lo = (r0 + ra < n) ? (((s[ra * 32 + (k >> 3)] >> (k & 7)) & 1u) ? kBfPlus1 : kBfMinus1) : 0u;
      const uint32_t hi = (r0 + rb < n) ? (((s[rb * 32 + (k >> 3)] >> (k & 7)) & 1u) ? kBfPlus1 : kBfMinus1) : 0u;
      w[e] = lo | (hi << 16);
    }
    dst[q] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// ---------------------------------------------------------------- training
// One warp per row of C logits (C % 128 == 0) with a set of S labels
// labels[r * S ..] (-1 entries unused; S = 1 is the usual one-hot target).
// With P = the softmax mass on the set, rows r < n with a label get
// loss[r] = -log P, dL = (softmax - softmax * [c in set] / P) * grad_scale and
// correct[r] = (argmax in the set); other rows get dL = 0, loss 0, correct 0.
__global__ void __launch_bounds__(256) k_softmax_xent(const float* __restrict__ logits, const int* __restrict__ labels,
                                                      int S, int n, int rows, int C, float grad_scale,
                                                      __nv_bfloat16* __restrict__ dL, float* __restrict__ loss,
                                                      int* __restrict__ correct) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const int r = warp;
  const int mine = (r < n && lane < S) ? labels[(size_t)r * S + lane] : -1;
  const bool any = __any_sync(0xffffffffu, mine >= 0);
  uint2* drow = reinterpret_cast<uint2*>(dL + (size_t)r * C);
  if (!any) {
    for (int c = lane; c < C / 4; c += 32) drow[c] = make_uint2(0, 0);
    if (lane == 0) {
      loss[r] = 0.f;
      correct[r] = 0;
    }
    return;
  }
  const float4* row = reinterpret_cast<const float4*>(logits + (size_t)r * C);
  float mx = -3.0e38f;
  int amax = 0;
  for (int c = lane; c < C / 4; c += 32) {
    const float4 v = row[c];
    if (v.x > mx) { mx = v.x; amax = 4 * c; }
    if (v.y > mx) { mx = v.y; amax = 4 * c + 1; }
    if (v.z > mx) { mx = v.z; amax = 4 * c + 2; }
    if (v.w > mx) { mx = v.w; amax = 4 * c + 3; }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const float om = __shfl_xor_sync(0xffffffffu, mx, o);
    const int oa = __shfl_xor_sync(0xffffffffu, amax, o);
    if (om > mx || (om == mx && oa < amax)) {
      mx = om;
      amax = oa;
    }
  }
  float sum = 0.f;
  for (int c = lane; c < C / 4; c += 32) {
    const float4 v = row[c];
    sum += __expf(v.x - mx) + __expf(v.y - mx) + __expf(v.z - mx) + __expf(v.w - mx);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  const float inv = 1.0f / sum;
  // the set's unnormalised mass
  const float em = mine >= 0 ? __expf(logits[(size_t)r * C + mine] - mx) : 0.f;
  float es = em;
#pragma unroll
  for (int o = 16; o; o >>= 1) es += __shfl_xor_sync(0xffffffffu, es, o);
  for (int c = lane; c < C / 4; c += 32) {
    const float4 v = row[c];
    const float p[4] = {__expf(v.x - mx) * inv, __expf(v.y - mx) * inv, __expf(v.z - mx) * inv,
                        __expf(v.w - mx) * inv};
    const __nv_bfloat162 a = __floats2bfloat162_rn(p[0] * grad_scale, p[1] * grad_scale);
    const __nv_bfloat162 b = __floats2bfloat162_rn(p[2] * grad_scale, p[3] * grad_scale);
    drow[c] = make_uint2(*reinterpret_cast<const uint32_t*>(&a), *reinterpret_cast<const uint32_t*>(&b));
  }
  __syncwarp();
  // label columns: p - p / P = p - e / es
  if (mine >= 0) dL[(size_t)r * C + mine] = __float2bfloat16_rn((em * inv - em / es) * grad_scale);
  const unsigned hit = __ballot_sync(0xffffffffu, mine == amax);
  if (lane == 0) {
    loss[r] = logf(sum) - logf(es);
    correct[r] = hit ? 1 : 0;
  }
}

// out[c][r] = in[r][c]; R % 32 == 0, C % 32 == 0.  32 x 32 tiles, 32 x 8 threads.
__global__ void __launch_bounds__(256) k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int R, int C,
                                                        __nv_bfloat16* __restrict__ out) {
  __shared__ uint16_t t[32][33];
  const uint16_t* src = reinterpret_cast<const uint16_t*>(in);
  uint16_t* dst = reinterpret_cast<uint16_t*>(out);
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) t[i][threadIdx.x] = src[(size_t)(r0 + i) * C + c0 + threadIdx.x];
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) dst[(size_t)(c0 + i) * R + r0 + threadIdx.x] = t[threadIdx.x][i];
}

// partial[chunk][c] = sum of in[r][c] over the chunk's rows (C % 64 == 0).
// grid (C / 64, chunks); 8 warps split the rows, lane holds two columns.
__global__ void __launch_bounds__(256) k_colsum_bf16(const __nv_bfloat16* __restrict__ in, int R, int C,
                                                     int rows_per_chunk, float* __restrict__ partial) {
  __shared__ float2 s[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * 64 + 2 * lane;
  const int rb = blockIdx.y * rows_per_chunk, re = min(R, rb + rows_per_chunk);
  float2 acc = make_float2(0.f, 0.f);
  for (int r = rb + warp; r < re; r += 8) {
    const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(in + (size_t)r * C + c);
    const float2 f = __bfloat1622float2(v);
    acc.x += f.x;
    acc.y += f.y;
  }
  s[warp][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    float2 t = s[0][lane];
    for (int w = 1; w < 8; w++) {
      t.x += s[w][lane].x;
      t.y += s[w][lane].y;
    }
    partial[(size_t)blockIdx.y * C + c] = t.x;
    partial[(size_t)blockIdx.y * C + c + 1] = t.y;
  }
}

// g = sum of nsplit partial gradients; Adam step on the fp32 master weights;
// bf16 copy for the GEMMs.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ partial, int nsplit, long long n, __nv_bfloat16* __restrict__ w_bf16,
                       AdamStep a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float g = 0.f;
  for (int s = 0; s < nsplit; s++) g += partial[(size_t)s * n + i];
  const float mi = a.b1 * m[i] + (1.f - a.b1) * g;
  const float vi = a.b2 * v[i] + (1.f - a.b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - a.lr * (mi * a.c1) / (sqrtf(vi * a.c2) + a.eps);
  w[i] = wi;
  if (w_bf16) w_bf16[i] = __float2bfloat16_rn(wi);
}

// w[i] = std * N(0, 1) from a counter-based hash (Box-Muller), bf16 copy.
__global__ void k_init_normal(float* __restrict__ w, long long n, float stddev, unsigned long long seed,
                              __nv_bfloat16* __restrict__ w_bf16) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t h1 = splitmix64(seed ^ (2ull * (uint64_t)i));
  const uint64_t h2 = splitmix64(seed ^ (2ull * (uint64_t)i + 1ull));
  const float z = sqrtf(-2.f * logf(u01(h1))) * cospif(2.f * u01(h2));
  w[i] = stddev * z;
  if (w_bf16) w_bf16[i] = __float2bfloat16_rn(w[i]);
}

// MLP weights that compute nearest-centroid scores: hidden unit j < 256 is
// relu(x_j), unit 256 + j is relu(-x_j) (the rest start at zero), so with
// s_c = +-1 centroid bits, logit_c = scale * sum_j s_cj (relu(x_j) - relu(-x_j))
// = scale * (256 - 2 * Hamming(x, centroid c)).
__global__ void k_init_centroid_mlp(const uint8_t* __restrict__ centroids, int C, int Hd, float scale,
                                    float* __restrict__ w1, float* __restrict__ b1, float* __restrict__ w2,
                                    float* __restrict__ b2, __nv_bfloat16* __restrict__ w1b,
                                    __nv_bfloat16* __restrict__ w2b) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n1 = (long long)Hd * 256, n2 = (long long)C * Hd;
  if (t < n1) {
    const int j = (int)(t / 256), k = (int)(t % 256);
    const float v = (j < 256 && j == k) ? 1.f : ((j >= 256 && j < 512 && j - 256 == k) ? -1.f : 0.f);
    w1[t] = v;
    w1b[t] = __float2bfloat16_rn(v);
  }
  if (t < n2) {
    const int c = (int)(t / Hd), j = (int)(t % Hd);
    float v = 0.f;
    if (j < 512) {
      const int k = j & 255;
      const float sbit = ((centroids[(size_t)c * 32 + (k >> 3)] >> (k & 7)) & 1u) ? 1.f : -1.f;
      v = j < 256 ? scale * sbit : -scale * sbit;
    }
    w2[t] = v;
    w2b[t] = __float2bfloat16_rn(v);
  }
  if (t < Hd) b1[t] = 0.f;
  if (t < C) b2[t] = 0.f;
}

// out[r] = a random database row with each bit flipped with probability
// p_r ~ U[flip_lo, flip_hi] (counter-based hash per row and bit).  One thread
// per (row, 32-bit word).
__global__ void k_perturb_rows(const uint8_t* __restrict__ db, int ndb, int n, unsigned long long seed, float flip_lo,
                               float flip_hi, uint8_t* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8ll * n) return;
  const int r = (int)(t >> 3), w = (int)(t & 7);
  const uint64_t hr = splitmix64(seed ^ (0x9E37ull << 40) ^ (uint64_t)r);
  const int src = (int)(hr % (uint64_t)ndb);
  const float p = fminf(flip_lo + (flip_hi - flip_lo) * u01(splitmix64(hr ^ 0x5bd1e995ull)), 0.99999994f);
  const uint32_t thr = (uint32_t)(fmaxf(p, 0.f) * 16777216.0f) << 8;  // p * 2^32, below 2^32
  uint32_t v = reinterpret_cast<const uint32_t*>(db)[(size_t)src * 8 + w];
  for (int b = 0; b < 32; b++) {
    const uint32_t h = (uint32_t)splitmix64(hr ^ ((uint64_t)(w * 32 + b) << 32));
    if (h < thr) v ^= 1u << b;
  }
  reinterpret_cast<uint32_t*>(out)[(size_t)r * 8 + w] = v;
}

// Spill lists: entry e < 2n is row e / 2 in cluster idx2[e] (its nearest, then
// second-nearest centroid from the k = 2 matcher).
// Lists from per-row cluster choices idx[row * per_row + j] (negative: none).
__global__ void k_count_spill(const int32_t* __restrict__ idx, int n, int per_row, int* __restrict__ counts) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (long long)n * per_row && idx[e] >= 0) atomicAdd(&counts[idx[e]], 1);
}
__global__ void k_scatter_spill(const int32_t* __restrict__ idx, int n, int per_row, int* __restrict__ cursor,
                                int* __restrict__ members) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (long long)n * per_row && idx[e] >= 0) members[atomicAdd(&cursor[idx[e]], 1)] = (int)(e / per_row);
}

// Stable list construction.  Entries e = row * per_row + j, in increasing e,
// go to their cluster's list in that order: block b of the histogram and the
// scatter owns entries [b * kStableEntries, + kStableEntries).
__global__ void __launch_bounds__(256) k_stable_hist(const int32_t* __restrict__ idx, long long total, int C,
                                                     int* __restrict__ hist) {
  extern __shared__ int s_h[];
  for (int c = threadIdx.x; c < C; c += blockDim.x) s_h[c] = 0;
  __syncthreads();
  const long long e0 = (long long)blockIdx.x * kStableEntries;
  const long long e1 = min(total, e0 + kStableEntries);
  for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int c = idx[e];
    if (c >= 0) atomicAdd(&s_h[c], 1);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) hist[(size_t)blockIdx.x * C + c] = s_h[c];
}

// hist[b][c] <- offsets[c] + entries of cluster c in blocks before b.
__global__ void k_stable_scan(int* __restrict__ hist, int nb, int C, const int* __restrict__ offsets) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  int run = offsets[c];
  for (int b = 0; b < nb; b++) {
    const int v = hist[(size_t)b * C + c];
    hist[(size_t)b * C + c] = run;
    run += v;
  }
}

// One warp per block of entries, 32 at a time in order: lanes with the same
// cluster take consecutive positions in lane order.
__global__ void __launch_bounds__(32) k_stable_scatter(const int32_t* __restrict__ idx, long long total, int per_row,
                                                       int C, const int* __restrict__ hist,
                                                       int* __restrict__ members) {
  extern __shared__ int s_cur[];
  const int lane = threadIdx.x;
  for (int c = lane; c < C; c += 32) s_cur[c] = hist[(size_t)blockIdx.x * C + c];
  __syncwarp();
  const long long e0 = (long long)blockIdx.x * kStableEntries;
  const long long e1 = min(total, e0 + kStableEntries);
  for (long long base = e0; base < e1; base += 32) {
    const long long e = base + lane;
    const int c = e < e1 ? idx[e] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (c >= 0) members[s_cur[c] + rank] = (int)(e / per_row);
    __syncwarp();
    if (c >= 0 && rank == 0) s_cur[c] += __popc(peers);
    __syncwarp();
  }
}

// One warp per row: the row's s <= 16 best columns from the GEMM's top-8 key
// lists (lists of 128 columns, 8 keys each, descending), written as column
// indices out[row * s + j] in decreasing key order (-1 past the keys).
__global__ void __launch_bounds__(256) k_select_topk(const uint32_t* __restrict__ keys, int n, int lists, int s,
                                                     int* __restrict__ out) {
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int nk = lists * kTopK;  // <= 256
  const int kpl = (nk + 31) >> 5;
  uint32_t mine[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int j = lane * kpl + i;
    mine[i] = (i < kpl && j < nk) ? keys[(size_t)r * nk + j] : 0u;
  }
#pragma unroll
  for (int a = 0; a < 7; a++)
#pragma unroll
    for (int b = 0; b < 7 - a; b++) {
      const uint32_t hi = max(mine[b], mine[b + 1]), lo = min(mine[b], mine[b + 1]);
      mine[b] = hi;
      mine[b + 1] = lo;
    }
  for (int i = 0; i < s; i++) {
    const uint32_t m = __reduce_max_sync(0xffffffffu, mine[0]);
    if (lane == 0) out[(size_t)r * s + i] = m ? top_key_col(m) : -1;
    if (mine[0] == m && m != 0u) {
#pragma unroll
      for (int k = 0; k < 7; k++) mine[k] = mine[k + 1];
      mine[7] = 0u;
    }
  }
}

// ---------------------------------------------------------------- k-majority
// assign[i] = nearest centroid (the k = 2 matcher's first index); counts per
// cluster; changed = number of rows whose cluster moved.
__global__ void k_assign(const int32_t* __restrict__ idx2, int n, int* __restrict__ assign, int* __restrict__ counts,
                         int* __restrict__ changed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = idx2[2 * i];
  if (assign[i] != c) atomicAdd(changed, 1);
  assign[i] = c;
  atomicAdd(&counts[c], 1);
}

// offsets[0..k] = exclusive scan of counts[0..k-1]; cursor = copy of offsets;
// optional items[0..k] = exclusive scan of ceil(counts / per_item).  One block
// of 1024 threads; k <= 1024 * 8.
__global__ void __launch_bounds__(1024) k_scan_counts(const int* __restrict__ counts, int k, int* __restrict__ offsets,
                                                      int* __restrict__ cursor, int per_item, int* __restrict__ items) {
  __shared__ int s_sum[1024], s_items[1024];
  const int t = threadIdx.x;
  const int per = (k + 1023) / 1024;
  int local = 0, local_items = 0;
  for (int j = 0; j < per; j++) {
    const int c = t * per + j;
    if (c < k) {
      local += counts[c];
      if (per_item > 0) local_items += (counts[c] + per_item - 1) / per_item;
    }
  }
  s_sum[t] = local;
  s_items[t] = local_items;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int a = t >= o ? s_sum[t - o] : 0;
    const int b = t >= o ? s_items[t - o] : 0;
    __syncthreads();
    s_sum[t] += a;
    s_items[t] += b;
    __syncthreads();
  }
  int run = s_sum[t] - local, run_items = s_items[t] - local_items;
  for (int j = 0; j < per; j++) {
    const int c = t * per + j;
    if (c < k) {
      offsets[c] = run;
      if (cursor) cursor[c] = run;
      if (per_item > 0) items[c] = run_items;
      run += counts[c];
      if (per_item > 0) run_items += (counts[c] + per_item - 1) / per_item;
    }
  }
  if (t == 1023) {
    offsets[k] = s_sum[1023];
    if (per_item > 0) items[k] = s_items[1023];
  }
}

__global__ void k_scatter_members(const int* __restrict__ assign, int n, int* __restrict__ cursor,
                                  int* __restrict__ members) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  members[atomicAdd(&cursor[assign[i]], 1)] = i;
}

// Bitwise majority of each cluster's members (ties keep the old bit); an empty
// cluster takes a database row chosen by a hash of (seed, iteration, cluster).
// One block of 256 threads per cluster, thread t counts bit t.
__global__ void __launch_bounds__(256) k_majority(const uint8_t* __restrict__ db, int n, const int* __restrict__ members,
                                                  const int* __restrict__ offsets, uint8_t* __restrict__ centroids,
                                                  unsigned long long seed, int iter) {
  const int c = blockIdx.x;
  const int t = threadIdx.x;
  const int beg = offsets[c], end = offsets[c + 1];
  __shared__ uint32_t s_bits[8];
  if (t < 8) s_bits[t] = 0u;
  __syncthreads();
  uint32_t bit;
  if (end == beg) {
    const int src = (int)(splitmix64(seed ^ ((uint64_t)iter << 32) ^ (uint64_t)c) % (uint64_t)n);
    bit = (db[(size_t)src * 32 + (t >> 3)] >> (t & 7)) & 1u;
  } else {
    int cnt = 0;
    for (int j = beg; j < end; j++) cnt += (db[(size_t)members[j] * 32 + (t >> 3)] >> (t & 7)) & 1;
    const int size = end - beg;
    const uint32_t old = (centroids[(size_t)c * 32 + (t >> 3)] >> (t & 7)) & 1u;
    bit = 2 * cnt > size ? 1u : (2 * cnt < size ? 0u : old);
  }
  if (bit) atomicOr(&s_bits[t >> 5], 1u << (t & 31));
  __syncthreads();
  if (t < 8) reinterpret_cast<uint32_t*>(centroids + (size_t)c * 32)[t] = s_bits[t];
}

// out[j] = db row members[j] (32 bytes), two threads per row.
__global__ void k_gather_rows(const uint8_t* __restrict__ db, const int* __restrict__ members, int n,
                              uint8_t* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2ll * n) return;
  const int j = (int)(t >> 1), h = (int)(t & 1);
  reinterpret_cast<uint4*>(out)[2 * (size_t)j + h] = reinterpret_cast<const uint4*>(db)[2 * (size_t)members[j] + h];
}

// out[j] = in[idx[j]]
__global__ void k_gather_i32(const int* __restrict__ in, const int* __restrict__ idx, int n, int width,
                             int* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * width) return;
  const int i = (int)(t / width), j = (int)(t - (long long)i * width);
  out[t] = in[(size_t)idx[i] * width + j];
}

__global__ void k_count(const int* __restrict__ assign, int n, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&counts[assign[i]], 1);
}

// acc[0] += sum of loss, acc[1] += sum of correct (one block of 256 per 256 * 8 rows)
__global__ void __launch_bounds__(256) k_accum_stats(const float* __restrict__ loss, const int* __restrict__ correct,
                                                     int n, float* __restrict__ acc) {
  __shared__ float s_l[8], s_c[8];
  float l = 0.f, c = 0.f;
  for (int i = blockIdx.x * 256 * 8 + threadIdx.x; i < min(n, (blockIdx.x + 1) * 256 * 8); i += 256) {
    l += loss[i];
    c += (float)correct[i];
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    l += __shfl_xor_sync(0xffffffffu, l, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_l[threadIdx.x >> 5] = l;
    s_c[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float tl = 0.f, tc = 0.f;
    for (int w = 0; w < 8; w++) {
      tl += s_l[w];
      tc += s_c[w];
    }
    atomicAdd(&acc[0], tl);
    atomicAdd(&acc[1], tc);
  }
}

// labels[i] = assign[nearest database row of training row i]
// Training labels: row i's S labels are the first S clusters row_sets lists
// for its exact nearest database row (its nearest cluster when S = 1).
__global__ void k_labels(const int32_t* __restrict__ idx2, int n, const int* __restrict__ row_sets, int set_width,
                         int S, int* __restrict__ labels) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * S) return;
  const int i = (int)(t / S), j = (int)(t - (long long)i * S);
  const int nn = idx2[2 * i];
  labels[t] = nn >= 0 ? row_sets[(size_t)nn * set_width + j] : -1;
}

// ---------------------------------------------------------------- search
// One warp per query: merge the GEMM's top-8 key lists (one per 128 columns,
// lists * 8 keys) into the query's n_probe best clusters.  margin = logit1 - logit2.  A query
// whose margin is below margin_thr probes nothing (the exact fallback answers
// it); otherwise its non-empty probed clusters are counted.  Every partial entry
// (per_slot per probe slot, per_slot <= 4) starts empty.
__global__ void __launch_bounds__(256) k_select_probes(const uint32_t* __restrict__ keys, int nq, int lists,
                                                       int n_probe, float margin_thr, const int* __restrict__ ivf_offsets,
                                                       int* __restrict__ probes, float* __restrict__ margin,
                                                       int* __restrict__ probe_counts, uint2* __restrict__ partial,
                                                       int per_slot) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= nq) return;
  const int nk = lists * kTopK;  // <= 256
  const int kpl = (nk + 31) >> 5;
  uint32_t mine[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int j = lane * kpl + i;
    mine[i] = (i < kpl && j < nk) ? keys[(size_t)q * nk + j] : 0u;
  }
  // the lane's keys in descending order
#pragma unroll
  for (int a = 0; a < 7; a++)
#pragma unroll
    for (int b = 0; b < 7 - a; b++) {
      const uint32_t hi = max(mine[b], mine[b + 1]), lo = min(mine[b], mine[b + 1]);
      mine[b] = hi;
      mine[b + 1] = lo;
    }
  uint32_t best[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) {
    const uint32_t m = __reduce_max_sync(0xffffffffu, mine[0]);
    best[i] = m;
    if (mine[0] == m && m != 0u) {
#pragma unroll
      for (int k = 0; k < 7; k++) mine[k] = mine[k + 1];
      mine[7] = 0u;
    }
  }
  const float l1 = order_bits_float(best[0] & ~((1u << kTopColBits) - 1u));
  const float l2 = order_bits_float(best[1] & ~((1u << kTopColBits) - 1u));
  const float mg = l1 - l2;
  const bool fb = mg < margin_thr;  // answered by the exact fallback: nothing to probe
  if (lane < kTopK * per_slot) partial[(size_t)q * kTopK * per_slot + lane] = make_uint2(kNoKeyShared, kNoKeyShared);
  if (lane == 0) margin[q] = mg;
  if (lane < kTopK) {
    int c = -1;
#pragma unroll
    for (int i = 0; i < kTopK; i++)
      if (i == lane) c = best[i] ? top_key_col(best[i]) : -1;
    if (lane >= n_probe || fb || c < 0 || ivf_offsets[c + 1] == ivf_offsets[c]) c = -1;
    probes[(size_t)q * kTopK + lane] = c;
    if (c >= 0) atomicAdd(&probe_counts[c], 1);
  }
}

// list[cursor[c]++] = q * 8 + slot for every live probe (q, slot) of cluster c
__global__ void k_fill_probe_lists(const int* __restrict__ probes, int nq, int* __restrict__ cursor,
                                   int* __restrict__ list) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq * kTopK) return;
  const int c = probes[t];
  if (c >= 0) list[atomicAdd(&cursor[c], 1)] = t;
}

constexpr int kRerankChunk = 256;

// One block per (cluster, up to 128 probing queries): each thread holds one
// query; the cluster's rows stream through shared memory; the exact top-2 of
// the cluster (keys = distance << 22 | database index) goes to the probe slot.
__global__ void __launch_bounds__(kRerankQ) k_rerank(const uint8_t* __restrict__ q_desc, const int* __restrict__ list,
                                                     const int* __restrict__ probe_offsets,
                                                     const int* __restrict__ item_offsets, int n_clusters,
                                                     const uint8_t* __restrict__ ivf_desc,
                                                     const int* __restrict__ ivf_members,
                                                     const int* __restrict__ ivf_offsets, uint2* __restrict__ partial) {
  __shared__ uint4 s_db[kRerankChunk * 2];
  __shared__ int s_id[kRerankChunk];
  const int item = blockIdx.x;
  if (item >= item_offsets[n_clusters]) return;
  // cluster c with item_offsets[c] <= item < item_offsets[c + 1]
  int lo = 0, hi = n_clusters;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (item_offsets[mid] <= item) lo = mid;
    else hi = mid;
  }
  const int c = lo;
  const int e0 = probe_offsets[c] + (item - item_offsets[c]) * kRerankQ;
  const int e1 = min(e0 + kRerankQ, probe_offsets[c + 1]);
  const int e = e0 + (int)threadIdx.x;
  const bool active = e < e1;
  const int slot = active ? list[e] : 0;
  uint32_t qw[8];
  {
    const uint4* qp = reinterpret_cast<const uint4*>(q_desc) + 2 * (size_t)(slot >> 3);
    const uint4 v0 = __ldg(qp), v1 = __ldg(qp + 1);
    qw[0] = v0.x; qw[1] = v0.y; qw[2] = v0.z; qw[3] = v0.w;
    qw[4] = v1.x; qw[5] = v1.y; qw[6] = v1.z; qw[7] = v1.w;
  }
  const int r_beg = ivf_offsets[c], r_end = ivf_offsets[c + 1];
  uint32_t k1 = kNoKeyShared, k2 = kNoKeyShared;
  const uint4* db4 = reinterpret_cast<const uint4*>(ivf_desc);
  for (int r0 = r_beg; r0 < r_end; r0 += kRerankChunk) {
    const int rows = min(kRerankChunk, r_end - r0);
    __syncthreads();
    for (int i = threadIdx.x; i < rows * 2; i += kRerankQ) s_db[i] = __ldg(db4 + 2 * (size_t)r0 + i);
    for (int i = threadIdx.x; i < rows; i += kRerankQ) s_id[i] = __ldg(ivf_members + r0 + i);
    __syncthreads();
    for (int j = 0; j < rows; j++) {
      const uint4 t0 = s_db[2 * j], t1 = s_db[2 * j + 1];
      const uint32_t d = __popc(qw[0] ^ t0.x) + __popc(qw[1] ^ t0.y) + __popc(qw[2] ^ t0.z) +
                         __popc(qw[3] ^ t0.w) + __popc(qw[4] ^ t1.x) + __popc(qw[5] ^ t1.y) +
                         __popc(qw[6] ^ t1.z) + __popc(qw[7] ^ t1.w);
      top2_push_shared(k1, k2, (d << kIdxBitsShared) | (uint32_t)s_id[j]);
    }
  }
  if (active) partial[slot] = make_uint2(k1, k2);
}

// Per query: top-2 over its probe slots' partial pairs (per_slot pairs per
// slot; a database row listed in two probed clusters is counted once).  Queries with margin < margin_thr or a best
// distance above max_dist go to the fallback list; the others get their result.
__global__ void k_merge_probes(const uint2* __restrict__ partial, int per_slot, int nq, const float* __restrict__ margin,
                               float margin_thr, int max_dist, uint32_t* __restrict__ dist2,
                               int32_t* __restrict__ idx2, int* __restrict__ fb_list, int* __restrict__ fb_count) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  uint32_t k1 = kNoKeyShared, k2 = kNoKeyShared;
  const int n = kTopK * per_slot;
  for (int s = 0; s < n; s++) {
    const uint2 p = partial[(size_t)q * n + s];
    if (p.x != k1 && p.x != k2) top2_push_shared(k1, k2, p.x);
    if (p.y != k1 && p.y != k2) top2_push_shared(k1, k2, p.y);
  }
  const bool far = k1 == kNoKeyShared || (int)(k1 >> kIdxBitsShared) > max_dist;
  if (margin[q] < margin_thr || far) {
    if (fb_list) {
      fb_list[atomicAdd(fb_count, 1)] = q;
      return;
    }
  }
  MatchArgs a{};
  a.dist2 = dist2;
  a.idx2 = idx2;
  finish_query_shared(a, q, k1, k2);
}

__global__ void k_gather_fallback(const uint8_t* __restrict__ q_desc, const int* __restrict__ fb_list,
                                  const int* __restrict__ fb_count, uint8_t* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if ((t >> 1) >= *fb_count) return;
  const int j = t >> 1, h = t & 1;
  reinterpret_cast<uint4*>(out)[2 * (size_t)j + h] =
      reinterpret_cast<const uint4*>(q_desc)[2 * (size_t)fb_list[j] + h];
}

__global__ void k_scatter_fallback(const int* __restrict__ fb_list, const int* __restrict__ fb_count,
                                   const uint32_t* __restrict__ fd, const int32_t* __restrict__ fi,
                                   uint32_t* __restrict__ dist2, int32_t* __restrict__ idx2) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= *fb_count) return;
  const int q = fb_list[j];
  dist2[2 * q] = fd[2 * j];
  dist2[2 * q + 1] = fd[2 * j + 1];
  idx2[2 * q] = fi[2 * j];
  idx2[2 * q + 1] = fi[2 * j + 1];
}

// (query, database row) pairs a rerank scans: sum over clusters of probing
// slots x listed rows.  One block of 1024 threads.
__global__ void __launch_bounds__(1024) k_probe_pairs(const int* __restrict__ probe_offsets,
                                                      const int* __restrict__ ivf_offsets, int C,
                                                      unsigned long long* __restrict__ out) {
  __shared__ unsigned long long s_sum[32];
  unsigned long long acc = 0;
  for (int c = threadIdx.x; c < C; c += blockDim.x)
    acc += (unsigned long long)(probe_offsets[c + 1] - probe_offsets[c]) * (unsigned)(ivf_offsets[c + 1] - ivf_offsets[c]);
  for (int d = 16; d >= 1; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
  if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < (blockDim.x >> 5) ? s_sum[threadIdx.x] : 0ull;
    for (int d = 16; d >= 1; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
    if (threadIdx.x == 0) *out = acc;
  }
}

// ---------------------------------------------------------------- padded lists
// Rows per cluster rounded up to the tensor-core rerank's 256-row tile.
__global__ void k_pad_counts(const int* __restrict__ ivf_offsets, int C, int* __restrict__ pad_counts) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < C) pad_counts[c] = (ivf_offsets[c + 1] - ivf_offsets[c] + 255) / 256 * 256;
}

// Cluster c's padded rows [pad_offsets[c], pad_offsets[c + 1]): its list's
// packed database rows with their database index, then zero rows with index
// -1.  One block per cluster, 16 bytes per thread and step.
__global__ void __launch_bounds__(256) k_fill_pad(const uint8_t* __restrict__ db, const int* __restrict__ ivf_members,
                                                  const int* __restrict__ ivf_offsets,
                                                  const int* __restrict__ pad_offsets, uint8_t* __restrict__ pad_desc,
                                                  int* __restrict__ pad_members) {
  const int c = blockIdx.x;
  const int m0 = ivf_offsets[c], n = ivf_offsets[c + 1] - m0;
  const int p0 = pad_offsets[c], np = pad_offsets[c + 1] - p0;
  uint4* out = reinterpret_cast<uint4*>(pad_desc) + (size_t)p0 * 2;
  const uint4* src = reinterpret_cast<const uint4*>(db);
  for (int i = threadIdx.x; i < np * 2; i += blockDim.x) {
    const int r = i >> 1;
    out[i] = r < n ? src[(size_t)ivf_members[m0 + r] * 2 + (i & 1)] : make_uint4(0u, 0u, 0u, 0u);
  }
  for (int r = threadIdx.x; r < np; r += blockDim.x) pad_members[p0 + r] = r < n ? ivf_members[m0 + r] : -1;
}

// ---------------------------------------------------------------- LSH ablation
// Random-projection buckets: bucket = sign bits of the first nbits projections.
// Probes: the own bucket, then single-bit flips of the least confident bits
// (smallest |projection|), in that order.
__global__ void k_lsh_probes(const float* __restrict__ proj, int rows_stride, int n, int nbits, int n_probe,
                             const int* __restrict__ ivf_offsets, int* __restrict__ probes, int* __restrict__ probe_counts,
                             int* __restrict__ bucket_out, float* __restrict__ margin, uint2* __restrict__ partial,
                             int per_slot) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float* p = proj + (size_t)q * rows_stride;
  int b = 0;
  float conf[16];
  int order[16];
  for (int i = 0; i < nbits; i++) {
    const float v = p[i];
    if (v > 0.f) b |= 1 << i;
    conf[i] = fabsf(v);
    order[i] = i;
  }
  if (bucket_out) bucket_out[q] = b;
  if (!probes) return;
  // selection of the n_probe - 1 least confident bits
  for (int i = 0; i < nbits; i++)
    for (int j = i + 1; j < nbits; j++)
      if (conf[order[j]] < conf[order[i]]) {
        const int t = order[i];
        order[i] = order[j];
        order[j] = t;
      }
  margin[q] = 3.0e38f;
  for (int s = 0; s < kTopK * per_slot; s++) partial[(size_t)q * kTopK * per_slot + s] = make_uint2(kNoKeyShared, kNoKeyShared);
  for (int s = 0; s < kTopK; s++) {
    int c = -1;
    if (s < n_probe) c = s == 0 ? b : (b ^ (1 << order[s - 1]));
    if (c >= 0 && ivf_offsets[c + 1] == ivf_offsets[c]) c = -1;
    probes[(size_t)q * kTopK + s] = c;
    if (c >= 0) atomicAdd(&probe_counts[c], 1);
  }
}

}  // namespace orbx
