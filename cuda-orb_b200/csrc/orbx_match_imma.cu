// Brute-force k = 2 Hamming matching on the 5th-generation tensor cores.
//
// A 256-bit descriptor b is expanded to 256 int8 values s_k = 2*b_k - 1 (+-1),
// so for two descriptors dot(s, t) = 256 - 2 * Hamming(s, t), computed exactly
// by tcgen05.mma kind::i8 with int32 accumulation.  One block owns 128
// queries (the MMA's M) and walks 256-row database tiles (the MMA's N) with
// K = 256 = eight K=32 MMA steps per tile:
//   warp 0     TMA producer: the query tile once, database tiles through a
//              3-stage shared-memory ring (128-byte swizzle, no multicast);
//   warp 1     MMA issuer: one elected thread issues the eight MMAs of a tile
//              into one of two TMEM accumulators (2 x 256 columns) and commits
//              them to the ring's "empty" and the accumulator's "full" barriers;
//   warps 2-17 epilogue: each reads its 32 TMEM lanes (queries) over a quarter
//              of the columns into registers, hands the accumulator straight
//              back, and keeps a running best / second-best key per query.
// The block's result per query is the top-2 by (distance, index), the same
// keys as the XOR-popc kernel (orbx_match.cu), so both forms agree bit for bit.
// Every barrier wait is bounded by a clock deadline; on expiry the block
// records kErrImmaTimeout, drains its in-flight copies, frees TMEM and exits.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "orbx_device.cuh"
#include "orbx_internal.cuh"

namespace orbx {

constexpr int kIBM = 128;  // queries per block (MMA M)
constexpr int kIBN = 256;  // database rows per tile (MMA N)
constexpr int kIK = 256;   // bytes per expanded descriptor (MMA K)
constexpr int kIStages = 3;
constexpr int kIEpiWarps = 16;  // four per TMEM lane quarter, 64 columns each
constexpr int kIThreads = (2 + kIEpiWarps) * 32;
constexpr uint32_t kIHalfA = kIBM * 128;  // one 128-byte-wide K half of the query tile
constexpr uint32_t kIHalfB = kIBN * 128;
constexpr uint32_t kIATile = 2 * kIHalfA;
constexpr uint32_t kIBTile = 2 * kIHalfB;
constexpr uint32_t kINumBars = 1 + 2 * kIStages + 4;
// 1024 bytes of alignment slack, the query tile, the ring, the barriers, TMEM base + abort flag;
// the end-of-block merge scratch reuses ring stage 0 (free once the last MMA completed)
constexpr uint32_t kISmemBytes = 1024 + kIATile + kIStages * kIBTile + 8 * kINumBars + 16;
// dynamic tiles + the static s_last and per-row bounds (4 x kIBM 16-bit)
static_assert(kISmemBytes + 16 + 4 * kIBM * 2 <= 232448, "exceeds the 227 KB shared-memory opt-in");
static_assert(3 * kIBM * sizeof(uint2) <= kIBTile, "merge scratch must fit in one ring stage");
constexpr uint32_t kITmemCols = 512;
constexpr long long kIDeadlineCycles = 4000000000ll;  // ~2 s at 2 GHz

// instruction descriptor: S32 accumulate, S8 x S8, both K-major, N = 256, M = 128
constexpr uint32_t kIDesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kIBN >> 3) << 17) |
                            ((uint32_t)(kIBM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// A waiting thread is suspended by the barrier unit (woken when the phase
// completes, or after this many nanoseconds) instead of spinning on the
// ALU pipe that the epilogue warps need.
constexpr uint32_t kTryWaitSuspendNs = 20000;
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(kTryWaitSuspendNs)
      : "memory");
  return ok != 0;
}

// Bounded wait: false once the block's deadline has passed or another role aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long deadline,
                                          volatile int* abort_flag) {
  while (!mbar_try(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() > deadline) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// Dot value given to database columns past the end of the set (never selected).
constexpr int kMaskedDot = -65536;

// Three-input max of float bit patterns, without flushing denormals.
__device__ __forceinline__ float fmax3_bits(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Whether any of 32 dot products exceeds thr.  With thr >= 0 the values are
// reduced as float bit patterns by three-input max: a non-negative int32 is a
// zero or denormal float and keeps its order, a negative one is a NaN, which
// max ignores (it cannot exceed a non-negative thr anyway); 16 instructions
// instead of the 31 of an integer max.  A negative thr takes the integer max.
__device__ __forceinline__ bool any_exceeds32(const int* v, int thr) {
  if (thr >= 0) {
    float m[12];
#pragma unroll
    for (int i = 0; i < 10; i++)
      m[i] = fmax3_bits(__int_as_float(v[3 * i]), __int_as_float(v[3 * i + 1]), __int_as_float(v[3 * i + 2]));
    m[10] = __int_as_float(v[30]);
    m[11] = __int_as_float(v[31]);
    const float r0 = fmax3_bits(m[0], m[1], m[2]), r1 = fmax3_bits(m[3], m[4], m[5]);
    const float r2 = fmax3_bits(m[6], m[7], m[8]), r3 = fmax3_bits(m[9], m[10], m[11]);
    const float r = fmax3_bits(r0, r1, fmax3_bits(r2, r3, r3));
    const int rb = __float_as_int(r);
    return rb > thr && rb < 0x7F800000;  // all 32 negative: the result is a NaN
  }
  int m = v[0];
#pragma unroll
  for (int j = 1; j < 32; j++) m = max(m, v[j]);
  return m > thr;
}

// Maxima of the column groups 0-8, 9-17, 18-26 and 27-31 of a 32-column chunk,
// as float bit patterns (the reduction any_exceeds32 uses, for thr >= 0).
__device__ __forceinline__ void group_max4(const int* v, float* r) {
  float m[12];
#pragma unroll
  for (int i = 0; i < 10; i++)
    m[i] = fmax3_bits(__int_as_float(v[3 * i]), __int_as_float(v[3 * i + 1]), __int_as_float(v[3 * i + 2]));
  m[10] = __int_as_float(v[30]);
  m[11] = __int_as_float(v[31]);
  r[0] = fmax3_bits(m[0], m[1], m[2]);
  r[1] = fmax3_bits(m[3], m[4], m[5]);
  r[2] = fmax3_bits(m[6], m[7], m[8]);
  r[3] = fmax3_bits(m[9], m[10], m[11]);
}
// Whether a group maximum from group_max4 exceeds thr >= 0 (a NaN maximum
// means every value of the group was negative).
__device__ __forceinline__ bool bits_exceed(float r, int thr) {
  const int rb = __float_as_int(r);
  return rb > thr && rb < 0x7F800000;
}

// Global key (distance << 22 | index) of a chunk-local key (dot << 5 | 31 - column).
__device__ __forceinline__ uint32_t local_to_key(int lk, int g_chunk) {
  const int dot = lk >> 5;
  const int col = 31 - (lk & 31);
  return ((uint32_t)((256 - dot) >> 1) << kIdxBitsShared) | (uint32_t)(g_chunk + col);
}

// Top two of columns B .. E-1 of a chunk on local keys (dot << 5 | 31 - column),
// ties keeping the lower column, pushed into (k1, k2).
template <int B, int E>
__device__ __forceinline__ void chunk_top2_push(const int* vc, int gc, uint32_t& k1, uint32_t& k2) {
  int a1 = INT_MIN, a2 = INT_MIN;
#pragma unroll
  for (int j = B; j < E; j++) {
    const int lk = (vc[j] << 5) | (31 - j);
    a2 = max(a2, min(a1, lk));
    a1 = max(a1, lk);
  }
  if ((a1 >> 5) > kMaskedDot) top2_push_shared(k1, k2, local_to_key(a1, gc));
  if ((a2 >> 5) > kMaskedDot) top2_push_shared(k1, k2, local_to_key(a2, gc));
}

// Expand 256-bit descriptors to +-1 int8 rows; rows at or past the count are zero.
__global__ void k_expand_pm1(const uint8_t* __restrict__ bits, int n_host, const int* d_n, int rows,
                             int8_t* __restrict__ out) {
  __shared__ unsigned long long lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    unsigned long long v = 0;
    for (int j = 0; j < 8; j++) v |= (unsigned long long)(((i >> j) & 1) ? 0x01u : 0xFFu) << (8 * j);
    lut[i] = v;
  }
  __syncthreads();
  const int n = d_n ? min(*d_n, rows) : min(n_host, rows);
  const long long total = (long long)rows * 32;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long r = idx >> 5;
    const unsigned long long v = (r < n) ? lut[bits[idx]] : 0ull;
    reinterpret_cast<unsigned long long*>(out)[idx] = v;
  }
}

// Warp-uniform bounded wait: lane 0 polls, the result is broadcast.
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, long long deadline,
                                          volatile int* abort_flag) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, deadline, abort_flag) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__global__ void __launch_bounds__(kIThreads, 1)
    k_match_imma(const __grid_constant__ CUtensorMap tmQ, const __grid_constant__ CUtensorMap tmD, MatchArgs a,
                 MatchWork w, int splits, int* err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  uint8_t* sA = smem;
  uint8_t* sB = sA + kIATile;
  int* s_merge = reinterpret_cast<int*>(sB);  // used only after the last tile
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + kIStages * kIBTile);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + kINumBars);
  volatile int* s_abort = reinterpret_cast<volatile int*>(s_tmem + 1);
  __shared__ unsigned int s_last;
  // each column group's current second-best distance per query row (0xFFFF:
  // none yet): two keys at or below it exist, so it bounds what the other
  // column groups keep for that row (1 KB: the dynamic tiles leave 1.9 KB)
  __shared__ uint16_t s_d2[4][kIBM];

  const int nq = min(a.d_nq ? *a.d_nq : a.nq, w.nq_cap);
  const int ndb = a.d_ndb ? *a.d_ndb : a.ndb;
  const int qtiles = (nq + kIBM - 1) / kIBM;
  // With the query count on the device, the grid is sized for the capacity;
  // when fewer query tiles are live, their database scans are split further
  // (up to the merge scratch's splits_cap) so that the whole grid works.
  if (a.d_nq && w.splits_cap > splits && qtiles > 0) splits = max(splits, min(w.splits_cap, (int)gridDim.x / qtiles));
  const int qb = blockIdx.x / splits;
  const int sp = blockIdx.x - qb * splits;
  if (qb >= qtiles) return;  // uniform over the block: before any barrier or TMEM use
  const int dbtiles = (ndb + kIBN - 1) / kIBN;
  const int t_beg = (int)((long long)dbtiles * sp / splits);
  const int t_end = (int)((long long)dbtiles * (sp + 1) / splits);
  const int ntiles = t_end - t_beg;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t bar0 = smem_u32(bars);
  const uint32_t BAR_A = bar0;
#define BAR_BFULL(s) (bar0 + 8u * (1 + (s)))
#define BAR_BEMPTY(s) (bar0 + 8u * (1 + kIStages + (s)))
#define BAR_ACCFULL(s) (bar0 + 8u * (1 + 2 * kIStages + (s)))
#define BAR_ACCEMPTY(s) (bar0 + 8u * (3 + 2 * kIStages + (s)))

  for (int i = threadIdx.x; i < 4 * kIBM; i += blockDim.x) (&s_d2[0][0])[i] = 0xFFFFu;
  if (threadIdx.x == 0) {
    mbar_init(BAR_A, 1);
    for (int s = 0; s < kIStages; s++) {
      mbar_init(BAR_BFULL(s), 1);
      mbar_init(BAR_BEMPTY(s), 1);
    }
    for (int s = 0; s < 2; s++) {
      mbar_init(BAR_ACCFULL(s), 1);
      mbar_init(BAR_ACCEMPTY(s), kIEpiWarps);
    }
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(kITmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *s_tmem;
  const long long deadline = clock64() + kIDeadlineCycles;

  // epilogue state (warps 2..17): best and second-best key of this row
  const int quarter = warp & 3;
  const int colgrp = (warp >= 2) ? ((warp - 2) >> 2) : 0;
  uint32_t k1 = kNoKeyShared, k2 = kNoKeyShared;

  if (warp == 0) {
    if (lane == 0) {
      // TMA producer
      int issued[kIStages];
      for (int s = 0; s < kIStages; s++) issued[s] = 0;
      bool ok = true;
      mbar_expect_tx(BAR_A, kIATile);
      tma_load_2d(smem_u32(sA), &tmQ, 0, qb * kIBM, BAR_A);
      tma_load_2d(smem_u32(sA + kIHalfA), &tmQ, 128, qb * kIBM, BAR_A);
      for (int i = 0; i < ntiles; i++) {
        const int s = i % kIStages;
        const int use = i / kIStages;
        if (use > 0 && !mbar_wait(BAR_BEMPTY(s), (use - 1) & 1, deadline, s_abort)) {
          ok = false;
          break;
        }
        const int row = (t_beg + i) * kIBN;
        mbar_expect_tx(BAR_BFULL(s), kIBTile);
        tma_load_2d(smem_u32(sB + s * kIBTile), &tmD, 0, row, BAR_BFULL(s));
        tma_load_2d(smem_u32(sB + s * kIBTile + kIHalfB), &tmD, 128, row, BAR_BFULL(s));
        issued[s]++;
      }
      if (!ok) {
        *s_abort = 1;
        atomicOr(err, kErrImmaTimeout);
      }
      // Drain before the block may exit: every issued copy has landed and every
      // MMA that read a stage has completed (its commit arrived on "empty").
      long long dl = clock64() + kIDeadlineCycles;
      while (!mbar_try(BAR_A, 0) && clock64() < dl) {
      }
      for (int s = 0; s < kIStages; s++) {
        if (issued[s] == 0) continue;
        const uint32_t par = (uint32_t)(issued[s] - 1) & 1u;
        dl = clock64() + kIDeadlineCycles;
        while (!mbar_try(BAR_BFULL(s), par) && clock64() < dl) {
        }
        dl = clock64() + kIDeadlineCycles;
        while (!mbar_try(BAR_BEMPTY(s), par) && clock64() < dl) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer: eight K=32 steps per tile into accumulator (tile & 1)
      bool ok = mbar_wait(BAR_A, 0, deadline, s_abort);
      const uint32_t a_lo = smem_u32(sA);
      for (int i = 0; ok && i < ntiles; i++) {
        const int s = i % kIStages;
        const int acc = i & 1;
        if (!mbar_wait(BAR_BFULL(s), (uint32_t)(i / kIStages) & 1u, deadline, s_abort)) {
          ok = false;
          break;
        }
        if (i >= 2 && !mbar_wait(BAR_ACCEMPTY(acc), (uint32_t)((i - 2) >> 1) & 1u, deadline, s_abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + (uint32_t)(acc * kIBN);
        const uint32_t b_lo = smem_u32(sB + s * kIBTile);
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int h = k >> 2, kk = k & 3;
          const uint64_t da = sw128_desc(a_lo + h * kIHalfA) + (uint64_t)(2 * kk);
          const uint64_t db = sw128_desc(b_lo + h * kIHalfB) + (uint64_t)(2 * kk);
          umma_i8(d, da, db, kIDesc, k > 0 ? 1u : 0u);
        }
        umma_commit(BAR_BEMPTY(s));
        umma_commit(BAR_ACCFULL(acc));
      }
      if (!ok) {
        *s_abort = 1;
        atomicOr(err, kErrImmaTimeout);
      }
    }
  } else {
    // epilogue: TMEM lanes 32*(warp&3).. (one query per lane), columns [64*colgrp, +64)
    bool ok = true;
    for (int i = 0; i < ntiles; i++) {
      const int acc = i & 1;
      if (!warp_wait(BAR_ACCFULL(acc), (uint32_t)(i >> 1) & 1u, deadline, s_abort)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int g0 = (t_beg + i) * kIBN + colgrp * 64;
      const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kIBN + colgrp * 64);
      int v[64];
      tmem_ld32(taddr, v);
      tmem_ld32(taddr + 32u, v + 32);
      tmem_wait_ld();
      // the values are in registers: hand the accumulator back to the MMA warp now
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(BAR_ACCEMPTY(acc));
      if (g0 + 64 > ndb) {
#pragma unroll
        for (int j = 0; j < 64; j++)
          if (g0 + j >= ndb) v[j] = kMaskedDot;
      }
      // the other column groups' second best for this row: a column can reach the
      // row's final top two only at or below its distance (its index may be lower)
      const int row = quarter * 32 + lane;
      unsigned gbd = 0xFFFFu;
#pragma unroll
      for (int g = 0; g < 4; g++)
        if (g != colgrp) gbd = min(gbd, (unsigned)reinterpret_cast<volatile uint16_t*>(&s_d2[g][0])[row]);
      const int thr_gb = (gbd == 0xFFFFu) ? kMaskedDot : 256 - 2 * (int)gbd - 1;
      auto next_thr = [&]() {
        return max(thr_gb, (k2 == kNoKeyShared) ? kMaskedDot : 256 - 2 * (int)(k2 >> kIdxBitsShared));
      };
      int thr = next_thr();
#pragma unroll
      for (int c = 0; c < 2; c++) {
        // columns arrive in increasing index order, so only a strictly larger dot
        // than the current second best can enter the top two
        const int* vc = v + 32 * c;
        const int gc = g0 + 32 * c;
        if (__any_sync(0xffffffffu, thr < 0)) {  // a lane has no second best yet: the whole chunk (warp-uniform)
          chunk_top2_push<0, 32>(vc, gc, k1, k2);
          thr = next_thr();
          continue;
        }
        float gm[4];
        group_max4(vc, gm);
        const float cm = fmax3_bits(gm[0], gm[1], fmax3_bits(gm[2], gm[3], gm[3]));
        if (!__any_sync(0xffffffffu, bits_exceed(cm, thr))) continue;
        // only the column groups with a value above the threshold, in column
        // order, the threshold tightening as the top two improve
        if (__any_sync(0xffffffffu, bits_exceed(gm[0], thr))) {
          chunk_top2_push<0, 9>(vc, gc, k1, k2);
          thr = next_thr();
        }
        if (__any_sync(0xffffffffu, bits_exceed(gm[1], thr))) {
          chunk_top2_push<9, 18>(vc, gc, k1, k2);
          thr = next_thr();
        }
        if (__any_sync(0xffffffffu, bits_exceed(gm[2], thr))) {
          chunk_top2_push<18, 27>(vc, gc, k1, k2);
          thr = next_thr();
        }
        if (__any_sync(0xffffffffu, bits_exceed(gm[3], thr))) {
          chunk_top2_push<27, 32>(vc, gc, k1, k2);
          thr = next_thr();
        }
      }
      if (k2 != kNoKeyShared) reinterpret_cast<volatile uint16_t*>(&s_d2[colgrp][0])[row] = (uint16_t)(k2 >> kIdxBitsShared);
    }
    if (!ok) {
      *s_abort = 1;
      if (lane == 0) atomicOr(err, kErrImmaTimeout);
    }
    if (colgrp > 0) reinterpret_cast<uint2*>(s_merge)[(colgrp - 1) * kIBM + quarter * 32 + lane] = make_uint2(k1, k2);
  }
#undef BAR_BFULL
#undef BAR_BEMPTY
#undef BAR_ACCFULL
#undef BAR_ACCEMPTY

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kITmemCols)
                 : "memory");
  }
  if (warp >= 2 && colgrp == 0) {
    // merge the four column groups of each row
    const int row = quarter * 32 + lane;
    for (int g = 0; g < 3; g++) {
      const uint2 pk = reinterpret_cast<const uint2*>(s_merge)[g * kIBM + row];
      top2_push_shared(k1, k2, pk.x);
      top2_push_shared(k1, k2, pk.y);
    }
    const int q = qb * kIBM + row;
    if (q < nq) {
      if (splits == 1)
        finish_query_shared(a, q, k1, k2);
      else
        reinterpret_cast<uint2*>(w.part)[(size_t)sp * w.nq_cap + q] = make_uint2(k1, k2);
    }
  }
  if (splits == 1) return;
  // the last block of this query tile to finish merges the partial top-2 of all splits
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&w.tile_done[qb], 1u) == (unsigned)(splits - 1)) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) w.tile_done[qb] = 0u;
  if (threadIdx.x >= kIBM) return;
  const int q = qb * kIBM + threadIdx.x;
  if (q >= nq) return;
  const uint2* part = reinterpret_cast<const uint2*>(w.part);
  uint32_t m1 = kNoKeyShared, m2 = kNoKeyShared;
  for (int s2 = 0; s2 < splits; s2++) {
    const uint2 pk = __ldcg(part + (size_t)s2 * w.nq_cap + q);
    top2_push_shared(m1, m2, pk.x);
    top2_push_shared(m1, m2, pk.y);
  }
  finish_query_shared(a, q, m1, m2);
}

// ---------------------------------------------------------------------------
// Probe rerank of the learned proposal on the tensor cores
//
// A work item is one cluster c with up to 128 of the query slots that probe it
// (list[probe_offsets[c] ..], grouped by cluster; slot = query * 8 + probe).
// The cluster's rows are kept packed (32 bytes each, padded per cluster to
// 256-row tiles) and expanded in shared memory, so HBM carries an eighth of
// the bytes expanded rows would.  The blocks are persistent and claim items
// from a global counter (items differ widely in size); the producer thread
// claims them and passes them to the other roles through a small queue:
//   warp 0      producer: each tile's 8 KB of packed rows by cp.async.bulk
//               into a 4-stage ring;
//   warp 1      MMA issuer, as in k_match_imma, into two 256-column
//               accumulators; commits release the expanded stage, the
//               accumulator and, after an item's last tile, its query tile;
//   warps 2-9   expanders: at an item's start they gather its slots' queries
//               as +-1 rows (two threads per row) into one of two query tiles,
//               then expand each packed tile to 0 / 1 rows into one of two
//               database tiles, one row per thread, in the 128-byte swizzled
//               K-major layout the TMA writes;
//   warps 10-25 epilogue: warp w reads TMEM lanes 32 * (w % 4) and 64 columns,
//               keeps the top-2 keys (distance << 22 | database index) of each
//               slot over the item's tiles (distance = popcount(query) - dot')
//               and writes them to partial[slot * 4 + column group].
// Each cluster's list is in increasing database index, so column order is
// index order and ties resolve as in the other matchers.  Every wait is bounded (kIDeadlineCycles per
// wait); on expiry the block records kErrImmaTimeout, drains its copies and
// exits.
// ---------------------------------------------------------------------------
constexpr int kRrExpWarps = 8;
constexpr int kRrThreads = (2 + kRrExpWarps + kIEpiWarps) * 32;
constexpr uint32_t kRrPStages = 4;
constexpr uint32_t kRrPTile = kIBN * 32;  // packed rows of one tile
constexpr uint32_t kRrQueue = 8;  // claimed items in flight between the producer and the other roles
constexpr uint32_t kRrNumBars = 2 + 2 + 2 * kRrPStages + 2 + 2 + 2 + 2 + 2 * kRrQueue;
// the item queue's consumers: the MMA thread, the expander and the epilogue warps
constexpr uint32_t kRrQueueReaders = 1 + kRrExpWarps + kIEpiWarps;
constexpr uint32_t kRrSmemBytes =
    1024 + 2 * kIATile + 2 * kIBTile + kRrPStages * kRrPTile + 8 * kRrNumBars + 4 * kRrQueue + 16;
static_assert(kRrSmemBytes + 16 <= 232448, "exceeds the 227 KB shared-memory opt-in");
static_assert(kRrExpWarps * 32 == kIBN && kRrExpWarps * 32 == 2 * kIBM, "one expander thread per row, two per query");

struct RrItem {
  int c;      // cluster
  int e0;     // first slot in list
  int rows;   // slots in this item (1..128)
  int nrow;   // the cluster's database rows
  int pbase;  // first padded row of the cluster
  int tiles;  // 256-row tiles
};

__device__ __forceinline__ RrItem rr_item(const RerankImmaArgs& a, int it) {
  int lo = 0, hi = a.n_clusters;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(a.item_offsets + mid) <= it) lo = mid;
    else hi = mid;
  }
  RrItem r;
  r.c = lo;
  r.e0 = __ldg(a.probe_offsets + lo) + (it - __ldg(a.item_offsets + lo)) * kIBM;
  r.rows = min(kIBM, __ldg(a.probe_offsets + lo + 1) - r.e0);
  r.nrow = __ldg(a.ivf_offsets + lo + 1) - __ldg(a.ivf_offsets + lo);
  r.pbase = __ldg(a.pad_offsets + lo);
  r.tiles = (r.nrow + kIBN - 1) / kIBN;
  return r;
}

// Bounded wait with a fresh deadline: false on expiry or when another role aborted.
__device__ __forceinline__ bool rr_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  return mbar_wait(bar, parity, clock64() + kIDeadlineCycles, abort_flag);
}
__device__ __forceinline__ bool rr_warp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = rr_wait(bar, parity, abort_flag) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// Four +-1 bytes from four bits: byte j is +1 where bit j of n is set, else -1
// (the expansion k_expand_pm1 makes).  The multiply spreads bit j to bit 8j
// without carries (bit positions j + 7i are distinct for j, i < 4).
__device__ __forceinline__ uint32_t pm1_nibble(uint32_t n) {
  return 0xFFFFFFFFu ^ (((n * 0x00204081u) & 0x01010101u) * 0xFEu);
}

// 16-byte chunk cc (K bytes 16 cc .. 16 cc + 15) of a +-1 row from its packed
// 32-bit word w = words[cc >> 1]: bits 16 (cc & 1) .. + 15.
__device__ __forceinline__ uint4 pm1_chunk(uint32_t w, int cc) {
  const uint32_t h = w >> ((cc & 1) * 16);
  return make_uint4(pm1_nibble(h & 0xFu), pm1_nibble((h >> 4) & 0xFu), pm1_nibble((h >> 8) & 0xFu),
                    pm1_nibble((h >> 12) & 0xFu));
}

// The same chunk as 0 / 1 bytes (byte j = bit j): a database row in this form
// gives dot' = sum of the query's +-1 values where the row has a one, and
// Hamming(q, row) = popcount(q) - dot'.
__device__ __forceinline__ uint32_t b01_nibble(uint32_t n) { return (n * 0x00204081u) & 0x01010101u; }
__device__ __forceinline__ uint4 b01_chunk(uint32_t w, int cc) {
  const uint32_t h = w >> ((cc & 1) * 16);
  return make_uint4(b01_nibble(h & 0xFu), b01_nibble((h >> 4) & 0xFu), b01_nibble((h >> 8) & 0xFu),
                    b01_nibble((h >> 12) & 0xFu));
}

// Swizzled address of chunk cc of row r in a K-major tile of `rows` rows
// (two 128-byte K halves, each rows x 128 bytes).
__device__ __forceinline__ uint8_t* sw128_chunk(uint8_t* tile, uint32_t half_bytes, int r, int cc) {
  return tile + (cc >> 3) * half_bytes + r * 128 + (((cc & 7) ^ (r & 7)) << 4);
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// The next claimed item of the queue (-1 when none is left), for a whole warp;
// one arrival per warp frees the entry.  False on a timeout.
__device__ __forceinline__ bool rr_next_item(uint32_t qfull, uint32_t qempty, volatile int* s_queue, uint32_t qs,
                                             uint32_t parity, volatile int* abort_flag, int* it) {
  if (!rr_warp_wait(qfull, parity, abort_flag)) return false;
  *it = s_queue[qs];
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive(qempty);
  return true;
}

__global__ void __launch_bounds__(kRrThreads, 1) k_rerank_imma(RerankImmaArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  uint8_t* sA = smem;               // two query tiles
  uint8_t* sX = sA + 2 * kIATile;   // two expanded database tiles
  uint8_t* sP = sX + 2 * kIBTile;   // ring of packed database tiles
  uint64_t* bars = reinterpret_cast<uint64_t*>(sP + kRrPStages * kRrPTile);
  volatile int* s_queue = reinterpret_cast<volatile int*>(bars + kRrNumBars);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(const_cast<int*>(s_queue) + kRrQueue);
  volatile int* s_abort = reinterpret_cast<volatile int*>(s_tmem + 1);

  const int n_items = __ldg(a.item_offsets + a.n_clusters);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t bar0 = smem_u32(bars);
#define RR_AFULL(b) (bar0 + 8u * (b))
#define RR_AEMPTY(b) (bar0 + 8u * (2 + (b)))
#define RR_PFULL(s) (bar0 + 8u * (4 + (s)))
#define RR_PEMPTY(s) (bar0 + 8u * (4 + kRrPStages + (s)))
#define RR_XFULL(x) (bar0 + 8u * (4 + 2 * kRrPStages + (x)))
#define RR_XEMPTY(x) (bar0 + 8u * (6 + 2 * kRrPStages + (x)))
#define RR_ACCFULL(x) (bar0 + 8u * (8 + 2 * kRrPStages + (x)))
#define RR_ACCEMPTY(x) (bar0 + 8u * (10 + 2 * kRrPStages + (x)))
#define RR_QFULL(k) (bar0 + 8u * (12 + 2 * kRrPStages + (k)))
#define RR_QEMPTY(k) (bar0 + 8u * (12 + 2 * kRrPStages + kRrQueue + (k)))

  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; b++) {
      mbar_init(RR_AFULL(b), kRrExpWarps);
      mbar_init(RR_AEMPTY(b), 1);
      mbar_init(RR_XFULL(b), kRrExpWarps);
      mbar_init(RR_XEMPTY(b), 1);
      mbar_init(RR_ACCFULL(b), 1);
      mbar_init(RR_ACCEMPTY(b), kIEpiWarps);
    }
    for (uint32_t st = 0; st < kRrPStages; st++) {
      mbar_init(RR_PFULL(st), 1);
      mbar_init(RR_PEMPTY(st), kRrExpWarps);
    }
    for (uint32_t k = 0; k < kRrQueue; k++) {
      mbar_init(RR_QFULL(k), 1);
      mbar_init(RR_QEMPTY(k), kRrQueueReaders);
    }
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(kITmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // producer: the packed rows of every tile of every item of this block, in order
      uint32_t issued[kRrPStages];
      for (uint32_t st = 0; st < kRrPStages; st++) issued[st] = 0u;
      uint32_t g = 0, k = 0;
      bool ok = true;
      while (ok) {
        // claim the next item and hand it to the other roles (-1: none left)
        const uint32_t qs = k % kRrQueue;
        if (k >= kRrQueue && !rr_wait(RR_QEMPTY(qs), ((k / kRrQueue) - 1) & 1u, s_abort)) {
          ok = false;
          break;
        }
        int it = atomicAdd(a.item_counter, 1);
        if (it >= n_items) it = -1;
        s_queue[qs] = it;
        mbar_arrive(RR_QFULL(qs));
        k++;
        if (it < 0) break;
        const RrItem r = rr_item(a, it);
        for (int t = 0; t < r.tiles; t++, g++) {
          const uint32_t st = g % kRrPStages;
          if (g >= kRrPStages && !rr_wait(RR_PEMPTY(st), ((g / kRrPStages) - 1) & 1u, s_abort)) {
            ok = false;
            break;
          }
          mbar_expect_tx(RR_PFULL(st), kRrPTile);
          bulk_load(smem_u32(sP + st * kRrPTile), a.pad_desc + (size_t)(r.pbase + t * kIBN) * 32, kRrPTile,
                    RR_PFULL(st));
          issued[st]++;
        }
      }
      if (!ok) {
        *s_abort = 1;
        atomicOr(a.err, kErrImmaTimeout);
      }
      // drain: every issued copy has landed and been read
      for (uint32_t st = 0; st < kRrPStages; st++) {
        if (issued[st] == 0) continue;
        const uint32_t par = (issued[st] - 1) & 1u;
        long long dl = clock64() + kIDeadlineCycles;
        while (!mbar_try(RR_PFULL(st), par) && clock64() < dl) {
        }
        dl = clock64() + kIDeadlineCycles;
        while (!mbar_try(RR_PEMPTY(st), par) && clock64() < dl && !*s_abort) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      uint32_t g = 0, na = 0, k = 0;
      bool ok = true;
      while (ok) {
        const uint32_t qs = k % kRrQueue;
        if (!rr_wait(RR_QFULL(qs), (k / kRrQueue) & 1u, s_abort)) {
          ok = false;
          break;
        }
        const int it = s_queue[qs];
        mbar_arrive(RR_QEMPTY(qs));
        k++;
        if (it < 0) break;
        const RrItem r = rr_item(a, it);
        if (r.tiles == 0) continue;
        const uint32_t b = na & 1u;
        if (!rr_wait(RR_AFULL(b), (na >> 1) & 1u, s_abort)) {
          ok = false;
          break;
        }
        const uint32_t a_lo = smem_u32(sA + b * kIATile);
        for (int t = 0; t < r.tiles; t++, g++) {
          const uint32_t x = g & 1u;
          if (!rr_wait(RR_XFULL(x), (g >> 1) & 1u, s_abort) ||
              (g >= 2 && !rr_wait(RR_ACCEMPTY(x), ((g >> 1) - 1) & 1u, s_abort))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem_base + x * (uint32_t)kIBN;
          const uint32_t b_lo = smem_u32(sX + x * kIBTile);
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const int h = k >> 2, kk = k & 3;
            const uint64_t da = sw128_desc(a_lo + h * kIHalfA) + (uint64_t)(2 * kk);
            const uint64_t db = sw128_desc(b_lo + h * kIHalfB) + (uint64_t)(2 * kk);
            umma_i8(d, da, db, kIDesc, k > 0 ? 1u : 0u);
          }
          umma_commit(RR_XEMPTY(x));
          umma_commit(RR_ACCFULL(x));
        }
        if (!ok) break;
        umma_commit(RR_AEMPTY(b));
        na++;
      }
      if (!ok) {
        *s_abort = 1;
        atomicOr(a.err, kErrImmaTimeout);
      }
    }
  } else if (warp < 2 + kRrExpWarps) {
    // expanders: thread e (0..255)
    const int e = threadIdx.x - 64;
    uint32_t na = 0, g = 0, k = 0;
    bool ok = true;
    while (ok) {
      int it;
      const uint32_t qs = k % kRrQueue;
      if (!rr_next_item(RR_QFULL(qs), RR_QEMPTY(qs), s_queue, qs, (k / kRrQueue) & 1u, s_abort, &it)) {
        ok = false;
        break;
      }
      k++;
      if (it < 0) break;
      const RrItem ri = rr_item(a, it);
      if (ri.tiles == 0) continue;
      // the item's queries: row e >> 1, K half e & 1
      const uint32_t b = na & 1u;
      if (na >= 2 && !rr_warp_wait(RR_AEMPTY(b), ((na >> 1) - 1) & 1u, s_abort)) {
        ok = false;
        break;
      }
      {
        const int r = e >> 1, half = e & 1;
        uint4 w = make_uint4(0u, 0u, 0u, 0u);
        if (r < ri.rows) {
          const int q = __ldg(a.list + ri.e0 + r) >> 3;
          w = __ldg(reinterpret_cast<const uint4*>(a.q_bits) + 2 * (size_t)q + half);
        }
        const uint32_t wd[4] = {w.x, w.y, w.z, w.w};
        uint8_t* tile = sA + b * kIATile;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int cc = 8 * half + j;
          const uint4 v = (r < ri.rows) ? pm1_chunk(wd[j >> 1], cc) : make_uint4(0u, 0u, 0u, 0u);
          *reinterpret_cast<uint4*>(sw128_chunk(tile, kIHalfA, r, cc)) = v;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(RR_AFULL(b));
      na++;
      // the item's database tiles: row e of each
      for (int t = 0; t < ri.tiles; t++, g++) {
        const uint32_t st = g % kRrPStages, x = g & 1u;
        if (!rr_warp_wait(RR_PFULL(st), (g / kRrPStages) & 1u, s_abort) ||
            (g >= 2 && !rr_warp_wait(RR_XEMPTY(x), ((g >> 1) - 1) & 1u, s_abort))) {
          ok = false;
          break;
        }
        const uint4* src = reinterpret_cast<const uint4*>(sP + st * kRrPTile) + 2 * e;
        const uint4 w0 = src[0], w1 = src[1];
        const uint32_t wd[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
        __syncwarp();
        if (lane == 0) mbar_arrive(RR_PEMPTY(st));
        uint8_t* tile = sX + x * kIBTile;
#pragma unroll
        for (int cc = 0; cc < 16; cc++)
          *reinterpret_cast<uint4*>(sw128_chunk(tile, kIHalfB, e, cc)) = b01_chunk(wd[cc >> 1], cc);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(RR_XFULL(x));
      }
    }
    if (!ok) {
      *s_abort = 1;
      if (lane == 0) atomicOr(a.err, kErrImmaTimeout);
    }
  } else {
    // epilogue
    const int ew = warp - 2 - kRrExpWarps;
    const int quarter = warp & 3;
    const int colgrp = ew >> 2;
    const int row = quarter * 32 + lane;
    uint32_t g = 0, k = 0;
    bool ok = true;
    while (ok) {
      int it;
      const uint32_t qs = k % kRrQueue;
      if (!rr_next_item(RR_QFULL(qs), RR_QEMPTY(qs), s_queue, qs, (k / kRrQueue) & 1u, s_abort, &it)) {
        ok = false;
        break;
      }
      k++;
      if (it < 0) break;
      const RrItem ri = rr_item(a, it);
      // this lane's slot and its query's popcount
      int slot = -1, pc = 0;
      if (row < ri.rows) {
        slot = __ldg(a.list + ri.e0 + row);
        const uint4* qp = reinterpret_cast<const uint4*>(a.q_bits) + 2 * (size_t)(slot >> 3);
        const uint4 w0 = __ldg(qp), w1 = __ldg(qp + 1);
        pc = __popc(w0.x) + __popc(w0.y) + __popc(w0.z) + __popc(w0.w) + __popc(w1.x) + __popc(w1.y) +
             __popc(w1.z) + __popc(w1.w);
      }
      uint32_t k1 = kNoKeyShared, k2 = kNoKeyShared;
      for (int t = 0; t < ri.tiles; t++, g++) {
        const uint32_t acc = g & 1u;
        if (!rr_warp_wait(RR_ACCFULL(acc), (g >> 1) & 1u, s_abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        // the query's bound from its other items so far (any stale value is a valid, looser bound)
        const uint32_t gb = slot >= 0 ? __ldcg(a.q_bound + (slot >> 3)) : kNoKeyShared;
        const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + acc * (uint32_t)kIBN + colgrp * 64;
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
          int v[32];
          tmem_ld32(taddr + 32u * c, v);
          tmem_wait_ld();
          if (c == 1) {
            // every column of this group is in registers: hand the accumulator back
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(RR_ACCEMPTY(acc));
          }
          const int col0 = t * kIBN + colgrp * 64 + 32 * c;  // first column's row within the cluster
          const int valid = ri.nrow - col0;
          if (valid < 32) {
#pragma unroll
            for (int j = 0; j < 32; j++)
              if (j >= valid) v[j] = kMaskedDot;
          }
          // The cluster's list is in increasing database index and the columns
          // arrive in list order, so only a strictly larger dot' (a strictly
          // smaller distance) than the current second best's can enter.
          int thr = (k2 == kNoKeyShared) ? kMaskedDot : pc - (int)(k2 >> kIdxBitsShared);
          // another item of the same query may already hold a closer second best:
          // columns farther than it cannot reach the query's top two (equal
          // distances stay, their index decides)
          if (gb != kNoKeyShared) thr = max(thr, pc - (int)(gb >> kIdxBitsShared) - 1);
          if (__any_sync(0xffffffffu, any_exceeds32(v, thr))) {
            // the chunk's best two on local keys (dot' << 5 | 31 - column): ties keep the lower column
            int a1 = INT_MIN, a2 = INT_MIN;
#pragma unroll
            for (int j = 0; j < 32; j++) {
              const int lk = (v[j] << 5) | (31 - j);
              a2 = max(a2, min(a1, lk));
              a1 = max(a1, lk);
            }
            if ((a1 >> 5) > thr) {
              const int m1 = __ldg(a.pad_members + ri.pbase + col0 + 31 - (a1 & 31));
              top2_push_shared(k1, k2, ((uint32_t)(pc - (a1 >> 5)) << kIdxBitsShared) | (uint32_t)m1);
              if ((a2 >> 5) > thr) {
                const int m2 = __ldg(a.pad_members + ri.pbase + col0 + 31 - (a2 & 31));
                top2_push_shared(k1, k2, ((uint32_t)(pc - (a2 >> 5)) << kIdxBitsShared) | (uint32_t)m2);
              }
            }
          }
        }
      }
      if (!ok) break;
      if (slot >= 0) {
        a.partial[(size_t)slot * kRrGroups + colgrp] = make_uint2(k1, k2);
        // two distinct rows at or below k2: the query's final second best is no worse
        if (k2 != kNoKeyShared) atomicMin(a.q_bound + (slot >> 3), k2);
      }
    }
    if (!ok) {
      *s_abort = 1;
      if (lane == 0) atomicOr(a.err, kErrImmaTimeout);
    }
  }
#undef RR_AFULL
#undef RR_AEMPTY
#undef RR_PFULL
#undef RR_PEMPTY
#undef RR_XFULL
#undef RR_XEMPTY
#undef RR_ACCFULL
#undef RR_ACCEMPTY
#undef RR_QFULL
#undef RR_QEMPTY

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kITmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

static bool make_rows_map(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kIK, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kIK};
  cuuint32_t box[2] = {128u, box_rows};
  cuuint32_t es[2] = {1u, 1u};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int imma_rows_q(int n) { return (n + kIBM - 1) / kIBM * kIBM; }

// Database splits per query tile so that the grid fills the 148 SMs in whole
// waves (one 227 KB block per SM): 512 query tiles -> 2 splits -> 1024 blocks.
int imma_default_splits(int nq_cap) {
  const int qt = (nq_cap + kIBM - 1) / kIBM;
  int best = 1;
  double best_eff = 0.0;
  for (int s = 1; s <= 16; s++) {
    const long long blocks = (long long)qt * s;
    const long long waves = (blocks + 147) / 148;
    const double eff = (double)blocks / (double)(waves * 148);
    if (eff > best_eff + 0.02) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}
int imma_rows_db(int n) { return (n + kIBN - 1) / kIBN * kIBN; }

cudaError_t launch_expand_pm1(const uint8_t* bits, int n, const int* d_n, int rows, int8_t* out, cudaStream_t s) {
  if (rows <= 0) return cudaSuccess;
  k_expand_pm1<<<4 * 148, 256, 0, s>>>(bits, n, d_n, rows, out);
  return cudaGetLastError();
}

cudaError_t launch_match_imma(const ImmaLaunch& L, cudaStream_t s) {
  if (L.nq_cap <= 0) return cudaSuccess;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_match_imma, cudaFuncAttributeMaxDynamicSharedMemorySize, kISmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int qrows = imma_rows_q(L.nq_cap);
  const int dbrows = imma_rows_db(L.ndb_cap > 0 ? L.ndb_cap : 1);
  {
    const int blocks = 4 * 148;
    if (!L.q_ready) k_expand_pm1<<<blocks, 256, 0, s>>>(L.args.q, L.args.nq, L.args.d_nq, qrows, L.q_pm1);
    if (L.ndb_cap > 0 && !L.db_ready)
      k_expand_pm1<<<blocks, 256, 0, s>>>(L.args.db, L.args.ndb, L.args.d_ndb, dbrows, L.db_pm1);
  }
  CUtensorMap tq, td;
  if (!make_rows_map(&tq, L.q_pm1, (uint64_t)qrows, kIBM)) return cudaErrorInvalidValue;
  if (!make_rows_map(&td, L.db_pm1, (uint64_t)dbrows, kIBN)) return cudaErrorInvalidValue;
  const int qtiles = qrows / kIBM;
  k_match_imma<<<qtiles * L.splits, kIThreads, kISmemBytes, s>>>(tq, td, L.args, L.work, L.splits, L.err);
  return cudaGetLastError();
}

cudaError_t launch_rerank_imma(const RerankImmaArgs& a, int max_items, cudaStream_t s) {
  if (max_items <= 0) return cudaSuccess;
  if (!a.pad_desc || (reinterpret_cast<uintptr_t>(a.pad_desc) & 15u)) return cudaErrorInvalidValue;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_rerank_imma, cudaFuncAttributeMaxDynamicSharedMemorySize, kRrSmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return cudaErrorInvalidValue;
  const int blocks = max_items < sms ? max_items : sms;  // persistent: one block per SM
  k_rerank_imma<<<blocks, kRrThreads, kRrSmemBytes, s>>>(a);
  return cudaGetLastError();
}

}  // namespace orbx
