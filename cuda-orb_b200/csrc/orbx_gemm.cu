// BF16 GEMM on the 5th-generation tensor cores for the learned matching
// proposal: C[M x N] = A[M x K] * B[N x K]^T with fp32 accumulation in TMEM.
//
// A and B are row-major bf16 with K contiguous (K-major).  The kernel is
// persistent: one block per SM walks the work items (128 x 256 output tile,
// K split) blockIdx.x, blockIdx.x + gridDim.x, ...
//   warp 0     TMA producer: 64-wide K blocks of A and B through a 4-stage
//              shared-memory ring (128-byte swizzle, no multicast);
//   warp 1     MMA issuer: tcgen05.mma.kind::f16, four K = 16 steps per K
//              block, into one of two 256-column TMEM accumulators, so the
//              next tile's MMAs run while the epilogue drains this one;
//   warps 2-9  epilogue: warp w reads TMEM lanes 32 * (w % 4) (one output row
//              per lane) and columns [128 * ((w - 2) / 4), +128) of the tile,
//              then applies GemmArgs::mode (orbx_learned.cuh).
// A work item is one output tile, or for kTop8Row an M tile with a run of N
// tiles, whose rows keep running top-8 lists across the run.
// M must be a multiple of 128, N of 256, K of 64 * splits; callers pad.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "orbx_device.cuh"
#include "orbx_internal.cuh"
#include "orbx_learned.cuh"

namespace orbx {

constexpr int kGBM = 128;
constexpr int kGBN = 256;
constexpr int kGBK = 64;  // 128 bytes of bf16: one swizzle atom row
constexpr int kGStages = 4;
constexpr int kGEpiWarps = 8;
constexpr int kGThreads = (2 + kGEpiWarps) * 32;
constexpr uint32_t kGATile = kGBM * kGBK * 2;  // 16 KB
constexpr uint32_t kGBTile = kGBN * kGBK * 2;  // 32 KB
constexpr uint32_t kGStage = kGATile + kGBTile;
constexpr uint32_t kGNumBars = 2 * kGStages + 4;  // full, empty per stage; acc full, acc empty per accumulator
constexpr uint32_t kGSmemBytes = 1024 + kGStages * kGStage + 8 * kGNumBars + 16;
static_assert(kGSmemBytes + 16 <= 232448, "exceeds the 227 KB shared-memory opt-in");
constexpr int kGTmemCols = 2 * kGBN;
constexpr long long kGDeadlineCycles = 4000000000ll;  // per wait, about 2 s
// instruction descriptor: F32 accumulate, BF16 x BF16, both K-major, N = 256, M = 128
constexpr uint32_t kGDesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kGBN >> 3) << 17) | ((uint32_t)(kGBM >> 4) << 24);

namespace {
__device__ __forceinline__ uint32_t g_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t g_sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

__device__ __forceinline__ void g_mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void g_mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// A waiting thread is suspended by the barrier unit (woken when the phase
// completes, or after this many nanoseconds) instead of spinning on the
// ALU pipe that the epilogue warps need.
constexpr uint32_t kTryWaitSuspendNs = 20000;
__device__ __forceinline__ bool g_mbar_try(uint32_t bar, uint32_t parity) {
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
// Bounded wait: gives up after kGDeadlineCycles or when another role aborted.
__device__ __forceinline__ bool g_mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  const long long deadline = clock64() + kGDeadlineCycles;
  while (!g_mbar_try(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() > deadline) return false;
  }
  return true;
}
__device__ __forceinline__ void g_mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Warp-uniform bounded wait: lane 0 polls, the result is broadcast.
__device__ __forceinline__ bool g_warp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = g_mbar_wait(bar, parity, abort_flag) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}
__device__ __forceinline__ void g_tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void g_umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                            uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z)
      : "memory");
}
__device__ __forceinline__ void g_umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// 32 consecutive accumulator columns of this lane's row (waits for the load)
__device__ __forceinline__ void g_tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
}  // namespace

// Epilogue of 32 columns [n0, n0 + 32) of row m (values in v).
__device__ __forceinline__ void g_epilogue_chunk(const GemmArgs& g, int split, int m, int n0, float* v, uint32_t* top) {
  if (g.bias && g.splits == 1) {
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = __fadd_rn(v[j], __ldg(g.bias + n0 + j));
  }
  const size_t off = (size_t)m * g.N + (size_t)n0;
  if (g.mode == kStoreF32) {
    float4* dst = reinterpret_cast<float4*>(g.c_f32 + (size_t)split * g.M * g.N + off);
#pragma unroll
    for (int j = 0; j < 8; j++) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    return;
  }
  if (g.mode == kTop8 || g.mode == kTop8Row) {
    float mx = v[0];
#pragma unroll
    for (int j = 1; j < 32; j++) mx = fmaxf(mx, v[j]);
    if (!__any_sync(0xffffffffu, top_key(mx, n0) > top[kTopK - 1])) return;  // no column of this chunk can enter
    // a key above the 8th needs a logit at least the 8th's (truncated) value
    float f8 = top[kTopK - 1] ? order_bits_float(top[kTopK - 1] & ~((1u << kTopColBits) - 1u)) : -INFINITY;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (v[j] >= f8) {
        uint32_t key = top_key(v[j], n0 + j);
        if (key > top[kTopK - 1]) {
#pragma unroll
          for (int i = 0; i < kTopK; i++) {
            const uint32_t hi = max(top[i], key);
            key = min(top[i], key);
            top[i] = hi;
          }
          if (top[kTopK - 1]) f8 = order_bits_float(top[kTopK - 1] & ~((1u << kTopColBits) - 1u));
        }
      }
    }
    return;
  }
  if (g.mode == kBiasReluBF16) {
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = fmaxf(v[j], 0.f);
  } else if (g.mode == kMaskBF16) {
    const uint4* aux = reinterpret_cast<const uint4*>(g.aux + off);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint4 w = __ldg(aux + j);
      const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int e = 0; e < 4; e++) {
        // bf16 > 0: sign bit clear and not zero
        if ((ws[e] & 0x8000u) || !(ws[e] & 0x7FFFu)) v[8 * j + 2 * e] = 0.f;
        if ((ws[e] & 0x80000000u) || !(ws[e] & 0x7FFF0000u)) v[8 * j + 2 * e + 1] = 0.f;
      }
    }
  }
  uint4* dst = reinterpret_cast<uint4*>(g.c_bf16 + off);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    uint32_t w[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const __nv_bfloat162 pr = __floats2bfloat162_rn(v[8 * j + 2 * e], v[8 * j + 2 * e + 1]);
      w[e] = *reinterpret_cast<const uint32_t*>(&pr);
    }
    dst[j] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Work item -> (M tile, first N tile, K split, part): one tile per item, or
// kTop8Row's M tile with `tpi` consecutive N tiles.
struct GItem {
  int tm, tn0, split, part;
};
__device__ __forceinline__ GItem g_item(const GemmArgs& g, int item, int n_tiles, int parts, int tpi) {
  GItem r;
  if (g.mode == kTop8Row) {
    r.tm = item / parts;
    r.part = item - r.tm * parts;
    r.tn0 = r.part * tpi;
    r.split = 0;
  } else {
    r.split = item % g.splits;
    const int tile = item / g.splits;
    r.tm = tile / n_tiles;
    r.tn0 = tile - r.tm * n_tiles;
    r.part = 0;
  }
  return r;
}

__global__ void __launch_bounds__(kGThreads, 1)
    k_gemm_bf16(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = g_smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kGStages * kGStage);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + kGNumBars);
  volatile int* s_abort = reinterpret_cast<volatile int*>(s_tmem + 1);

  const int n_tiles = g.N / kGBN;
  const bool row_top = g.mode == kTop8Row;
  const int parts = row_top ? gemm_top_parts(n_tiles) : 1;
  const int tpi = row_top ? n_tiles / parts : 1;  // N tiles per work item
  const int items = row_top ? (g.M / kGBM) * parts : (g.M / kGBM) * n_tiles * g.splits;
  const int kblocks = g.K / kGBK / g.splits;
  const int my_items = blockIdx.x < items ? (items - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bar0 = g_smem_u32(bars);
#define GBAR_FULL(s) (bar0 + 8u * (s))
#define GBAR_EMPTY(s) (bar0 + 8u * (kGStages + (s)))
#define GBAR_ACCFULL(a) (bar0 + 8u * (2 * kGStages + (a)))
#define GBAR_ACCEMPTY(a) (bar0 + 8u * (2 * kGStages + 2 + (a)))

  if (threadIdx.x == 0) {
    for (int s = 0; s < kGStages; s++) {
      g_mbar_init(GBAR_FULL(s), 1);
      g_mbar_init(GBAR_EMPTY(s), 1);
    }
    for (int a = 0; a < 2; a++) {
      g_mbar_init(GBAR_ACCFULL(a), 1);
      g_mbar_init(GBAR_ACCEMPTY(a), kGEpiWarps);
    }
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(g_smem_u32(s_tmem)),
                 "r"(kGTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // TMA producer over every K block of every item of this block
      int issued[kGStages];
      for (int s = 0; s < kGStages; s++) issued[s] = 0;
      long long gkb = 0;
      bool ok = true;
      for (int j = 0; ok && j < my_items; j++) {
        const GItem it = g_item(g, (int)blockIdx.x + j * (int)gridDim.x, n_tiles, parts, tpi);
        for (int t = 0; ok && t < tpi; t++) {
          const int tn = it.tn0 + t;
          for (int kb = 0; kb < kblocks; kb++, gkb++) {
            const int s = (int)(gkb % kGStages);
            const long long use = gkb / kGStages;
            if (use > 0 && !g_mbar_wait(GBAR_EMPTY(s), (uint32_t)((use - 1) & 1), s_abort)) {
              ok = false;
              break;
            }
            uint8_t* st = smem + s * kGStage;
            const int kx = (it.split * kblocks + kb) * kGBK;
            g_mbar_expect_tx(GBAR_FULL(s), kGStage);
            g_tma_load_2d(g_smem_u32(st), &tmA, kx, it.tm * kGBM, GBAR_FULL(s));
            g_tma_load_2d(g_smem_u32(st + kGATile), &tmB, kx, tn * kGBN, GBAR_FULL(s));
            issued[s]++;
          }
        }
      }
      if (!ok) {
        *s_abort = 1;
        atomicOr(g.err, kErrImmaTimeout);
      }
      // drain before exit: copies landed and the MMAs that read them completed
      for (int s = 0; s < kGStages; s++) {
        if (!issued[s]) continue;
        const uint32_t par = (uint32_t)(issued[s] - 1) & 1u;
        long long dl = clock64() + kGDeadlineCycles;
        while (!g_mbar_try(GBAR_FULL(s), par) && clock64() < dl) {
        }
        dl = clock64() + kGDeadlineCycles;
        while (!g_mbar_try(GBAR_EMPTY(s), par) && clock64() < dl) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      long long gkb = 0;
      bool ok = true;
      const int my_tiles = my_items * tpi;
      for (int j = 0; ok && j < my_tiles; j++) {
        const int acc = j & 1;
        if (j >= 2 && !g_mbar_wait(GBAR_ACCEMPTY(acc), (uint32_t)(((j >> 1) - 1) & 1), s_abort)) {
          ok = false;
          break;
        }
        const uint32_t d = tmem + (uint32_t)(acc * kGBN);
        for (int kb = 0; kb < kblocks; kb++, gkb++) {
          const int s = (int)(gkb % kGStages);
          if (!g_mbar_wait(GBAR_FULL(s), (uint32_t)((gkb / kGStages) & 1), s_abort)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a_lo = g_smem_u32(smem + s * kGStage);
          const uint32_t b_lo = a_lo + kGATile;
#pragma unroll
          for (int k = 0; k < kGBK / 16; k++) {
            g_umma_bf16(d, g_sw128_desc(a_lo) + (uint64_t)(2 * k), g_sw128_desc(b_lo) + (uint64_t)(2 * k), kGDesc,
                        (kb > 0 || k > 0) ? 1u : 0u);
          }
          g_umma_commit(GBAR_EMPTY(s));
        }
        if (ok) g_umma_commit(GBAR_ACCFULL(acc));
      }
      if (!ok) {
        *s_abort = 1;
        atomicOr(g.err, kErrImmaTimeout);
      }
    }
  } else {
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    bool ok = true;
    int gt = 0;  // tiles of this block so far: accumulator gt & 1
    for (int j = 0; ok && j < my_items; j++) {
      const GItem it = g_item(g, (int)blockIdx.x + j * (int)gridDim.x, n_tiles, parts, tpi);
      const int m = it.tm * kGBM + quarter * 32 + lane;
      uint32_t top[kTopK];
#pragma unroll
      for (int i = 0; i < kTopK; i++) top[i] = 0u;
      for (int t = 0; t < tpi; t++, gt++) {
        const int acc = gt & 1;
        const int tn = it.tn0 + t;
        if (!g_warp_wait(GBAR_ACCFULL(acc), (uint32_t)((gt >> 1) & 1), s_abort)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (g.mode == kTop8) {
#pragma unroll
          for (int i = 0; i < kTopK; i++) top[i] = 0u;
        }
        const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kGBN + half * 128);
#pragma unroll 1
        for (int c = 0; c < 4; c++) {
          float v[32];
          g_tmem_ld32(tbase + (uint32_t)(c * 32), v);
          if (c == 3) {
            // every column of this half is in registers: hand the accumulator back
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) g_mbar_arrive(GBAR_ACCEMPTY(acc));
          }
          g_epilogue_chunk(g, it.split, m, tn * kGBN + half * 128 + c * 32, v, top);
        }
        if (g.mode == kTop8) {
          uint4* dst = reinterpret_cast<uint4*>(g.top_keys + ((size_t)m * (2 * n_tiles) + 2 * tn + half) * kTopK);
          dst[0] = make_uint4(top[0], top[1], top[2], top[3]);
          dst[1] = make_uint4(top[4], top[5], top[6], top[7]);
        }
      }
      if (ok && row_top) {
        uint4* dst = reinterpret_cast<uint4*>(g.top_keys + ((size_t)m * (2 * parts) + 2 * it.part + half) * kTopK);
        dst[0] = make_uint4(top[0], top[1], top[2], top[3]);
        dst[1] = make_uint4(top[4], top[5], top[6], top[7]);
      }
    }
    if (!ok) {
      *s_abort = 1;
      if (lane == 0) atomicOr(g.err, kErrImmaTimeout);
    }
  }
#undef GBAR_FULL
#undef GBAR_EMPTY
#undef GBAR_ACCFULL
#undef GBAR_ACCEMPTY
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGTmemCols) : "memory");
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 gemm_encoder() {
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

static bool make_bf16_map(CUtensorMap* m, const void* base, uint64_t rows, uint64_t k, uint32_t box_rows) {
  auto enc = gemm_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(k * 2)};
  cuuint32_t box[2] = {(cuuint32_t)kGBK, box_rows};
  cuuint32_t es[2] = {1u, 1u};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_gemm_bf16(const GemmArgs& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return cudaSuccess;
  if (g.splits < 1 || (g.splits > 1 && g.mode != kStoreF32)) return cudaErrorInvalidValue;
  if (g.M % kGBM || g.N % kGBN || g.K % (kGBK * g.splits)) return cudaErrorInvalidValue;
  if ((g.mode == kTop8 || g.mode == kTop8Row) && g.N > (1 << kTopColBits)) return cudaErrorInvalidValue;
  if (!g.err) return cudaErrorInvalidValue;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  CUtensorMap ta, tb;
  if (!make_bf16_map(&ta, g.a, (uint64_t)g.M, (uint64_t)g.K, kGBM)) return cudaErrorInvalidValue;
  if (!make_bf16_map(&tb, g.b, (uint64_t)g.N, (uint64_t)g.K, kGBN)) return cudaErrorInvalidValue;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return cudaErrorInvalidValue;
  const int items = g.mode == kTop8Row ? (g.M / kGBM) * gemm_top_parts(g.N / kGBN) : (g.M / kGBM) * (g.N / kGBN) * g.splits;
  const int blocks = items < sms ? items : sms;  // persistent: one block per SM
  k_gemm_bf16<<<blocks, kGThreads, kGSmemBytes, s>>>(ta, tb, g);
  return cudaGetLastError();
}

}  // namespace orbx
