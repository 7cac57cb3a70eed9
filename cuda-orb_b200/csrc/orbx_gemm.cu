// BF16 GEMM on the 5th-generation tensor cores for the learned matching
// proposal: C[M x N] = A[M x K] * B[N x K]^T with fp32 accumulation in TMEM.
//
// A and B are row-major bf16 with K contiguous (K-major).  One block computes a
// 128 x 256 tile of C (for one K split): warp 0 streams 64-wide K blocks of A
// and B through a 4-stage TMA ring (128-byte swizzle, no multicast), warp 1
// issues tcgen05.mma.kind::f16 (four K = 16 steps per block) into a 256-column
// TMEM accumulator, and warps 2-5 read the accumulator back (one row per
// thread) and apply the epilogue chosen by GemmArgs::mode (orbx_learned.cuh).
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
constexpr int kGThreads = 6 * 32;
constexpr uint32_t kGATile = kGBM * kGBK * 2;  // 16 KB
constexpr uint32_t kGBTile = kGBN * kGBK * 2;  // 32 KB
constexpr uint32_t kGStage = kGATile + kGBTile;
constexpr uint32_t kGNumBars = 2 * kGStages + 1;
constexpr uint32_t kGSmemBytes = 1024 + kGStages * kGStage + 8 * kGNumBars + 16;
static_assert(kGSmemBytes + 16 <= 232448, "exceeds the 227 KB shared-memory opt-in");
constexpr long long kGDeadlineCycles = 4000000000ll;
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
__device__ __forceinline__ bool g_mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool g_mbar_wait(uint32_t bar, uint32_t parity, long long deadline,
                                            volatile int* abort_flag) {
  while (!g_mbar_try(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() > deadline) return false;
  }
  return true;
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

__global__ void __launch_bounds__(kGThreads, 1)
    k_gemm_bf16(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = g_smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kGStages * kGStage);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + kGNumBars);
  volatile int* s_abort = reinterpret_cast<volatile int*>(s_tmem + 1);

  const int n_tiles = g.N / kGBN;
  const int split = blockIdx.x % g.splits;
  const int tile = blockIdx.x / g.splits;
  const int tm = tile / n_tiles;
  const int tn = tile - tm * n_tiles;
  const int kblocks = g.K / kGBK / g.splits;
  const int kb0 = split * kblocks;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bar0 = g_smem_u32(bars);
#define GBAR_FULL(s) (bar0 + 8u * (s))
#define GBAR_EMPTY(s) (bar0 + 8u * (kGStages + (s)))
#define GBAR_ACC (bar0 + 8u * (2 * kGStages))

  if (threadIdx.x == 0) {
    for (int s = 0; s < kGStages; s++) {
      g_mbar_init(GBAR_FULL(s), 1);
      g_mbar_init(GBAR_EMPTY(s), 1);
    }
    g_mbar_init(GBAR_ACC, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(g_smem_u32(s_tmem)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *s_tmem;
  const long long deadline = clock64() + kGDeadlineCycles;

  if (warp == 0) {
    if (lane == 0) {
      int issued[kGStages];
      for (int s = 0; s < kGStages; s++) issued[s] = 0;
      for (int kb = 0; kb < kblocks; kb++) {
        const int s = kb % kGStages;
        const int use = kb / kGStages;
        if (use > 0 && !g_mbar_wait(GBAR_EMPTY(s), (use - 1) & 1, deadline, s_abort)) {
          *s_abort = 1;
          atomicOr(g.err, kErrImmaTimeout);
          break;
        }
        uint8_t* st = smem + s * kGStage;
        g_mbar_expect_tx(GBAR_FULL(s), kGStage);
        g_tma_load_2d(g_smem_u32(st), &tmA, (kb0 + kb) * kGBK, tm * kGBM, GBAR_FULL(s));
        g_tma_load_2d(g_smem_u32(st + kGATile), &tmB, (kb0 + kb) * kGBK, tn * kGBN, GBAR_FULL(s));
        issued[s]++;
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
      bool ok = true;
      for (int kb = 0; kb < kblocks; kb++) {
        const int s = kb % kGStages;
        if (!g_mbar_wait(GBAR_FULL(s), (uint32_t)(kb / kGStages) & 1u, deadline, s_abort)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_lo = g_smem_u32(smem + s * kGStage);
        const uint32_t b_lo = a_lo + kGATile;
#pragma unroll
        for (int k = 0; k < kGBK / 16; k++) {
          g_umma_bf16(tmem, g_sw128_desc(a_lo) + (uint64_t)(2 * k), g_sw128_desc(b_lo) + (uint64_t)(2 * k), kGDesc,
                      (kb > 0 || k > 0) ? 1u : 0u);
        }
        g_umma_commit(GBAR_EMPTY(s));
      }
      if (ok) {
        g_umma_commit(GBAR_ACC);
      } else {
        *s_abort = 1;
        atomicOr(g.err, kErrImmaTimeout);
      }
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32*(w&3).., row m = tm*128 + lane quarter
    const int quarter = warp & 3;
    int ok = 0;
    if (lane == 0) ok = g_mbar_wait(GBAR_ACC, 0, deadline, s_abort) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m = tm * kGBM + quarter * 32 + lane;
      const size_t crow = (size_t)m * g.N + (size_t)tn * kGBN;
      const bool use_bias = g.bias && g.splits == 1;
      uint32_t top[kTopK];
#pragma unroll
      for (int i = 0; i < kTopK; i++) top[i] = 0u;
#pragma unroll 1
      for (int c = 0; c < kGBN / 32; c++) {
        float v[32];
        g_tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(c * 32), v);
        const int n0 = tn * kGBN + c * 32;
        if (use_bias) {
#pragma unroll
          for (int j = 0; j < 32; j++) v[j] = __fadd_rn(v[j], __ldg(g.bias + n0 + j));
        }
        if (g.mode == kStoreF32) {
          float4* dst = reinterpret_cast<float4*>(g.c_f32 + (size_t)split * g.M * g.N + crow + c * 32);
#pragma unroll
          for (int j = 0; j < 8; j++) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        } else if (g.mode == kTop8) {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            uint32_t key = top_key(v[j], n0 + j);
            if (key > top[kTopK - 1]) {
#pragma unroll
              for (int i = 0; i < kTopK; i++) {
                const uint32_t hi = max(top[i], key);
                key = min(top[i], key);
                top[i] = hi;
              }
            }
          }
        } else {
          if (g.mode == kBiasReluBF16) {
#pragma unroll
            for (int j = 0; j < 32; j++) v[j] = fmaxf(v[j], 0.f);
          } else if (g.mode == kMaskBF16) {
            const uint4* aux = reinterpret_cast<const uint4*>(g.aux + crow + c * 32);
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
          uint4* dst = reinterpret_cast<uint4*>(g.c_bf16 + crow + c * 32);
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
      }
      if (g.mode == kTop8) {
        uint4* dst = reinterpret_cast<uint4*>(g.top_keys + ((size_t)m * n_tiles + tn) * kTopK);
        dst[0] = make_uint4(top[0], top[1], top[2], top[3]);
        dst[1] = make_uint4(top[4], top[5], top[6], top[7]);
      }
    } else if (lane == 0) {
      atomicOr(g.err, kErrImmaTimeout);
    }
  }
#undef GBAR_FULL
#undef GBAR_EMPTY
#undef GBAR_ACC
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
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
  if (g.mode == kTop8 && g.N > (1 << kTopColBits)) return cudaErrorInvalidValue;
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
  const int blocks = (g.M / kGBM) * (g.N / kGBN) * g.splits;
  k_gemm_bf16<<<blocks, kGThreads, kGSmemBytes, s>>>(ta, tb, g);
  return cudaGetLastError();
}

}  // namespace orbx
