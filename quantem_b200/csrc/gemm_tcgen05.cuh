// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (sm_100a).
//
//   C[M, N] (op)= A[M, K] * B[N, K]^T (+ bias[N]) (ReLU)
//
// A and B are K-major (row-major with K contiguous, leading dimensions lda/ldb in
// elements, multiples of 8 so that every row starts on a 16-byte boundary).
//
// One CTA of 128 threads computes a 128 x BN tile:
//   * warp 0, one lane: TMA producer.  Each k-block (64 bf16 = one 128-byte
//     swizzle row) of A (128 x 64) and B (BN x 64) is copied by
//     cp.async.bulk.tensor into a 4-stage ring with the 128-byte swizzle; an
//     mbarrier per stage counts the transaction bytes.
//   * warp 1, one lane: MMA issuer.  tcgen05.mma.cta_group::1.kind::f16 with
//     M = 128, N = BN, K = 16 (four per k-block), BF16 operands read from shared
//     memory through matrix descriptors, FP32 accumulator in tensor memory
//     (TMEM, BN columns x 128 lanes).  tcgen05.commit frees a stage when its
//     MMAs have read it, and signals the epilogue after the last k-block.
//   * warp 2 allocates / frees the TMEM columns.
//   * all four warps: epilogue.  Warp w reads TMEM lanes 32w..32w+31 (tile rows)
//     with tcgen05.ld.32x32b, applies bias / ReLU and stores FP32 or BF16, or
//     adds FP32 atomically (split-K).
// Out-of-range rows / columns / k of the tile are zero-filled by TMA and masked
// in the epilogue, so M, N, K need no padding.
//
// Every mbarrier wait is bounded by the global timer; on expiry the CTA records
// a status code, still drains what it issued, frees TMEM and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnn_act.cuh"

namespace qb {
namespace gemm {

constexpr int BM = 128;
constexpr int BK = 64;  // bf16 per 128-byte swizzle row
constexpr int STAGES = 4;
constexpr int THREADS = 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s bound on any single wait

// EPI_RELU is activation 1; bits EPI_ACT_SHIFT.. hold any activation id (qb::ACT_*)
enum : int { EPI_BF16 = 1, EPI_RELU = 2, EPI_ATOMIC = 4, EPI_ACT_SHIFT = 8, EPI_ACT_MASK = 0xF00 };
enum : int { GEMM_TIMEOUT = 1 };

struct Epilogue {
  void* out;          // FP32 or BF16 [M][ldc]
  const float* bias;  // [N] or null
  int ldc;
  int flags;
  int act;  // qb::ACT_* applied to acc + bias
};

template <int BN>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int BAR_OFF = STAGES * STAGE_BYTES;
  static constexpr int BYTES = BAR_OFF + 256 + 1024;  // barriers + 1 KB alignment slack
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase with the given parity to complete; false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (true) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of
// 128 bytes, 8-row core groups 1024 bytes apart (SBO), descriptor version 1.
__device__ __forceinline__ uint64_t sdesc_k128(const void* tile) {
  const uint64_t addr = (smem_u32(tile) >> 4) & 0x3FFFull;
  return addr | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major.
template <int BN>
__host__ __device__ constexpr uint32_t idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_bf16_tn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M,
                        int N, int K, int kb_per_split, Epilogue epi, int* status) {
  static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN: TMEM allocation is a power of two >= 32");
  using L = Smem<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(done + 1);
  int* fail_flag = reinterpret_cast<int*>(tmem_holder + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nkb_all = (K + BK - 1) / BK;
  const int kb0 = blockIdx.z * kb_per_split;
  const int kb1 = min(nkb_all, kb0 + kb_per_split);
  const int nkb = kb1 - kb0;  // >= 1 (host sizes the split)

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *fail_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;

  if (warp == 0 && lane == 0) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (i / STAGES) & 1;
      if (!mbar_wait(&empty[s], ph ^ 1)) {
        atomicExch(fail_flag, 1);
        break;
      }
      uint8_t* sa = smem + s * L::STAGE_BYTES;
      mbar_expect_tx(&full[s], L::STAGE_BYTES);
      tma_load_2d(sa, &tmA, &full[s], (kb0 + i) * BK, m0);
      tma_load_2d(sa + L::A_BYTES, &tmB, &full[s], (kb0 + i) * BK, n0);
    }
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = idesc_bf16<BN>();
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (i / STAGES) & 1;
      if (!mbar_wait(&full[s], ph)) {
        atomicExch(fail_flag, 1);
        break;
      }
      tc_fence_after();
      const uint8_t* sa = smem + s * L::STAGE_BYTES;
      const uint64_t ad = sdesc_k128(sa), bd = sdesc_k128(sa + L::A_BYTES);
#pragma unroll
      for (int k = 0; k < BK / 16; ++k)  // +32 bytes along the swizzled row per K = 16 step
        umma_bf16(tmem, ad + 2 * k, bd + 2 * k, idesc, (i | k) != 0 ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);  // also after a failure: completes once every issued MMA has finished
  }
  __syncwarp();

  const bool ok = mbar_wait(done, 0);
  tc_fence_after();
  if (!ok) atomicExch(fail_flag, 1);
  __syncthreads();
  const bool good = (*fail_flag == 0);
  if (good) {
    const int row = m0 + warp * 32 + lane;
    const bool add_bias = epi.bias != nullptr && (!(epi.flags & EPI_ATOMIC) || blockIdx.z == 0);
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      __syncwarp();
      tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);  // warp-collective
      const int col0 = n0 + c0;
      if (col0 >= N) break;  // uniform across the CTA
      if (row >= M) continue;
      const int ncols = min(16, N - col0);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        if (add_bias && j < ncols) v[j] += epi.bias[col0 + j];
        v[j] = act_forward(epi.act, v[j]);
      }
      const size_t off = size_t(row) * epi.ldc + col0;
      if (epi.flags & EPI_ATOMIC) {
        float* o = static_cast<float*>(epi.out) + off;
        for (int j = 0; j < ncols; ++j) atomicAdd(o + j, v[j]);
      } else if (epi.flags & EPI_BF16) {
        __nv_bfloat16* o = static_cast<__nv_bfloat16*>(epi.out) + off;
        if (ncols == 16 && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
          uint4 pk[2];
          __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
          for (int j = 0; j < 8; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
          reinterpret_cast<uint4*>(o)[0] = pk[0];
          reinterpret_cast<uint4*>(o)[1] = pk[1];
        } else {
          for (int j = 0; j < ncols; ++j) o[j] = __float2bfloat16_rn(v[j]);
        }
      } else {
        float* o = static_cast<float*>(epi.out) + off;
        if (ncols == 16 && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            reinterpret_cast<float4*>(o)[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        } else {
          for (int j = 0; j < ncols; ++j) o[j] = v[j];
        }
      }
    }
  } else if (threadIdx.x == 0 && status) {
    atomicOr(status, GEMM_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
  }
}

}  // namespace gemm
}  // namespace qb
