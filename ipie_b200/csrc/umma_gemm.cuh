// Generic tcgen05 GEMM for the mixed-precision walker step.
//
// One CTA computes a 128 x BN tile of
//     D_a = sum_k A_a[m, k] B[n, k]          a = 0 .. NA-1   (NA left operands share B)
// with A_a and B K-major fp32 in global memory, read through TMA into
// 128B-swizzled shared memory and multiplied as TF32 on the 5th-gen tensor
// cores.  NSPLIT = 3 adds the hi/lo correction products A_hi B_lo + A_lo B_hi
// (each operand pre-split into a TF32 head and remainder, ~2^-22 relative);
// NSPLIT = 1 is plain TF32.
//
// Accumulation in chunks: the tensor core's FP32 accumulator loses about half
// an ulp per accumulation step, always toward zero, so a long K sum in TMEM
// comes out shrunk by a relative ~(K/8) * 2^-24 (measured: -1.7e-5 at
// K = 1600, -3.8e-5 at K = 6400).  Here the MMAs accumulate only KCHUNK k-blocks
// (32 K each) into one of two TMEM buffers; the epilogue warps drain each
// finished chunk into FP32 registers (round-to-nearest adds) while the tensor
// cores fill the other buffer, which bounds the shrink to that of one chunk.
//
// Roles (192 threads): warp 4 lane 0 issues TMA loads into a STAGES-deep ring
// (full/empty mbarriers); warp 5 lane 0 issues tcgen05.mma; warps 0-3 (TMEM
// lanes 0-127, one output row per thread) drain the chunks (chunk_full /
// chunk_empty mbarriers) and run the epilogue on the summed row of NA*BN
// values.  Epilogues synchronise with bar.sync 1, 128 (epi_sync), never with
// __syncthreads.
//
// Batching: grid.z indexes a batch; the tile's first A row is
// z * a_rows_per_batch + blockIdx.y * 128 and its first B row
// z * b_rows_per_batch + blockIdx.x * BN (rows past a batch's own extent read
// the next batch or TMA's zero fill; the epilogue drops them).
#pragma once

#include "umma.cuh"

namespace ipie_b200 {
namespace umma {

struct GemmMaps {
  CUtensorMap a_hi[2];
  CUtensorMap a_lo[2];
  CUtensorMap b_hi;
  CUtensorMap b_lo;
};

constexpr int kBM = 128;
constexpr int kBK = 32;  // fp32 per 128-byte row

__host__ __device__ constexpr int tmem_cols_for(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512; }

constexpr int kGemmThreads = 192;
constexpr int kChunkKB = 2;  // k-blocks (of 32) accumulated in TMEM before a drain

// named barrier of the 128 epilogue threads (warps 0-3)
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }
// AND of pred over the 128 epilogue threads (named barrier 1)
__device__ __forceinline__ bool epi_all(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.and.pred q, 1, 128, p;\nselp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)pred)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void mbar_arrive_cta(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

template <int BN, int NA, int NSPLIT, int STAGES>
struct GemmShape {
  static constexpr int A_TILE = kBM * kBK * 4;
  static constexpr int B_TILE = BN * kBK * 4;
  static constexpr int NAT = NA * (NSPLIT == 3 ? 2 : 1);
  static constexpr int NBT = NSPLIT == 3 ? 2 : 1;
  static constexpr int STAGE_BYTES = NAT * A_TILE + NBT * B_TILE;
  static constexpr int BUF_COLS = tmem_cols_for(NA * BN);  // one accumulator buffer
  static constexpr int TMEM_COLS = 2 * BUF_COLS;
  static constexpr int SMEM_BYTES = 1024 + STAGES * STAGE_BYTES + 256;
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN must be a multiple of 32 in [32, 256]");
  static_assert(2 * NA * BN <= 512, "two accumulator buffers exceed TMEM");
  static_assert(STAGE_BYTES % 1024 == 0, "stage must keep 1024-byte alignment");
};

template <int BN, int NA, int NSPLIT, int STAGES, class Epi>
__global__ void __launch_bounds__(kGemmThreads, 1)
    umma_gemm_kernel(const __grid_constant__ GemmMaps maps, int K, int a_rows_per_batch, int b_rows_per_batch, Epi epi,
                     unsigned* status) {
  using S = GemmShape<BN, NA, NSPLIT, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * S::STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* cfull = empty + STAGES;  // [2] chunk accumulated (MMA commit)
  uint64_t* cempty = cfull + 2;      // [2] chunk drained (128 epilogue arrivals)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(cempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&cfull[b], 1);
      mbar_init(&cempty[b], 128);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, S::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int nk = (K + kBK - 1) / kBK;
  const int nchunks = (nk + kChunkKB - 1) / kChunkKB;
  const int z = blockIdx.z;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
  const int arow = z * a_rows_per_batch + m0;
  const int brow = z * b_rows_per_batch + n0;

  if (warp == 4) {
    if (lane == 0) {
      for (int a = 0; a < NA; ++a) {
        tma_prefetch_desc(&maps.a_hi[a]);
        if (NSPLIT == 3) tma_prefetch_desc(&maps.a_lo[a]);
      }
      tma_prefetch_desc(&maps.b_hi);
      if (NSPLIT == 3) tma_prefetch_desc(&maps.b_lo);
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES, r = kb / STAGES;
        if (r > 0 && !mbar_wait(&empty[s], (r - 1) & 1, abort_flag, status)) break;
        mbar_expect_tx(&full[s], S::STAGE_BYTES);
        uint8_t* st = smem + s * S::STAGE_BYTES;
        const int k = kb * kBK;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          tma_load_2d(st + (a * (S::NAT / NA)) * S::A_TILE, &maps.a_hi[a], k, arow, &full[s]);
          if (NSPLIT == 3) tma_load_2d(st + (a * 2 + 1) * S::A_TILE, &maps.a_lo[a], k, arow, &full[s]);
        }
        tma_load_2d(st + S::NAT * S::A_TILE, &maps.b_hi, k, brow, &full[s]);
        if (NSPLIT == 3) tma_load_2d(st + S::NAT * S::A_TILE + S::B_TILE, &maps.b_lo, k, brow, &full[s]);
      }
    }
    __syncwarp();
  } else if (warp == 5) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(kBM, BN);
      bool ok = true;
      for (int kb = 0; kb < nk && ok; ++kb) {
        const int c = kb / kChunkKB, buf = c & 1;
        const bool first = (kb % kChunkKB) == 0;
        if (first && c >= 2 && !mbar_wait(&cempty[buf], ((c >> 1) - 1) & 1, abort_flag, status)) break;
        const int s = kb % STAGES, r = kb / STAGES;
        if (!mbar_wait(&full[s], r & 1, abort_flag, status)) break;
        tc_fence_after();
        uint8_t* st = smem + s * S::STAGE_BYTES;
        const uint64_t db_hi = desc_kmajor_sw128(st + S::NAT * S::A_TILE);
        const uint64_t db_lo = desc_kmajor_sw128(st + S::NAT * S::A_TILE + S::B_TILE);
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const uint64_t da_hi = desc_kmajor_sw128(st + (a * (S::NAT / NA)) * S::A_TILE);
          const uint64_t da_lo = desc_kmajor_sw128(st + (a * 2 + 1) * S::A_TILE);
          const uint32_t d = tmem + (uint32_t)(buf * S::BUF_COLS + a * BN);
#pragma unroll
          for (int kk = 0; kk < kBK / 8; ++kk) {
            // 8 tf32 = 32 bytes per MMA: advance the start address by 2 (16-byte units)
            mma_tf32(d, da_hi + 2 * kk, db_hi + 2 * kk, idesc, (!first || kk > 0) ? 1u : 0u);
            if (NSPLIT == 3) {
              mma_tf32(d, da_hi + 2 * kk, db_lo + 2 * kk, idesc, 1u);
              mma_tf32(d, da_lo + 2 * kk, db_hi + 2 * kk, idesc, 1u);
            }
          }
        }
        mma_commit(&empty[s]);
        if ((kb % kChunkKB) == kChunkKB - 1 || kb == nk - 1) mma_commit(&cfull[buf]);
      }
    }
    __syncwarp();
  } else {
    // drain every chunk into FP32 registers (round-to-nearest), then the epilogue
    float v[NA * BN];
#pragma unroll
    for (int i = 0; i < NA * BN; ++i) v[i] = 0.0f;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      const int buf = c & 1;
      if (ok && !mbar_wait(&cfull[buf], (c >> 1) & 1, abort_flag, status)) ok = false;
      // tcgen05.ld is warp-collective: decide per warp
      ok = __all_sync(0xffffffffu, ok) != 0;
      if (!ok) break;
      tc_fence_after();
#pragma unroll
      for (int q = 0; q < NA * BN / 32; ++q) {
        float t[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * S::BUF_COLS + q * 32), t);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[q * 32 + i] += t[i];
      }
      tc_fence_before();
      mbar_arrive_cta(&cempty[buf]);
    }
    // epilogues may synchronise the 128 epilogue threads: decide for all four warps together
    if (epi_all(ok && !*abort_flag)) epi(z, m0 + warp * 32 + lane, n0, v, smem);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, S::TMEM_COLS);
}

}  // namespace umma
}  // namespace ipie_b200
