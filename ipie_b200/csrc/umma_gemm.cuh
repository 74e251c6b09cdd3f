// Generic tcgen05 GEMM for the mixed-precision walker step.
//
// One CTA computes a 128 x BN tile of
//     D_a = sum_k A_a[m, k] B[n, k]          a = 0 .. NA-1   (NA left operands share B)
// with A_a and B K-major in global memory, read through TMA into 128B-swizzled
// shared memory and multiplied on the 5th-gen tensor cores, either as TF32
// (fp32 words, KIND_TF32) or as FP16 (KIND_F16: half the bytes per K and twice
// the tensor rate; operands carry a power-of-two scale that the epilogue
// removes).  NSPLIT = 3 adds the hi/lo correction products A_hi B_lo + A_lo B_hi
// (each operand pre-split into a head and remainder, ~2^-22 relative for TF32
// and for in-range FP16); NSPLIT = 1 is a single product.
//
// Accumulation in chunks: the tensor core's FP32 accumulator loses about half
// an ulp per accumulation step, always toward zero, so a long K sum in TMEM
// comes out shrunk by a relative ~(K/8) * 2^-24 (measured: -1.7e-5 at
// K = 1600, -3.8e-5 at K = 6400).  Here the MMAs accumulate only KCHUNK k-blocks
// (32 K each) into one of two TMEM buffers; the epilogue warps drain each
// finished chunk into FP32 registers (round-to-nearest adds) while the tensor
// cores fill the other buffer, which bounds the shrink to that of one chunk.
//
// Roles: 4 epilogue warps per 128 accumulator columns (warp w: TMEM lane
// quarter w % 4, i.e. one output row per thread, and column group w / 4) drain
// the chunks (chunk_full / chunk_empty mbarriers) and run the epilogue on their
// group's summed 128 values (a tile of BN = 256 is handed to the epilogue as two
// 128-column tiles); then one warp whose lane 0 issues TMA loads into a
// STAGES-deep ring (full/empty mbarriers) and one whose lane 0 issues
// tcgen05.mma.  One-group epilogues may synchronise with bar.sync 1, 128
// (epi_sync), never with __syncthreads.
//
// CTA pairs (CG = 2, clusters of two): a tile is 256 x BN; the even CTA of the pair (the
// leader) issues tcgen05.mma.cta_group::2 for both, each CTA stages its own 128 rows of A and
// BN / 2 rows of B (so each SM loads and reads half of B per product), and each CTA's epilogue
// drains its own 128 rows of D from its own TMEM.  Both producers' copies complete on the
// leader's full barrier (which expects both stages' bytes), the MMA commits arrive on the empty
// and chunk-full barriers of both CTAs, and both epilogues arrive on the leader's chunk-empty
// barrier.
//
// Tiles: TileOrder numbers the (128 CG) x BN output tiles of nz batches; a tile
// (z, mt, nt) reads A rows from z * a_rows_per_batch + mt * 128 and B rows from
// z * b_rows_per_batch + nt * BN (rows past a batch's own extent read the next
// batch or TMA's zero fill; the epilogue drops them).  The CTAs are persistent:
// one per SM, each walking the tile list with stride gridDim.x.
#pragma once

#include "umma.cuh"

namespace ipie_b200 {
namespace umma {

struct GemmMaps {
  CUtensorMap a_hi[2];
  CUtensorMap a_lo[2];
  CUtensorMap b_hi;
  CUtensorMap b_lo;
  CUtensorMap out[4];  // output maps of epilogues that store through TMA (EpiUsesMaps)
  // 1: a_hi / b_hi are 3-D maps whose second plane is the remainder (lo at a fixed offset from
  // hi in one allocation), so one copy of depth 2 brings both tiles (a_lo / b_lo unused): every
  // copy a thread issues costs it about as much time whatever its size
  int a_planes, b_planes;
};

constexpr int kBM = 128;
constexpr int kBK = 32;  // fp32 per 128-byte row

// Operand kinds: a stage holds 128-byte K rows of either
constexpr int KIND_TF32 = 0;  // fp32 words read as TF32 (32 per row, kind::tf32)
constexpr int KIND_F16 = 1;   // FP16 (64 per row, kind::f16)
constexpr int KIND_F16_K32 = 2;  // FP16, 32 per 64-byte row (64B swizzle): half-size stages, twice as many
__host__ __device__ constexpr int kblock_elems(int kind) { return kind == KIND_F16 ? 64 : 32; }
__host__ __device__ constexpr int row_bytes(int kind) { return kind == KIND_F16_K32 ? 64 : 128; }
// k-blocks accumulated in TMEM before a drain: 128 FP16 / 64 TF32 elements of K either way
__host__ __device__ constexpr int chunk_kb(int kind) { return kind == KIND_F16_K32 ? 4 : 2; }

__host__ __device__ constexpr int tmem_cols_for(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512; }

// Epilogue warps: one group of 4 (the four TMEM lane quarters) per 128 accumulator
// columns; then a producer and an MMA warp.
template <int NA, int BN>
struct GemmRoles {
  static constexpr int kGroups = (NA * BN + 127) / 128;
  static constexpr int kGroupCols = NA * BN / kGroups;
  static constexpr int kEpiThreads = 128 * kGroups;
  static constexpr int kThreads = kEpiThreads + 64;
  static constexpr int kProducerWarp = 4 * kGroups, kMmaWarp = 4 * kGroups + 1;
  static_assert(NA * BN % kGroups == 0 && kGroupCols % 32 == 0, "column groups of whole 32-column loads");
};

// named barrier of the 128 epilogue threads of a one-group tile (warps 0-3)
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }
// AND of pred over the nthreads epilogue threads (named barrier 2)
__device__ __forceinline__ bool epi_all(bool pred, int nthreads) {
  uint32_t r;
  asm volatile(
      "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.and.pred q, 2, %2, p;\nselp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(nthreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void mbar_arrive_cta(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Order of the output tiles: tile l (of nm x nn x nz) has batch z = l / (nm * nn); inside the
// batch either the column-tile index runs fastest, or (m_fast) the row tiles are taken in
// groups of m_group: within a group the row-tile index runs fastest over the group's row
// tiles for every column tile in turn.  The CTAs resident at one time take consecutive tiles,
// so the operand swept along the fast index should fit in L2: a whole row-tile group of A
// stays there while the column tiles of B stream past it once per group.
struct TileOrder {
  int nm, nn, nz;
  int m_fast;
  int m_group;  // row tiles per group (m_fast); nm or more: one group
  __host__ __device__ int count() const { return nm * nn * nz; }
  __device__ void decode(int l, int& z, int& mt, int& nt) const {
    const int per = nm * nn;
    z = l / per;
    const int r = l - z * per;
    if (m_fast) {
      const int span = m_group * nn;  // tiles of one full group
      const int g = r / span;
      const int m0 = g * m_group;
      const int gm = min(m_group, nm - m0);  // the last group may be shorter
      const int rem = r - g * span;          // < gm * nn
      mt = m0 + rem % gm;
      nt = rem / gm;
    } else {
      nt = r % nn;
      mt = r / nn;
    }
  }
};

// Epilogues declare the shared memory they use (kSmemBytes): it is a region of its own, since in
// a persistent CTA the TMA ring is already refilled for the next tile while an epilogue runs.
template <class Epi, class = void>
struct EpiSmem {
  static constexpr int value = 0;
};
template <class Epi>
struct EpiSmem<Epi, decltype((void)Epi::kSmemBytes)> {
  static constexpr int value = Epi::kSmemBytes;
};

// Epilogues with kUsesMaps = true take the kernel's GemmMaps as a sixth argument (their TMA
// stores name maps.out) and have thread 0 wait for its bulk stores before the CTA exits.
template <class Epi, class = void>
struct EpiUsesMaps {
  static constexpr bool value = false;
};
template <class Epi>
struct EpiUsesMaps<Epi, decltype((void)Epi::kUsesMaps)> {
  static constexpr bool value = Epi::kUsesMaps;
};

template <int BN, int NA, int NSPLIT, int STAGES, int EPI_SMEM = 0, int KIND = KIND_TF32, int CG = 1>
struct GemmShape {
  static constexpr int A_TILE = kBM * row_bytes(KIND);
  static constexpr int B_TILE = BN / CG * row_bytes(KIND);  // this CTA's rows of B
  static constexpr int NAT = NA * (NSPLIT == 3 ? 2 : 1);
  static constexpr int NBT = NSPLIT == 3 ? 2 : 1;
  static constexpr int STAGE_BYTES = NAT * A_TILE + NBT * B_TILE;
  static constexpr int BUF_COLS = tmem_cols_for(NA * BN);  // one accumulator buffer
  static constexpr int TMEM_COLS = 2 * BUF_COLS;
  static constexpr int EPI_OFFSET = STAGES * STAGE_BYTES;
  static constexpr int BAR_OFFSET = EPI_OFFSET + ((EPI_SMEM + 15) / 16) * 16;
  static constexpr int SMEM_BYTES = 1024 + BAR_OFFSET + 256;
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN must be a multiple of 32 in [32, 256]");
  static_assert(2 * NA * BN <= 512, "two accumulator buffers exceed TMEM");
  static_assert(STAGE_BYTES % 1024 == 0, "stage must keep 1024-byte alignment");
  static_assert(SMEM_BYTES <= 232448, "shared memory per CTA exceeded");
  static_assert(CG == 1 || (CG == 2 && NA == 1 && KIND != KIND_TF32 && BN % 32 == 0),
                "CTA pairs: one left operand, FP16, BN / 2 a multiple of 16");
};

// Persistent CTAs: CTA b computes tiles b, b + gridDim.x, ...; the stage ring, the chunk counter
// and the two TMEM buffers run on across tiles, so one tile's epilogue overlaps the next tile's
// loads and first MMAs.
template <int BN, int NA, int NSPLIT, int STAGES, class Epi, int KIND = KIND_TF32, int CG = 1>
__global__ void __launch_bounds__(GemmRoles<NA, BN>::kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ GemmMaps maps, int K, int a_rows_per_batch, int b_rows_per_batch,
                     TileOrder order, Epi epi, unsigned* status) {
  using S = GemmShape<BN, NA, NSPLIT, STAGES, EpiSmem<Epi>::value, KIND, CG>;
  using R = GemmRoles<NA, BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* epi_smem = smem + S::EPI_OFFSET;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  uint64_t* cfull = empty + STAGES;  // [2] chunk accumulated (MMA commit)
  uint64_t* cempty = cfull + 2;      // [2] chunk drained (one arrival per epilogue thread)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(cempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // CTA pairs: rank in the pair, the pair's index and count
  const uint32_t rank = CG == 2 ? cluster_ctarank() : 0u;
  const int unit = CG == 2 ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int nunits = CG == 2 ? (int)(gridDim.x >> 1) : (int)gridDim.x;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&cfull[b], 1);
      mbar_init(&cempty[b], CG * R::kEpiThreads);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    if constexpr (CG == 2)
      tmem_alloc_pair(tmem_slot, S::TMEM_COLS);
    else
      tmem_alloc(tmem_slot, S::TMEM_COLS);
  }
  tc_fence_before();
  __syncthreads();
  if constexpr (CG == 2) cluster_sync_all();  // the peer's barriers are initialised before any arrive
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  constexpr int KB = kblock_elems(KIND);  // K elements per k-block (one row of the tile)
  constexpr int KK = row_bytes(KIND) / 32;  // MMAs per k-block: 32 bytes of K each
  constexpr int CKB = chunk_kb(KIND);
  const int nk = (K + KB - 1) / KB;
  const int nchunks = (nk + CKB - 1) / CKB;
  const int ntiles = order.count();

  if (warp == R::kProducerWarp) {
    if (lane == 0) {
      for (int a = 0; a < NA; ++a) {
        tma_prefetch_desc(&maps.a_hi[a]);
        if (NSPLIT == 3) tma_prefetch_desc(&maps.a_lo[a]);
      }
      tma_prefetch_desc(&maps.b_hi);
      if (NSPLIT == 3) tma_prefetch_desc(&maps.b_lo);
      uint32_t g = 0;  // stage uses so far (all tiles)
      bool ok = true;
      for (int l = unit; l < ntiles && ok; l += nunits) {
        int z, mt, nt;
        order.decode(l, z, mt, nt);
        const int arow = z * a_rows_per_batch + mt * (kBM * CG) + (int)rank * kBM;
        const int brow = z * b_rows_per_batch + nt * BN + (int)rank * (BN / CG);
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const uint32_t s = g % STAGES, r = g / STAGES;
          if (r > 0 && !mbar_wait(&empty[s], (r - 1) & 1, abort_flag, status)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + s * S::STAGE_BYTES;
          const int k = kb * KB;
          if constexpr (CG == 2) {
            // both CTAs' copies complete on the leader's full barrier, which expects both stages
            if (rank == 0) mbar_expect_tx(&full[s], 2 * S::STAGE_BYTES);
            const uint32_t fb = mapa_shared(&full[s], 0);
            if (NSPLIT == 3 && maps.a_planes) {
              tma_load_3d_pair(st, &maps.a_hi[0], k, arow, 0, fb);
            } else {
              tma_load_2d_pair(st, &maps.a_hi[0], k, arow, fb);
              if (NSPLIT == 3) tma_load_2d_pair(st + S::A_TILE, &maps.a_lo[0], k, arow, fb);
            }
            if (NSPLIT == 3 && maps.b_planes) {
              tma_load_3d_pair(st + S::NAT * S::A_TILE, &maps.b_hi, k, brow, 0, fb);
            } else {
              tma_load_2d_pair(st + S::NAT * S::A_TILE, &maps.b_hi, k, brow, fb);
              if (NSPLIT == 3) tma_load_2d_pair(st + S::NAT * S::A_TILE + S::B_TILE, &maps.b_lo, k, brow, fb);
            }
            continue;
          }
          mbar_expect_tx(&full[s], S::STAGE_BYTES);
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            if (NSPLIT == 3 && maps.a_planes) {
              tma_load_3d(st + (a * 2) * S::A_TILE, &maps.a_hi[a], k, arow, 0, &full[s]);
            } else {
              tma_load_2d(st + (a * (S::NAT / NA)) * S::A_TILE, &maps.a_hi[a], k, arow, &full[s]);
              if (NSPLIT == 3) tma_load_2d(st + (a * 2 + 1) * S::A_TILE, &maps.a_lo[a], k, arow, &full[s]);
            }
          }
          if (NSPLIT == 3 && maps.b_planes) {
            tma_load_3d(st + S::NAT * S::A_TILE, &maps.b_hi, k, brow, 0, &full[s]);
          } else {
            tma_load_2d(st + S::NAT * S::A_TILE, &maps.b_hi, k, brow, &full[s]);
            if (NSPLIT == 3) tma_load_2d(st + S::NAT * S::A_TILE + S::B_TILE, &maps.b_lo, k, brow, &full[s]);
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == R::kMmaWarp) {
    if (lane == 0 && rank == 0) {
      constexpr uint32_t idesc = KIND != KIND_TF32 ? idesc_f16(kBM * CG, BN) : idesc_tf32(kBM, BN);
      uint32_t g = 0, c = 0;  // stage uses and chunks so far (all tiles)
      bool ok = true;
      for (int l = unit; l < ntiles && ok; l += nunits) {
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const bool first = (kb % CKB) == 0;
          const bool last = (kb % CKB) == CKB - 1 || kb == nk - 1;
          const uint32_t buf = c & 1;
          if (first && c >= 2 && !mbar_wait(&cempty[buf], ((c >> 1) - 1) & 1, abort_flag, status)) {
            ok = false;
            break;
          }
          const uint32_t s = g % STAGES, r = g / STAGES;
          if (!mbar_wait(&full[s], r & 1, abort_flag, status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          uint8_t* st = smem + s * S::STAGE_BYTES;
          const uint64_t db_hi = desc_kmajor<KIND>(st + S::NAT * S::A_TILE);
          const uint64_t db_lo = desc_kmajor<KIND>(st + S::NAT * S::A_TILE + S::B_TILE);
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            const uint64_t da_hi = desc_kmajor<KIND>(st + (a * (S::NAT / NA)) * S::A_TILE);
            const uint64_t da_lo = desc_kmajor<KIND>(st + (a * 2 + 1) * S::A_TILE);
            const uint32_t d = tmem + (uint32_t)(buf * S::BUF_COLS + a * BN);
#pragma unroll
            for (int kk = 0; kk < KK; ++kk) {
              // K steps wholly past K multiply TMA's zero fill: skip them
              if (kk > 0 && kb * KB + kk * (KB / KK) >= K) break;
              // 32 bytes of K per MMA (8 tf32 or 16 fp16): advance the start address by 2 (16-byte units)
              if constexpr (CG == 2) {
                mma_f16_pair(d, da_hi + 2 * kk, db_hi + 2 * kk, idesc, (!first || kk > 0) ? 1u : 0u);
                if (NSPLIT == 3) {
                  mma_f16_pair(d, da_hi + 2 * kk, db_lo + 2 * kk, idesc, 1u);
                  mma_f16_pair(d, da_lo + 2 * kk, db_hi + 2 * kk, idesc, 1u);
                }
              } else if constexpr (KIND != KIND_TF32) {
                mma_f16(d, da_hi + 2 * kk, db_hi + 2 * kk, idesc, (!first || kk > 0) ? 1u : 0u);
                if (NSPLIT == 3) {
                  mma_f16(d, da_hi + 2 * kk, db_lo + 2 * kk, idesc, 1u);
                  mma_f16(d, da_lo + 2 * kk, db_hi + 2 * kk, idesc, 1u);
                }
              } else {
                mma_tf32(d, da_hi + 2 * kk, db_hi + 2 * kk, idesc, (!first || kk > 0) ? 1u : 0u);
                if (NSPLIT == 3) {
                  mma_tf32(d, da_hi + 2 * kk, db_lo + 2 * kk, idesc, 1u);
                  mma_tf32(d, da_lo + 2 * kk, db_hi + 2 * kk, idesc, 1u);
                }
              }
            }
          }
          if constexpr (CG == 2) {
            mma_commit_pair(&empty[s]);
            if (last) {
              mma_commit_pair(&cfull[buf]);
              ++c;
            }
          } else {
            mma_commit(&empty[s]);
            if (last) {
              mma_commit(&cfull[buf]);
              ++c;
            }
          }
        }
      }
    }
    __syncwarp();
  } else {
    // drain every chunk into FP32 registers (round-to-nearest), then the epilogue; warp w
    // reads TMEM lane quarter w % 4 and column group w / 4
    const int quarter = warp & 3, group = warp >> 2;
    uint32_t c = 0;  // chunks so far (all tiles)
    bool ok = true;
    // chunk-empty arrivals of a pair go to the leader's barriers (the peer's own are unused)
    const uint32_t ce_remote[2] = {CG == 2 ? mapa_shared(&cempty[0], 0) : 0u, CG == 2 ? mapa_shared(&cempty[1], 0) : 0u};
    for (int l = unit; l < ntiles; l += nunits) {
      int z, mt, nt;
      order.decode(l, z, mt, nt);
      float v[R::kGroupCols];
#pragma unroll
      for (int i = 0; i < R::kGroupCols; ++i) v[i] = 0.0f;
      for (int ch = 0; ch < nchunks && ok; ++ch, ++c) {
        const uint32_t buf = c & 1;
        if (!mbar_wait(&cfull[buf], (c >> 1) & 1, abort_flag, status)) ok = false;
        // tcgen05.ld is warp-collective: decide per warp
        ok = __all_sync(0xffffffffu, ok) != 0;
        if (!ok) break;
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < R::kGroupCols / 32; ++q) {
          float t[32];
          tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) +
                        (uint32_t)(buf * S::BUF_COLS + group * R::kGroupCols + q * 32),
                    t);
#pragma unroll
          for (int i = 0; i < 32; ++i) v[q * 32 + i] += t[i];
        }
        tc_fence_before();
        if constexpr (CG == 2)
          mbar_arrive_cluster(ce_remote[buf]);
        else
          mbar_arrive_cta(&cempty[buf]);
      }
      // every epilogue thread takes this vote once per tile, so all of them leave together;
      // a column group hands its columns to the epilogue as a tile starting at its own offset
      if (!epi_all(ok && !*abort_flag, R::kEpiThreads)) break;
      const int row = mt * (kBM * CG) + (int)rank * kBM + quarter * 32 + lane;
      if constexpr (EpiUsesMaps<Epi>::value)
        epi(z, row, nt * BN + group * (R::kGroupCols / NA), v, epi_smem, &maps);
      else
        epi(z, row, nt * BN + group * (R::kGroupCols / NA), v, epi_smem);
    }
  }
  if constexpr (EpiUsesMaps<Epi>::value) {
    if (threadIdx.x == 0) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if constexpr (CG == 2) {
    // neither CTA frees its TMEM or leaves while the pair's MMAs, copies or arrivals may still
    // reach it
    cluster_sync_all();
    tc_fence_after();
    if (warp == 0) tmem_dealloc_pair(tmem, S::TMEM_COLS);
  } else {
    if (warp == 0) tmem_dealloc(tmem, S::TMEM_COLS);
  }
}

}  // namespace umma
}  // namespace ipie_b200
