// Fused mixed-precision orbital update of one spin block on FP16 operands, one
// walker per CTA at a time (persistent CTAs):
//
//     phi <- phi + (E - I) phi                  (one-body, FP64 add of the product)
//     T_0 = phi;  T_k = V T_{k-1} / k;  phi += T_k   (k = 1 .. nmax, Taylor series of exp(V))
//     phi <- phi + (E - I) phi                  (one-body)
//
// Every product is a 3-pass FP16 tcgen05 GEMM (A_hi B_hi + A_hi B_lo + A_lo B_hi,
// kind::f16, FP32 accumulators in TMEM) of operands split into binary16 head and
// remainder after a power-of-two scale: E - I by e_scale and V by v_scale (fixed
// per call, chosen by the caller), and the right operand B (the walker's current
// T_k or phi) by a per-walker power of two: the walker's starting orbitals by their
// exact scale, 2^(14 - e) for max|phi| = f 2^e, f in [0.5, 1) (a CTA-wide max, once
// per walker), every later B by that scale / 16.  The split carries ~2^-22 relative
// accuracy of every entry down to ~2^-13 of the orbitals' largest, and an absolute
// error near 2^-35 of it below; a B entry beyond 2^5 times it (far beyond any
// Taylor term of a convergent series) raises the non-finite status bit.  phi
// accumulates in TMEM as head/tail float pairs (~2^-47 relative) between the
// first one-body factor, read from FP64 global memory, and the last, written to
// it in FP64.
//
// What stays on chip: B (planar rows -- Re of orbital n at row n, Im at row
// BN/2 + n -- FP16 head and remainder) lives in shared memory, double-buffered:
// each term's epilogue writes the next term's operand straight into the other
// buffer, in the 128B-swizzled K-major layout the MMA reads, so T_k never goes to
// global memory, and the next term's MMAs start on the k-blocks of the first
// 128-row tile while the epilogue still works on the second.  Only the left
// operands stream through TMA: the walker's VHS planes (re/im, hi/lo; 3-D tensor
// map, rows and columns past M zero-filled without traffic; the same ~0.3 MB for
// every term, so after the first term they come from L2) and the shared E - I.
//
// Roles (BN = 64: 576 threads): warps 0..4G-1 epilogue (warp w: TMEM lane quarter
// w % 4, i.e. one output row per thread, and orbital group w / 4 of G = BN / 16
// groups of 8), then one warp whose lane 0 is the TMA producer and one whose lane
// 0 issues the MMAs.  Barriers: full/empty per stage (TMA <-> MMA), accb[mt]
// (MMA -> epilogue, once per 128-row tile and term), bready[h] (epilogue -> MMA,
// one arrival per epilogue thread per term and 128-row half of B: that half
// written and that tile's accumulator read), and the named barrier 1 of the
// epilogue threads around the CTA-wide max of each walker's starting orbitals.
// Every mbarrier wait is bounded (umma.cuh); a timeout raises the status bit and
// all roles leave their loops (the epilogue threads still meet at their named
// barrier in the same order), then TMEM is released.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <string.h>

#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"
#include "umma.cuh"

namespace ipie_b200 {
namespace umma {

cudaError_t make_map_f16(CUtensorMap* m, const void* base, long long rows, long long k, long long ld, int box_rows);
cudaError_t make_map_f16_batched(CUtensorMap* m, const void* base, long long batch, long long rows, long long k,
                                 long long ld, int box_rows);
cudaError_t make_map_f16_tail4(CUtensorMap* m, const void* base, long long batch, long long rows, long long k,
                               long long ld, long long plane, int box_rows);

namespace {

struct Chain16Maps {
  CUtensorMap e_hi, e_lo;  // E - I (M x Mp halves), box 128 x 64
  CUtensorMap v[4];        // VHS planes re_hi, im_hi, re_lo, im_lo (W, M, Mp halves), box 1 x 128 x 64
  CUtensorMap vt;          // the four planes as one 4-D map, box 16 x rows x 1 x 4 (tail4)
  int tail_plane[4];       // position of plane v[i] in vt's plane order
  int tail4;               // vt is valid: the planes are equally spaced in one allocation
};

constexpr int kATile = 128 * 128;        // bytes: 128 rows x 64 halves
constexpr int kStageBytes = 2 * kATile;  // re and im planes of one part (hi or lo)
constexpr int kMaxM = 256;
constexpr int kKB = kMaxM / 64;          // k-blocks of 64 reserved for B (M <= 256)

template <int BN>
struct Chain16Roles {
  static constexpr int kGroups = BN / 16;
  static constexpr int kEpiWarps = 4 * kGroups;
  static constexpr int kEpiThreads = 32 * kEpiWarps;
  static constexpr int kProducerWarp = kEpiWarps, kMmaWarp = kEpiWarps + 1;
  static constexpr int kThreads = kEpiThreads + 64;
  // stages of the left-operand ring next to the two B buffers (2 x 2 x kKB x BN x 128 bytes)
  static constexpr int kStages = BN == 64 ? 3 : 5;
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// byte offset of B element (row n, k) inside one B region (hi or lo): k-block tiles of BN rows x
// 128 bytes (64 halves), 16-byte chunks (8 halves) XOR-swizzled with the row (TMA's 128B pattern)
template <int BN>
__device__ __forceinline__ uint32_t b16_offset(int n, int k) {
  const int kb = k >> 6, kc = k & 63;
  return (uint32_t)(kb * BN * 128 + n * 128 + ((((kc >> 3) ^ (n & 7)) << 4) | ((kc & 7) << 1)));
}

// B element = binary16 head and remainder of x * s (s a power of two)
template <int BN>
__device__ __forceinline__ void put_b16(uint8_t* bhi, uint8_t* blo, int n, int k, float x, float s) {
  const uint32_t o = b16_offset<BN>(n, k);
  const float y = x * s;
  const __half h = __float2half_rn(y);
  *reinterpret_cast<__half*>(bhi + o) = h;
  *reinterpret_cast<__half*>(blo + o) = __float2half_rn(y - __half2float(h));
}

// Writes the binary16 head and remainder of v x s for an 8 x 8 block of B: on entry lane l of
// the warp holds v[q] for K index k_base + l and orbital row n0 + q; groups of 8 lanes transpose
// their 8 x 8 block with shuffles (three butterfly stages, each swapping the off-diagonal
// halves), after which lane 8g + r holds orbital row n0 + r at K indices k_base + 8g .. + 7, one
// 16-byte chunk of the K-major swizzled layout per plane.
template <int BN>
__device__ __forceinline__ void put_b16_block(uint8_t* bhi, uint8_t* blo, int n0, int k_base, float (&v)[8],
                                              float s) {
  const int lane = threadIdx.x & 31, r = lane & 7;
#pragma unroll
  for (int st = 4; st >= 1; st >>= 1) {
    const bool upper = (r & st) != 0;
#pragma unroll
    for (int q0 = 0; q0 < 8; ++q0) {
      if (q0 & st) continue;
      const int q1 = q0 | st;
      const float x = upper ? v[q0] : v[q1];
      const float y = __shfl_xor_sync(0xffffffffu, x, st);
      if (upper)
        v[q0] = y;
      else
        v[q1] = y;
    }
  }
  uint32_t hw[4], lw[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float y0 = v[2 * i] * s, y1 = v[2 * i + 1] * s;
    const __half h0 = __float2half_rn(y0), h1 = __float2half_rn(y1);
    const __half l0 = __float2half_rn(y0 - __half2float(h0)), l1 = __float2half_rn(y1 - __half2float(h1));
    hw[i] = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
    lw[i] = (uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
  }
  const uint32_t o = b16_offset<BN>(n0 + r, k_base + (lane & ~7));
  *reinterpret_cast<uint4*>(bhi + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *reinterpret_cast<uint4*>(blo + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// (a, b) += x for a head/tail float pair a + b (|b| <= ulp(a)/2): Knuth's two-sum of a and x,
// then the tail folded back; ~2^-47 relative, enough to accumulate the FP32 Taylor terms
// of phi without a round trip through FP64 global memory.
__device__ __forceinline__ void ff_add(float& a, float& b, float x) {
  const float s = a + x;
  const float v = s - a;
  const float e = (a - (s - v)) + (x - v);
  const float t = b + e;
  a = s + t;
  b = t - (a - s);
}

// scale of a new B from its largest magnitude: 2^(14 - e) for max = f 2^e, f in [0.5, 1); capped
// at 2^64 (a term below 2^-51 of unit orbitals stays smaller than the ideal range, and the
// unscaling factor 1 / (k v_scale s) stays a normal float)
__device__ __forceinline__ float b_scale_for(float mx) {
  if (!(mx > 0.0f) || !isfinite(mx)) return 1.0f;
  int e;
  frexpf(mx, &e);
  return ldexpf(1.0f, 14 - max(e, -50));
}

// CTA-wide max of |v| and AND of ok over the nthreads epilogue threads, in one barrier (named
// barrier 1, which also orders the shared-memory atomics before the read).  Slot u % 3 of smax
// takes this max; slot (u + 2) % 3 is cleared for the one after next (its last reader passed
// the barrier before this one).  Every epilogue thread takes part every time, so a failed wait
// anywhere makes all of them leave at the same point.
__device__ __forceinline__ bool epi_max_vote(float v, bool ok, unsigned* smax, uint32_t& u, int nthreads,
                                             float& mx) {
  const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(fabsf(v)));
  if ((threadIdx.x & 31) == 0) atomicMax(&smax[u % 3], bits);
  uint32_t r;
  asm volatile(
      "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.and.pred q, 1, %2, p;\nselp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)ok), "r"(nthreads)
      : "memory");
  mx = __uint_as_float(*reinterpret_cast<volatile unsigned*>(&smax[u % 3]));
  if (threadIdx.x == 0) smax[(u + 2) % 3] = 0u;
  ++u;
  return r != 0;
}

template <int BN>
__global__ void __launch_bounds__(Chain16Roles<BN>::kThreads, 1)
    orbital_chain16_kernel(const __grid_constant__ Chain16Maps maps, float e_scale, float v_scale,
                           const double2* __restrict__ phi_in, double2* __restrict__ phi_out, int W, int M, int N,
                           int nmax, unsigned* status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int KB = (M + 63) / 64, MT = (M + 127) / 128;
  constexpr int kBTile = BN * 128;
  constexpr int kBRegion = kKB * kBTile;  // one of hi / lo of one buffer
  constexpr int kH = BN / 2;              // Im rows start here
  using R = Chain16Roles<BN>;
  constexpr int kEpiThreads = R::kEpiThreads, kThreads = R::kThreads;
  constexpr int kProducerWarp = R::kProducerWarp, kMmaWarp = R::kMmaWarp;
  constexpr int kSt = R::kStages;
  // two B buffers (hi, lo each): the epilogue of term g writes buffer (g + 1) & 1 while the MMAs
  // of term g read buffer g & 1
  uint8_t* bbuf = smem;
  uint8_t* stg = smem + 4 * kBRegion;
  uint64_t* full = reinterpret_cast<uint64_t*>(stg + kSt * kStageBytes);
  uint64_t* empty = full + kSt;
  uint64_t* accb = empty + kSt;  // one per 128-row tile (M <= 256)
  uint64_t* bready = accb + 2;   // one per 128-row half of B (its rows come from that tile)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bready + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned* smax = reinterpret_cast<unsigned*>(tmem_slot + 2);  // [3]: the walkers' starting maxima
  unsigned* tmax = smax + 3;  // [4]: max |B| of global term g in slot g % 4
  // TMEM columns: accumulators 2 m-tiles x 2 left operands x BN, then phi as head/tail float
  // pairs (2 m-tiles x [head BN | tail BN])
  constexpr uint32_t kTmemCols = 8 * BN;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kSt; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accb[0], 1);
    mbar_init(&accb[1], 1);
    mbar_init(&bready[0], kEpiThreads);
    mbar_init(&bready[1], kEpiThreads);
    *abort_flag = 0;
    smax[0] = smax[1] = smax[2] = 0u;
    tmax[0] = tmax[1] = tmax[2] = tmax[3] = 0u;
    mbar_fence_init();
  }
  // rows n >= N (and kH + n >= kH + N) and k >= M of both B buffers stay zero for the whole kernel
  for (int i = threadIdx.x; i < 4 * kBRegion / 16; i += kThreads)
    reinterpret_cast<int4*>(smem)[i] = make_int4(0, 0, 0, 0);
  fence_proxy_async_smem();
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nterms = nmax + 2;

  if (warp == kProducerWarp) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      tma_prefetch_desc(&maps.e_hi);
      tma_prefetch_desc(&maps.e_lo);
      for (int i = 0; i < 4; ++i) tma_prefetch_desc(&maps.v[i]);
      uint32_t g = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < W && ok; w += gridDim.x)
        for (int t = 0; t < nterms && ok; ++t) {
          const bool onebody = (t == 0 || t == nterms - 1);
          for (int mt = 0; mt < MT && ok; ++mt)
            for (int kb = 0; kb < KB && ok; ++kb)
              for (int part = 0; part < 2; ++part, ++g) {
                const uint32_t s = g % kSt, r = g / kSt;
                if (r > 0 && !mbar_wait(&empty[s], (r - 1) & 1, abort_flag, status)) {
                  ok = false;
                  break;
                }
                uint8_t* st = stg + s * kStageBytes;
                if (onebody) {
                  mbar_expect_tx(&full[s], kATile);
                  tma_load_2d(st, part ? &maps.e_lo : &maps.e_hi, kb * 64, mt * 128, &full[s]);
                } else {
                  // rows and columns past M of the walker's matrix are zero-filled by TMA (no traffic)
                  mbar_expect_tx(&full[s], 2 * kATile);
                  tma_load_3d(st, &maps.v[2 * part], kb * 64, mt * 128, w, &full[s]);
                  tma_load_3d(st + kATile, &maps.v[2 * part + 1], kb * 64, mt * 128, w, &full[s]);
                }
              }
        }
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_f16(128, BN);
      uint32_t g = 0, term = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < W && ok; w += gridDim.x)
        for (int t = 0; t < nterms && ok; ++t, ++term) {
          const bool onebody = (t == 0 || t == nterms - 1);
          uint8_t* b_hi = bbuf + (term & 1) * 2 * kBRegion;
          uint8_t* b_lo = b_hi + kBRegion;
          for (int mt = 0; mt < MT && ok; ++mt)
            for (int kb = 0; kb < KB && ok; ++kb) {
              // B's k-blocks 0-1 are rows 0..127 of the previous term's output (tile 0), k-blocks
              // 2-3 rows 128..255 (tile 1): start on a half as soon as the epilogue has written it
              if (mt == 0 && (kb & 1) == 0) {
                if (!mbar_wait(&bready[kb >> 1], term & 1, abort_flag, status)) {
                  ok = false;
                  break;
                }
                tc_fence_after();
              }
              for (int part = 0; part < 2; ++part, ++g) {
                const uint32_t s = g % kSt, r = g / kSt;
                if (!mbar_wait(&full[s], r & 1, abort_flag, status)) {
                  ok = false;
                  break;
                }
                tc_fence_after();
                uint8_t* st = stg + s * kStageBytes;
                const uint64_t a0 = desc_kmajor_sw128(st), a1 = desc_kmajor_sw128(st + kATile);
                const uint64_t bh = desc_kmajor_sw128(b_hi + kb * kBTile), bl = desc_kmajor_sw128(b_lo + kb * kBTile);
                const uint32_t d0 = tmem + (uint32_t)((mt * 2 + 0) * BN), d1 = tmem + (uint32_t)((mt * 2 + 1) * BN);
                // K steps of 16 past M are all zero: skip them
                const int kk_end = min(4, (M - kb * 64 + 15) / 16);
                for (int kk = 0; kk < kk_end; ++kk) {
                  const uint32_t acc = (kb > 0 || kk > 0 || part > 0) ? 1u : 0u;
                  if (part == 0) {
                    mma_f16(d0, a0 + 2 * kk, bh + 2 * kk, idesc, acc);
                    mma_f16(d0, a0 + 2 * kk, bl + 2 * kk, idesc, 1u);
                    if (!onebody) {
                      mma_f16(d1, a1 + 2 * kk, bh + 2 * kk, idesc, acc);
                      mma_f16(d1, a1 + 2 * kk, bl + 2 * kk, idesc, 1u);
                    }
                  } else {
                    mma_f16(d0, a0 + 2 * kk, bh + 2 * kk, idesc, 1u);
                    if (!onebody) mma_f16(d1, a1 + 2 * kk, bh + 2 * kk, idesc, 1u);
                  }
                }
                mma_commit(&empty[s]);
                if (kb == KB - 1 && part == 1) mma_commit(&accb[mt]);
              }
            }
        }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue warps
    constexpr int kHalf = kH / R::kGroups;
    static_assert(kHalf == 8, "one group of 8 orbitals per epilogue warp");
    const int quarter = warp & 3, half = warp >> 2;  // lane quarter, orbital group
    const int c0 = half * kHalf;                     // this warp's first orbital
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    uint32_t term = 0, u = 0;
    bool ok = true;
    // the walker loop ends only through the vote, which every epilogue thread takes together
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
      const double2* pin = phi_in + (size_t)w * M * N;
      double2* pout = phi_out + (size_t)w * M * N;
      // prologue: B = planar split of the walker's starting orbitals x their exact scale, read
      // coalesced (consecutive threads take consecutive elements of the row-major M x N block);
      // the second read comes from cache
      float pmax = 0.0f;
      for (int i = threadIdx.x; i < M * N; i += kEpiThreads) {
        const double2 z = pin[i];
        pmax = fmaxf(pmax, fmaxf(fabsf((float)z.x), fabsf((float)z.y)));
      }
      float mx;
      if (!epi_max_vote(pmax, ok && !*abort_flag, smax, u, kEpiThreads, mx)) break;
      const float s_in = b_scale_for(mx);
      // The scale of every later B is chosen before it is computed, so that the next term's
      // products can start as soon as the first half of B is written (no CTA-wide maximum on the
      // critical path).  It comes from the exact maxima of the earlier B's of the walker, which
      // the epilogue threads reduce into tmax while they write them: phi after the first one-body
      // factor takes s_in / 2; T_1 = V phi the scale of 2^5 x max|phi|; T_t (t >= 2) that of
      // max|T_(t-1)| x 4 x the last growth ratio max|T_(t-1)| / max|T_(t-2)| (the ratios of a
      // Taylor series fall like (t-1)/t); phi before the last one-body factor that of 2 x the sum
      // of the maxima.  A scale that comes out too small for its B costs a few bits below the
      // entries at 2^-13 of the largest (their absolute error stays near 2^-30 of it); one too
      // large for its B is caught (|B x scale| >= 2^15 raises the non-finite status bit).
      float s_cur = s_in, m_prev = 0.0f, m_sum = 0.0f;
      {
        uint8_t* b_hi = bbuf + (term & 1) * 2 * kBRegion;
        uint8_t* b_lo = b_hi + kBRegion;
        for (int i = threadIdx.x; i < M * N; i += kEpiThreads) {
          const int m = i / N, n = i - m * N;
          const double2 z = pin[i];
          put_b16<BN>(b_hi, b_lo, n, m, (float)z.x, s_in);
          put_b16<BN>(b_hi, b_lo, kH + n, m, (float)z.y, s_in);
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(&bready[0]);
      mbar_arrive(&bready[1]);
      bool overflow = false;
      for (int t = 0; t < nterms; ++t, ++term) {
        const bool onebody = (t == 0 || t == nterms - 1);
        const bool last = t == nterms - 1;
        // every epilogue thread has written this term's B and reduced its maximum into
        // tmax[term % 4] (the wait returns at once; it orders those writes before the reads here)
        if (ok && !mbar_wait(&bready[1], term & 1, abort_flag, status)) ok = false;
        const float m_cur = __uint_as_float(*reinterpret_cast<volatile unsigned*>(&tmax[term & 3]));
        if (threadIdx.x == 0) tmax[(term + 2) & 3] = 0u;  // for the B two terms ahead
        const float sb = s_cur;  // scale of the B this term multiplies
        // the accumulator holds the product of the scaled operands
        const float unscale = onebody ? 1.0f / (e_scale * sb) : 1.0f / ((float)t * v_scale * sb);
        // scale of the B this term's epilogue writes
        float s_next;
        if (t == 0) {
          s_next = s_in * 0.5f;
        } else if (t == 1) {
          s_next = b_scale_for(m_cur * 32.0f);
          m_sum = m_cur;
        } else {
          const float pred = m_cur * 4.0f * fmaxf(m_cur / fmaxf(m_prev, 1e-30f), 1e-6f);
          s_next = t < nmax ? b_scale_for(pred) : b_scale_for(2.0f * (m_sum + m_cur + pred));
          m_sum += m_cur;
        }
        m_prev = m_cur;
        uint8_t* n_hi = bbuf + ((term + 1) & 1) * 2 * kBRegion;  // the next term's B
        uint8_t* n_lo = n_hi + kBRegion;
        float lmax = 0.0f;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          if (mt >= MT) break;
          // each 128-row tile has its own accumulator barrier, so the first tile's epilogue
          // overlaps the second tile's MMAs; a failed wait skips the work, not the arrivals
          if (ok && !mbar_wait(&accb[mt], term & 1, abort_flag, status)) ok = false;
          ok = __all_sync(0xffffffffu, ok) != 0;
          if (ok) tc_fence_after();
          // a warp whose 32 rows all lie past M, or whose orbitals all lie past N, has nothing to do
          if (ok && mt * 128 + quarter * 32 < M && c0 < N) {
            const int m = mt * 128 + quarter * 32 + lane;
            const bool row_ok = m < M;
            const uint32_t dc0 = lane_base + (uint32_t)((mt * 2 + 0) * BN);
            const uint32_t dc1 = lane_base + (uint32_t)((mt * 2 + 1) * BN);
            const uint32_t ac = lane_base + (uint32_t)(4 * BN + mt * 2 * BN);  // phi: head [0, BN), tail [BN, 2BN)
            // real parts, then imaginary parts; TMEM reads/writes are warp-collective, so every
            // lane takes part and rows past M only skip their global and shared-memory writes
#pragma unroll
            for (int p = 0; p < 2; ++p) {
              // p = 0: Re = D0[n] - D1[kH + n]; p = 1: Im = D0[kH + n] + D1[n]
              // (one-body: D0[n] and D0[kH + n] with the real left operand E - I)
              const int cx = (p ? kH : 0) + c0, cy = (p ? 0 : kH) + c0;
              uint32_t x[8], y[8], ha[8], ta[8];
              tmem_ld8(tmem + dc0 + cx, x);
              if (!onebody) tmem_ld8(tmem + dc1 + cy, y);
              if (t > 0) {
                tmem_ld8(tmem + ac + cx, ha);
                tmem_ld8(tmem + ac + BN + cx, ta);
              }
              tmem_wait_ld();
              reg_after_wait(x);
              if (!onebody) reg_after_wait(y);
              if (t > 0) {
                reg_after_wait(ha);
                reg_after_wait(ta);
              }
              double base[8];
              if (t == 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                  const double* src = reinterpret_cast<const double*>(pin + (size_t)m * N + c0 + q) + p;
                  base[q] = (row_ok && c0 + q < N) ? *src : 0.0;
                }
              }
              float nbv[8];  // this lane's next-B values (row m, orbitals c0..c0+7)
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const int n = c0 + q;
                float uq = __uint_as_float(x[q]);
                if (!onebody) uq = p ? uq + __uint_as_float(y[q]) : uq - __uint_as_float(y[q]);
                const float vq = uq * unscale;  // (E - I) phi, or T_t
                const bool live = row_ok && n < N;
                float nb = 0.0f;  // the next B value
                if (t == 0) {
                  // phi after the first one-body factor, kept as a head/tail float pair
                  const double o = base[q] + (double)vq;
                  const float hh = (float)o;
                  ha[q] = __float_as_uint(hh);
                  ta[q] = __float_as_uint((float)(o - (double)hh));
                  nb = hh;
                } else if (last) {
                  const double o = (double)__uint_as_float(ha[q]) + (double)__uint_as_float(ta[q]) + (double)vq;
                  if (live) reinterpret_cast<double*>(pout + (size_t)m * N + n)[p] = o;
                } else {
                  float a = __uint_as_float(ha[q]), b = __uint_as_float(ta[q]);
                  ff_add(a, b, vq);
                  ha[q] = __float_as_uint(a);
                  ta[q] = __float_as_uint(b);
                  nb = t < nmax ? vq : a + b;
                }
                if (!live) nb = 0.0f;
                overflow |= !(fabsf(nb * s_next) < 32768.0f);
                lmax = fmaxf(lmax, fabsf(nb));
                nbv[q] = nb;
              }
              if (!last) {
                // rows past M and orbitals past N hold zeros, which is what B keeps there
                put_b16_block<BN>(n_hi, n_lo, (p ? kH : 0) + c0, mt * 128 + quarter * 32, nbv, s_next);
                tmem_st8(tmem + ac + cx, ha);
                tmem_st8(tmem + ac + BN + cx, ta);
              }
            }
          }
          if (!last) {
            if (mt == MT - 1) {
              // the next B's maximum, complete once every epilogue thread has arrived below
              const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(lmax));
              if (lane == 0 && bits) atomicMax(&tmax[(term + 1) & 3], bits);
            }
            // this half of the next B is written and this tile's accumulator read: the MMAs of
            // the next term may start on it (and overwrite the accumulator)
            tc_fence_before();
            fence_proxy_async_smem();
            mbar_arrive(&bready[mt]);
          }
        }
        if (MT == 1 && !last) mbar_arrive(&bready[1]);
        tmem_wait_st();
        s_cur = s_next;
      }
      // a Taylor term beyond binary16's range at the fixed scale: the walker's orbitals are wrong
      if (overflow) flag(status, STATUS_NONFINITE);
      tc_fence_before();
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// ---------------------------------------------------------------------------------------------
// The same orbital update with the operand roles transposed (M <= 208): every product is
//
//     D[r][m] = sum_k' A[r][k'] B[m][k']   (tcgen05 kind::f16, M = 128 rows, N = Mp = M rounded up to 16)
//
// with the walker's current orbitals as A and the walker's VHS planes (or E - I) as B, so that
// one MMA covers every row of V (N = 208 at M = 200) instead of 64 orbital columns: an MMA issues
// in ~70 cycles whatever its size, which bound the 128 x 64 x 16 products of the kernel above, and
// a 128 x 208 x 16 product runs ~100 cycles on the tensor core.
//
// A (shared memory, 128 rows x K' = 2 Mp, binary16, 32B-swizzled K-major 16-column k-blocks):
// row 32 q + n holds orbital n, q = 2 h + c for the head (h = 0) or remainder (h = 1) of the split
// and the output component c (0 = real, 1 = imaginary); its K' = [0, Mp) half is the real-part
// operand and [Mp, 2 Mp) the imaginary-part one:
//     real-output rows: [Re T | -Im T],   imaginary-output rows: [Im T | Re T]
// against B = [Re V | Im V] along K' (the planes of one k-block loaded as separate stages), so that
// D's lane 32 q + n, column m holds the head or remainder part of Re or Im (V T)[m][n] (for E - I
// only the real half of K' runs: Re T x (E - I) and Im T x (E - I)).  Each product is four MMAs
// per K step (A x B_head and A x B_remainder for both planes), the remainder x remainder term
// riding along.  The epilogue adds lanes 32 q + n and 32 (q + 2) + n through a shared-memory
// staging tile (different warps own those TMEM lanes).
//
// Pipeline: the epilogue of term g handles the output in 64-row chunks (the K chunks of the next
// product): it loads the chunk's accumulator columns into the staging tile, writes the next
// operand's rows of that chunk into A and arrives on aready[chunk]; the MMAs of term g + 1 start
// on a chunk as soon as it is written.  D is double-buffered in TMEM (columns 0 and 256), so the
// MMAs of term g + 1 run while the epilogue of term g still reads its buffer.  phi accumulates in
// FP64 in phi_out (global memory, read back by the same thread every term); the binary16 scales of
// the operands follow the kernel above (a predicted scale per Taylor term).
constexpr int kTMaxM = 208;
constexpr int kTEpiWarps = 16, kTEpiThreads = 32 * kTEpiWarps;
constexpr int kTProducerWarp = kTEpiWarps, kTMmaWarp = kTEpiWarps + 1;
constexpr int kTThreads = kTEpiThreads + 64;
constexpr int kTStages = 3;
constexpr int kTPitch = 68;  // floats per staging row: 64 columns + 4 (bank spread)
constexpr int kTStagingBytes = 128 * kTPitch * 4;
__host__ __device__ constexpr int t_a_bytes(int mp) { return 128 * 2 * mp * 2; }
__host__ __device__ constexpr int t_stage_bytes(int mp) { return mp * 128; }
__host__ __device__ constexpr size_t t_smem_bytes(int mp) {
  return 1024 + (size_t)t_a_bytes(mp) + (size_t)kTStages * t_stage_bytes(mp) + kTStagingBytes + 256;
}

// byte offset of A element (row r, K' index k): 16-column k-blocks of 128 rows x 32 bytes, the two
// 16-byte halves of a row swapped on every other group of 4 rows (TMA's and the MMA's 32B pattern)
__device__ __forceinline__ uint32_t t_a_offset(int r, int k) {
  return (uint32_t)((k >> 4) * 4096 + r * 32 + ((((k >> 3) & 1) ^ ((r >> 2) & 1)) << 4) + ((k & 7) << 1));
}
// binary16 head and remainder of v x s, four values packed per 8 bytes
__device__ __forceinline__ void t_split4(const float (&v)[4], float s, uint2& hi, uint2& lo) {
  uint32_t h[2], l[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float y0 = v[2 * i] * s, y1 = v[2 * i + 1] * s;
    const __half h0 = __float2half_rn(y0), h1 = __float2half_rn(y1);
    const __half l0 = __float2half_rn(y0 - __half2float(h0)), l1 = __float2half_rn(y1 - __half2float(h1));
    h[i] = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
    l[i] = (uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
  }
  hi = make_uint2(h[0], h[1]);
  lo = make_uint2(l[0], l[1]);
}
__device__ __forceinline__ uint2 t_neg(uint2 x) { return make_uint2(x.x ^ 0x80008000u, x.y ^ 0x80008000u); }
__device__ __forceinline__ void t_put(uint8_t* a, int r, int k, uint2 v) {
  *reinterpret_cast<uint2*>(a + t_a_offset(r, k)) = v;
}
// the next operand's entries for orbital n at rows m0 .. m0 + 3 (values x s, split): all eight
// places they take in A
__device__ __forceinline__ void t_put_a4(uint8_t* a, int mp, int n, int m0, const float (&tr)[4],
                                         const float (&ti)[4], float s) {
  uint2 rh, rl, ih, il;
  t_split4(tr, s, rh, rl);
  t_split4(ti, s, ih, il);
  t_put(a, n, m0, rh);
  t_put(a, n, mp + m0, t_neg(ih));
  t_put(a, 32 + n, m0, ih);
  t_put(a, 32 + n, mp + m0, rh);
  t_put(a, 64 + n, m0, rl);
  t_put(a, 64 + n, mp + m0, t_neg(il));
  t_put(a, 96 + n, m0, il);
  t_put(a, 96 + n, mp + m0, rl);
}
// AND of ok over the epilogue threads (named barrier 1), which also orders their shared-memory writes
__device__ __forceinline__ bool t_epi_all(bool ok) {
  uint32_t r;
  asm volatile(
      "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.and.pred q, 1, %2, p;\nselp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)ok), "r"(kTEpiThreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void t_epi_sync() { asm volatile("bar.sync 2, %0;\n" ::"r"(kTEpiThreads) : "memory"); }

__global__ void __launch_bounds__(kTThreads, 1)
    orbital_chain_t16_kernel(const __grid_constant__ Chain16Maps maps, float e_scale, float v_scale,
                             const double2* __restrict__ phi_in, double2* __restrict__ phi_out, int W, int M, int N,
                             int nmax, unsigned* status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int Mp = (M + 15) & ~15;  // N of every product; K of each half of K'
  const int KB16 = Mp / 16;       // 16-column k-blocks of A per half of K'
  const int C = (Mp + 63) / 64;   // 64-row chunks of the output (64-column k-blocks of B)
  const int stage_bytes = t_stage_bytes(Mp);
  const bool tail4 = maps.tail4 != 0 && Mp - 64 * (C - 1) == 16;
  uint8_t* abuf = smem;
  uint8_t* stg = smem + t_a_bytes(Mp);
  float* staging = reinterpret_cast<float*>(stg + kTStages * stage_bytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(staging) + kTStagingBytes);
  uint64_t* empty = full + kTStages;
  uint64_t* accfull = empty + kTStages;  // [2] D buffer complete (MMA commit)
  uint64_t* accempty = accfull + 2;      // [2] D buffer read (every epilogue thread)
  uint64_t* aready = accempty + 2;       // [4] chunk of A written (every epilogue thread)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(aready + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned* smax = reinterpret_cast<unsigned*>(tmem_slot + 2);  // [3]: the walkers' starting maxima
  unsigned* tmax = smax + 3;  // [4]: max |operand| of global term g in slot g % 4
  constexpr uint32_t kTmemCols = 512;  // D buffers at columns 0 and 256

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accfull[b], 1);
      mbar_init(&accempty[b], kTEpiThreads);
    }
    for (int c = 0; c < 4; ++c) mbar_init(&aready[c], kTEpiThreads);
    *abort_flag = 0;
    smax[0] = smax[1] = smax[2] = 0u;
    tmax[0] = tmax[1] = tmax[2] = tmax[3] = 0u;
    mbar_fence_init();
  }
  // A's rows of orbitals past N and columns past M stay zero for the whole kernel
  for (int i = threadIdx.x; i < t_a_bytes(Mp) / 16; i += kTThreads)
    reinterpret_cast<int4*>(abuf)[i] = make_int4(0, 0, 0, 0);
  fence_proxy_async_smem();
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nterms = nmax + 2;

  if (warp == kTProducerWarp) {
    // ------------------------------------------------------------ TMA producer
    // lane p issues the loads of stages p, p + kProducers, ... (producer_lanes)
    constexpr int kProducers = producer_lanes(kTStages);
    if (lane < kProducers) {
      if (lane == 0) {
        tma_prefetch_desc(&maps.e_hi);
        tma_prefetch_desc(&maps.e_lo);
        for (int i = 0; i < 4; ++i) tma_prefetch_desc(&maps.v[i]);
      }
      uint32_t g = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < W && ok; w += gridDim.x)
        for (int t = 0; t < nterms && ok; ++t) {
          const bool onebody = (t == 0 || t == nterms - 1);
          const int nparts = onebody ? 1 : 2;
          for (int c = 0; c < C && ok; ++c) {
            // a Taylor term's last chunk of 16 columns: all four planes in one stage (tail4)
            const bool t4 = tail4 && !onebody && c == C - 1;
            const int nst = t4 ? 1 : 2 * nparts;
            for (int q = 0; q < nst; ++q, ++g) {
              const int p = q >> 1, h = q & 1;
              if ((int)(g % kProducers) != lane) continue;
              const uint32_t s = g % kTStages, r = g / kTStages;
              if (r > 0 && !mbar_wait(&empty[s], (r - 1) & 1, abort_flag, status)) {
                ok = false;
                break;
              }
              uint8_t* dst = stg + s * stage_bytes;
              // 64 columns x Mp rows x 2 bytes either way (t4: 16 columns x 4 planes)
              mbar_expect_tx(&full[s], stage_bytes);
              // rows and columns past M are zero-filled by TMA (no traffic)
              if (t4)
                tma_load_4d(dst, &maps.vt, c * 64, 0, w, 0, &full[s]);
              else if (onebody)
                tma_load_2d(dst, h ? &maps.e_lo : &maps.e_hi, c * 64, 0, &full[s]);
              else  // maps.v: re_hi, im_hi, re_lo, im_lo
                tma_load_3d(dst, &maps.v[2 * h + p], c * 64, 0, w, &full[s]);
            }
          }
        }
    }
    __syncwarp();
  } else if (warp == kTMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(128, Mp);
      uint32_t g = 0, term = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < W && ok; w += gridDim.x)
        for (int t = 0; t < nterms && ok; ++t, ++term) {
          const bool onebody = (t == 0 || t == nterms - 1);
          const int nparts = onebody ? 1 : 2;
          const uint32_t buf = term & 1;
          if (term >= 2 && !mbar_wait(&accempty[buf], ((term >> 1) - 1) & 1, abort_flag, status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + buf * 256;
          bool first = true;
          for (int c = 0; c < C && ok; ++c) {
            if (!mbar_wait(&aready[c], term & 1, abort_flag, status)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const int kkc = min(4, (Mp - 64 * c) / 16);
            if (tail4 && !onebody && c == C - 1) {
              // one stage: plane v[2h + p] at position tail_plane[2h + p], 32-byte rows
              const uint32_t s = g % kTStages, r = g / kTStages;
              if (!mbar_wait(&full[s], r & 1, abort_flag, status)) {
                ok = false;
                break;
              }
              tc_fence_after();
              for (int p = 0; p < 2; ++p)
                for (int h = 0; h < 2; ++h) {
                  const uint64_t bdesc =
                      desc_kmajor_sw32(stg + s * stage_bytes + maps.tail_plane[2 * h + p] * Mp * 32);
                  const uint64_t adesc = desc_kmajor_sw32(abuf + (p * KB16 + 4 * c) * 4096);
                  mma_f16(d, adesc, bdesc, idesc, first ? 0u : 1u);
                  first = false;
                }
              mma_commit(&empty[s]);
              ++g;
              continue;
            }
            for (int p = 0; p < nparts && ok; ++p)
              for (int h = 0; h < 2; ++h, ++g) {
                const uint32_t s = g % kTStages, r = g / kTStages;
                if (!mbar_wait(&full[s], r & 1, abort_flag, status)) {
                  ok = false;
                  break;
                }
                tc_fence_after();
                const uint64_t bdesc = desc_kmajor_sw128(stg + s * stage_bytes);
                for (int kk = 0; kk < kkc; ++kk) {
                  const uint64_t adesc = desc_kmajor_sw32(abuf + (p * KB16 + 4 * c + kk) * 4096);
                  mma_f16(d, adesc, bdesc + 2 * kk, idesc, first ? 0u : 1u);
                  first = false;
                }
                mma_commit(&empty[s]);
              }
          }
          if (ok) mma_commit(&accfull[buf]);
        }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue warps
    // TMEM loads: warp w reads lane quarter w % 4, columns 16 (w / 4) .. + 15 of each chunk;
    // outputs: thread (w, n = lane) takes rows 4 w .. 4 w + 3 of each chunk for orbital n
    const int q = warp & 3, j = warp >> 2;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t term = 0, u = 0;
    bool ok = true;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
      const double2* pin = phi_in + (size_t)w * M * N;
      double2* pout = phi_out + (size_t)w * M * N;
      float pmax = 0.0f;
      for (int i = threadIdx.x; i < M * N; i += kTEpiThreads) {
        const double2 z = pin[i];
        pmax = fmaxf(pmax, fmaxf(fabsf((float)z.x), fabsf((float)z.y)));
      }
      float mx;
      if (!epi_max_vote(pmax, ok && !*abort_flag, smax, u, kTEpiThreads, mx)) break;
      const float s_in = b_scale_for(mx);
      // the first operand: the walker's starting orbitals x their exact scale
      for (int c = 0; c < C; ++c) {
        const int m0 = 64 * c + 4 * warp;
        if (m0 < Mp) {
          float tr[4], ti[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int m = m0 + i;
            const double2 z = (m < M && lane < N) ? pin[(size_t)m * N + lane] : make_double2(0.0, 0.0);
            tr[i] = (float)z.x;
            ti[i] = (float)z.y;
          }
          t_put_a4(abuf, Mp, lane, m0, tr, ti, s_in);
        }
      }
      fence_proxy_async_smem();
      for (int c = 0; c < C; ++c) mbar_arrive(&aready[c]);
      float s_cur = s_in, m_prev = 0.0f, m_sum = 0.0f;
      bool overflow = false;
      for (int t = 0; t < nterms; ++t, ++term) {
        const bool onebody = (t == 0 || t == nterms - 1);
        const bool last = t == nterms - 1;
        const uint32_t buf = term & 1;
        // every epilogue thread has written this term's operand and reduced its maximum into
        // tmax[term % 4] before its last arrival (the wait orders those writes before the read)
        if (ok && !mbar_wait(&aready[C - 1], term & 1, abort_flag, status)) ok = false;
        const float m_cur = __uint_as_float(*reinterpret_cast<volatile unsigned*>(&tmax[term & 3]));
        if (threadIdx.x == 0) tmax[(term + 2) & 3] = 0u;  // for the operand two terms ahead
        const float sb = s_cur;
        const float unscale = onebody ? 1.0f / (e_scale * sb) : 1.0f / ((float)t * v_scale * sb);
        // the scale of the operand this term writes (predicted as in the kernel above)
        float s_next;
        if (t == 0) {
          s_next = s_in * 0.5f;
        } else if (t == 1) {
          s_next = b_scale_for(m_cur * 32.0f);
          m_sum = m_cur;
        } else {
          const float pred = m_cur * 4.0f * fmaxf(m_cur / fmaxf(m_prev, 1e-30f), 1e-6f);
          s_next = t < nmax ? b_scale_for(pred) : b_scale_for(2.0f * (m_sum + m_cur + pred));
          m_sum += m_cur;
        }
        m_prev = m_cur;
        if (ok && !mbar_wait(&accfull[buf], (term >> 1) & 1, abort_flag, status)) ok = false;
        float lmax = 0.0f;
        for (int c = 0; c < C; ++c) {
          // this thread's FP64 orbitals of the chunk (phi, or the running sum), loaded before the
          // staging round so that their latency passes behind it
          const int m0 = 64 * c + 4 * warp;
          double2 pv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int m = m0 + i;
            const size_t o = (size_t)m * N + lane;
            pv[i] = (m0 < Mp && m < M && lane < N) ? (t == 0 ? pin[o] : pout[o]) : make_double2(0.0, 0.0);
          }
          // accumulator columns of this chunk -> staging (tcgen05.ld is warp-collective)
          ok = __all_sync(0xffffffffu, ok) != 0;
          const int col = 64 * c + 16 * j;
          if (ok && col < Mp) {
            tc_fence_after();
            uint32_t x[16];
            tmem_ld16(tmem + lane_base + buf * 256 + (uint32_t)col, x);
            tmem_wait_ld();
            reg_after_wait(x);
            float4* dst = reinterpret_cast<float4*>(staging + (q * 32 + lane) * kTPitch + 16 * j);
#pragma unroll
            for (int i = 0; i < 4; ++i)
              dst[i] = make_float4(__uint_as_float(x[4 * i]), __uint_as_float(x[4 * i + 1]),
                                   __uint_as_float(x[4 * i + 2]), __uint_as_float(x[4 * i + 3]));
          }
          if (c == C - 1) {
            // the buffer is read: the MMAs two terms ahead may overwrite it
            tc_fence_before();
            mbar_arrive(&accempty[buf]);
          }
          if (!t_epi_all(ok && !*abort_flag)) {
            ok = false;
            break;
          }
          if (m0 < Mp) {
            const float4 rh = *reinterpret_cast<const float4*>(staging + lane * kTPitch + 4 * warp);
            const float4 ih = *reinterpret_cast<const float4*>(staging + (32 + lane) * kTPitch + 4 * warp);
            const float4 rl = *reinterpret_cast<const float4*>(staging + (64 + lane) * kTPitch + 4 * warp);
            const float4 il = *reinterpret_cast<const float4*>(staging + (96 + lane) * kTPitch + 4 * warp);
            const float vr[4] = {(rh.x + rl.x) * unscale, (rh.y + rl.y) * unscale, (rh.z + rl.z) * unscale,
                                 (rh.w + rl.w) * unscale};
            const float vi[4] = {(ih.x + il.x) * unscale, (ih.y + il.y) * unscale, (ih.z + il.z) * unscale,
                                 (ih.w + il.w) * unscale};
            float nr[4], ni[4];  // the next operand (orbital lane, rows m0 ..)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int m = m0 + i;
              const bool live = m < M && lane < N;
              nr[i] = 0.0f;
              ni[i] = 0.0f;
              if (!live) continue;
              // t = 0: phi after the first one-body factor, where the FP64 sum starts
              const double2 a = make_double2(pv[i].x + (double)vr[i], pv[i].y + (double)vi[i]);
              pout[(size_t)m * N + lane] = a;
              if (t == 0) {
                nr[i] = (float)a.x;
                ni[i] = (float)a.y;
              } else if (!last) {
                nr[i] = t < nmax ? vr[i] : (float)a.x;
                ni[i] = t < nmax ? vi[i] : (float)a.y;
              }
              overflow |= !(fabsf(nr[i] * s_next) < 32768.0f) || !(fabsf(ni[i] * s_next) < 32768.0f);
              lmax = fmaxf(lmax, fmaxf(fabsf(nr[i]), fabsf(ni[i])));
            }
            if (!last) t_put_a4(abuf, Mp, lane, m0, nr, ni, s_next);
          }
          if (!last) {
            if (c == C - 1) {
              // the next operand's maximum, complete once every epilogue thread has arrived
              const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(lmax));
              if (lane == 0 && bits) atomicMax(&tmax[(term + 1) & 3], bits);
            }
            fence_proxy_async_smem();
            mbar_arrive(&aready[c]);
          }
          t_epi_sync();  // the staging tile is free for the next chunk
        }
        if (!ok) break;
        s_cur = s_next;
      }
      // a Taylor term beyond binary16's range at its predicted scale: the walker's orbitals are wrong
      if (overflow) flag(status, STATUS_NONFINITE);
      tc_fence_before();
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

cudaError_t launch_chain_t16(const Chain16Maps& maps, float e_scale, float v_scale, const double2* phi_in,
                             double2* phi_out, int W, int M, int N, int nmax, unsigned* status, cudaStream_t st) {
  const int Mp = (M + 15) & ~15;
  const size_t smem = t_smem_bytes(Mp);
  cudaError_t e =
      cudaFuncSetAttribute(orbital_chain_t16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int grid = W < sms ? W : sms;
  orbital_chain_t16_kernel<<<grid, kTThreads, smem, st>>>(maps, e_scale, v_scale, phi_in, phi_out, W, M, N, nmax,
                                                          status);
  note_launch();
  return cudaGetLastError();
}

template <int BN>
cudaError_t launch_chain16(const Chain16Maps& maps, float e_scale, float v_scale, const double2* phi_in,
                           double2* phi_out, int W, int M, int N, int nmax, unsigned* status, cudaStream_t st) {
  const size_t smem = 1024 + 4 * (size_t)kKB * BN * 128 + Chain16Roles<BN>::kStages * kStageBytes + 256;
  auto kern = orbital_chain16_kernel<BN>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int grid = W < sms ? W : sms;
  kern<<<grid, Chain16Roles<BN>::kThreads, smem, st>>>(maps, e_scale, v_scale, phi_in, phi_out, W, M, N, nmax, status);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

bool orbital_chain16_fits(int M, int N) { return M >= 1 && M <= kMaxM && N >= 1 && N <= 32; }

// One launch for the whole mixed orbital update of one spin block (see the file comment).
// e_hi/e_lo: (E - I) x e_scale (M, f16_ld(M)) binary16; v_*: VHS planes x v_scale (W, M, f16_ld(M)).
cudaError_t mixed_orbital_chain16(const void* e_hi, const void* e_lo, float e_scale, const void* v_re_hi,
                                  const void* v_re_lo, const void* v_im_hi, const void* v_im_lo, float v_scale,
                                  const double2* phi_in, double2* phi_out, int W, int M, int N, int nmax,
                                  unsigned* status, cudaStream_t st) {
  if (!orbital_chain16_fits(M, N) || nmax < 1 || phi_in == phi_out || W <= 0 || !(e_scale > 0.0f) ||
      !(v_scale > 0.0f))
    return cudaErrorInvalidValue;
  const int ld = f16_ld(M);
  // M <= 208: the transposed kernel (every row of V in one MMA); else the 128-row tile kernel
  const bool transposed = M <= kTMaxM;
  const int box_rows = transposed ? (M + 15) & ~15 : 128;
  Chain16Maps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  if ((e = make_map_f16(&maps.e_hi, e_hi, M, M, ld, box_rows)) != cudaSuccess) return e;
  if ((e = make_map_f16(&maps.e_lo, e_lo, M, M, ld, box_rows)) != cudaSuccess) return e;
  const void* planes[4] = {v_re_hi, v_im_hi, v_re_lo, v_im_lo};
  for (int i = 0; i < 4; ++i)
    if ((e = make_map_f16_batched(&maps.v[i], planes[i], W, M, M, ld, box_rows)) != cudaSuccess) return e;
  if (transposed) {
    // planes equally spaced in one allocation (in any order): the 4-D map of their last columns
    uintptr_t a[4], lo = ~uintptr_t(0);
    for (int i = 0; i < 4; ++i) {
      a[i] = reinterpret_cast<uintptr_t>(planes[i]);
      lo = a[i] < lo ? a[i] : lo;
    }
    uintptr_t stride = 0;
    for (int i = 0; i < 4; ++i)
      if (a[i] != lo && (stride == 0 || a[i] - lo < stride)) stride = a[i] - lo;
    int seen = 0;
    bool even = stride > 0 && stride % 16 == 0;
    for (int i = 0; i < 4 && even; ++i) {
      const uintptr_t d = a[i] - lo;
      const int pos = (int)(d / stride);
      even = d % stride == 0 && pos < 4 && !(seen & (1 << pos));
      seen |= 1 << pos;
      maps.tail_plane[i] = pos;
    }
    maps.tail4 = even && make_map_f16_tail4(&maps.vt, reinterpret_cast<const void*>(lo), W, M, M, ld,
                                            (long long)(stride / 2), box_rows) == cudaSuccess;
    return launch_chain_t16(maps, e_scale, v_scale, phi_in, phi_out, W, M, N, nmax, status, st);
  }
  if (2 * N <= 32) return launch_chain16<32>(maps, e_scale, v_scale, phi_in, phi_out, W, M, N, nmax, status, st);
  return launch_chain16<64>(maps, e_scale, v_scale, phi_in, phi_out, W, M, N, nmax, status, st);
}

}  // namespace umma
}  // namespace ipie_b200
