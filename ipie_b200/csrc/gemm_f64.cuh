// FP64 tensor-core GEMM core for the plain (FP64) walker step.
//
// One CTA computes a BM x BN tile of C = sum_k A[m][k] B[k][n] with
// warp-level DMMA (mma.sync m8n8k4 f64).  Operands are staged through shared
// memory in k-contiguous tiles sA[m][k], sB[n][k] (row stride BK + 4 doubles,
// which makes the fragment reads conflict-free); a per-use *loader* functor
// fills the tiles from global memory with whatever layout the operand has
// (row-major, walker-major complex, complex 2x2 embedding ...), and a
// per-use *epilogue* functor consumes accumulator pairs (C[m][n], C[m][n+1]).
// The pair maps to (re, im) of one complex output whenever the n axis is the
// interleaved complex axis, so complex outputs are written by one thread.
//
// The k loop is double-buffered: the loader for tile k+1 runs into registers
// (loader-owned) before the MMAs of tile k, and is committed to the other
// shared buffer afterwards.
#pragma once

#include "common.cuh"

namespace ipie_b200 {

template <int BM_, int BN_, int BK_, int WARPS_M_, int WARPS_N_>
struct TileCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_;
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = WARPS_N_;
  static constexpr int THREADS = 32 * WARPS_M * WARPS_N;
  static constexpr int LDS = BK + 4;
  static constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;  // warp tile
  static constexpr int FM = WTM / 8, FN = WTN / 8;              // mma tiles per warp
  static constexpr int SMEM_DOUBLES = 2 * (BM + BN) * LDS;
  static_assert(BK % 4 == 0, "BK must be a multiple of 4");
  static_assert(WTM % 8 == 0 && WTN % 8 == 0, "warp tile must be a multiple of 8");
};

// ---------------------------------------------------------------------------
// Loaders.  Each loader stages `E` elements per thread in registers:
//   fetch(batch, r0, k0, rows, K)  -> global loads into regs (zero outside)
//   commit(sT)                     -> regs into the k-contiguous smem tile
// `r` is the tile's row axis (m for A, n for B).
// ---------------------------------------------------------------------------

// Row-major real operand, element (r, k) at p[batch*bs + r*ld + k] (k contiguous).
template <class Cfg, int ROWS>
struct LoadRowK {
  const double* p;
  long long bs, ld;
  static constexpr int E = ROWS * Cfg::BK / Cfg::THREADS;
  double v[E];
  __device__ __forceinline__ void fetch(int b, int r0, int k0, int rows, int K) {
    const double* q = p + (long long)b * bs;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int r = r0 + e / Cfg::BK, k = k0 + e % Cfg::BK;
      v[i] = (r < rows && k < K) ? __ldg(q + (long long)r * ld + k) : 0.0;
    }
  }
  __device__ __forceinline__ void commit(double* s) const {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      s[(e / Cfg::BK) * Cfg::LDS + e % Cfg::BK] = v[i];
    }
  }
};

// Real operand stored with the row axis contiguous: element (r, k) at p[b*bs + k*ld + r].
template <class Cfg, int ROWS>
struct LoadRowR {
  const double* p;
  long long bs, ld;
  static constexpr int E = ROWS * Cfg::BK / Cfg::THREADS;
  double v[E];
  __device__ __forceinline__ void fetch(int b, int r0, int k0, int rows, int K) {
    const double* q = p + (long long)b * bs;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int r = r0 + e % ROWS, k = k0 + e / ROWS;
      v[i] = (r < rows && k < K) ? __ldg(q + (long long)k * ld + r) : 0.0;
    }
  }
  __device__ __forceinline__ void commit(double* s) const {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      s[(e % ROWS) * Cfg::LDS + e / ROWS] = v[i];
    }
  }
};

// Complex right operand embedded as a real 2x2 block per element so that a
// complex row-major left operand (interleaved, read as real M x 2K) times it
// gives the interleaved complex product:
//   B''[2k][2n] = re, B''[2k+1][2n] = -im, B''[2k][2n+1] = im, B''[2k+1][2n+1] = re.
// Source: complex B[k][n] at p[b*bs + k*ld + n] (double2 units, n contiguous).
template <class Cfg, int ROWS>
struct LoadCplxEmbed {
  const double2* p;
  long long bs, ld;
  static constexpr int CR = ROWS / 2, CK = Cfg::BK / 2;  // complex tile extent
  static constexpr int E = CR * CK / Cfg::THREADS > 0 ? CR * CK / Cfg::THREADS : 1;
  double2 v[E];
  __device__ __forceinline__ void fetch(int b, int r0, int k0, int rows, int K) {
    const double2* q = p + (long long)b * bs;
    int n0 = r0 / 2, kc0 = k0 / 2, nrows = rows / 2, kc = K / 2;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int n = n0 + e % CR, k = kc0 + e / CR;
      v[i] = (e < CR * CK && n < nrows && k < kc) ? q[(long long)k * ld + n] : make_double2(0.0, 0.0);
    }
  }
  __device__ __forceinline__ void commit(double* s) const {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      if (e < CR * CK) {
        int n = e % CR, k = e / CR;
        double* r0 = s + (2 * n) * Cfg::LDS + 2 * k;
        double* r1 = r0 + Cfg::LDS;
        r0[0] = v[i].x;
        r0[1] = -v[i].y;
        r1[0] = v[i].y;
        r1[1] = v[i].x;
      }
    }
  }
};

// Walker-major complex operand read as real rows (w, c): element
// (r = 2w + c, k) at p[w*ld + 2k + c] (ld in doubles).  Used for the
// half-rotated Green's functions G[w][k] as the right operand of
// rchol . G^T, so the output pair (n, n+1) is (re, im) of walker w.
template <class Cfg, int ROWS>
struct LoadWalkerCplx {
  const double* p;
  long long ld;
  static constexpr int E = ROWS * Cfg::BK / Cfg::THREADS;
  double v[E];
  __device__ __forceinline__ void fetch(int b, int r0, int k0, int rows, int K) {
    int w0 = r0 / 2;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int wl = e / (2 * Cfg::BK), rem = e % (2 * Cfg::BK);
      int k = k0 + rem / 2, c = rem & 1, w = w0 + wl;
      v[i] = (2 * w < rows && k < K) ? __ldg(p + (long long)w * ld + 2 * k + c) : 0.0;
    }
  }
  __device__ __forceinline__ void commit(double* s) const {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int wl = e / (2 * Cfg::BK), rem = e % (2 * Cfg::BK);
      s[(2 * wl + (rem & 1)) * Cfg::LDS + rem / 2] = v[i];
    }
  }
};

// ---------------------------------------------------------------------------
// Main loop (device function, reused by kernels with their own epilogues).
// ---------------------------------------------------------------------------
template <class Cfg>
struct Acc {
  double v[Cfg::FM][Cfg::FN][2];
};

template <class Cfg, class LA, class LB>
__device__ __forceinline__ void dmma_mainloop(int b, int m0, int n0, int M, int N, int K, LA& la, LB& lb,
                                              double* smem, Acc<Cfg>& acc) {
  double* sA[2] = {smem, smem + (Cfg::BM + Cfg::BN) * Cfg::LDS};
  double* sB[2] = {smem + Cfg::BM * Cfg::LDS, smem + (Cfg::BM + Cfg::BN) * Cfg::LDS + Cfg::BM * Cfg::LDS};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp / Cfg::WARPS_N) * Cfg::WTM, wn0 = (warp % Cfg::WARPS_N) * Cfg::WTN;
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) acc.v[i][j][0] = acc.v[i][j][1] = 0.0;

  const int nk = (K + Cfg::BK - 1) / Cfg::BK;
  la.fetch(b, m0, 0, M, K);
  lb.fetch(b, n0, 0, N, K);
  la.commit(sA[0]);
  lb.commit(sB[0]);
  __syncthreads();
  for (int kt = 0; kt < nk; ++kt) {
    const int cur = kt & 1;
    if (kt + 1 < nk) {
      la.fetch(b, m0, (kt + 1) * Cfg::BK, M, K);
      lb.fetch(b, n0, (kt + 1) * Cfg::BK, N, K);
    }
    const double* a_s = sA[cur];
    const double* b_s = sB[cur];
#pragma unroll
    for (int kk = 0; kk < Cfg::BK; kk += 4) {
      double af[Cfg::FM], bf[Cfg::FN];
#pragma unroll
      for (int i = 0; i < Cfg::FM; ++i) af[i] = a_s[(wm0 + 8 * i + g) * Cfg::LDS + kk + t];
#pragma unroll
      for (int j = 0; j < Cfg::FN; ++j) bf[j] = b_s[(wn0 + 8 * j + g) * Cfg::LDS + kk + t];
#pragma unroll
      for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
        for (int j = 0; j < Cfg::FN; ++j) dmma884(acc.v[i][j], af[i], bf[j]);
    }
    if (kt + 1 < nk) {
      la.commit(sA[cur ^ 1]);
      lb.commit(sB[cur ^ 1]);
    }
    __syncthreads();
  }
}

// Accumulator element (i, j, q) of this thread sits at tile row / column:
template <class Cfg>
__device__ __forceinline__ int acc_row(int i) {
  const int warp = threadIdx.x >> 5, g = (threadIdx.x & 31) >> 2;
  return (warp / Cfg::WARPS_N) * Cfg::WTM + 8 * i + g;
}
template <class Cfg>
__device__ __forceinline__ int acc_col(int j) {
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 3;
  return (warp % Cfg::WARPS_N) * Cfg::WTN + 8 * j + 2 * t;
}

// ---------------------------------------------------------------------------
// Generic kernel with a pointwise-pair epilogue.  Grid: x -> n tiles,
// y -> m tiles, z -> batch.
// ---------------------------------------------------------------------------
template <class Cfg, class LA, class LB, class Epi>
__global__ void __launch_bounds__(Cfg::THREADS) dmma_gemm_kernel(int M, int N, int K, LA la, LB lb, Epi epi) {
  extern __shared__ double smem[];
  const int b = blockIdx.z;
  const int m0 = blockIdx.y * Cfg::BM, n0 = blockIdx.x * Cfg::BN;
  Acc<Cfg> acc;
  dmma_mainloop<Cfg>(b, m0, n0, M, N, K, la, lb, smem, acc);
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) {
      int row = m0 + acc_row<Cfg>(i);
      int col = n0 + acc_col<Cfg>(j);
      if (row < M && col < N) epi(b, row, col, acc.v[i][j][0], acc.v[i][j][1]);
    }
}

template <class Kern>
inline cudaError_t set_smem(Kern kern, size_t smem) {
  if (smem > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaSuccess;
}

template <class Cfg, class LA, class LB, class Epi>
inline cudaError_t launch_dmma_gemm(int M, int N, int K, int batch, LA la, LB lb, Epi epi, cudaStream_t st) {
  size_t smem = Cfg::SMEM_DOUBLES * sizeof(double);
  auto kern = dmma_gemm_kernel<Cfg, LA, LB, Epi>;
  cudaError_t e = set_smem(kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid((N + Cfg::BN - 1) / Cfg::BN, (M + Cfg::BM - 1) / Cfg::BM, batch);
  kern<<<grid, Cfg::THREADS, smem, st>>>(M, N, K, la, lb, epi);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200
