// GEMM-shaped stages of the FP64 walker step on the f64 tensor cores
// (DMMA): force bias, VHS assembly, one-body propagation, the Taylor series
// of exp(VHS), and the fused exchange energy.
#include "gemm_f64.cuh"
#include "kernels.h"

namespace ipie_b200 {

// Large GEMMs (force bias, VHS, exchange): 128 x 64 CTA tile, 8 warps.
using CfgBig = TileCfg<128, 64, 16, 4, 2>;
// Batched per-walker GEMMs: 64-row tile; the column tile follows 2N.
using CfgW64 = TileCfg<64, 64, 16, 2, 4>;
using CfgW32 = TileCfg<64, 32, 16, 4, 2>;
using CfgW16 = TileCfg<64, 16, 16, 4, 2>;

// ---------------------------------------------------------------------------
// Force bias: vbias[w][x] (+)= sum_k rchol[x][k] Ghalf[w][k]  (rchol real).
// M = X rows, N = 2W interleaved (re, im) columns, K = N_s * M_basis.
// ---------------------------------------------------------------------------
struct EpiVbias {
  double2* v;
  int X;
  int accumulate;
  double scale;  // 2 for spin-aliased walkers: exactly t + t
  __device__ __forceinline__ void operator()(int, int x, int col, double v0, double v1) const {
    const size_t idx = (size_t)(col >> 1) * X + x;
    double2 r = make_double2(scale * v0, scale * v1);
    if (accumulate) r = cadd(r, v[idx]);
    v[idx] = r;
  }
};

cudaError_t launch_force_bias(const double* rchol, const double2* ghalf, int W, int X, int K, double2* vbias,
                              int accumulate, cudaStream_t st, double scale) {
  using C = CfgBig;
  LoadRowK<C, C::BM> la{rchol, 0, K};
  LoadWalkerCplx<C, C::BN> lb{reinterpret_cast<const double*>(ghalf), 2LL * K};
  return launch_dmma_gemm<C>(X, 2 * W, K, 1, la, lb, EpiVbias{vbias, X, accumulate, scale}, st);
}

// ---------------------------------------------------------------------------
// VHS: VHS_packed[p][(w,c)] = sum_x L_packed[p][x] xshifted[x][(w,c)], scaled
// by i sqrt(dt) and scattered to both triangles of the symmetric (W, M, M).
// ---------------------------------------------------------------------------
struct EpiVHS {
  double2* vhs;
  const int* ii;
  const int* jj;
  int M;
  double sdt;
  __device__ __forceinline__ void operator()(int, int p, int col, double v0, double v1) const {
    const int w = col >> 1;
    const double2 val = make_double2(-sdt * v1, sdt * v0);
    const int i = ii[p], j = jj[p];
    double2* base = vhs + (size_t)w * M * M;
    base[(size_t)i * M + j] = val;
    base[(size_t)j * M + i] = val;
  }
};

cudaError_t launch_vhs(const double* chol_packed, const int* idx_i, const int* idx_j, int P, int X, int M,
                       const double2* xshifted, int W, double sqrt_dt, double2* vhs, cudaStream_t st) {
  using C = CfgBig;
  LoadRowK<C, C::BM> la{chol_packed, 0, X};
  LoadRowR<C, C::BN> lb{reinterpret_cast<const double*>(xshifted), 0, 2LL * W};
  return launch_dmma_gemm<C>(P, 2 * W, X, 1, la, lb, EpiVHS{vhs, idx_i, idx_j, M, sqrt_dt}, st);
}

// ---------------------------------------------------------------------------
// One-body: phi_out[w] = expH1 . phi_in[w]; expH1 real (M x M) or complex.
// ---------------------------------------------------------------------------
struct EpiStoreC {
  double2* out;
  long long bs;
  int ld;  // complex row stride
  __device__ __forceinline__ void operator()(int b, int row, int col, double v0, double v1) const {
    out[(size_t)b * bs + (size_t)row * ld + (col >> 1)] = make_double2(v0, v1);
  }
};

template <class C>
static cudaError_t one_body_cfg(const double* expH1, int cplx, const double2* phi_in, double2* phi_out, int W, int M,
                                int N, cudaStream_t st) {
  EpiStoreC epi{phi_out, (long long)M * N, N};
  if (!cplx) {
    LoadRowK<C, C::BM> la{expH1, 0, M};
    LoadRowR<C, C::BN> lb{reinterpret_cast<const double*>(phi_in), 2LL * M * N, 2LL * N};
    return launch_dmma_gemm<C>(M, 2 * N, M, W, la, lb, epi, st);
  }
  LoadRowK<C, C::BM> la{expH1, 0, 2LL * M};
  LoadCplxEmbed<C, C::BN> lb{phi_in, (long long)M * N, N};
  return launch_dmma_gemm<C>(M, 2 * N, 2 * M, W, la, lb, epi, st);
}

cudaError_t launch_one_body(const double* expH1, int cplx, const double2* phi_in, double2* phi_out, int W, int M, int N,
                            cudaStream_t st) {
  if (2 * N > 32) return one_body_cfg<CfgW64>(expH1, cplx, phi_in, phi_out, W, M, N, st);
  if (2 * N > 16) return one_body_cfg<CfgW32>(expH1, cplx, phi_in, phi_out, W, M, N, st);
  return one_body_cfg<CfgW16>(expH1, cplx, phi_in, phi_out, W, M, N, st);
}

// ---------------------------------------------------------------------------
// Taylor series of exp(VHS) applied to phi:
//   T_0 = phi_in;  T_n = VHS T_{n-1} / n;  phi_out = phi_in + sum_{n=1..nmax} T_n
// One batched complex GEMM per term (VHS complex natural layout as the left
// operand, T embedded 2x2 as the right operand), phi_out updated in the
// epilogue.  t0/t1 are ping-pong buffers of the size of phi.
// ---------------------------------------------------------------------------
struct EpiTaylor {
  double2* tout;
  const double2* phi_in;
  double2* phi_out;
  long long bs;
  int ld;
  double inv_n;
  int first;
  __device__ __forceinline__ void operator()(int b, int row, int col, double v0, double v1) const {
    const size_t idx = (size_t)b * bs + (size_t)row * ld + (col >> 1);
    const double2 t = make_double2(v0 * inv_n, v1 * inv_n);
    if (tout) tout[idx] = t;
    const double2 base = first ? phi_in[idx] : phi_out[idx];
    phi_out[idx] = cadd(base, t);
  }
};

template <class C>
static cudaError_t taylor_cfg(const double2* vhs, const double2* phi_in, double2* phi_out, double2* t0, double2* t1,
                              int W, int M, int N, int nmax, cudaStream_t st) {
  const double2* src = phi_in;
  double2* bufs[2] = {t0, t1};
  for (int n = 1; n <= nmax; ++n) {
    double2* dst = (n == nmax) ? nullptr : bufs[n & 1];
    LoadRowK<C, C::BM> la{reinterpret_cast<const double*>(vhs), 2LL * M * M, 2LL * M};
    LoadCplxEmbed<C, C::BN> lb{src, (long long)M * N, N};
    EpiTaylor epi{dst, phi_in, phi_out, (long long)M * N, N, 1.0 / n, n == 1};
    cudaError_t e = launch_dmma_gemm<C>(M, 2 * N, 2 * M, W, la, lb, epi, st);
    if (e != cudaSuccess) return e;
    src = dst;
  }
  return cudaSuccess;
}

cudaError_t launch_taylor(const double2* vhs, const double2* phi_in, double2* phi_out, double2* t0, double2* t1, int W,
                          int M, int N, int nmax, cudaStream_t st) {
  if (nmax < 1) return cudaErrorInvalidValue;
  if (2 * N > 32) return taylor_cfg<CfgW64>(vhs, phi_in, phi_out, t0, t1, W, M, N, nmax, st);
  if (2 * N > 16) return taylor_cfg<CfgW32>(vhs, phi_in, phi_out, t0, t1, W, M, N, nmax, st);
  return taylor_cfg<CfgW16>(vhs, phi_in, phi_out, t0, t1, W, M, N, nmax, st);
}

// ---------------------------------------------------------------------------
// Fused exchange:  raw_w = sum_x sum_ij T_ij T_ji,  T = rchol_x (N x M) Ghalf_w^T.
// GEMM rows (x, i) over X*NP (i padded to NP in {8,16,32}), columns
// (w, j, c) over 2*W*NP, K = M.  The CTA tile holds complete NP x NP blocks
// (x, w); the epilogue parks the tile in shared memory, forms the bilinear
// trace per block and writes one partial per (x-tile, walker) -- T itself
// never reaches global memory.
// ---------------------------------------------------------------------------
template <class C, int NP>
struct LoadExchA {  // rows (x, i): rchol[x][i*M + m], zero for i >= N
  const double* p;
  int N, M;
  static constexpr int E = C::BM * C::BK / C::THREADS;
  double v[E];
  __device__ __forceinline__ void fetch(int, int r0, int k0, int rows, int K) {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      int e = threadIdx.x + q * C::THREADS;
      int r = r0 + e / C::BK, k = k0 + e % C::BK;
      int x = r / NP, i = r % NP;
      v[q] = (r < rows && i < N && k < K) ? __ldg(p + ((size_t)x * N + i) * M + k) : 0.0;
    }
  }
  __device__ __forceinline__ void commit(double* s) const {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      int e = threadIdx.x + q * C::THREADS;
      s[(e / C::BK) * C::LDS + e % C::BK] = v[q];
    }
  }
};

template <class C, int NP>
struct LoadExchB {  // rows (w, j, c): Ghalf[w][j][m].c, zero for j >= N
  const double* p;
  int N, M;
  static constexpr int E = C::BN * C::BK / C::THREADS;
  double v[E];
  __device__ __forceinline__ void fetch(int, int r0, int k0, int rows, int K) {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      int e = threadIdx.x + q * C::THREADS;
      int pl = e / (2 * C::BK), rem = e % (2 * C::BK);
      int k = k0 + rem / 2, c = rem & 1;
      int pr = r0 / 2 + pl;  // (w, j) pair index
      int w = pr / NP, j = pr % NP;
      v[q] = (2 * pr < rows && j < N && k < K) ? __ldg(p + (((size_t)w * N + j) * M + k) * 2 + c) : 0.0;
    }
  }
  __device__ __forceinline__ void commit(double* s) const {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      int e = threadIdx.x + q * C::THREADS;
      int pl = e / (2 * C::BK), rem = e % (2 * C::BK);
      s[(2 * pl + (rem & 1)) * C::LDS + rem / 2] = v[q];
    }
  }
};

template <class C, int NP>
__global__ void __launch_bounds__(C::THREADS) exchange_kernel(const double* __restrict__ rchol,
                                                              const double* __restrict__ ghalf, int W, int X, int M,
                                                              int N, double2* __restrict__ part) {
  extern __shared__ double smem[];
  constexpr int XB = C::BM / NP;        // x values per tile
  constexpr int WB = C::BN / (2 * NP);  // walkers per tile
  const int m0 = blockIdx.y * C::BM, n0 = blockIdx.x * C::BN;
  const int rows = X * NP, cols = 2 * W * NP;
  LoadExchA<C, NP> la{rchol, N, M};
  LoadExchB<C, NP> lb{ghalf, N, M};
  Acc<C> acc;
  dmma_mainloop<C>(0, m0, n0, rows, cols, M, la, lb, smem, acc);
  // park the tile: sC[r][c] with row stride BN + 2
  constexpr int LDC = C::BN + 2;
  double* sC = smem;
#pragma unroll
  for (int i = 0; i < C::FM; ++i)
#pragma unroll
    for (int j = 0; j < C::FN; ++j) {
      int r = acc_row<C>(i), c = acc_col<C>(j);
      sC[r * LDC + c] = acc.v[i][j][0];
      sC[r * LDC + c + 1] = acc.v[i][j][1];
    }
  __syncthreads();
  // Each warp reduces (x_l, w_l) blocks: sum_{i,j<N} T_ij T_ji.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = C::THREADS / 32;
  __shared__ double2 wpart[XB * WB];
  for (int blk = warp; blk < XB * WB; blk += nw) {
    const int xl = blk / WB, wl = blk % WB;
    double2 s = make_double2(0.0, 0.0);
    const bool valid = (blockIdx.y * XB + xl) < X && (blockIdx.x * WB + wl) < W;
    if (valid) {
      for (int e = lane; e < N * N; e += 32) {
        const int i = e / N, j = e % N;
        const double* tij = sC + (xl * NP + i) * LDC + 2 * (wl * NP + j);
        const double* tji = sC + (xl * NP + j) * LDC + 2 * (wl * NP + i);
        s.x += tij[0] * tji[0] - tij[1] * tji[1];
        s.y += tij[0] * tji[1] + tij[1] * tji[0];
      }
    }
    s = warp_sum2(s);
    if (lane == 0) wpart[blk] = s;
  }
  __syncthreads();
  if (threadIdx.x < WB) {
    const int w = blockIdx.x * WB + threadIdx.x;
    if (w < W) {
      double2 s = make_double2(0.0, 0.0);
      for (int xl = 0; xl < XB; ++xl) s = cadd(s, wpart[xl * WB + threadIdx.x]);
      part[(size_t)blockIdx.y * W + w] = s;
    }
  }
}

template <int NP>
static cudaError_t exchange_np(const double* rchol, const double2* ghalf, int W, int X, int M, int N, double2* part,
                               int* ntiles, cudaStream_t st) {
  using C = CfgBig;  // 128 x 64
  static_assert(C::BM % NP == 0 && C::BN % (2 * NP) == 0, "tile must hold whole blocks");
  constexpr int XB = C::BM / NP, WB = C::BN / (2 * NP);
  const int gx = (W + WB - 1) / WB, gy = (X + XB - 1) / XB;
  *ntiles = gy;
  if (part == nullptr) return cudaSuccess;
  size_t smem = C::SMEM_DOUBLES * sizeof(double);
  size_t need = (size_t)C::BM * (C::BN + 2) * sizeof(double);
  if (need > smem) smem = need;
  auto kern = exchange_kernel<C, NP>;
  cudaError_t e = set_smem(kern, smem);
  if (e != cudaSuccess) return e;
  kern<<<dim3(gx, gy), C::THREADS, smem, st>>>(rchol, reinterpret_cast<const double*>(ghalf), W, X, M, N, part);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_exchange(const double* rchol, const double2* ghalf, int W, int X, int M, int N, double2* part,
                            int* ntiles, cudaStream_t st) {
  if (N <= 0) {
    *ntiles = 0;
    return cudaSuccess;
  }
  if (N <= 8) return exchange_np<8>(rchol, ghalf, W, X, M, N, part, ntiles, st);
  if (N <= 16) return exchange_np<16>(rchol, ghalf, W, X, M, N, part, ntiles, st);
  if (N <= 32) return exchange_np<32>(rchol, ghalf, W, X, M, N, part, ntiles, st);
  return cudaErrorInvalidValue;
}

}  // namespace ipie_b200
