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
// Complex-Cholesky pieces (ipie's GenericComplexChol), each built from real-operand
// GEMMs of the same core: a complex operand R = R_re + i R_im enters as two launches,
// the second scaled by i in the epilogue.
//
// Force bias / Coulomb vector: out[w][xoff + x] (+)= (sr + i si) sum_k R_part[x][k] Ghalf[w][k],
// out rows of `ld` complex.
// ---------------------------------------------------------------------------
struct EpiVbiasC {
  double2* v;
  int ld, xoff;
  int accumulate;
  double sr, si;
  __device__ __forceinline__ void operator()(int, int x, int col, double v0, double v1) const {
    const size_t idx = (size_t)(col >> 1) * ld + xoff + x;
    double2 r = make_double2(sr * v0 - si * v1, sr * v1 + si * v0);
    if (accumulate) r = cadd(r, v[idx]);
    v[idx] = r;
  }
};

cudaError_t launch_force_bias_c(const double* rpart, const double2* ghalf, int W, int X, int K, double2* out, int ld,
                                int xoff, int accumulate, double sr, double si, cudaStream_t st) {
  using C = CfgBig;
  LoadRowK<C, C::BM> la{rpart, 0, K};
  LoadWalkerCplx<C, C::BN> lb{reinterpret_cast<const double*>(ghalf), 2LL * K};
  return launch_dmma_gemm<C>(X, 2 * W, K, 1, la, lb, EpiVbiasC{out, ld, xoff, accumulate, sr, si}, st);
}

// VHS of a complex Cholesky: V_w = i sqrt(dt) C . xs_w with C = [A | B] (M*M, F) complex and
// xs (F, W) complex, as two launches on C_re (mode 0: write) and C_im (mode 1: accumulate i x):
//   C xs = (P0 - Q1) + i (P1 + Q0),  (P0, P1) = C_re (xs_re, xs_im),  (Q0, Q1) = C_im (xs_re, xs_im),
//   V = i sqrt(dt) C xs:  Re V = -sdt (P1 + Q0),  Im V = sdt (P0 - Q1).
// Rows p = i M + j of C map to V_w[i][j] directly (no symmetry).
struct EpiVHSFull {
  double2* vhs;
  int M;
  double sdt;
  int mode;
  __device__ __forceinline__ void operator()(int, int p, int col, double v0, double v1) const {
    const int w = col >> 1;
    double2* dst = vhs + (size_t)w * M * M + p;
    if (mode == 0) {
      *dst = make_double2(-sdt * v1, sdt * v0);
    } else {
      const double2 o = *dst;
      *dst = make_double2(o.x - sdt * v0, o.y - sdt * v1);
    }
  }
};

cudaError_t launch_vhs_full(const double* cpart, int M, int F, const double2* xshifted, int W, double sqrt_dt,
                            double2* vhs, int mode, cudaStream_t st) {
  using C = CfgBig;
  LoadRowK<C, C::BM> la{cpart, 0, F};
  LoadRowR<C, C::BN> lb{reinterpret_cast<const double*>(xshifted), 0, 2LL * W};
  return launch_dmma_gemm<C>(M * M, 2 * W, F, 1, la, lb, EpiVHSFull{vhs, M, sqrt_dt, mode}, st);
}

// Local energy of the complex-Cholesky form, one CTA per walker:
//   e1b = sum_s Ghalf_s . rH1_s + ecore,  ecoul = 1/2 sum_x X1[x] X2[x],  e2b = ecoul - exx.
__global__ void __launch_bounds__(256) energy_complex_kernel(const double2* __restrict__ ga,
                                                              const double2* __restrict__ gb, int NMa, int NMb,
                                                              const double2* __restrict__ rh1a,
                                                              const double2* __restrict__ rh1b, double ecore,
                                                              const double2* __restrict__ x1,
                                                              const double2* __restrict__ x2, int X,
                                                              const double2* __restrict__ exx,
                                                              double2* __restrict__ energy) {
  __shared__ double2 red[2][8];
  const int w = blockIdx.x, tid = threadIdx.x;
  double2 e1 = make_double2(0.0, 0.0), ec = make_double2(0.0, 0.0);
  for (int k = tid; k < NMa; k += 256) e1 = cadd(e1, cmul(ga[(size_t)w * NMa + k], rh1a[k]));
  for (int k = tid; k < NMb; k += 256) e1 = cadd(e1, cmul(gb[(size_t)w * NMb + k], rh1b[k]));
  for (int x = tid; x < X; x += 256) ec = cadd(ec, cmul(x1[(size_t)w * X + x], x2[(size_t)w * X + x]));
  e1 = warp_sum2(e1);
  ec = warp_sum2(ec);
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = e1;
    red[1][tid >> 5] = ec;
  }
  __syncthreads();
  if (tid == 0) {
    double2 a = make_double2(ecore, 0.0), c = make_double2(0.0, 0.0);
    for (int k = 0; k < 8; ++k) {
      a = cadd(a, red[0][k]);
      c = cadd(c, red[1][k]);
    }
    const double2 e2 = csub(cscale(c, 0.5), exx[w]);
    energy[(size_t)w * 3 + 0] = cadd(a, e2);
    energy[(size_t)w * 3 + 1] = a;
    energy[(size_t)w * 3 + 2] = e2;
  }
}

// out[w] (accumulate: +=) coef * sum_t part[t][w]
__global__ void scaled_row_sum_kernel(const double2* __restrict__ part, int rows, int W, double2 coef,
                                      double2* __restrict__ out, int accumulate) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int t = 0; t < rows; ++t) acc = cadd(acc, part[(size_t)t * W + w]);
  const double2 r = cmul(coef, acc);
  out[w] = accumulate ? cadd(out[w], r) : r;
}

cudaError_t launch_scaled_row_sum(const double2* part, int rows, int W, double2 coef, double2* out, int accumulate,
                                  cudaStream_t st) {
  scaled_row_sum_kernel<<<(W + 127) / 128, 128, 0, st>>>(part, rows, W, coef, out, accumulate);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_energy_complex(const double2* ga, const double2* gb, int W, int NMa, int NMb, const double2* rh1a,
                                  const double2* rh1b, double ecore, const double2* x1, const double2* x2, int X,
                                  const double2* exx, double2* energy, cudaStream_t st) {
  energy_complex_kernel<<<W, 256, 0, st>>>(ga, gb, NMa, NMb, rh1a, rh1b, ecore, x1, x2, X, exx, energy);
  note_launch();
  return cudaGetLastError();
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
