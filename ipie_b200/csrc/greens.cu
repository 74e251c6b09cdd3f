// Green's function and overlap for spin blocks of N <= 32 electrons, one
// 128-thread CTA per walker with a small shared-memory footprint (~34 KB) so
// that several walkers share an SM:
//
//   O = phi^T psi*  (N x N): phi and psi* stream through shared memory in
//       16-row chunks; each thread accumulates a 2 x 4 block of O in registers;
//   P O = L U: partial pivoting on |.| in shared memory (warp 0 picks the
//       pivot, all threads update);  log|det O| = sum log|U_kk|,
//       phase = (-1)^swaps prod U_kk / |U_kk|;
//   Ghalf[:, m] = O^{-1} phi[m, :]^T: thread m loads its row of phi in pivot
//       order straight into registers and runs both triangular solves there
//       (L and U are read as shared-memory broadcasts), then stores column m.
// ovlp_w = prod_s phase_s * exp(sum_s log|det O_s| - log_shift_w).
// Same contract as gf_overlap_kernel (walkers.cu), which keeps N > 32.
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

namespace {

constexpr int kThreads = 128;
constexpr int kChunk = 16;  // rows of phi / psi* per shared-memory chunk
constexpr int kNP = 33;     // row stride of O in shared memory

struct SpinLU32 {
  double logabs;
  double2 phase;
};

// Factor one spin block; leaves L\U (unit L) in sO, the row order in sPerm, 1/U_kk in sInv.
__device__ SpinLU32 factor_block(const double2* __restrict__ phi, const double2* __restrict__ psic, int M, int N,
                                 double2 (*sO)[kNP], double2 (*sPhi)[32], double2 (*sPsi)[32], int* sPerm,
                                 double2* sInv, double2* red, unsigned* status) {
  const int tid = threadIdx.x;
  // ---- O = phi^T psi*: thread (ti, tj) owns rows {ti, ti+16} x columns {tj + 8q}
  const int ti = tid >> 3, tj = tid & 7;
  double2 acc[2][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[a][q] = make_double2(0.0, 0.0);
  for (int m0 = 0; m0 < M; m0 += kChunk) {
    const int mc = min(kChunk, M - m0);
    __syncthreads();
    for (int e = tid; e < kChunk * 32; e += kThreads) {
      const int r = e >> 5, c = e & 31;
      const bool in = r < mc && c < N;
      sPhi[r][c] = in ? phi[(size_t)(m0 + r) * N + c] : make_double2(0.0, 0.0);
      sPsi[r][c] = in ? psic[(size_t)(m0 + r) * N + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < kChunk; ++r) {
      const double2 a0 = sPhi[r][ti], a1 = sPhi[r][ti + 16];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 b = sPsi[r][tj + 8 * q];
        acc[0][q].x += a0.x * b.x - a0.y * b.y;
        acc[0][q].y += a0.x * b.y + a0.y * b.x;
        acc[1][q].x += a1.x * b.x - a1.y * b.y;
        acc[1][q].y += a1.x * b.y + a1.y * b.x;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) sO[ti + 16 * a][tj + 8 * q] = acc[a][q];
  if (tid < 32) sPerm[tid] = tid;
  __syncthreads();
  // ---- LU with partial pivoting
  int swaps = 0;
  for (int k = 0; k < N; ++k) {
    if (tid < 32) {
      double best = -1.0;
      int bi = k;
      if (tid >= k && tid < N) {
        best = cabs2(sO[tid][k]);
        bi = tid;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      // swap rows k and bi (all N columns) and the row order
      if (bi != k && tid < N) {
        const double2 t = sO[k][tid];
        sO[k][tid] = sO[bi][tid];
        sO[bi][tid] = t;
      }
      if (bi != k && tid == 0) {
        const int t = sPerm[k];
        sPerm[k] = sPerm[bi];
        sPerm[bi] = t;
      }
      if (tid == 0) red[4] = make_double2((double)bi, 0.0);
      __syncwarp();
      if (tid == 0) {
        const double2 pv = sO[k][k];
        if (pv.x == 0.0 && pv.y == 0.0) flag(status, STATUS_SINGULAR);
        sInv[k] = cdiv(make_double2(1.0, 0.0), pv);
      }
    }
    __syncthreads();
    if ((int)red[4].x != k) ++swaps;
    const double2 ip = sInv[k];
    const int rem = N - k - 1;
    // column k of L, then the trailing update (each thread recomputes its multiplier)
    for (int e = tid; e < rem * rem; e += kThreads) {
      const int r = k + 1 + e / rem, c = k + 1 + e % rem;
      const double2 l = cmul(sO[r][k], ip);
      sO[r][c] = csub(sO[r][c], cmul(l, sO[k][c]));
    }
    __syncthreads();
    for (int r = k + 1 + tid; r < N; r += kThreads) sO[r][k] = cmul(sO[r][k], ip);
    __syncthreads();
  }
  SpinLU32 out;
  if (tid == 0) {
    double la = 0.0;
    double2 ph = make_double2((swaps & 1) ? -1.0 : 1.0, 0.0);
    for (int k = 0; k < N; ++k) {
      const double2 u = sO[k][k];
      const double a = cabs_(u);
      la += log(a);
      ph = cmul(ph, make_double2(u.x / a, u.y / a));
    }
    red[0] = make_double2(la, 0.0);
    red[1] = ph;
  }
  __syncthreads();
  out.logabs = red[0].x;
  out.phase = red[1];
  return out;
}

// Ghalf (N, M) of one spin block from the factors in shared memory.
__device__ void solve_block(const double2* __restrict__ phi, int M, int N, double2 (*sO)[kNP], const int* sPerm,
                            const double2* sInv, double2* __restrict__ ghalf, double2* __restrict__ ghalf2) {
  for (int m = threadIdx.x; m < M; m += kThreads) {
    double2 y[32];
    const double2* row = phi + (size_t)m * N;
#pragma unroll
    for (int i = 0; i < 32; ++i) y[i] = i < N ? row[sPerm[i]] : make_double2(0.0, 0.0);
    // L y = P b (unit lower); square loops with compile-time bounds keep y in registers
#pragma unroll
    for (int i = 1; i < 32; ++i) {
      if (i < N) {
        double2 s = y[i];
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (j < i) s = csub(s, cmul(sO[i][j], y[j]));
        y[i] = s;
      }
    }
    // U x = y
#pragma unroll
    for (int ii = 0; ii < 32; ++ii) {
      const int i = 31 - ii;
      if (i < N) {
        double2 s = y[i];
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (j > i && j < N) s = csub(s, cmul(sO[i][j], y[j]));
        y[i] = cmul(s, sInv[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (i < N) {
        ghalf[(size_t)i * M + m] = y[i];
        if (ghalf2 != nullptr) ghalf2[(size_t)i * M + m] = y[i];
      }
  }
}

template <bool WITH_GHALF>
__global__ void __launch_bounds__(kThreads) gf_lu32_kernel(const double2* __restrict__ phia,
                                                           const double2* __restrict__ phib, int M, int na, int nb,
                                                           const double2* __restrict__ psia_c,
                                                           const double2* __restrict__ psib_c,
                                                           const double* __restrict__ log_shift,
                                                           double2* __restrict__ ghalfa, double2* __restrict__ ghalfb,
                                                           double2* __restrict__ ovlp, double2* __restrict__ logdet,
                                                           unsigned* status) {
  __shared__ double2 sO[32][kNP];
  __shared__ double2 sPhi[kChunk][32];
  __shared__ double2 sPsi[kChunk][32];
  __shared__ double2 sInv[32];
  __shared__ double2 red[8];
  __shared__ int sPerm[32];
  const int w = blockIdx.x;
  // spin aliasing: phib == phia with nb == na is one block counted twice
  const bool alias = (phib == phia) && (nb == na);
  double logsum = 0.0;
  double2 phase = make_double2(1.0, 0.0);
  for (int s = 0; s < 2; ++s) {
    const int N = s == 0 ? na : nb;
    if (N == 0) continue;
    if (s == 1 && alias) {
      logsum += red[2].x;
      phase = cmul(phase, red[3]);
      if (logdet != nullptr && threadIdx.x == 0) logdet[(size_t)w * 2 + 1] = logdet[(size_t)w * 2];
      continue;
    }
    const double2* phi = (s == 0 ? phia : phib) + (size_t)w * M * N;
    const SpinLU32 lu = factor_block(phi, s == 0 ? psia_c : psib_c, M, N, sO, sPhi, sPsi, sPerm, sInv, red, status);
    logsum += lu.logabs;
    phase = cmul(phase, lu.phase);
    if (threadIdx.x == 0) {
      red[2] = make_double2(lu.logabs, 0.0);
      red[3] = lu.phase;
      if (logdet != nullptr) logdet[(size_t)w * 2 + s] = make_double2(lu.logabs, atan2(lu.phase.y, lu.phase.x));
    }
    if (WITH_GHALF) {
      double2* g1 = (s == 0 ? ghalfa : ghalfb) + (size_t)w * N * M;
      double2* g2 = (s == 0 && alias && nb > 0 && ghalfb != ghalfa) ? ghalfb + (size_t)w * N * M : nullptr;
      solve_block(phi, M, N, sO, sPerm, sInv, g1, g2);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double2 o = cscale(phase, exp(logsum - log_shift[w]));
    if (!finite2(o)) flag(status, STATUS_NONFINITE);
    ovlp[w] = o;
  }
}

}  // namespace

bool gf_lu32_fits(int na, int nb) { return na >= 1 && na <= 32 && nb >= 0 && nb <= 32; }

cudaError_t launch_gf_lu32(const double2* phia, const double2* phib, int W, int M, int na, int nb,
                           const double2* psia_c, const double2* psib_c, const double* log_shift, double2* ghalfa,
                           double2* ghalfb, double2* ovlp, double2* logdet, unsigned* status, cudaStream_t st) {
  if (!gf_lu32_fits(na, nb) || M <= 0 || W <= 0) return cudaErrorInvalidValue;
  if (ghalfa != nullptr)
    gf_lu32_kernel<true><<<W, kThreads, 0, st>>>(phia, phib, M, na, nb, psia_c, psib_c, log_shift, ghalfa, ghalfb,
                                                 ovlp, logdet, status);
  else
    gf_lu32_kernel<false><<<W, kThreads, 0, st>>>(phia, phib, M, na, nb, psia_c, psib_c, log_shift, nullptr,
                                                  nullptr, ovlp, logdet, status);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200
