// Green's function and overlap for spin blocks of N <= 32 electrons, one
// 128-thread CTA per walker (42 KB of shared memory, four walkers per SM: two Ghalf columns per
// lane and pass keep a thread within 128 registers; measured 12% faster than three):
//
//   O = phi^T psi*  (N x N): phi and psi* stream through shared memory in
//       8-row chunks, a three-deep ring of cp.async copies issued two chunks
//       ahead (one barrier per chunk); each thread accumulates a 2 x 4 block of
//       O in registers;
//   X = (P O)^-1 by Gauss-Jordan elimination in place in shared memory with
//       partial pivoting on |.| (warp 0 picks the pivot, all threads update) --
//       the pivots are those of the LU factorisation, so
//       log|det O| = sum log|pivot_k|, phase = (-1)^swaps prod pivot_k / |pivot_k|
//       (one pivot per lane of warp 0, reduced with shuffles);
//   Ghalf[i, m] = sum_r X[i, r] phi[m, perm(r)] (= (O^-1 phi^T)[i, m]): a
//       register-tiled product -- warp w takes rows 8w..8w+7, lane l the
//       columns l + 32q (q < 2, so 64 columns per pass), phi staged in shared
//       memory 4 permuted columns at a time, transposed, through a four-deep
//       cp.async ring issued three steps ahead -- instead of one latency-bound
//       pair of triangular solves per column.
// ovlp_w = prod_s phase_s * exp(sum_s log|det O_s| - log_shift_w).
// Same contract as gf_overlap_kernel (walkers.cu), which keeps N > 32.
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

namespace {

constexpr int kThreads = 128;
constexpr int kChunk = 8;   // rows of phi / psi* per shared-memory chunk of the O product
constexpr int kORing = 3;   // chunks in the O product's copy ring
constexpr int kNP = 33;     // row stride of O in shared memory
constexpr int kRC = 4;      // permuted columns of phi per staged step of the Ghalf product
constexpr int kMQ = 2;      // columns of Ghalf per lane and pass (64 per pass)
constexpr int kMS = 32 * kMQ + 1;  // row stride of the staged phi^T step (odd in 16-byte units)
constexpr int kGRing = 4;   // steps in the Ghalf product's copy ring
constexpr int kOStage = 2 * kChunk * 32;  // double2 per O chunk (phi and psi*)
constexpr int kGStage = kRC * kMS;        // double2 per Ghalf step
constexpr int kStage = kORing * kOStage > kGRing * kGStage ? kORing * kOStage : kGRing * kGStage;
static_assert(kChunk * 32 % kThreads == 0 && kRC * 32 * kMQ % kThreads == 0, "whole copies per thread");

struct SpinDet32 {
  double logabs;
  double2 phase;
};

// sO = phi^T psi* (or, GRAM, the Gram matrix phi^H phi: psic unused) of one spin block.  phi and
// psi* stream through shared memory in 8-row chunks, a three-deep ring of cp.async copies issued
// two chunks ahead (one barrier per chunk); thread (ti, tj) accumulates rows {ti, ti+16} x
// columns {tj + 8q} in registers.  The caller synchronises before reading sO.
template <bool GRAM>
__device__ void o_product(const double2* __restrict__ phi, const double2* __restrict__ psic, int M, int N,
                          double2 (*sO)[kNP], double2* sStage) {
  const int tid = threadIdx.x;
  const int ti = tid >> 3, tj = tid & 7;
  double2 acc[2][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[a][q] = make_double2(0.0, 0.0);
  const int nch = (M + kChunk - 1) / kChunk;
  // chunk ch (rows 8 ch ..) into ring slot ch % kORing: phi rows then psi* rows, zeros past M / N
  auto issue = [&](int ch) {
    if (ch < nch) {
      double2* st = sStage + (ch % kORing) * kOStage;
#pragma unroll
      for (int u = 0; u < kChunk * 32 / kThreads; ++u) {
        const int e = tid + u * kThreads, r = e >> 5, c = e & 31, m = ch * kChunk + r;
        const bool in = m < M && c < N;
        const size_t off = in ? (size_t)m * N + c : 0;
        cp_async16(st + e, phi + off, in ? 16 : 0);
        if (!GRAM) cp_async16(st + kChunk * 32 + e, psic + off, in ? 16 : 0);
      }
    }
    cp_async_commit();  // (an empty group past the end keeps the group count per chunk)
  };
  issue(0);
  issue(1);
  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait<1>();  // this thread's copies of chunk ch have landed
    __syncthreads();     // everyone's have, and everyone is done with chunk ch - 1
    issue(ch + 2);       // into the slot of chunk ch - 1
    const double2(*sPhi)[32] = reinterpret_cast<const double2(*)[32]>(sStage + (ch % kORing) * kOStage);
    const double2(*sPsi)[32] =
        GRAM ? sPhi : reinterpret_cast<const double2(*)[32]>(sStage + (ch % kORing) * kOStage + kChunk * 32);
#pragma unroll
    for (int r = 0; r < kChunk; ++r) {
      double2 a0 = sPhi[r][ti], a1 = sPhi[r][ti + 16];
      if (GRAM) {
        a0.y = -a0.y;
        a1.y = -a1.y;
      }
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
  cp_async_wait<0>();
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) sO[ti + 16 * a][tj + 8 * q] = acc[a][q];
}

// O = phi^T psi* for one spin block into sO; then its inverse (of the row-permuted O) in place,
// the row order in sPerm and log|det|, phase from the pivots.
__device__ SpinDet32 invert_block(const double2* __restrict__ phi, const double2* __restrict__ psic, int M, int N,
                                  double2 (*sO)[kNP], double2* sStage, int* sPerm, double2* sPiv, double2* red,
                                  unsigned* status) {
  const int tid = threadIdx.x;
  o_product<false>(phi, psic, M, N, sO, sStage);
  if (tid < 32) sPerm[tid] = tid;
  __syncthreads();
  // ---- Gauss-Jordan with partial pivoting, in place: after step k row k holds the k-th row of
  // the reduced inverse and column k the multipliers.  Two barriers per step: warp 0 picks the
  // pivot (one redux.sync on a 32-bit key: the float bits of |a|^2 above the row index, so a
  // pivot within ~2e-6 of the largest, the lowest row on ties), swaps it into row k and scales
  // that row by 1/p (1/p = conj(p) / |p|^2, one reciprocal); then all threads update the rest with
  // the scaled row (thread: column tid % 32, rows tid / 32 + 4r), the owners of column k-1 first
  // applying that column's -1/p_{k-1} to their rows (deferred from step k-1: it commutes with the
  // row swap and the row scaling; warp 0 applies it to row k's entry with the row scaling), which
  // keeps a load-multiply-store off warp 0's serial chain.
  int swaps = 0;
  const int uj = tid & 31, ui = tid >> 5;
  double2 pinv_prev = make_double2(0.0, 0.0);
  for (int k = 0; k < N; ++k) {
    if (tid < 32) {
      unsigned key = 0u;
      if (tid >= k && tid < N)
        key = (__float_as_uint((float)cabs2(sO[tid][k])) & ~31u) | (unsigned)(31 - tid);
      const int bi = 31 - (int)(__reduce_max_sync(0xffffffffu, key) & 31u);
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
      if (bi != k) ++swaps;  // warp-uniform: every lane of warp 0 counts
      __syncwarp();
      // row k x 1/p, a_kk = 1/p
      const double2 pv = sO[k][k];
      const double rn = __drcp_rn(pv.x * pv.x + pv.y * pv.y);
      const double2 pinv = make_double2(pv.x * rn, -pv.y * rn);
      if (tid < N && tid != k) {
        double2 v = cmul(sO[k][tid], pinv);
        // row k's entry of column k-1 also takes that column's deferred -1/p_{k-1}
        if (tid == k - 1) v = cmul(v, make_double2(-pinv_prev.x, -pinv_prev.y));
        sO[k][tid] = v;
      }
      if (tid == 0) {
        if (pv.x == 0.0 && pv.y == 0.0) flag(status, STATUS_SINGULAR);
        sPiv[k] = pv;
        sO[k][k] = pinv;
        red[5] = pinv;
      }
    }
    __syncthreads();
    // a_ij -= a_ik (a_kj / a_kk) for i, j != k (the scaled row k; column k is only read here).
    // All of a thread's loads first: interleaved, each row's store could alias (for the compiler)
    // the next row's loads, which made the eight rows a serial chain.
    const double2 pk = red[5];
    if (uj < N && uj != k) {
      const double2 akj = sO[k][uj];
      double2 a[8], f[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = ui + 4 * r;
        a[r] = sO[i][uj];
        f[r] = sO[i][k];
      }
      if (uj == k - 1) {
        // column k-1 x -1/p_{k-1} for rows other than k-1 (row k's entry: warp 0 above)
        const double2 m = make_double2(-pinv_prev.x, -pinv_prev.y);
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (ui + 4 * r != k - 1) a[r] = cmul(a[r], m);
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = ui + 4 * r;
        if (i < N && i != k) sO[i][uj] = csub(a[r], cmul(f[r], akj));
      }
    }
    pinv_prev = pk;
    __syncthreads();
  }
  // column N-1 x -1/p_{N-1} (rows other than N-1)
  if (N > 0 && uj == N - 1) {
    const double2 m = make_double2(-pinv_prev.x, -pinv_prev.y);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = ui + 4 * r;
      if (i < N && i != N - 1) sO[i][uj] = cmul(sO[i][uj], m);
    }
  }
  __syncthreads();
  // ---- log|det| and phase from the pivots, one per lane of warp 0
  if (tid < 32) {
    double la = 0.0;
    double2 ph = make_double2(1.0, 0.0);
    if (tid < N) {
      const double2 u = sPiv[tid];
      const double a = cabs_(u);
      la = log(a);
      ph = make_double2(u.x / a, u.y / a);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      la += __shfl_xor_sync(0xffffffffu, la, o);
      const double2 q = make_double2(__shfl_xor_sync(0xffffffffu, ph.x, o), __shfl_xor_sync(0xffffffffu, ph.y, o));
      ph = cmul(ph, q);
    }
    if (tid == 0) {
      red[0] = make_double2(la, 0.0);
      red[1] = (swaps & 1) ? make_double2(-ph.x, -ph.y) : ph;
    }
  }
  __syncthreads();
  SpinDet32 out;
  out.logabs = red[0].x;
  out.phase = red[1];
  return out;
}

// Ghalf (N, M) of one spin block from X = (P O)^-1 in sO: Ghalf[i, m] = sum_r X[i, r] phi[m, perm(r)].
// The steps (pass of 64 columns m, group of kRC permuted columns) run in one sequence through
// the copy ring, passes included.
__device__ void ghalf_block(const double2* __restrict__ phi, int M, int N, double2 (*sO)[kNP], const int* sPerm,
                            double2* sStage, double2* __restrict__ ghalf, double2* __restrict__ ghalf2) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i0 = warp * 8;  // this warp's rows
  // the next step to copy: columns from im0, permuted columns from ir0 (im0 >= M: none left)
  int im0 = 0, ir0 = 0, slot = 0;
  // phi[im0 + ml][perm(ir0 + rr)] as sPT[rr][ml] (consecutive threads take consecutive rr)
  auto issue = [&]() {
    if (im0 < M) {
      double2* sPT = sStage + slot * kGStage;
#pragma unroll
      for (int u = 0; u < kRC * 32 * kMQ / kThreads; ++u) {
        const int e = tid + u * kThreads, rr = e % kRC, ml = e / kRC;
        const int r = ir0 + rr, m = im0 + ml;
        const bool in = r < N && m < M;
        cp_async16(sPT + rr * kMS + ml, phi + (in ? (size_t)m * N + sPerm[r] : 0), in ? 16 : 0);
      }
      ir0 += kRC;
      if (ir0 >= N) {
        ir0 = 0;
        im0 += 32 * kMQ;
      }
    }
    cp_async_commit();
    slot = slot == kGRing - 1 ? 0 : slot + 1;
  };
  issue();
  issue();
  issue();
  int cur = 0;  // ring slot of the step being multiplied
  for (int m0 = 0; m0 < M; m0 += 32 * kMQ) {
    double2 acc[8][kMQ];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int q = 0; q < kMQ; ++q) acc[a][q] = make_double2(0.0, 0.0);
    for (int r0 = 0; r0 < N; r0 += kRC) {
      cp_async_wait<2>();
      __syncthreads();
      issue();  // into the slot of the previous step
      const double2* sPT = sStage + cur * kGStage;
      cur = cur == kGRing - 1 ? 0 : cur + 1;
#pragma unroll
      for (int rr = 0; rr < kRC; ++rr) {
        double2 x[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) x[a] = sO[i0 + a][min(r0 + rr, 31)];
        if (r0 + rr >= N) continue;  // uniform
#pragma unroll
        for (int q = 0; q < kMQ; ++q) {
          if (q > 0 && m0 + 32 * q >= M) break;  // a column group wholly past M (uniform): the last pass
          const double2 b = sPT[rr * kMS + lane + 32 * q];
#pragma unroll
          for (int a = 0; a < 8; ++a) {
            acc[a][q].x += x[a].x * b.x - x[a].y * b.y;
            acc[a][q].y += x[a].x * b.y + x[a].y * b.x;
          }
        }
      }
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int i = i0 + a;
      if (i >= N) break;
#pragma unroll
      for (int q = 0; q < kMQ; ++q) {
        const int m = m0 + lane + 32 * q;
        if (m < M) {
          ghalf[(size_t)i * M + m] = acc[a][q];
          if (ghalf2 != nullptr) ghalf2[(size_t)i * M + m] = acc[a][q];
        }
      }
    }
  }
  cp_async_wait<0>();
}

template <bool WITH_GHALF>
__global__ void __launch_bounds__(kThreads, 4) gf_lu32_kernel(const double2* __restrict__ phia,
                                                              const double2* __restrict__ phib, int M, int na,
                                                              int nb, const double2* __restrict__ psia_c,
                                                              const double2* __restrict__ psib_c,
                                                              const double* __restrict__ log_shift,
                                                              double2* __restrict__ ghalfa,
                                                              double2* __restrict__ ghalfb,
                                                              double2* __restrict__ ovlp, double2* __restrict__ logdet,
                                                              unsigned* status) {
  __shared__ double2 sO[32][kNP];
  __shared__ __align__(16) double2 sStage[kStage];  // the O product's chunk ring, then the Ghalf step ring
  __shared__ double2 sPiv[32];
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
    const SpinDet32 d = invert_block(phi, s == 0 ? psia_c : psib_c, M, N, sO, sStage, sPerm, sPiv, red, status);
    logsum += d.logabs;
    phase = cmul(phase, d.phase);
    if (threadIdx.x == 0) {
      red[2] = make_double2(d.logabs, 0.0);
      red[3] = d.phase;
      if (logdet != nullptr) logdet[(size_t)w * 2 + s] = make_double2(d.logabs, atan2(d.phase.y, d.phase.x));
    }
    if (WITH_GHALF) {
      double2* g1 = (s == 0 ? ghalfa : ghalfb) + (size_t)w * N * M;
      double2* g2 = (s == 0 && alias && nb > 0 && ghalfb != ghalfa) ? ghalfb + (size_t)w * N * M : nullptr;
      ghalf_block(phi, M, N, sO, sPerm, sStage, g1, g2);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double2 o = cscale(phase, exp(logsum - log_shift[w]));
    if (!finite2(o)) flag(status, STATUS_NONFINITE);
    ovlp[w] = o;
  }
}

// ---------------------------------------------------------------------------------------------
// Reorthogonalisation of spin blocks of N <= 32 orbitals by Cholesky QR, the same unique thin QR
// (positive real diag R) as Gram-Schmidt or a sign-fixed Householder factorisation:
//   S = phi^H phi (o_product<true>), S = R^H R (Cholesky, right-looking, in shared memory; warp 0
//   scales the pivot row, all threads update the trailing upper triangle), X = R^-1 (warp 0,
//   lane i solving row i of X R = I, kept in the lower triangle of sO transposed plus the
//   diagonal), phi <- phi X in place (16-row chunks of phi through the copy ring; lane i forms
//   column i of four rows per warp, so each output row is one coalesced 512-byte store).
// log det R = sum log R_kk.  Its error is that of the Gram matrix, ~cond(phi)^2 eps: walkers are
// reorthogonalised every few steps, so phi stays close to orthonormal and cond(phi) near 1.
__device__ __noinline__ double cholqr_block(double2* __restrict__ phi, int M, int N, double2 (*sO)[kNP], double2* sStage,
                               double2* sDinv, double* sSpread, unsigned* status) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  o_product<true>(phi, nullptr, M, N, sO, sStage);
  __syncthreads();
  // ---- S = R^H R in the upper triangle of sO
  const int uj = tid & 31, ui = tid >> 5;
  for (int k = 0; k < N; ++k) {
    if (tid < 32) {
      const double skk = sO[k][k].x;
      __syncwarp();  // every lane has read the pivot before lane 0 replaces it
      if (!(skk > 0.0)) flag(status, STATUS_ZERO_NORM);
      const double d = sqrt(skk), dinv = 1.0 / d;
      if (lane > k && lane < N) sO[k][lane] = cscale(sO[k][lane], dinv);
      if (lane == 0) {
        sO[k][k] = make_double2(d, 0.0);
        sDinv[k] = make_double2(dinv, 0.0);
      }
    }
    __syncthreads();
    // S_ij -= conj(R_ki) R_kj for k < i <= j (loads first, as in the Gauss-Jordan update)
    if (uj > k && uj < N) {
      const double2 rkj = sO[k][uj];
      double2 a[8], f[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = ui + 4 * r;
        a[r] = sO[i][uj];
        f[r] = sO[k][i];
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = ui + 4 * r;
        if (i > k && i <= uj) sO[i][uj] = csub(a[r], cmulc(f[r], rkj));
      }
    }
    __syncthreads();
  }
  double logsum = 0.0;
  if (tid < 32) {
    // ---- X = R^-1 (upper): lane i, row i: X_ii = 1 / R_ii, X_ij = -(sum_{i<=k<j} X_ik R_kj) / R_jj
    double2 x[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < j; ++k) {
        const double2 rkj = sO[k][j];  // the same for every lane: a broadcast
        acc.x += x[k].x * rkj.x - x[k].y * rkj.y;
        acc.y += x[k].x * rkj.y + x[k].y * rkj.x;
      }
      const double di = j < N ? sDinv[j].x : 0.0;
      x[j] = lane == j ? make_double2(di, 0.0) : (lane < j ? make_double2(-acc.x * di, -acc.y * di)
                                                           : make_double2(0.0, 0.0));
    }
    // X_ij (i < j) to sO[j][i], below the diagonal: R is no longer read after the barrier
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (lane < j && j < N) sO[j][lane] = x[j];
    double rmax = 0.0, rmin = 1.0e300;
    if (lane < N) {
      const double r = sO[lane][lane].x;
      logsum = log(r);
      rmax = rmin = r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      logsum += __shfl_xor_sync(0xffffffffu, logsum, o);
      rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
      rmin = fmin(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
    }
    if (lane == 0) *sSpread = rmax / rmin;  // a lower bound on cond(phi); NaN when a pivot failed
  }
  __syncthreads();
  // ---- phi <- phi X: lane i = column i, rows m0 + 4 warp + a
  const int nch = (M + 15) / 16;
  auto issue = [&](int ch) {
    if (ch < nch) {
      double2* st = sStage + (ch % kORing) * kOStage;
#pragma unroll
      for (int u = 0; u < 16 * 32 / kThreads; ++u) {
        const int e = tid + u * kThreads, r = e >> 5, c = e & 31, m = ch * 16 + r;
        const bool in = m < M && c < N;
        cp_async16(st + e, phi + (in ? (size_t)m * N + c : 0), in ? 16 : 0);
      }
    }
    cp_async_commit();
  };
  issue(0);
  issue(1);
  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait<1>();
    __syncthreads();
    issue(ch + 2);  // rows ahead of the ones rewritten below
    const double2(*sPhi)[32] = reinterpret_cast<const double2(*)[32]>(sStage + (ch % kORing) * kOStage);
    double2 acc[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) acc[a] = make_double2(0.0, 0.0);
#pragma unroll 8
    for (int r = 0; r < 32; ++r) {
      // X[r][lane]: below the diagonal of sO transposed, the diagonal in sDinv, zero for r > lane
      const double2 xr = r < lane ? sO[lane][r] : (r == lane && r < N ? sDinv[r] : make_double2(0.0, 0.0));
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const double2 p = sPhi[4 * warp + a][r];
        acc[a].x += p.x * xr.x - p.y * xr.y;
        acc[a].y += p.x * xr.y + p.y * xr.x;
      }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int m = ch * 16 + 4 * warp + a;
      if (m < M && lane < N) phi[(size_t)m * N + lane] = acc[a];
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  return logsum;  // valid in warp 0
}

constexpr double kCholQR2 = 20.0;  // R-diagonal spread above which a block gets a second pass

// One CTA per walker: both spin blocks (the alpha block once when phib aliases it), then
// detR = exp(sum log R_kk - detR_shift), log_detR += log detR, ovlp /= detR (the contract of
// reortho_kernel in walkers.cu, which keeps N > 32).
__global__ void __launch_bounds__(kThreads, 4) reortho_chol32_kernel(double2* __restrict__ phia,
                                                                     double2* __restrict__ phib, int M, int na,
                                                                     int nb, const double* __restrict__ detR_shift,
                                                                     double* __restrict__ detR,
                                                                     double* __restrict__ log_detR,
                                                                     double2* __restrict__ ovlp, unsigned* status) {
  __shared__ double2 sO[32][kNP];
  __shared__ __align__(16) double2 sStage[kStage];
  __shared__ double2 sDinv[32];
  __shared__ double sSpread;
  const int w = blockIdx.x;
  const bool alias = (phib == phia) && (nb == na);
  double logsum = 0.0, log_a = 0.0;
  for (int s = 0; s < 2; ++s) {
    const int N = s == 0 ? na : nb;
    if (N == 0) continue;
    if (s == 1 && alias) {
      logsum += log_a;
      continue;
    }
    double2* phi = (s == 0 ? phia : phib) + (size_t)w * M * N;
    double l = cholqr_block(phi, M, N, sO, sStage, sDinv, &sSpread, status);
    // CholQR2: a second pass over the (now nearly orthonormal) result when R's diagonal spreads
    // by more than kCholQR2 (the first pass's error grows like cond(phi)^2 eps); R = R2 R1, so
    // the log-determinants add
    if (!(sSpread <= kCholQR2)) l += cholqr_block(phi, M, N, sO, sStage, sDinv, &sSpread, status);
    logsum += l;
    if (s == 0) log_a = l;
  }
  if (threadIdx.x == 0) {
    const double d = exp(logsum - detR_shift[w]);
    detR[w] = d;
    log_detR[w] += log(d);
    ovlp[w] = cscale(ovlp[w], 1.0 / d);
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

cudaError_t launch_reortho_chol32(double2* phia, double2* phib, int W, int M, int na, int nb,
                                  const double* detR_shift, double* detR, double* log_detR, double2* ovlp,
                                  unsigned* status, cudaStream_t st) {
  if (na < 1 || na > 32 || nb < 0 || nb > 32 || M <= 0 || W <= 0) return cudaErrorInvalidValue;
  reortho_chol32_kernel<<<W, kThreads, 0, st>>>(phia, phib, M, na, nb, detR_shift, detR, log_detR, ovlp, status);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200
