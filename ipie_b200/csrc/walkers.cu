// Per-walker kernels of the FP64 walker step: Green's function / overlap
// (batched LU), weight update, field shift, reorthogonalisation (modified
// Gram-Schmidt), population-control copies and small energy reductions.
//
// One CTA owns one walker (both spin blocks) for the kernels that need the
// walker's whole Slater matrix; its M x N orbitals live in shared memory.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

// Shared-memory row stride (in double2) for an M x N walker block: N + 1 keeps
// the column walks of the LU solve and Gram-Schmidt bank-conflict free.
__host__ __device__ inline int pad_n(int n) { return n + 1; }

size_t gf_smem_bytes(int M, int N) {
  const int NP = pad_n(N);
  // walker block + overlap matrix + trial chunk (32 rows) + pivots/inverse diagonal
  return sizeof(double2) * ((size_t)M * NP + (size_t)N * NP + 32 * (size_t)N + N) + sizeof(int) * N + 64 * sizeof(double2);
}

// ---------------------------------------------------------------------------
// Green's function + overlap.
//   O = phi^T psi*  (N x N);  P O = L U  (partial pivoting on |.|);
//   log|det O| = sum log|U_kk|,  phase = (-1)^swaps prod U_kk/|U_kk|;
//   Ghalf = O^{-1} phi^T  (N x M), solved column by column from the LU.
// ovlp_w = prod_s phase_s * exp(sum_s log|det O_s| - log_shift_w)
// ---------------------------------------------------------------------------
struct SpinLU {
  double logabs;
  double2 phase;
};

// Factor the overlap of one spin block already loaded in sY (M x N, stride NP).
__device__ SpinLU overlap_lu(const double2* __restrict__ psic, int M, int N, double2* sY, double2* sO,
                             double2* sPsi, int* sPiv, double2* sInvDiag, double2* red, unsigned* status) {
  const int NP = pad_n(N);
  const int tid = threadIdx.x, nth = blockDim.x;
  // O[i][j] = sum_m phi[m][i] psic[m][j], psic streamed through smem in 32-row chunks.
  for (int e = tid; e < N * N; e += nth) sO[(e / N) * NP + e % N] = make_double2(0.0, 0.0);
  // each thread owns a fixed set of (i, j) entries across chunks
  for (int m0 = 0; m0 < M; m0 += 32) {
    const int mc = min(32, M - m0);
    __syncthreads();
    for (int e = tid; e < mc * N; e += nth) sPsi[e] = psic[(size_t)(m0 + e / N) * N + e % N];
    __syncthreads();
    for (int e = tid; e < N * N; e += nth) {
      const int i = e / N, j = e % N;
      double2 s = sO[i * NP + j];
      for (int mm = 0; mm < mc; ++mm) {
        double2 a = sY[(m0 + mm) * NP + i], b = sPsi[mm * N + j];
        s.x += a.x * b.x - a.y * b.y;
        s.y += a.x * b.y + a.y * b.x;
      }
      sO[i * NP + j] = s;
    }
  }
  __syncthreads();
  // LU with partial pivoting.  Warp 0 finds the pivot; all threads update.
  int swaps = 0;
  for (int k = 0; k < N; ++k) {
    if (tid < 32) {
      double best = -1.0;
      int bi = k;
      for (int r = k + tid; r < N; r += 32) {
        double a = cabs2(sO[r * NP + k]);
        if (a > best) { best = a; bi = r; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (tid == 0) sPiv[k] = bi;
    }
    __syncthreads();
    const int piv = sPiv[k];
    if (piv != k) {
      for (int c = tid; c < N; c += nth) {
        double2 tmp = sO[k * NP + c];
        sO[k * NP + c] = sO[piv * NP + c];
        sO[piv * NP + c] = tmp;
      }
      swaps++;
    }
    __syncthreads();
    const double2 pv = sO[k * NP + k];
    if (tid == 0) {
      if (pv.x == 0.0 && pv.y == 0.0) flag(status, STATUS_SINGULAR);
      sInvDiag[k] = cdiv(make_double2(1.0, 0.0), pv);
    }
    __syncthreads();
    const double2 ip = sInvDiag[k];
    for (int r = k + 1 + tid; r < N; r += nth) sO[r * NP + k] = cmul(sO[r * NP + k], ip);
    __syncthreads();
    const int rem = N - k - 1;
    for (int e = tid; e < rem * rem; e += nth) {
      const int r = k + 1 + e / rem, c = k + 1 + e % rem;
      sO[r * NP + c] = csub(sO[r * NP + c], cmul(sO[r * NP + k], sO[k * NP + c]));
    }
    __syncthreads();
  }
  SpinLU out;
  if (tid == 0) {
    double la = 0.0;
    double2 ph = make_double2((swaps & 1) ? -1.0 : 1.0, 0.0);
    for (int k = 0; k < N; ++k) {
      double2 u = sO[k * NP + k];
      double a = cabs_(u);
      la += log(a);
      ph = cmul(ph, make_double2(u.x / a, u.y / a));
    }
    red[0] = make_double2(la, 0.0);
    red[1] = ph;
  }
  __syncthreads();
  out.logabs = red[0].x;
  out.phase = red[1];
  __syncthreads();
  return out;
}

// Ghalf = O^{-1} phi^T from the LU in sO; thread m solves for column m.
// ghalf2 (may be null) receives a second copy (spin-aliased walkers).
__device__ void solve_ghalf(int M, int N, double2* sY, const double2* sO, const int* sPiv, const double2* sInvDiag,
                            double2* __restrict__ ghalf, double2* __restrict__ ghalf2) {
  const int NP = pad_n(N);
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    double2* y = sY + m * NP;
    for (int k = 0; k < N; ++k) {
      int p = sPiv[k];
      if (p != k) {
        double2 t = y[k];
        y[k] = y[p];
        y[p] = t;
      }
    }
    for (int i = 1; i < N; ++i) {
      double2 s = y[i];
      for (int j = 0; j < i; ++j) s = csub(s, cmul(sO[i * NP + j], y[j]));
      y[i] = s;
    }
    for (int i = N - 1; i >= 0; --i) {
      double2 s = y[i];
      for (int j = i + 1; j < N; ++j) s = csub(s, cmul(sO[i * NP + j], y[j]));
      y[i] = cmul(s, sInvDiag[i]);
    }
    for (int i = 0; i < N; ++i) ghalf[(size_t)i * M + m] = y[i];
    if (ghalf2 != nullptr)
      for (int i = 0; i < N; ++i) ghalf2[(size_t)i * M + m] = y[i];
  }
}

template <bool WITH_GHALF>
__global__ void __launch_bounds__(256) gf_overlap_kernel(const double2* __restrict__ phia, const double2* __restrict__ phib,
                                                         int M, int na, int nb, const double2* __restrict__ psia_c,
                                                         const double2* __restrict__ psib_c,
                                                         const double* __restrict__ log_shift, double2* __restrict__ ghalfa,
                                                         double2* __restrict__ ghalfb, double2* __restrict__ ovlp,
                                                         double2* __restrict__ logdet, unsigned* status) {
  extern __shared__ double2 sm[];
  const int w = blockIdx.x;
  const int Nmax = max(na, nb), NP = pad_n(Nmax);
  double2* sY = sm;
  double2* sO = sY + (size_t)M * NP;
  double2* sPsi = sO + (size_t)Nmax * NP;
  double2* sInvDiag = sPsi + 32 * Nmax;
  double2* red = sInvDiag + Nmax;
  int* sPiv = reinterpret_cast<int*>(red + 64);
  // Spin aliasing: phib == phia (with nb == na) means the beta block is an exact
  // copy of the alpha block; it is factored once and counted twice.
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
    const int np = pad_n(N);
    __syncthreads();
    for (int e = threadIdx.x; e < M * N; e += blockDim.x) sY[(e / N) * np + e % N] = phi[e];
    __syncthreads();
    SpinLU lu = overlap_lu(s == 0 ? psia_c : psib_c, M, N, sY, sO, sPsi, sPiv, sInvDiag, red, status);
    logsum += lu.logabs;
    phase = cmul(phase, lu.phase);
    if (threadIdx.x == 0) {
      red[2] = make_double2(lu.logabs, 0.0);
      red[3] = lu.phase;
    }
    if (logdet != nullptr && threadIdx.x == 0) logdet[(size_t)w * 2 + s] = make_double2(lu.logabs, atan2(lu.phase.y, lu.phase.x));
    if (WITH_GHALF) {
      double2* g1 = (s == 0 ? ghalfa : ghalfb) + (size_t)w * N * M;
      double2* g2 = (s == 0 && alias && nb > 0 && ghalfb != ghalfa) ? ghalfb + (size_t)w * N * M : nullptr;
      solve_ghalf(M, N, sY, sO, sPiv, sInvDiag, g1, g2);
    }
  }
  if (threadIdx.x == 0) {
    double2 o = cscale(phase, exp(logsum - log_shift[w]));
    if (!finite2(o)) flag(status, STATUS_NONFINITE);
    ovlp[w] = o;
  }
}

cudaError_t launch_gf_overlap(const double2* phia, const double2* phib, int W, int M, int na, int nb,
                              const double2* psia_c, const double2* psib_c, const double* log_shift, double2* ghalfa,
                              double2* ghalfb, double2* ovlp, double2* logdet, unsigned* status, cudaStream_t st) {
  const int Nmax = max(na, nb);
  if (Nmax <= 0 || M <= 0 || W <= 0) return cudaErrorInvalidValue;
  // N <= 32: small-footprint kernel (greens.cu), several walkers per SM; larger blocks below
  if (gf_lu32_fits(na, nb))
    return launch_gf_lu32(phia, phib, W, M, na, nb, psia_c, psib_c, log_shift, ghalfa, ghalfb, ovlp, logdet, status,
                          st);
  size_t smem = gf_smem_bytes(M, Nmax);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  if (ghalfa != nullptr) {
    auto k = gf_overlap_kernel<true>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<W, 256, smem, st>>>(phia, phib, M, na, nb, psia_c, psib_c, log_shift, ghalfa, ghalfb, ovlp, logdet, status);
  note_launch();
  } else {
    auto k = gf_overlap_kernel<false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<W, 256, smem, st>>>(phia, phib, M, na, nb, psia_c, psib_c, log_shift, nullptr, nullptr, ovlp, logdet, status);
  note_launch();
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Field shift: from the force bias to the shifted fields of the VHS.
//   xbar = -sqrt(dt) (i vbias - mf);  |xbar| > bound -> xbar/|xbar|
//   xs = xi - xbar;  cmf = -sqrt(dt) sum_x xs mf;  cfb = sum_x xi xbar - xbar^2/2
// One CTA per 32 walkers; the (X, W) transposed store goes through smem.
// ---------------------------------------------------------------------------
// FP16 head and remainder of the scaled x, both rounded to nearest (the 3-pass operand split)
__device__ __forceinline__ void split_store_f16(__half* hi, __half* lo, size_t i, double x) {
  const double y = x * kFieldScaleF16;
  const __half h = __double2half(y);
  hi[i] = h;
  lo[i] = __double2half(y - (double)__half2float(h));
}

// xs_hi/xs_lo (optional): the shifted fields x kFieldScaleF16 as planar (W, 2, ldx) FP16
// head/remainder, the right operand of the mixed-precision VHS product.
__global__ void __launch_bounds__(256) field_shift_kernel(const double2* __restrict__ vbias, const double* __restrict__ xi,
                                                          const double2* __restrict__ mf, int W, int X, double sqrt_dt,
                                                          double bound, double2* __restrict__ xshifted,
                                                          double2* __restrict__ cmf, double2* __restrict__ cfb,
                                                          __half* __restrict__ xs_hi, __half* __restrict__ xs_lo) {
  __shared__ double2 tile[32][33];
  const int ldx = f16_ld(X);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w0 = blockIdx.x * 32;
  double2 acc_mf[4], acc_fb[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) acc_mf[q] = acc_fb[q] = make_double2(0.0, 0.0);
  for (int x0 = 0; x0 < X; x0 += 32) {
    const int x = x0 + lane;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int wl = warp * 4 + q, w = w0 + wl;
      double2 xs = make_double2(0.0, 0.0);
      if (w < W && x < X) {
        const double2 v = vbias[(size_t)w * X + x];
        const double2 m = mf[x];
        double2 xb = make_double2(-sqrt_dt * (-v.y - m.x), -sqrt_dt * (v.x - m.y));
        const double a = cabs_(xb);
        if (a > bound && a > 1e-13) xb = make_double2(xb.x / a, xb.y / a);
        const double r = xi[(size_t)w * X + x];
        xs = make_double2(r - xb.x, -xb.y);
        if (xs_hi != nullptr) {
          split_store_f16(xs_hi, xs_lo, ((size_t)w * 2) * ldx + x, xs.x);
          split_store_f16(xs_hi, xs_lo, ((size_t)w * 2 + 1) * ldx + x, xs.y);
        }
        acc_mf[q] = cadd(acc_mf[q], cmul(xs, m));
        double2 xb2 = cmul(xb, xb);
        acc_fb[q] = cadd(acc_fb[q], make_double2(r * xb.x - 0.5 * xb2.x, r * xb.y - 0.5 * xb2.y));
      }
      tile[lane][wl] = xs;
    }
    __syncthreads();
    // transposed store: row x, 32 consecutive walkers
    if (xshifted != nullptr)
      for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int xl = e / 32, wl = e % 32;
        if (x0 + xl < X && w0 + wl < W) xshifted[(size_t)(x0 + xl) * W + w0 + wl] = tile[xl][wl];
      }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double2 a = warp_sum2(acc_mf[q]), b = warp_sum2(acc_fb[q]);
    const int w = w0 + warp * 4 + q;
    if (lane == 0 && w < W) {
      cmf[w] = cscale(a, -sqrt_dt);
      cfb[w] = b;
    }
  }
}

// The same shift without the (X, W) transposed copy: four warps per walker (two walkers per
// block) walk its row of vbias / xi with coalesced loads, write the binary16 split and reduce cmf,
// cfb with shuffles and shared memory (the mixed form, which needs no FP64 transposed fields; one
// warp per walker left ~14 warps per SM, too few to cover the loads' latency).
constexpr int kShiftWarps = 4;  // warps per walker
__global__ void __launch_bounds__(256) field_shift_rows_kernel(const double2* __restrict__ vbias,
                                                               const double* __restrict__ xi,
                                                               const double2* __restrict__ mf, int W, int X,
                                                               double sqrt_dt, double bound, double2* __restrict__ cmf,
                                                               double2* __restrict__ cfb, __half* __restrict__ xs_hi,
                                                               __half* __restrict__ xs_lo) {
  __shared__ double2 part[8][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, sub = warp % kShiftWarps;
  const int w = blockIdx.x * (8 / kShiftWarps) + warp / kShiftWarps;
  const bool live = w < W;
  const int ldx = f16_ld(X);
  double2 acc_mf = make_double2(0.0, 0.0), acc_fb = make_double2(0.0, 0.0);
  for (int x = sub * 32 + lane; live && x < X; x += 32 * kShiftWarps) {
    const double2 v = vbias[(size_t)w * X + x];
    const double2 m = mf[x];
    double2 xb = make_double2(-sqrt_dt * (-v.y - m.x), -sqrt_dt * (v.x - m.y));
    const double a = cabs_(xb);
    if (a > bound && a > 1e-13) xb = make_double2(xb.x / a, xb.y / a);
    const double r = xi[(size_t)w * X + x];
    const double2 xs = make_double2(r - xb.x, -xb.y);
    if (xs_hi != nullptr) {
      split_store_f16(xs_hi, xs_lo, ((size_t)w * 2) * ldx + x, xs.x);
      split_store_f16(xs_hi, xs_lo, ((size_t)w * 2 + 1) * ldx + x, xs.y);
    }
    acc_mf = cadd(acc_mf, cmul(xs, m));
    const double2 xb2 = cmul(xb, xb);
    acc_fb = cadd(acc_fb, make_double2(r * xb.x - 0.5 * xb2.x, r * xb.y - 0.5 * xb2.y));
  }
  acc_mf = warp_sum2(acc_mf);
  acc_fb = warp_sum2(acc_fb);
  if (lane == 0) {
    part[warp][0] = acc_mf;
    part[warp][1] = acc_fb;
  }
  __syncthreads();
  if (live && sub == 0 && lane == 0) {
    for (int k = 1; k < kShiftWarps; ++k) {
      acc_mf = cadd(acc_mf, part[warp + k][0]);
      acc_fb = cadd(acc_fb, part[warp + k][1]);
    }
    cmf[w] = cscale(acc_mf, -sqrt_dt);
    cfb[w] = acc_fb;
  }
}

cudaError_t launch_field_shift(const double2* vbias, const double* xi, const double2* mf, int W, int X, double sqrt_dt,
                               double bound, double2* xshifted, double2* cmf, double2* cfb, cudaStream_t st,
                               void* xs_hi, void* xs_lo) {
  if (xshifted == nullptr)
    field_shift_rows_kernel<<<(W + 1) / 2, 256, 0, st>>>(vbias, xi, mf, W, X, sqrt_dt, bound, cmf, cfb,
                                                         static_cast<__half*>(xs_hi), static_cast<__half*>(xs_lo));
  else
    field_shift_kernel<<<(W + 31) / 32, 256, 0, st>>>(vbias, xi, mf, W, X, sqrt_dt, bound, xshifted, cmf, cfb,
                                                      static_cast<__half*>(xs_hi), static_cast<__half*>(xs_lo));
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Weight update (hybrid energy, importance function, cosine projection) and
// the driver's weight clip.  Scalars that change between steps (eshift,
// weight bound) are read from device memory so a captured step stays valid.
// ---------------------------------------------------------------------------
__global__ void update_weight_kernel(int W, const double2* __restrict__ ovlp_new, const double2* __restrict__ cfb,
                                     const double2* __restrict__ cmf, const double* __restrict__ eshift_p, double dt,
                                     double ebound, const double* __restrict__ wbound_p, double2* __restrict__ ovlp,
                                     double2* __restrict__ ehyb_prev, double* __restrict__ weight, unsigned* status) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const double eshift = *eshift_p;
  const double2 r = cdiv(ovlp_new[w], ovlp[w]);
  const double2 lr = make_double2(log(hypot(r.x, r.y)), atan2(r.y, r.x));
  const double2 f = cfb[w], c = cmf[w];
  double2 eh = make_double2(-(lr.x + f.x + c.x) / dt, -(lr.y + f.y + c.y) / dt);
  if (fabs(eshift) >= 1e-10) eh.x = fmin(fmax(eh.x, eshift - ebound), eshift + ebound);
  const double2 ep = ehyb_prev[w];
  const double2 arg = make_double2(-dt * (0.5 * (eh.x + ep.x) - eshift), -dt * (0.5 * (eh.y + ep.y)));
  const double magn = exp(arg.x);
  const double dtheta = -dt * eh.y - f.y;
  const double cosf = fmax(cos(dtheta), 0.0);
  double wn = weight[w] * magn * cosf;
  if (wbound_p != nullptr) {
    const double wb = *wbound_p;
    if (wb >= 0.0) wn = fmin(fmax(wn, -wb), wb);
  }
  if (!isfinite(wn)) flag(status, STATUS_NONFINITE);
  weight[w] = wn;
  ehyb_prev[w] = eh;
  ovlp[w] = ovlp_new[w];
}

cudaError_t launch_update_weight(int W, const double2* ovlp_new, const double2* cfb, const double2* cmf,
                                 const double* eshift, double dt, double ebound, const double* wbound, double2* ovlp,
                                 double2* ehyb, double* weight, unsigned* status, cudaStream_t st) {
  update_weight_kernel<<<(W + 127) / 128, 128, 0, st>>>(W, ovlp_new, cfb, cmf, eshift, dt, ebound, wbound, ovlp, ehyb,
                                                        weight, status);
  note_launch();
  return cudaGetLastError();
}

__global__ void clip_weight_kernel(int W, const double* __restrict__ wbound_p, double* __restrict__ weight) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const double wb = *wbound_p;
  weight[w] = fmin(fmax(weight[w], -wb), wb);
}

cudaError_t launch_clip_weight(int W, const double* wbound, double* weight, cudaStream_t st) {
  clip_weight_kernel<<<(W + 127) / 128, 128, 0, st>>>(W, wbound, weight);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Reorthogonalisation: modified Gram-Schmidt per spin block (unique thin QR
// with positive real diag(R), the sign-fixed Householder result), then
// detR = exp(sum log R_ii - detR_shift), log_detR += log detR, ovlp /= detR.
// ---------------------------------------------------------------------------
__device__ double mgs_block(double2* sY, int M, int N, double2* red, unsigned* status) {
  const int NP = pad_n(N);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double logsum = 0.0;
  for (int j = 0; j < N; ++j) {
    double s = 0.0;
    for (int m = threadIdx.x; m < M; m += blockDim.x) s += cabs2(sY[m * NP + j]);
    double2 t = block_sum2(make_double2(s, 0.0), red);
    const double nrm = sqrt(t.x);
    if (nrm == 0.0) flag(status, STATUS_ZERO_NORM);
    logsum += log(nrm);
    const double inv = 1.0 / nrm;
    for (int m = threadIdx.x; m < M; m += blockDim.x) sY[m * NP + j] = cscale(sY[m * NP + j], inv);
    __syncthreads();
    for (int k = j + 1 + warp; k < N; k += nw) {
      double2 d = make_double2(0.0, 0.0);
      for (int m = lane; m < M; m += 32) d = cadd(d, cmulc(sY[m * NP + j], sY[m * NP + k]));
      d = warp_sum2(d);
      for (int m = lane; m < M; m += 32) sY[m * NP + k] = csub(sY[m * NP + k], cmul(d, sY[m * NP + j]));
    }
    __syncthreads();
  }
  return logsum;
}

__global__ void __launch_bounds__(256) reortho_kernel(double2* __restrict__ phia, double2* __restrict__ phib, int M, int na,
                                                      int nb, const double* __restrict__ detR_shift,
                                                      double* __restrict__ detR, double* __restrict__ log_detR,
                                                      double2* __restrict__ ovlp, unsigned* status) {
  extern __shared__ double2 sm[];
  const int w = blockIdx.x;
  double2* red = sm;
  double2* sY = sm + 64;
  const bool alias = (phib == phia) && (nb == na);  // beta block is the alpha block: orthogonalise once
  double logsum = 0.0, log_a = 0.0;
  for (int s = 0; s < 2; ++s) {
    const int N = s == 0 ? na : nb;
    if (N == 0) continue;
    if (s == 1 && alias) {
      logsum += log_a;
      continue;
    }
    double2* phi = (s == 0 ? phia : phib) + (size_t)w * M * N;
    const int np = pad_n(N);
    __syncthreads();
    for (int e = threadIdx.x; e < M * N; e += blockDim.x) sY[(e / N) * np + e % N] = phi[e];
    __syncthreads();
    const double l = mgs_block(sY, M, N, red, status);
    logsum += l;
    if (s == 0) log_a = l;
    for (int e = threadIdx.x; e < M * N; e += blockDim.x) phi[e] = sY[(e / N) * np + e % N];
  }
  if (threadIdx.x == 0) {
    const double d = exp(logsum - detR_shift[w]);
    detR[w] = d;
    log_detR[w] += log(d);
    ovlp[w] = cscale(ovlp[w], 1.0 / d);
  }
}

cudaError_t launch_reortho(double2* phia, double2* phib, int W, int M, int na, int nb, const double* detR_shift,
                           double* detR, double* log_detR, double2* ovlp, unsigned* status, cudaStream_t st) {
  // blocks of at most 32 orbitals: Cholesky QR (greens.cu); larger ones by Gram-Schmidt below
  if (na >= 1 && na <= 32 && nb >= 0 && nb <= 32)
    return launch_reortho_chol32(phia, phib, W, M, na, nb, detR_shift, detR, log_detR, ovlp, status, st);
  const int Nmax = max(na, nb);
  size_t smem = sizeof(double2) * ((size_t)M * pad_n(Nmax) + 64);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaFuncSetAttribute(reortho_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  reortho_kernel<<<W, 256, smem, st>>>(phia, phib, M, na, nb, detR_shift, detR, log_detR, ovlp, status);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Population-control copies: walker dst receives walker src[dst] (src < 0: keep).
// The per-walker scalars travel with the orbitals, as in ipie's walker buffer.
// ---------------------------------------------------------------------------
__global__ void walker_copy_kernel(const int* __restrict__ src, int W, int M, int na, int nb, double2* phia,
                                   double2* phib, double* weight, double* unscaled_weight, double2* ehyb,
                                   double2* ovlp, double2* phase, double2* ghalfa, double2* ghalfb) {
  const int dst = blockIdx.x;
  const int s = src[dst];
  if (s < 0 || s == dst) return;
  const size_t sa = (size_t)M * na, sb = (size_t)M * nb;
  for (size_t e = threadIdx.x; e < sa; e += blockDim.x) phia[dst * sa + e] = phia[s * sa + e];
  if (phib != phia)
    for (size_t e = threadIdx.x; e < sb; e += blockDim.x) phib[dst * sb + e] = phib[s * sb + e];
  // Green's functions travel with the orbitals (they are functions of them)
  if (ghalfa != nullptr)
    for (size_t e = threadIdx.x; e < sa; e += blockDim.x) ghalfa[dst * sa + e] = ghalfa[s * sa + e];
  if (ghalfb != nullptr && ghalfb != ghalfa)
    for (size_t e = threadIdx.x; e < sb; e += blockDim.x) ghalfb[dst * sb + e] = ghalfb[s * sb + e];
  if (threadIdx.x == 0) {
    weight[dst] = weight[s];
    unscaled_weight[dst] = unscaled_weight[s];
    ehyb[dst] = ehyb[s];
    ovlp[dst] = ovlp[s];
    if (phase) phase[dst] = phase[s];
  }
}

cudaError_t launch_walker_copy(const int* src, int W, int M, int na, int nb, double2* phia, double2* phib,
                               double* weight, double* unscaled_weight, double2* ehyb, double2* ovlp, double2* phase,
                               double2* ghalfa, double2* ghalfb, cudaStream_t st) {
  walker_copy_kernel<<<W, 256, 0, st>>>(src, W, M, na, nb, phia, phib, weight, unscaled_weight, ehyb, ovlp, phase,
                                        ghalfa, ghalfb);
  note_launch();
  return cudaGetLastError();
}

// Out-of-place resampling (stochastic reconfiguration): walker d of the output
// arrays is walker src[d] of the input arrays, for every d; the weight is set by
// the caller.  Sources may repeat, so the copy cannot run in place.

__global__ void walker_gather_kernel(const int* __restrict__ src, int M, int na, int nb, WalkerArrays in,
                                     WalkerArrays out) {
  const int d = blockIdx.x;
  const int s = src[d];
  const size_t sa = (size_t)M * na, sb = (size_t)M * nb;
  for (size_t e = threadIdx.x; e < sa; e += blockDim.x) out.phia[d * sa + e] = in.phia[s * sa + e];
  if (in.phib != in.phia)
    for (size_t e = threadIdx.x; e < sb; e += blockDim.x) out.phib[d * sb + e] = in.phib[s * sb + e];
  if (in.ghalfa != nullptr)
    for (size_t e = threadIdx.x; e < sa; e += blockDim.x) out.ghalfa[d * sa + e] = in.ghalfa[s * sa + e];
  if (in.ghalfb != nullptr && in.ghalfb != in.ghalfa)
    for (size_t e = threadIdx.x; e < sb; e += blockDim.x) out.ghalfb[d * sb + e] = in.ghalfb[s * sb + e];
  if (threadIdx.x == 0) {
    out.ehyb[d] = in.ehyb[s];
    out.ovlp[d] = in.ovlp[s];
    if (in.phase) out.phase[d] = in.phase[s];
    out.unscaled_weight[d] = in.unscaled_weight[s];
  }
}

cudaError_t launch_walker_gather(const int* src, int W, int M, int na, int nb, const WalkerArrays& in,
                                 const WalkerArrays& out, cudaStream_t st) {
  walker_gather_kernel<<<W, 256, 0, st>>>(src, M, na, nb, in, out);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Energy pieces that are per-walker reductions.
//   e1b_w = sum_k Ghalfa[w,k] rH1a[k] + sum_k Ghalfb[w,k] rH1b[k] + ecore
//   ecoul_w = 1/2 sum_x X[w,x]^2  (X = rchol_a.Ghalfa + rchol_b.Ghalfb, no conjugate)
//   exx_w = sum over x-tiles of the fused exchange partials
// energy[w] = (e1b + ecoul - exx, e1b, ecoul - exx) with the RHF/UHF factors applied.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) energy_combine_kernel(int W, int X, int Ka, int Kb, const double2* __restrict__ ga,
                                                             const double2* __restrict__ gb, const double2* __restrict__ rh1a,
                                                             const double2* __restrict__ rh1b, double ecore,
                                                             const double2* __restrict__ xv, const double2* __restrict__ exx_part,
                                                             int ntiles, double f1, double fc, double fx,
                                                             double2* __restrict__ energy, unsigned* status) {
  __shared__ double2 red[32];
  const int w = blockIdx.x;
  double2 e1 = make_double2(0.0, 0.0), ec = make_double2(0.0, 0.0), ex = make_double2(0.0, 0.0);
  for (int k = threadIdx.x; k < Ka; k += blockDim.x) e1 = cadd(e1, cmul(ga[(size_t)w * Ka + k], rh1a[k]));
  if (gb != nullptr)
    for (int k = threadIdx.x; k < Kb; k += blockDim.x) e1 = cadd(e1, cmul(gb[(size_t)w * Kb + k], rh1b[k]));
  for (int x = threadIdx.x; x < X; x += blockDim.x) {
    double2 v = xv[(size_t)w * X + x];
    ec = cadd(ec, cmul(v, v));
  }
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) ex = cadd(ex, exx_part[(size_t)t * W + w]);
  e1 = block_sum2(e1, red);
  ec = block_sum2(ec, red);
  ex = block_sum2(ex, red);
  if (threadIdx.x == 0) {
    double2 e1b = make_double2(f1 * e1.x + ecore, f1 * e1.y);
    double2 e2b = make_double2(fc * ec.x - fx * ex.x, fc * ec.y - fx * ex.y);
    double2 tot = cadd(e1b, e2b);
    if (!finite2(tot)) flag(status, STATUS_NONFINITE);
    energy[(size_t)w * 3 + 0] = tot;
    energy[(size_t)w * 3 + 1] = e1b;
    energy[(size_t)w * 3 + 2] = e2b;
  }
}

cudaError_t launch_energy_combine(int W, int X, int Ka, int Kb, const double2* ga, const double2* gb,
                                  const double2* rh1a, const double2* rh1b, double ecore, const double2* xv,
                                  const double2* exx_part, int ntiles, double f1, double fc, double fx, double2* energy,
                                  unsigned* status, cudaStream_t st) {
  energy_combine_kernel<<<W, 256, 0, st>>>(W, X, Ka, Kb, ga, gb, rh1a, rh1b, ecore, xv, exx_part, ntiles, f1, fc, fx,
                                           energy, status);
  note_launch();
  return cudaGetLastError();
}

// GHF determinants (W, 2M, N), N = na + nb: the spin-diagonal blocks that the one-body
// factors and exp(VHS) act on -- rows 0..M-1 x columns 0..na-1 and rows M..2M-1 x columns
// na..N-1 -- copied to (W, M, na) and (W, M, nb) arrays (scatter = 0) or back (scatter = 1;
// the off-diagonal blocks of phi are not touched).  One thread per element.
__global__ void ghf_blocks_kernel(double2* __restrict__ phi, int W, int M, int na, int nb, double2* __restrict__ pa,
                                  double2* __restrict__ pb, int scatter) {
  const int N = na + nb;
  const long long na_el = (long long)M * na, nb_el = (long long)M * nb;
  const long long per = na_el + nb_el;
  const long long n = (long long)W * per;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long w = e / per;
    long long r = e - w * per;
    size_t pi, qi;
    double2* q;
    if (r < na_el) {
      const long long m = r / na, i = r - m * na;
      pi = ((size_t)w * 2 * M + m) * N + i;
      qi = ((size_t)w * M + m) * na + i;
      q = pa;
    } else {
      r -= na_el;
      const long long m = r / nb, j = r - m * nb;
      pi = ((size_t)w * 2 * M + M + m) * N + na + j;
      qi = ((size_t)w * M + m) * nb + j;
      q = pb;
    }
    if (scatter)
      phi[pi] = q[qi];
    else
      q[qi] = phi[pi];
  }
}

cudaError_t launch_ghf_blocks(double2* phi, int W, int M, int na, int nb, double2* pa, double2* pb, int scatter,
                              cudaStream_t st) {
  if (W <= 0 || M <= 0 || na < 0 || nb < 0 || na + nb == 0 || (na > 0 && pa == nullptr) || (nb > 0 && pb == nullptr))
    return cudaErrorInvalidValue;
  long long blocks = ((long long)W * M * (na + nb) + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  ghf_blocks_kernel<<<(unsigned)blocks, 256, 0, st>>>(phi, W, M, na, nb, pa, pb, scatter);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200
