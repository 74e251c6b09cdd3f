// Hand-written adjoint of the local energy with respect to the one-body
// Hamiltonian: e1b_w = sum_s tr(G_s^w h1_s) with the mixed Green's function
// G_s^w = psi_s^* Ghalf_s^w (M x M), so for upstream gradients g_w
//     dL/dh1_s = sum_w g_w G_s^w = psi_s^* (sum_w g_w Ghalf_s^w).
// With g_w = w_w / sum w this is the mixed-estimator one-body density matrix.
#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

// acc[k] = sum_w coeff[w] * ghalf[w][k]   (k over N*M), fixed summation order.
__global__ void weighted_walker_sum_kernel(const double2* __restrict__ ghalf, const double* __restrict__ coeff, int W,
                                           int K, double2* __restrict__ acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double2 s = make_double2(0.0, 0.0);
  for (int w = 0; w < W; ++w) {
    const double2 g = ghalf[(size_t)w * K + k];
    const double c = coeff[w];
    s.x += c * g.x;
    s.y += c * g.y;
  }
  acc[k] = s;
}

// out[p][q] (+)= sum_i psi_c[p][i] * A[i][q]   (psi_c (M, N), A (N, M), out (M, M))
__global__ void expand_half_kernel(const double2* __restrict__ psi_c, const double2* __restrict__ A, int M, int N,
                                   double2* __restrict__ out, int accumulate) {
  const int p = blockIdx.y, q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= M) return;
  double2 s = make_double2(0.0, 0.0);
  for (int i = 0; i < N; ++i) s = cadd(s, cmul(psi_c[(size_t)p * N + i], A[(size_t)i * M + q]));
  const size_t o = (size_t)p * M + q;
  out[o] = accumulate ? cadd(out[o], s) : s;
}

// rH1[i][q] = sum_p psi_c[p][i] * h1[p][q]   (psi_c (M, N), h1 (M, M) real, rH1 (N, M) complex)
__global__ void rotate_onebody_kernel(const double2* __restrict__ psi_c, const double* __restrict__ h1, int M, int N,
                                      double2* __restrict__ rh1) {
  const int i = blockIdx.y, q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= M) return;
  double2 s = make_double2(0.0, 0.0);
  for (int p = 0; p < M; ++p) {
    const double2 c = psi_c[(size_t)p * N + i];
    const double h = h1[(size_t)p * M + q];
    s.x += c.x * h;
    s.y += c.y * h;
  }
  rh1[(size_t)i * M + q] = s;
}


// Vector-Jacobian product of the single-determinant local energy with respect to one spin's
// half-rotated Green's function G (N, M):
//     E = f1 sum G . rH1 + fc (sum_x X_x^2) - fx sum_x tr(T_x T_x) + (other spin, ecore),
//     X_x = sum_s L_s,x . G_s,   T_x = L_x G^T (N, N),   L_x (N, M) row x of rchol,
//     dE/dG = f1 rH1 + 2 fc sum_x X_x L_x - 2 fx sum_x T_x L_x,
// gbar = ebar[w] * dE/dG.  One CTA per walker runs the sum over x: L_x and G in shared memory,
// T_x in shared memory, the accumulator (N M complex) in registers, 16 entries per thread at most.
constexpr int kVjpThreads = 512;
constexpr int kVjpPer = 16;  // N * M <= 8192
__global__ void __launch_bounds__(kVjpThreads, 1)
    energy_vjp_kernel(const double* __restrict__ rchol, const double2* __restrict__ ghalf,
                      const double2* __restrict__ rh1, const double2* __restrict__ xv, const double2* __restrict__ ebar,
                      int X, int M, int N, double f1, double fc2, double fx2, double2* __restrict__ gbar) {
  extern __shared__ double vjp_smem[];
  const int NM = N * M, w = blockIdx.x;
  double2* g = reinterpret_cast<double2*>(vjp_smem);  // (N, M)
  double* l = vjp_smem + 2 * NM;                      // (N, M)
  double2* t = reinterpret_cast<double2*>(l + NM);    // (N, N)
  const double2* gw = ghalf + (size_t)w * NM;
  for (int e = threadIdx.x; e < NM; e += kVjpThreads) g[e] = gw[e];
  double2 acc[kVjpPer];
#pragma unroll
  for (int r = 0; r < kVjpPer; ++r) acc[r] = make_double2(0.0, 0.0);
  for (int x = 0; x < X; ++x) {
    __syncthreads();  // the previous L_x and T_x are consumed
    const double* lx = rchol + (size_t)x * NM;
    for (int e = threadIdx.x; e < NM; e += kVjpThreads) l[e] = lx[e];
    __syncthreads();
    for (int q = threadIdx.x; q < N * N; q += kVjpThreads) {
      const int j = q / N, i = q - j * N;
      double2 s = make_double2(0.0, 0.0);
      for (int p = 0; p < M; ++p) {
        const double a = l[j * M + p];
        const double2 b = g[i * M + p];
        s.x += a * b.x;
        s.y += a * b.y;
      }
      t[q] = s;
    }
    __syncthreads();
    const double2 c = xv[(size_t)w * X + x];
#pragma unroll
    for (int r = 0; r < kVjpPer; ++r) {
      const int e = threadIdx.x + r * kVjpThreads;
      if (e < NM) {
        const int j = e / M, p = e - j * M;
        double2 s = make_double2(0.0, 0.0);
        for (int i = 0; i < N; ++i) {
          const double2 tj = t[j * N + i];
          const double li = l[i * M + p];
          s.x += tj.x * li;
          s.y += tj.y * li;
        }
        const double lv = l[e];
        acc[r].x += fc2 * c.x * lv - fx2 * s.x;
        acc[r].y += fc2 * c.y * lv - fx2 * s.y;
      }
    }
  }
  const double2 eb = ebar[w];
#pragma unroll
  for (int r = 0; r < kVjpPer; ++r) {
    const int e = threadIdx.x + r * kVjpThreads;
    if (e < NM) {
      const double2 h = rh1[e];
      const double2 d = make_double2(f1 * h.x + acc[r].x, f1 * h.y + acc[r].y);
      gbar[(size_t)w * NM + e] = cmul(eb, d);
    }
  }
}

cudaError_t launch_energy_vjp(const double* rchol, const double2* ghalf, const double2* rh1, const double2* xv,
                              const double2* ebar, int W, int X, int M, int N, double f1, double fc, double fx,
                              double2* gbar, cudaStream_t st) {
  const int NM = N * M;
  if (NM > kVjpPer * kVjpThreads || W <= 0 || X <= 0) return cudaErrorInvalidValue;
  const size_t smem = (size_t)NM * 24 + (size_t)N * N * 16;
  if (smem > 232448) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(energy_vjp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  energy_vjp_kernel<<<W, kVjpThreads, smem, st>>>(rchol, ghalf, rh1, xv, ebar, X, M, N, f1, 2.0 * fc, 2.0 * fx,
                                                  gbar);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" int ipie_b200_onebody_adjoint(int W, int M, int na, int nb, const void* ghalfa, const void* ghalfb,
                                         const void* psia_conj, const void* psib_conj, const double* coeff, void* work,
                                         void* rdm, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  double2* acc = reinterpret_cast<double2*>(work);
  double2* out = reinterpret_cast<double2*>(rdm);
  const void* g[2] = {ghalfa, ghalfb};
  const void* p[2] = {psia_conj, psib_conj};
  const int n[2] = {na, nb};
  for (int s = 0; s < 2; ++s) {
    double2* o = out + (size_t)s * M * M;
    if (n[s] == 0) {
      cudaMemsetAsync(o, 0, sizeof(double2) * M * M, st);
      continue;
    }
    const int K = n[s] * M;
    weighted_walker_sum_kernel<<<(K + 255) / 256, 256, 0, st>>>(reinterpret_cast<const double2*>(g[s]), coeff, W, K,
                                                                 acc);
    note_launch();
    expand_half_kernel<<<dim3((M + 127) / 128, M), 128, 0, st>>>(reinterpret_cast<const double2*>(p[s]), acc, M, n[s],
                                                                  o, 0);
    note_launch();
  }
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_rotate_onebody(const void* psi_conj, const double* h1, int M, int N, void* rh1, void* stream) {
  if (N == 0) return 0;
  rotate_onebody_kernel<<<dim3((M + 127) / 128, N), 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(psi_conj), h1, M, N, reinterpret_cast<double2*>(rh1));
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_local_energy_vjp(int rhf, const double* rchola, const double* rcholb, const void* rH1a,
                                          const void* rH1b, const void* ghalfa, const void* ghalfb, int W, int X,
                                          int M, int na, int nb, const void* ebar, void* work, void* gbara,
                                          void* gbarb, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (W <= 0 || X <= 0 || M <= 0 || na <= 0 || (!rhf && nb < 0)) return (int)cudaErrorInvalidValue;
  double2* xv = reinterpret_cast<double2*>(work);
  const double2* ga = reinterpret_cast<const double2*>(ghalfa);
  const double2* gb = reinterpret_cast<const double2*>(ghalfb);
  const double2* eb = reinterpret_cast<const double2*>(ebar);
  // the factors of ipie_b200_local_energy_single_det_batch: UHF f1 = 1, fc = 1/2, fx = 1/2;
  // RHF (alpha only, doubled) f1 = 2, fc = 2, fx = 1
  const double f1 = rhf ? 2.0 : 1.0, fc = rhf ? 2.0 : 0.5, fx = rhf ? 1.0 : 0.5;
  const bool alias = !rhf && nb == na && rcholb == rchola && ghalfb == ghalfa;
  const bool use_b = !rhf && nb > 0;
  // X_x = sum over the spins in the energy of L_s,x . G_s
  cudaError_t e = launch_force_bias(rchola, ga, W, X, na * M, xv, 0, st, alias ? 2.0 : 1.0);
  if (e == cudaSuccess && use_b && !alias) e = launch_force_bias(rcholb, gb, W, X, nb * M, xv, 1, st);
  if (e == cudaSuccess)
    e = launch_energy_vjp(rchola, ga, reinterpret_cast<const double2*>(rH1a), xv, eb, W, X, M, na, f1, fc, fx,
                          reinterpret_cast<double2*>(gbara), st);
  if (e != cudaSuccess || !use_b) return (int)e;
  if (alias) {
    if (gbarb != gbara)
      e = cudaMemcpyAsync(gbarb, gbara, (size_t)W * na * M * sizeof(double2), cudaMemcpyDeviceToDevice, st);
    return (int)e;
  }
  return (int)launch_energy_vjp(rcholb, gb, reinterpret_cast<const double2*>(rH1b), xv, eb, W, X, M, nb, f1, fc, fx,
                                reinterpret_cast<double2*>(gbarb), st);
}
