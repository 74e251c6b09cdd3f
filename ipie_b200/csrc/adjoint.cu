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
