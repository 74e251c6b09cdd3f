// Particle-hole multi-determinant trial: the sums over determinants of the
// overlap, the Green's function and the local energy.
//
// For a trial sum_j c_j |D_j> of basis-orbital determinants, the library's
// single-determinant kernels give each D_j's overlap O_j, half-rotated Green's
// function (the rows occ_j[i] of D_j's full Green's function) and local energy
// E_j; these kernels accumulate
//
//   S = sum_j c_j^* O_j,  G_s = sum_j c_j^* O_j G_j,s,  E = sum_j c_j^* O_j E_j
//
// determinant by determinant (in the trial's order, as ipie's loops do) and
// divide by S at the end (estimators/greens_function_multi_det.py:17-72,
// estimators/local_energy_batch.py:78-131; the Wick's-theorem routines
// greens_function_multi_det.py:1113 and local_energy_wicks.py:864 evaluate the
// same sums).
#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

// One CTA per walker.  ghalf_s (W, n_s, M); energy (W, 3) or NULL; acc_g_s (W, M, M) or NULL.
__global__ void multidet_accumulate_kernel(int M, int na, int nb, double2 coeff_conj, const int* __restrict__ occa,
                                           const int* __restrict__ occb, const double2* __restrict__ ovlp,
                                           const double2* __restrict__ energy, const double2* __restrict__ ghalfa,
                                           const double2* __restrict__ ghalfb, double2* __restrict__ acc_ovlp,
                                           double2* __restrict__ acc_energy, double2* __restrict__ acc_ga,
                                           double2* __restrict__ acc_gb) {
  const int w = blockIdx.x;
  const double2 wt = cmul(coeff_conj, ovlp[w]);
  if (threadIdx.x == 0) {
    acc_ovlp[w] = cadd(acc_ovlp[w], wt);
    if (energy != nullptr && acc_energy != nullptr)
      for (int k = 0; k < 3; ++k) acc_energy[3 * w + k] = cadd(acc_energy[3 * w + k], cmul(wt, energy[3 * w + k]));
  }
  const size_t MM = (size_t)M * M;
  if (acc_ga != nullptr)
    for (int e = threadIdx.x; e < na * M; e += blockDim.x) {
      const int i = e / M, q = e % M;
      double2* d = acc_ga + w * MM + (size_t)occa[i] * M + q;
      *d = cadd(*d, cmul(wt, ghalfa[((size_t)w * na + i) * M + q]));
    }
  if (acc_gb != nullptr)
    for (int e = threadIdx.x; e < nb * M; e += blockDim.x) {
      const int i = e / M, q = e % M;
      double2* d = acc_gb + w * MM + (size_t)occb[i] * M + q;
      *d = cadd(*d, cmul(wt, ghalfb[((size_t)w * nb + i) * M + q]));
    }
}

// One CTA per walker: energy and Green's functions divided by the walker's total overlap.
__global__ void multidet_finalize_kernel(int M, const double2* __restrict__ acc_ovlp, double2* __restrict__ energy,
                                         double2* __restrict__ ga, double2* __restrict__ gb, unsigned* status) {
  const int w = blockIdx.x;
  const double2 s = acc_ovlp[w];
  if (!(cabs2(s) > 0.0)) {
    if (threadIdx.x == 0) flag(status, STATUS_NONFINITE);
    return;
  }
  if (energy != nullptr && threadIdx.x < 3) energy[3 * w + threadIdx.x] = cdiv(energy[3 * w + threadIdx.x], s);
  const size_t MM = (size_t)M * M;
  for (size_t e = threadIdx.x; e < MM; e += blockDim.x) {
    if (ga != nullptr) ga[w * MM + e] = cdiv(ga[w * MM + e], s);
    if (gb != nullptr) gb[w * MM + e] = cdiv(gb[w * MM + e], s);
  }
}

}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" int ipie_b200_multidet_accumulate(int W, int M, int na, int nb, double coeff_re, double coeff_im,
                                             const int* occa, const int* occb, const void* ovlp, const void* energy,
                                             const void* ghalfa, const void* ghalfb, void* acc_ovlp, void* acc_energy,
                                             void* acc_ga, void* acc_gb, void* stream) {
  if (W <= 0 || M <= 0 || na < 0 || nb < 0 || ovlp == nullptr || acc_ovlp == nullptr) return (int)cudaErrorInvalidValue;
  multidet_accumulate_kernel<<<W, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      M, na, nb, make_double2(coeff_re, -coeff_im), occa, occb, reinterpret_cast<const double2*>(ovlp),
      reinterpret_cast<const double2*>(energy), reinterpret_cast<const double2*>(ghalfa),
      reinterpret_cast<const double2*>(ghalfb), reinterpret_cast<double2*>(acc_ovlp),
      reinterpret_cast<double2*>(acc_energy), reinterpret_cast<double2*>(acc_ga), reinterpret_cast<double2*>(acc_gb));
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_multidet_finalize(int W, int M, const void* acc_ovlp, void* energy, void* ga, void* gb,
                                           unsigned int* status, void* stream) {
  if (W <= 0 || M <= 0 || acc_ovlp == nullptr) return (int)cudaErrorInvalidValue;
  multidet_finalize_kernel<<<W, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      M, reinterpret_cast<const double2*>(acc_ovlp), reinterpret_cast<double2*>(energy), reinterpret_cast<double2*>(ga),
      reinterpret_cast<double2*>(gb), status);
  note_launch();
  return (int)cudaGetLastError();
}
