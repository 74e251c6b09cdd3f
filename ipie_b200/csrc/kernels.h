// Internal launcher declarations (C++), wrapped by the C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace ipie_b200 {

size_t gf_smem_bytes(int M, int N);

bool gf_lu32_fits(int na, int nb);
cudaError_t launch_gf_lu32(const double2* phia, const double2* phib, int W, int M, int na, int nb,
                           const double2* psia_c, const double2* psib_c, const double* log_shift, double2* ghalfa,
                           double2* ghalfb, double2* ovlp, double2* logdet, unsigned* status, cudaStream_t st);
cudaError_t launch_gf_overlap(const double2* phia, const double2* phib, int W, int M, int na, int nb,
                              const double2* psia_c, const double2* psib_c, const double* log_shift, double2* ghalfa,
                              double2* ghalfb, double2* ovlp, double2* logdet, unsigned* status, cudaStream_t st);
// Fixed power-of-two scale of the FP16 field operand of the mixed VHS product (|xs| < 1023 fits).
constexpr double kFieldScaleF16 = 64.0;
// FP16 operand rows are padded to a multiple of 8 halves (16-byte TMA strides).
__host__ __device__ inline int f16_ld(int k) { return (k + 7) & ~7; }
// xs_hi/xs_lo (binary16, optional): the shifted fields x kFieldScaleF16, planar (W, 2, f16_ld(X)).
cudaError_t launch_field_shift(const double2* vbias, const double* xi, const double2* mf, int W, int X, double sqrt_dt,
                               double bound, double2* xshifted, double2* cmf, double2* cfb, cudaStream_t st,
                               void* xs_hi = nullptr, void* xs_lo = nullptr);
cudaError_t launch_update_weight(int W, const double2* ovlp_new, const double2* cfb, const double2* cmf,
                                 const double* eshift, double dt, double ebound, const double* wbound, double2* ovlp,
                                 double2* ehyb, double* weight, unsigned* status, cudaStream_t st);
cudaError_t launch_clip_weight(int W, const double* wbound, double* weight, cudaStream_t st);
// Cholesky-QR reorthogonalisation for spin blocks of at most 32 orbitals (greens.cu)
cudaError_t launch_reortho_chol32(double2* phia, double2* phib, int W, int M, int na, int nb,
                                  const double* detR_shift, double* detR, double* log_detR, double2* ovlp,
                                  unsigned* status, cudaStream_t st);
cudaError_t launch_reortho(double2* phia, double2* phib, int W, int M, int na, int nb, const double* detR_shift,
                           double* detR, double* log_detR, double2* ovlp, unsigned* status, cudaStream_t st);
cudaError_t launch_ghf_blocks(double2* phi, int W, int M, int na, int nb, double2* pa, double2* pb, int scatter,
                              cudaStream_t st);
cudaError_t launch_walker_copy(const int* src, int W, int M, int na, int nb, double2* phia, double2* phib,
                               double* weight, double* unscaled_weight, double2* ehyb, double2* ovlp, double2* phase,
                               double2* ghalfa, double2* ghalfb, cudaStream_t st);
// per-walker arrays moved by the out-of-place resampling gather
struct WalkerArrays {
  double2 *phia, *phib, *ghalfa, *ghalfb, *ehyb, *ovlp, *phase;
  double* unscaled_weight;
};
cudaError_t launch_walker_gather(const int* src, int W, int M, int na, int nb, const WalkerArrays& in,
                                 const WalkerArrays& out, cudaStream_t st);
cudaError_t launch_energy_combine(int W, int X, int Ka, int Kb, const double2* ga, const double2* gb,
                                  const double2* rh1a, const double2* rh1b, double ecore, const double2* xv,
                                  const double2* exx_part, int ntiles, double f1, double fc, double fx, double2* energy,
                                  unsigned* status, cudaStream_t st);

cudaError_t launch_force_bias(const double* rchol, const double2* ghalf, int W, int X, int K, double2* vbias,
                              int accumulate, cudaStream_t st, double scale = 1.0);
cudaError_t launch_vhs(const double* chol_packed, const int* idx_i, const int* idx_j, int P, int X, int M,
                       const double2* xshifted, int W, double sqrt_dt, double2* vhs, cudaStream_t st);
cudaError_t launch_one_body(const double* expH1, int cplx, const double2* phi_in, double2* phi_out, int W, int M, int N,
                            cudaStream_t st);
cudaError_t launch_taylor(const double2* vhs, const double2* phi_in, double2* phi_out, double2* t0, double2* t1, int W,
                          int M, int N, int nmax, cudaStream_t st);
cudaError_t launch_force_bias_c(const double* rpart, const double2* ghalf, int W, int X, int K, double2* out, int ld,
                                int xoff, int accumulate, double sr, double si, cudaStream_t st);
cudaError_t launch_vhs_full(const double* cpart, int M, int F, const double2* xshifted, int W, double sqrt_dt,
                            double2* vhs, int mode, cudaStream_t st);
cudaError_t launch_scaled_row_sum(const double2* part, int rows, int W, double2 coef, double2* out, int accumulate,
                                  cudaStream_t st);
cudaError_t launch_energy_complex(const double2* ga, const double2* gb, int W, int NMa, int NMb, const double2* rh1a,
                                  const double2* rh1b, double ecore, const double2* x1, const double2* x2, int X,
                                  const double2* exx, double2* energy, cudaStream_t st);
cudaError_t launch_exchange(const double* rchol, const double2* ghalf, int W, int X, int M, int N, double2* part,
                            int* ntiles, cudaStream_t st);

cudaError_t launch_normal_fill_dev(double* out, long long n, unsigned long long seed, unsigned long long* counter,
                                   cudaStream_t st);
cudaError_t launch_normal_fill(double* out, long long n, unsigned long long seed, unsigned long long offset,
                               cudaStream_t st);
cudaError_t launch_walker_sums(int W, const double* weight, const double* unscaled, const double2* ehyb,
                               const double2* energy, double2* out, int accumulate, cudaStream_t st);

cudaError_t launch_propagate_fused(const double2* vhs, const double* expH1, int lda_e, const double2* phi_in,
                                   double2* phi_out, int W, int M, int N, int nmax, int pre, int post, cudaStream_t st);

namespace umma {
bool orbital_chain_fits(int M, int N);
cudaError_t mixed_orbital_chain(const float* e_hi, const float* e_lo, int lde, const float* v_re_hi,
                                const float* v_re_lo, const float* v_im_hi, const float* v_im_lo,
                                const double2* phi_in, double2* phi_out, int W, int M, int N, int nmax,
                                unsigned* status, cudaStream_t st);
bool orbital_chain16_fits(int M, int N);
cudaError_t mixed_orbital_chain16(const void* e_hi, const void* e_lo, float e_scale, const void* v_re_hi,
                                  const void* v_re_lo, const void* v_im_hi, const void* v_im_lo, float v_scale,
                                  const double2* phi_in, double2* phi_out, int W, int M, int N, int nmax,
                                  unsigned* status, cudaStream_t st);
cudaError_t mixed_orbitals(const float* e_hi, const float* e_lo, int Mp, const float* v_re_hi, const float* v_re_lo,
                           const float* v_im_hi, const float* v_im_lo, const double2* phi_in, double2* phi_out,
                           float* b0_hi, float* b0_lo, float* b1_hi, float* b1_lo, int W, int M, int N, int nmax,
                           unsigned* status, cudaStream_t st);
}  // namespace umma

}  // namespace ipie_b200
