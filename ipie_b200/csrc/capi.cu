// C ABI of the walker step (declared in include/ipie_b200.h).
#include "../../include/ipie_b200.h"
#include "kernels.h"

#include <atomic>

namespace ipie_b200 {
static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace ipie_b200

using namespace ipie_b200;

#define ST(s) reinterpret_cast<cudaStream_t>(s)
#define C2(p) reinterpret_cast<double2*>(p)
#define CC2(p) reinterpret_cast<const double2*>(p)

extern "C" {

const char* ipie_b200_version(void) { return "ipie_b200 0.1 (sm_100a)"; }

long long ipie_b200_launch_count(void) { return ipie_b200::g_launches.load(); }

int ipie_b200_greens_function_single_det_batch(const void* phia, const void* phib, int W, int M, int na, int nb,
                                               const void* psia_conj, const void* psib_conj, const double* log_shift,
                                               void* ghalfa, void* ghalfb, void* ovlp, void* logdet,
                                               unsigned int* status, void* stream) {
  if (ghalfa == nullptr || (nb > 0 && ghalfb == nullptr)) return (int)cudaErrorInvalidValue;
  return (int)launch_gf_overlap(CC2(phia), CC2(phib), W, M, na, nb, CC2(psia_conj), CC2(psib_conj), log_shift,
                                C2(ghalfa), C2(ghalfb), C2(ovlp), C2(logdet), status, ST(stream));
}

int ipie_b200_calc_overlap_single_det_uhf(const void* phia, const void* phib, int W, int M, int na, int nb,
                                          const void* psia_conj, const void* psib_conj, const double* log_shift,
                                          void* ovlp, unsigned int* status, void* stream) {
  return (int)launch_gf_overlap(CC2(phia), CC2(phib), W, M, na, nb, CC2(psia_conj), CC2(psib_conj), log_shift,
                                nullptr, nullptr, C2(ovlp), nullptr, status, ST(stream));
}

int ipie_b200_construct_force_bias_batch_single_det(const double* rchola, const double* rcholb, const void* ghalfa,
                                                    const void* ghalfb, int W, int X, int M, int na, int nb,
                                                    void* vbias, void* stream) {
  // Spin aliasing (rcholb == rchola, ghalfb == ghalfa, nb == na): one product, doubled (exactly t + t).
  const bool alias = nb == na && nb > 0 && rcholb == rchola && ghalfb == ghalfa;
  cudaError_t e = launch_force_bias(rchola, CC2(ghalfa), W, X, na * M, C2(vbias), 0, ST(stream), alias ? 2.0 : 1.0);
  if (e != cudaSuccess || nb == 0 || alias) return (int)e;
  return (int)launch_force_bias(rcholb, CC2(ghalfb), W, X, nb * M, C2(vbias), 1, ST(stream));
}

int ipie_b200_field_shift(const void* vbias, const double* xi, const void* mf_shift, int W, int X, double sqrt_dt,
                          double bound, void* xshifted, void* cmf, void* cfb, void* stream) {
  return (int)launch_field_shift(CC2(vbias), xi, CC2(mf_shift), W, X, sqrt_dt, bound, C2(xshifted), C2(cmf), C2(cfb),
                                 ST(stream));
}

int ipie_b200_construct_vhs(const double* chol_packed, const int* idx_i, const int* idx_j, int M, int X,
                            const void* xshifted, int W, double sqrt_dt, void* vhs, void* stream) {
  const int P = M * (M + 1) / 2;
  return (int)launch_vhs(chol_packed, idx_i, idx_j, P, X, M, CC2(xshifted), W, sqrt_dt, C2(vhs), ST(stream));
}

// ---- complex Cholesky (ipie's GenericComplexChol) ----
int ipie_b200_force_bias_complex(const double* r_re, const double* r_im, const void* ghalf, int W, int X, int K,
                                 void* out, int ld, int xoff, int accumulate, void* stream) {
  if (W <= 0 || X <= 0 || K <= 0 || ld < xoff + X || xoff < 0) return (int)cudaErrorInvalidValue;
  cudaError_t e = launch_force_bias_c(r_re, CC2(ghalf), W, X, K, C2(out), ld, xoff, accumulate, 1.0, 0.0, ST(stream));
  if (e != cudaSuccess) return (int)e;
  return (int)launch_force_bias_c(r_im, CC2(ghalf), W, X, K, C2(out), ld, xoff, 1, 0.0, 1.0, ST(stream));
}

int ipie_b200_construct_vhs_complex(const double* c_re, const double* c_im, int M, int F, const void* xshifted, int W,
                                    double sqrt_dt, void* vhs, void* stream) {
  if (M <= 0 || F <= 0 || W <= 0) return (int)cudaErrorInvalidValue;
  cudaError_t e = launch_vhs_full(c_re, M, F, CC2(xshifted), W, sqrt_dt, C2(vhs), 0, ST(stream));
  if (e != cudaSuccess) return (int)e;
  return (int)launch_vhs_full(c_im, M, F, CC2(xshifted), W, sqrt_dt, C2(vhs), 1, ST(stream));
}

int ipie_b200_energy_complex(const void* ghalfa, const void* ghalfb, int W, int NMa, int NMb, const void* rh1a,
                             const void* rh1b, double ecore, const void* x1, const void* x2, int X, const void* exx,
                             void* energy, void* stream) {
  if (W <= 0 || X <= 0 || NMa < 0 || NMb < 0) return (int)cudaErrorInvalidValue;
  return (int)launch_energy_complex(CC2(ghalfa), CC2(ghalfb), W, NMa, NMb, CC2(rh1a), CC2(rh1b), ecore, CC2(x1),
                                    CC2(x2), X, CC2(exx), C2(energy), ST(stream));
}

int ipie_b200_apply_exponential_batch(const void* vhs, const void* phi_in, void* phi_out, void* work, int W, int M,
                                      int N, int nmax, void* stream) {
  if (phi_in == phi_out) return (int)cudaErrorInvalidValue;
  double2* t0 = C2(work);
  double2* t1 = t0 + (size_t)W * M * N;
  return (int)launch_taylor(CC2(vhs), CC2(phi_in), C2(phi_out), t0, t1, W, M, N, nmax, ST(stream));
}

int ipie_b200_propagate_one_body(const void* expH1, int expH1_is_complex, const void* phi_in, void* phi_out, int W,
                                 int M, int N, void* stream) {
  if (phi_in == phi_out) return (int)cudaErrorInvalidValue;
  return (int)launch_one_body(reinterpret_cast<const double*>(expH1), expH1_is_complex, CC2(phi_in), C2(phi_out), W, M,
                              N, ST(stream));
}

int ipie_b200_propagate_orbitals(const void* vhs, const double* expH1, int lda_e, const void* phi_in, void* phi_out,
                                 int W, int M, int N, int nmax, int pre_one_body, int post_one_body, void* stream) {
  return (int)launch_propagate_fused(CC2(vhs), expH1, lda_e, CC2(phi_in), C2(phi_out), W, M, N, nmax, pre_one_body,
                                     post_one_body, ST(stream));
}

int ipie_b200_update_weight(int W, const void* ovlp_new, const void* cfb, const void* cmf, const double* eshift,
                            double dt, double ebound, const double* wbound, void* ovlp, void* hybrid_energy,
                            double* weight, unsigned int* status, void* stream) {
  return (int)launch_update_weight(W, CC2(ovlp_new), CC2(cfb), CC2(cmf), eshift, dt, ebound, wbound, C2(ovlp),
                                   C2(hybrid_energy), weight, status, ST(stream));
}

int ipie_b200_clip_weight(int W, const double* wbound, double* weight, void* stream) {
  return (int)launch_clip_weight(W, wbound, weight, ST(stream));
}

int ipie_b200_reortho(void* phia, void* phib, int W, int M, int na, int nb, const double* detR_shift, double* detR,
                      double* log_detR, void* ovlp, unsigned int* status, void* stream) {
  return (int)launch_reortho(C2(phia), C2(phib), W, M, na, nb, detR_shift, detR, log_detR, C2(ovlp), status,
                             ST(stream));
}

int ipie_b200_ghf_blocks(void* phi, int W, int M, int na, int nb, void* pa, void* pb, int scatter, void* stream) {
  return (int)launch_ghf_blocks(C2(phi), W, M, na, nb, C2(pa), C2(pb), scatter, ST(stream));
}

int ipie_b200_walker_copy(const int* src, int W, int M, int na, int nb, void* phia, void* phib, double* weight,
                          double* unscaled_weight, void* hybrid_energy, void* ovlp, void* phase, void* ghalfa,
                          void* ghalfb, void* stream) {
  return (int)launch_walker_copy(src, W, M, na, nb, C2(phia), C2(phib), weight, unscaled_weight, C2(hybrid_energy),
                                 C2(ovlp), C2(phase), C2(ghalfa), C2(ghalfb), ST(stream));
}

int ipie_b200_walker_gather(const int* src, int W, int M, int na, int nb, const void* phia, const void* phib,
                            const void* ghalfa, const void* ghalfb, const void* hybrid_energy, const void* ovlp,
                            const void* phase, const double* unscaled_weight, void* phia_out, void* phib_out,
                            void* ghalfa_out, void* ghalfb_out, void* hybrid_energy_out, void* ovlp_out,
                            void* phase_out, double* unscaled_weight_out, void* stream) {
  const bool alias_phi = phib == phia, alias_g = ghalfb == ghalfa;
  if ((nb > 0 && !alias_phi && (phib == nullptr || phib_out == nullptr)) || phia == phia_out ||
      (!alias_phi && phib != nullptr && phib == phib_out) || (ghalfa != nullptr && ghalfa == ghalfa_out) ||
      (phase != nullptr && phase_out == nullptr) || (ghalfa != nullptr && ghalfa_out == nullptr) ||
      (ghalfb != nullptr && !alias_g && ghalfb_out == nullptr))
    return (int)cudaErrorInvalidValue;
  using D = double2*;
  WalkerArrays in{(D)phia, (D)phib, (D)ghalfa, (D)ghalfb, (D)hybrid_energy, (D)ovlp, (D)phase,
                  const_cast<double*>(unscaled_weight)};
  WalkerArrays out{(D)phia_out, (D)phib_out, (D)ghalfa_out, (D)ghalfb_out, (D)hybrid_energy_out, (D)ovlp_out,
                   (D)phase_out, unscaled_weight_out};
  return (int)launch_walker_gather(src, W, M, na, nb, in, out, ST(stream));
}

int ipie_b200_exchange_rows(int W, int X, int M, int N) {
  int rows = 0;
  if (launch_exchange(nullptr, nullptr, W, X, M, N, nullptr, &rows, nullptr) != cudaSuccess) return -1;
  return rows;
}

int ipie_b200_exchange(const double* rchol, const void* ghalf, int W, int X, int M, int N, void* part, void* stream) {
  int rows = 0;
  if (part == nullptr) return (int)cudaErrorInvalidValue;
  return (int)launch_exchange(rchol, CC2(ghalf), W, X, M, N, C2(part), &rows, ST(stream));
}

// Exchange of one spin block of a complex-Cholesky Hamiltonian,
//   exx_w = 1/2 sum_x sum_ij T1_ij T2_ji,  T1 = (R_re + i R_im)_x G^T,  T2 = (S_re + i S_im)_x G^T
// (R = rchol, S = rcholbar), from the real exchange kernel by polarisation: with
// E(P) = sum_x sum_ij [P_x G^T]_ij [P_x G^T]_ji, the cross sum of real P and Q is
// (E(P + Q) - E(P - Q)) / 4, and T1_ij T2_ji expands into the four cross sums
// (R_re, S_re) - (R_im, S_im) + i (R_re, S_im) + i (R_im, S_re).  pol holds the eight real
// operands P +- Q in that order ((8, X, N*M) f64, rr+ rr- ii+ ii- ri+ ri- ir+ ir-).
int ipie_b200_exchange_complex(const double* pol, const void* ghalf, int W, int X, int M, int N, void* part,
                               void* exx, int accumulate, void* stream) {
  if (pol == nullptr || part == nullptr || W <= 0) return (int)cudaErrorInvalidValue;
  cudaStream_t st = ST(stream);
  const double2 coef[8] = {make_double2(0.125, 0.0),  make_double2(-0.125, 0.0), make_double2(-0.125, 0.0),
                           make_double2(0.125, 0.0),  make_double2(0.0, 0.125),  make_double2(0.0, -0.125),
                           make_double2(0.0, 0.125),  make_double2(0.0, -0.125)};
  const size_t stride = (size_t)X * N * M;
  for (int k = 0; k < 8; ++k) {
    int rows = 0;
    cudaError_t e = launch_exchange(pol + k * stride, CC2(ghalf), W, X, M, N, C2(part), &rows, st);
    if (e != cudaSuccess) return (int)e;
    e = launch_scaled_row_sum(CC2(part), rows, W, coef[k], C2(exx), (k > 0 || accumulate) ? 1 : 0, st);
    if (e != cudaSuccess) return (int)e;
  }
  return 0;
}

int ipie_b200_local_energy_single_det_batch(int rhf, const double* rchola, const double* rcholb, const void* rH1a,
                                            const void* rH1b, double ecore, const void* ghalfa, const void* ghalfb,
                                            int W, int X, int M, int na, int nb, void* work, void* energy,
                                            unsigned int* status, void* stream) {
  cudaStream_t st = ST(stream);
  double2* xv = C2(work);
  double2* part = xv + (size_t)W * X;
  const bool alias = !rhf && nb == na && nb > 0 && rcholb == rchola && ghalfb == ghalfa;
  const int use_b = (!rhf && nb > 0 && !alias);
  cudaError_t e = launch_force_bias(rchola, CC2(ghalfa), W, X, na * M, xv, 0, st, alias ? 2.0 : 1.0);
  if (e == cudaSuccess && use_b) e = launch_force_bias(rcholb, CC2(ghalfb), W, X, nb * M, xv, 1, st);
  if (e != cudaSuccess) return (int)e;
  int rows_a = 0, rows_b = 0;
  e = launch_exchange(rchola, CC2(ghalfa), W, X, M, na, part, &rows_a, st);
  if (e != cudaSuccess) return (int)e;
  if (use_b) {
    e = launch_exchange(rcholb, CC2(ghalfb), W, X, M, nb, part + (size_t)rows_a * W, &rows_b, st);
    if (e != cudaSuccess) return (int)e;
  }
  // UHF: e1b = Ga.rH1a + Gb.rH1b + ecore; ecoul = (Xa+Xb)^2 / 2; exx = raw / 2.
  // RHF: e1b = 2 Ga.rH1a + ecore;        ecoul = 2 Xa^2;         exx = raw.
  // Spin aliasing: the beta exchange equals the alpha one (raw_a + raw_b = 2 raw_a).
  const double f1 = rhf ? 2.0 : 1.0, fc = rhf ? 2.0 : 0.5, fx = (rhf || alias) ? 1.0 : 0.5;
  const bool e1_b = !rhf && nb > 0;
  return (int)launch_energy_combine(W, X, na * M, nb * M, CC2(ghalfa), e1_b ? CC2(ghalfb) : nullptr, CC2(rH1a),
                                    CC2(rH1b), ecore, xv, part, rows_a + rows_b, f1, fc, fx, C2(energy), status, st);
}

int ipie_b200_energy_combine(int W, int X, int M, int na, int nb, const void* ghalfa, const void* ghalfb,
                             const void* rH1a, const void* rH1b, double ecore, const void* xv, const void* part,
                             int nrows, double f1, double fc, double fx, void* energy, unsigned int* status,
                             void* stream) {
  return (int)launch_energy_combine(W, X, na * M, nb * M, CC2(ghalfa), CC2(ghalfb), CC2(rH1a), CC2(rH1b), ecore,
                                    CC2(xv), CC2(part), nrows, f1, fc, fx, C2(energy), status, ST(stream));
}

int ipie_b200_walker_sums(int W, const double* weight, const double* unscaled_weight, const void* hybrid_energy,
                          const void* energy, void* out, int accumulate, void* stream) {
  return (int)launch_walker_sums(W, weight, unscaled_weight, CC2(hybrid_energy), CC2(energy), C2(out), accumulate,
                                 ST(stream));
}

int ipie_b200_normal_fill(double* out, long long n, unsigned long long seed, unsigned long long offset, void* stream) {
  return (int)launch_normal_fill(out, n, seed, offset, ST(stream));
}

int ipie_b200_normal_fill_dev(double* out, long long n, unsigned long long seed, unsigned long long* counter,
                              void* stream) {
  return (int)launch_normal_fill_dev(out, n, seed, counter, ST(stream));
}

}  // extern "C"
