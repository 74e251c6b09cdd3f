/*
 * ipie_b200 -- C ABI of the B200 phaseless-AFQMC walker step.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (as void*, NULL = legacy default stream), enqueues its kernels on that
 * stream and returns immediately.
 *
 * Conventions
 *   - complex values are interleaved (re, im) doubles: numpy/torch complex128;
 *   - arrays are C-contiguous with ipie's shapes (noted per argument);
 *   - W walkers, M basis functions, na/nb electrons per spin, X Cholesky
 *     vectors, P = M(M+1)/2 packed pairs;
 *   - return value: 0 on success, otherwise the cudaError_t of the failed
 *     launch (cudaErrorInvalidValue = 1 for unsupported sizes);
 *   - `status` (optional, device unsigned int) collects numerical trouble
 *     bits: 1 non-finite value, 2 singular overlap pivot, 4 bad shape,
 *     8 zero column in Gram-Schmidt.  Kernels never trap; the caller reads
 *     the word (ipie raises Python exceptions at the matching places).
 *
 * Each function names the ipie routine (file:line inside the ipie project)
 * whose arithmetic it performs.
 */
#ifndef IPIE_B200_H
#define IPIE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Library version string. */
const char* ipie_b200_version(void);

/* Number of kernels this library has enqueued since it was loaded (host
 * counter; instrumentation for benchmarks, no counterpart in ipie). */
long long ipie_b200_launch_count(void);

/* Half-rotated Green's function and overlap of every walker with a
 * single-determinant trial.
 * replaces: estimators/greens_function_single_det.py:106-154
 *           (greens_function_single_det_batch; CPU twin :62-103)
 * phia (W,M,na) phib (W,M,nb) complex; psia_conj (M,na) psib_conj (M,nb)
 * complex = conj(trial orbitals); log_shift (W) double;
 * out: ghalfa (W,na,M) ghalfb (W,nb,M) complex, ovlp (W) complex,
 *      logdet (W,2) complex (log|det|, phase angle) per spin or NULL. */
int ipie_b200_greens_function_single_det_batch(const void* phia, const void* phib, int W, int M, int na, int nb,
                                               const void* psia_conj, const void* psib_conj, const double* log_shift,
                                               void* ghalfa, void* ghalfb, void* ovlp, void* logdet,
                                               unsigned int* status, void* stream);

/* Overlap only.
 * replaces: propagation/overlap.py:29-59 (calc_overlap_single_det_uhf) */
int ipie_b200_calc_overlap_single_det_uhf(const void* phia, const void* phib, int W, int M, int na, int nb,
                                          const void* psia_conj, const void* psib_conj, const double* log_shift,
                                          void* ovlp, unsigned int* status, void* stream);

/* Force bias vbias[w,x] = sum_s rchol_s[x,:] . Ghalf_s[w,:] (real rchol).
 * replaces: propagation/force_bias.py:79-121
 *           (construct_force_bias_batch_single_det, rhf=False branch)
 * rchola (X, na*M) rcholb (X, nb*M) double; ghalfa/b as above;
 * out: vbias (W, X) complex.  nb = 0 skips the beta block. */
int ipie_b200_construct_force_bias_batch_single_det(const double* rchola, const double* rcholb, const void* ghalfa,
                                                    const void* ghalfb, int W, int X, int M, int na, int nb,
                                                    void* vbias, void* stream);

/* Shifted fields from the force bias (capped at |xbar| <= bound), with the
 * per-walker constants cmf and cfb.
 * replaces: propagation/phaseless_base.py:284-306 (propagate_walkers_two_body
 *           up to the VHS) and :360-368 (apply_bound_force_bias)
 * vbias (W,X) complex, xi (W,X) double N(0,1) draws, mf_shift (X) complex;
 * out: xshifted (X,W) complex, cmf (W) complex, cfb (W) complex. */
int ipie_b200_field_shift(const void* vbias, const double* xi, const void* mf_shift, int W, int X, double sqrt_dt,
                          double bound, void* xshifted, void* cmf, void* cfb, void* stream);

/* VHS[w] = i sqrt(dt) sum_x L_x xshifted[x,w], symmetric (W,M,M).
 * replaces: propagation/phaseless_generic.py:66-97 (construct_VHS, real
 *           Cholesky) and utils/pack_numba_gpu.py:24-34 (unpack)
 * chol_packed (P,X) double; idx_i/idx_j (P) int = numpy.triu_indices(M);
 * xshifted (X,W) complex; out: vhs (W,M,M) complex. */
int ipie_b200_construct_vhs(const double* chol_packed, const int* idx_i, const int* idx_j, int M, int X,
                            const void* xshifted, int W, double sqrt_dt, void* vhs, void* stream);

/* phi_out = sum_{n=0..nmax} VHS^n phi_in / n! (recurrence T_n = VHS T_{n-1}/n).
 * replaces: propagation/operations.py:85-117 (apply_exponential_batch)
 * vhs (W,M,M) complex; phi_in/phi_out (W,M,N) complex (distinct buffers);
 * work: 2*W*M*N complex scratch. */
int ipie_b200_apply_exponential_batch(const void* vhs, const void* phi_in, void* phi_out, void* work, int W, int M,
                                      int N, int nmax, void* stream);

/* phi_out[w] = expH1 . phi_in[w].
 * replaces: propagation/operations.py:26-55 (propagate_one_body)
 * expH1 (M,M) double (expH1_is_complex = 0) or complex (1);
 * phi_in/phi_out (W,M,N) complex, distinct buffers. */
int ipie_b200_propagate_one_body(const void* expH1, int expH1_is_complex, const void* phi_in, void* phi_out, int W,
                                 int M, int N, void* stream);

/* Hybrid energy, importance function, cosine projection, then the driver's
 * weight clip when *wbound >= 0 (wbound may be NULL).
 * replaces: propagation/phaseless_base.py:340-358 (update_weight),
 *           :370-380 (apply_bound_hybrid), qmc/afqmc.py:581-585 (clip)
 * ovlp_new, cfb, cmf (W) complex; eshift, wbound: device doubles;
 * in/out: ovlp (W) complex, hybrid_energy (W) complex, weight (W) double. */
int ipie_b200_update_weight(int W, const void* ovlp_new, const void* cfb, const void* cmf, const double* eshift,
                            double dt, double ebound, const double* wbound, void* ovlp, void* hybrid_energy,
                            double* weight, unsigned int* status, void* stream);

/* weight = clip(weight, -*wbound, *wbound).  replaces: qmc/afqmc.py:581-585 */
int ipie_b200_clip_weight(int W, const double* wbound, double* weight, void* stream);

/* Thin QR of every spin block with positive diag(R) (in place), detR and
 * overlap rescale.
 * replaces: walkers/uhf_walkers.py:108-143 (reortho) / :145-161
 * in/out: phia, phib, ovlp, log_detR; out: detR (W) double. */
int ipie_b200_reortho(void* phia, void* phib, int W, int M, int na, int nb, const double* detR_shift, double* detR,
                      double* log_detR, void* ovlp, unsigned int* status, void* stream);

/* Population-control walker copies: walker d receives walker src[d]
 * (src[d] < 0 keeps it): orbitals, weight, unscaled weight, hybrid energy,
 * overlap and phase (phase may be NULL).
 * replaces: walkers/pop_controller.py:128-196 (get_buffer/set_buffer) and
 *           the send/receive loop :403-429 */
int ipie_b200_walker_copy(const int* src, int W, int M, int na, int nb, void* phia, void* phib, double* weight,
                          double* unscaled_weight, void* hybrid_energy, void* ovlp, void* phase, void* stream);

/* Exchange energy for callers that cannot allocate device memory (their device
 * memory is owned by their own pool allocator, or their loop cannot take the
 * implicit synchronisation of cudaMalloc/cudaFree).  No counterpart in ipie:
 * it is ipie_b200_exchange plus the sum over partial rows, with the partials in
 * a fixed 16 MiB file-scope device array instead of a caller workspace.
 * out: exx (W) complex = sum_x sum_ij T_ij T_ji.  Limit: ipie_b200_exchange_rows(W,X,M,N) * W
 * <= 1048576 (e.g. W=2048, X=1600, M=200, N=32 fits); larger calls return
 * cudaErrorInvalidValue (1) before any work.  The array is shared by all calls
 * and keeps the last call's partials; calls overlapping on the GPU race.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress,
 * that device current); make it before any stream capture on that device.
 * Allocates nothing. */
int ipie_b200_exchange_noalloc(const double* rchol, const void* ghalf, int W, int X, int M, int N, void* exx,
                               void* stream);

/* Number of partial rows the exchange kernel writes for one spin block
 * (the workspace for ipie_b200_exchange is rows * W complex). */
int ipie_b200_exchange_rows(int W, int X, int M, int N);

/* Exchange partials: part[t, w] summed over t gives sum_x sum_ij T_ij T_ji with
 * T = rchol_x (N x M) . Ghalf_w^T; T is never stored.
 * replaces: estimators/kernels/gpu/exchange.py:64-141 (exchange_reduction)
 *           with the T GEMM of estimators/local_energy_sd.py:1053-1070
 * rchol (X, N*M) double, ghalf (W,N,M) complex; out: part (rows, W) complex. */
int ipie_b200_exchange(const double* rchol, const void* ghalf, int W, int X, int M, int N, void* part, void* stream);

/* Local energy (W,3) complex [e1b+e2b, e1b, e2b] of single-determinant walkers.
 * rhf = 0 (UHF form, used by ipie in production):
 *   replaces estimators/local_energy_sd.py:358-403 (local_energy_single_det_uhf_batch)
 *   and :987-1080 (local_energy_single_det_batch_gpu);
 * rhf = 1 (spin-alpha only, doubled):
 *   replaces estimators/local_energy_sd.py:106-155 (local_energy_single_det_rhf_batch).
 * rH1a (na,M) rH1b (nb,M) complex; rchola/rcholb double;
 * work: W*X + (rows_a + rows_b)*W complex, rows_s = ipie_b200_exchange_rows(W,X,M,n_s).
 * out: energy (W,3) complex. */
int ipie_b200_local_energy_single_det_batch(int rhf, const double* rchola, const double* rcholb, const void* rH1a,
                                            const void* rH1b, double ecore, const void* ghalfa, const void* ghalfb,
                                            int W, int X, int M, int na, int nb, void* work, void* energy,
                                            unsigned int* status, void* stream);

/* Per-walker block sums (complex[7], accumulated into out when accumulate=1):
 * [sum w, sum w_unscaled, sum w*E_hyb, sum w*Re E0, sum w, sum w*Re E1, sum w*Re E2].
 * replaces: walkers/base_walkers.py:43-50 (WalkerAccumulator.update) and
 *           estimators/energy.py:156-165 (EnergyEstimator.compute_estimator sums)
 * unscaled_weight, hybrid_energy, energy (W,3) may be NULL. */
int ipie_b200_walker_sums(int W, const double* weight, const double* unscaled_weight, const void* hybrid_energy,
                          const void* energy, void* out, int accumulate, void* stream);

/* n standard normal draws (Philox4x32-10 + Box-Muller) for counter block
 * `offset` of stream `seed`; the throughput-mode replacement of
 * propagation/phaseless_base.py:296-298 (xp.random.normal).  The sequence
 * differs from numpy's MT19937 by construction. */
int ipie_b200_normal_fill(double* out, long long n, unsigned long long seed, unsigned long long offset, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IPIE_B200_H */
