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
 *   - spin aliasing: passing the same pointer for the alpha and beta arrays
 *     (phib == phia, ghalfb == ghalfa, rcholb == rchola, with nb == na)
 *     declares the beta block an exact copy of the alpha block (an RHF trial
 *     and walkers started from it); such blocks are computed once and counted
 *     twice, with the same results as two identical blocks;
 *   - `status` (optional, device unsigned int) collects numerical trouble
 *     bits: 1 non-finite value, 2 singular overlap pivot, 4 bad shape,
 *     8 zero column in Gram-Schmidt, 16 zero total weight in population
 *     control.  Kernels never trap; the caller reads
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

/* One launch for the orbital update of a step: phi_out = B exp(VHS) B phi_in per
 * walker, B = expH1 (each one-body factor optional), exp by the order-nmax
 * Taylor recurrence.  replaces the sequence ipie applies in
 * propagation/phaseless_base.py:321-327: propagate_walkers_one_body
 * (operations.py:26-55), apply_exponential_batch (operations.py:85-117),
 * propagate_walkers_one_body.
 * vhs (W,M,M) complex; expH1 real (M, lda_e) row-major with lda_e even >= M
 * (NULL when both flags are 0); phi_in/phi_out (W,M,N) complex, distinct.
 * Supports M <= 256, N <= 32 (cudaErrorInvalidValue otherwise). */
int ipie_b200_propagate_orbitals(const void* vhs, const double* expH1, int lda_e, const void* phi_in, void* phi_out,
                                 int W, int M, int N, int nmax, int pre_one_body, int post_one_body, void* stream);

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
 * overlap rescale: Cholesky QR for blocks of at most 32 orbitals (error ~cond(phi)^2
 * eps; walkers reorthogonalised every few steps stay near orthonormal), modified
 * Gram-Schmidt above.
 * replaces: walkers/uhf_walkers.py:108-143 (reortho) / :145-161
 * in/out: phia, phib, ovlp, log_detR; out: detR (W) double. */
int ipie_b200_reortho(void* phia, void* phib, int W, int M, int na, int nb, const double* detR_shift, double* detR,
                      double* log_detR, void* ovlp, unsigned int* status, void* stream);

/* Population-control walker copies: walker d receives walker src[d]
 * (src[d] < 0 keeps it): orbitals, weight, unscaled weight, hybrid energy,
 * overlap, phase and the half-rotated Green's functions (phase, ghalfa,
 * ghalfb may be NULL).
 * replaces: walkers/pop_controller.py:128-196 (get_buffer/set_buffer) and
 *           the send/receive loop :403-429 */
int ipie_b200_walker_copy(const int* src, int W, int M, int na, int nb, void* phia, void* phib, double* weight,
                          double* unscaled_weight, void* hybrid_energy, void* ovlp, void* phase, void* ghalfa,
                          void* ghalfb, void* stream);
/* Pair-branch population control decided on the device (no host round trip;
 * capturable in a CUDA graph).  Rescales weight by total |w| / target_weight
 * (unscaled_weight <- the weights before), sorts |w| stably, pairs walkers
 * inward from both ends while the lightest is below min_weight or the heaviest
 * above max_weight, and draws one uniform per pair (Philox4x32-10 keyed by
 * seed, counter block *counter, advanced by one per call) to choose the
 * survivor, which takes half the pair's weight.  out: src (W) int for
 * ipie_b200_walker_copy -- killed walkers receive the highest-index survivor
 * (paired = 0: ipie's single-process semantics) or their own pair's survivor
 * (paired = 1: ipie's semantics when pairs span ranks), others -1;
 * total_weight[0] = total |w|; wbound[0] = 0.1 total |w| (the next steps' weight
 * clip; may be NULL); uniforms (W/2 doubles, may be NULL) the draws of the
 * pairs formed, in pair order.  2 <= W <= 8192.  A total below 1e-8 leaves the
 * weights untouched and sets status bit 16 (ipie raises ValueError there).
 * replaces: walkers/pop_controller.py:78-125 (pop_control rescale) and
 *           :304-429 (pair_branch decisions) */
int ipie_b200_pair_branch(int W, double* weight, double* unscaled_weight, double target_weight, double min_weight,
                          double max_weight, unsigned long long seed, unsigned long long* counter, int paired, int* src,
                          double* total_weight, double* wbound, double* uniforms, unsigned int* status, void* stream);
/* Out-of-place resampling: walker d of the *_out arrays becomes walker src[d]
 * of the inputs (orbitals, half-rotated Green's functions, hybrid energy,
 * overlap, phase, unscaled weight; sources may repeat).  ghalf*, phase may be
 * NULL; phib == phia / ghalfb == ghalfa (spin-aliased blocks) copy once.
 * Inputs and outputs must not overlap.
 * replaces: the gather/scatter of stochastic_reconfiguration,
 *           walkers/pop_controller.py:432-475 */
int ipie_b200_walker_gather(const int* src, int W, int M, int na, int nb, const void* phia, const void* phib,
                            const void* ghalfa, const void* ghalfb, const void* hybrid_energy, const void* ovlp,
                            const void* phase, const double* unscaled_weight, void* phia_out, void* phib_out,
                            void* ghalfa_out, void* ghalfb_out, void* hybrid_energy_out, void* ovlp_out,
                            void* phase_out, double* unscaled_weight_out, void* stream);

/* GHF determinants phi (W, 2M, N), N = na + nb (rows 0..M-1 alpha, M..2M-1 beta spin
 * orbitals): scatter = 0 copies the spin-diagonal blocks phi[:, :M, :na] to pa (W, M, na)
 * and phi[:, M:, na:] to pb (W, M, nb); scatter = 1 writes them back (the off-diagonal
 * blocks are not touched).  These are the blocks ipie's GHF walkers propagate (their phia /
 * phib views).  replaces: walkers/ghf_walkers.py:63-77 (phia/phib views as used by
 * propagation/phaseless_generic.py:35-58 and phaseless_base.py:274-280). */
int ipie_b200_ghf_blocks(void* phi, int W, int M, int na, int nb, void* pa, void* pb, int scatter, void* stream);

/* ---- complex Cholesky Hamiltonians (ipie's GenericComplexChol: nfields = 2X, the first X
 * fields coupling to A = (L + L^H)/2, the rest to B = i (L - L^H)/2) ---- */

/* out[w][xoff + x] (accumulate: +=) sum_k (r_re + i r_im)[x][k] Ghalf[w][k]: one spin's term of
 * the force bias [rA . G ; rB . G] or of the Coulomb vectors X1 = sum_s rchol_s . G_s and
 * X2 = sum_s rcholbar_s . G_s; r_* (X, K) f64 with K = N*M, out rows of ld complex.
 * replaces: propagation/force_bias.py:124-150 and estimators/local_energy_sd.py:205-262 (X1, X2). */
int ipie_b200_force_bias_complex(const double* r_re, const double* r_im, const void* ghalf, int W, int X, int K,
                                 void* out, int ld, int xoff, int accumulate, void* stream);

/* VHS[w] = i sqrt(dt) (C . xshifted)[:, w] reshaped (M, M), C = [A | B] (M*M, F = 2X) complex
 * as its parts c_re, c_im (M*M, F) f64; xshifted (F, W) complex.  Not symmetric: written whole.
 * replaces: propagation/phaseless_generic.py:99-111. */
int ipie_b200_construct_vhs_complex(const double* c_re, const double* c_im, int M, int F, const void* xshifted, int W,
                                    double sqrt_dt, void* vhs, void* stream);

/* exx[w] (accumulate: +=) 1/2 sum_x sum_ij T1_ij T2_ji with T1 = rchol_x . Ghalf_w^T and
 * T2 = rcholbar_x . Ghalf_w^T for one spin block of a complex-Cholesky Hamiltonian, from the
 * real exchange kernel by polarisation: pol (8, X, N*M) f64 holds rchol_a +- rcholbar_b for
 * (a, b) = (re, re), (im, im), (re, im), (im, re) in that order, + before -; part: the
 * workspace of ipie_b200_exchange (rows * W complex).
 * replaces: estimators/local_energy_sd.py:307-355 (exx_kernel_batch_complex_rchol). */
int ipie_b200_exchange_complex(const double* pol, const void* ghalf, int W, int X, int M, int N, void* part,
                               void* exx, int accumulate, void* stream);

/* energy[w] = (e1b + e2b, e1b, e2b) with e1b = sum_s Ghalf_s . rH1_s + ecore,
 * e2b = 1/2 sum_x X1[w][x] X2[w][x] - exx[w] (X1, X2 (W, X) from ipie_b200_force_bias_complex;
 * exx (W) the exchange, see the Python estimator).
 * replaces: estimators/local_energy_sd.py:406-460. */
int ipie_b200_energy_complex(const void* ghalfa, const void* ghalfb, int W, int NMa, int NMb, const void* rh1a,
                             const void* rh1b, double ecore, const void* x1, const void* x2, int X, const void* exx,
                             void* energy, void* stream);

/* Exchange energy for callers that cannot allocate device memory (their device
 * memory is owned by their own pool allocator, or their loop cannot take the
 * implicit synchronisation of cudaMalloc/cudaFree).  No counterpart in ipie:
 * it is ipie_b200_exchange plus the sum over partial rows, with the partials in
 * a fixed 16 MiB file-scope device array instead of a caller workspace.
 * out: exx (W) complex = sum_x sum_ij T_ij T_ji.  Limit: ipie_b200_exchange_rows(W,X,M,N) * W
 * <= 1048576 (e.g. W=2048, X=1600, M=200, N=32 fits); larger calls return
 * cudaErrorInvalidValue (1) before any work.  The array is shared by all calls
 * and keeps the last call's partials; calls overlapping on the GPU race.  Every
 * call looks up the array's address on the current device (cudaGetSymbolAddress),
 * so a device reset does not leave a stale address; the first call on a device
 * also loads the library's device code there: make it before any stream capture
 * on that device.  Allocates nothing. */
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

/* Energy from its parts: energy[w] = (e1b + e2b, e1b, e2b) with
 * e1b = f1 (Ghalfa.rH1a + Ghalfb.rH1b) + ecore (ghalfb NULL: alpha only),
 * e2b = fc sum_x xv[w,x]^2 - fx sum_t part[t,w] (nrows = 0: no exchange term).
 * The local-energy entry points are this combine after their GEMMs; the
 * control variate uses it without the exchange. */
int ipie_b200_energy_combine(int W, int X, int M, int na, int nb, const void* ghalfa, const void* ghalfb,
                             const void* rH1a, const void* rH1b, double ecore, const void* xv, const void* part,
                             int nrows, double f1, double fc, double fx, void* energy, unsigned int* status,
                             void* stream);

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
/* The same draws with the counter block read from *counter (device memory), which is then
 * advanced by one on the stream: a step captured in a CUDA graph draws a new block on
 * every replay. */
int ipie_b200_normal_fill_dev(double* out, long long n, unsigned long long seed, unsigned long long* counter,
                              void* stream);

/* ---- mixed-precision form: tcgen05 tensor cores, FP32 accumulation ----
 * 3-pass products of operands split into head and remainder: FP16 (binary16,
 * scaled by powers of two) for the force bias, VHS and exchange, TF32 for the
 * orbital update.  FP64 stays in the overlap LU/determinant, the Green's
 * function solve, Gram-Schmidt, the weights/phases and the orbital accumulation. */

/* Force bias as a 3-pass FP16 product (FP32 accumulation, FP64 output), from the
 * padded half-rotated Cholesky split (ipie_b200_rchol_pad_split, its scale
 * r*_scale); the Green's function is split per walker with its own scale inside
 * gwork.  Same contract and spin-alias convention as
 * ipie_b200_construct_force_bias_batch_single_det; gwork: 2*W*2*32*M floats. */
int ipie_b200_construct_force_bias_mixed(const void* ra_hi, const void* ra_lo, double ra_scale, const void* rb_hi,
                                         const void* rb_lo, double rb_scale, const void* ghalfa, const void* ghalfb,
                                         float* gwork, int W, int X, int M, int na, int nb, void* vbias,
                                         unsigned int* status, void* stream);

/* ipie_b200_field_shift that also (or only: xshifted may be NULL) writes the
 * shifted fields x 64 as planar (W, 2, Xp) binary16 head/remainder pairs,
 * Xp = X rounded up to a multiple of 8 (the pad columns are not written). */
int ipie_b200_field_shift_mixed(const void* vbias, const double* xi, const void* mf_shift, int W, int X,
                                double sqrt_dt, double bound, void* xshifted, void* xs_hi, void* xs_lo, void* cmf,
                                void* cfb, void* stream);

/* VHS = i sqrt(dt) L . xshifted as a 3-pass FP16 tensor-core product (FP32
 * accumulation, ~2^-22 relative), written as four planar arrays Re/Im x head/
 * remainder: f16_planes = 0: fp32 TF32 head/remainder (W, M, M) (the operands of
 * ipie_b200_propagate_orbitals_mixed); f16_planes = 1: binary16 head/remainder
 * of V x v_scale (a power of two, > 0), (W, M, Mp) with Mp = M rounded up to a
 * multiple of 8 (the operands of ipie_b200_propagate_orbitals_mixed16).
 * cp_hi/cp_lo: packed Cholesky (P, Xp) x cp_scale (a power of two putting its
 * largest entry near 2^14) split into binary16 (ipie_b200_split_f16); xs_hi/xs_lo
 * from ipie_b200_field_shift_mixed.  replaces (mixed form):
 * propagation/phaseless_generic.py:66-97. */
int ipie_b200_construct_vhs_mixed(const void* cp_hi, const void* cp_lo, const int* idx_i, const int* idx_j, int M,
                                  int X, const void* xs_hi, const void* xs_lo, int W, double sqrt_dt, double cp_scale,
                                  int f16_planes, double v_scale, void* v_re_hi, void* v_re_lo, void* v_im_hi,
                                  void* v_im_lo, unsigned int* status, void* stream);

/* Number of 16 x 16 orbital-pair blocks (I <= J) of the block-tiled VHS operand:
 * nb (nb + 1) / 2 with nb = ceil(M / 16); the operand has 256 rows per block. */
int ipie_b200_vhs_blocks(int M);

/* Block-tiled Cholesky operand of ipie_b200_construct_vhs_blocks: row r (of
 * 256 * ipie_b200_vhs_blocks(M)) = packed Cholesky row rowmap[r] (-1: zeros) x scale,
 * split into binary16 head/remainder (R, Xp), Xp = X rounded up to 8.  Block k = (I, J),
 * row-major over I <= J; its row 16 a + b is the pair (16 I + a, 16 J + b) (a zero row
 * when either index is >= M). */
int ipie_b200_vhs_block_pack(const double* chol_packed, const int* rowmap, int M, int X, double scale, void* cb_hi,
                             void* cb_lo, void* stream);

/* The f16_planes output of ipie_b200_construct_vhs_mixed (same values and layout, and the
 * pad columns [M, Mp) written with zeros) from the block-tiled Cholesky operand: the
 * product runs with the fields as its left operand, so that a thread holds a 16 x 8 half
 * block of one walker's plane and writes it as 16-byte runs in both orientations.
 * flags bit 0: persistent CTAs.  replaces (mixed form): propagation/phaseless_generic.py:66-97. */
int ipie_b200_construct_vhs_blocks(const void* cb_hi, const void* cb_lo, int M, int X, const void* xs_hi,
                                   const void* xs_lo, int W, double sqrt_dt, double cb_scale, double v_scale,
                                   void* v_re_hi, void* v_re_lo, void* v_im_hi, void* v_im_lo, int flags,
                                   unsigned int* status, void* stream);

/* 1 when ipie_b200_propagate_orbitals_mixed16 takes this spin block (M <= 256, 1 <= N <= 32). */
int ipie_b200_orbital_chain16_fits(int M, int N);

/* phi_out = E exp(V) E phi_in per walker (Taylor order nmax) in one launch, every
 * product a 3-pass FP16 tensor-core product (FP32 accumulation); the walker's
 * Taylor terms stay on chip, each with its own exact power-of-two scale, and phi
 * accumulates as head/tail float pairs (~2^-47) between FP64 input and output.
 * e_hi/e_lo: (E - I) x e_scale (M, Mp) binary16 head/remainder (E real); v_*:
 * the f16_planes output of ipie_b200_construct_vhs_mixed with its v_scale.  When
 * the four planes lie equally spaced in one allocation (e.g. one (4, W, M, Mp)
 * array) the last 16 columns of all four come in one copy (faster when M rounded up
 * to a multiple of 16 ends 16 columns past a multiple of 64, as M = 200 does).
 * replaces (mixed form): propagation/phaseless_base.py:321-327. */
int ipie_b200_propagate_orbitals_mixed16(const void* e_hi, const void* e_lo, double e_scale, const void* v_re_hi,
                                         const void* v_re_lo, const void* v_im_hi, const void* v_im_lo,
                                         double v_scale, const void* phi_in, void* phi_out, int W, int M, int N,
                                         int nmax, unsigned int* status, void* stream);

/* phi_out = E exp(V) E phi_in per walker with every product a 3-pass TF32
 * tensor-core GEMM (E = expH1 hi/lo (M, lde) fp32, lde % 4 == 0; V planar from
 * ipie_b200_construct_vhs_mixed); phi accumulates in FP64.  work: 4*W*2N*M
 * floats.  M % 4 == 0, 2N <= 64.  replaces (mixed form):
 * propagation/phaseless_base.py:321-327. */
int ipie_b200_propagate_orbitals_mixed(const float* e_hi, const float* e_lo, int lde, const float* v_re_hi,
                                       const float* v_re_lo, const float* v_im_hi, const float* v_im_lo,
                                       const void* phi_in, void* phi_out, float* work, int W, int M, int N, int nmax,
                                       unsigned int* status, void* stream);

/* Half-rotated Cholesky rows (x, i) padded to NP = 8/16/32 >= N and columns padded
 * to Mp = M rounded up to a multiple of 8, times `scale` (a power of two; the
 * largest entry near 2^14), as binary16 head/remainder (X*NP, Mp) arrays (zeros
 * in the pads): the left operand of the mixed force bias and exchange. */
int ipie_b200_rchol_pad_split(const double* rchol, int X, int N, int M, double scale, void* hi, void* lo,
                              void* stream);

/* Exchange of one spin block in the mixed form: exx[w] (complex) = sum_x sum_ij T_ij T_ji,
 * T = rchol_x (N x M) . Ghalf_w^T, as 3-pass FP16 tensor-core products with FP64 bilinear
 * sums.  r_hi/r_lo: the padded split rows of ipie_b200_rchol_pad_split with its scale
 * r_scale (the first X Cholesky vectors of a larger array may be passed with a smaller
 * X); gwork: 2*W*2*32*M
 * floats; part: (ceil(X*NP/128) + 1) * W complex.  With the trial reference (ghalf_trial,
 * kmat, raw_trial[1]; see ipie_b200_local_energy_mixed) only G - G_T passes through the
 * tensor cores; ghalf_trial NULL disables it.
 * replaces (mixed form): estimators/local_energy_sd.py:263-303 (exx_kernel_batch_real_rchol). */
int ipie_b200_exchange_mixed(const void* r_hi, const void* r_lo, double r_scale, const void* ghalf,
                             const void* ghalf_trial, const void* kmat, const void* raw_trial, int W, int X, int M,
                             int N, float* gwork, void* part, void* exx, unsigned int* status, void* stream);

/* Local energy of the mixed form: the exchange as 3-pass FP16 tensor-core
 * products (T never stored, bilinear sums in FP64); e1b in FP64; the Coulomb
 * vector in FP64 without the trial reference, and with it as the trial's FP64
 * vector plus the 3-pass FP16 product of G - G_T.  Same contract and spin-alias convention as
 * ipie_b200_local_energy_single_det_batch; rchola/rcholb FP64, r*_hi/lo and
 * r*_scale from ipie_b200_rchol_pad_split; gwork: 2*W*2*32*M floats; work:
 * W*X + rows*W complex with rows = sum over spin blocks of ceil(X*NP/128)
 * (+1 per spin block with the trial reference).
 * Trial reference (optional; ghalf_trial_a NULL disables it): the trial's
 * Ghalf_s (N_s, M), the exchange gradient there K_s (N_s, M) and raw_trial[s]
 * = sum_x tr(T_s T_s) at the trial (complex); the tensor cores then only see
 * G - G_T and raw(G_T) + K.(G - G_T) is added in FP64, so the exchange error
 * scales with the walker's distance from the trial.
 * replaces (mixed form): estimators/local_energy_sd.py:987-1080. */
int ipie_b200_local_energy_mixed(int rhf, const double* rchola, const double* rcholb, const void* ra_hi,
                                 const void* ra_lo, double ra_scale, const void* rb_hi, const void* rb_lo,
                                 double rb_scale, const void* rH1a,
                                 const void* rH1b, double ecore, const void* ghalfa, const void* ghalfb,
                                 const void* ghalf_trial_a, const void* ghalf_trial_b, const void* kmat_a,
                                 const void* kmat_b, const void* raw_trial, int W, int X, int M, int na, int nb,
                                 float* gwork, void* work, void* energy, unsigned int* status, void* stream);

/* ---- learned control variate for the exchange energy (no counterpart in ipie) ----
 * MLP 16 -> H -> H -> 1 (SiLU), bf16 weights `wbf`, fp32 master copy/biases,
 * FP32 accumulation; parameter layout W1 (16,H), b1, W2 (H,H), b2, W3 (H,1), b3. */
/* out (B) = MLP(x (B,16)); acts: 4*B*H floats (pre/post activations kept for backward). */
int ipie_b200_mlp_forward(const float* x, int B, int F, int H, const void* wbf, const float* master, float* acts,
                          float* out, void* stream);
/* grad = d/dtheta mean((out - target)^2); work: B + 2*B*H floats; loss (+)= the batch loss. */
int ipie_b200_mlp_backward(const float* x, const float* target, int B, int F, int H, const void* wbf,
                           const float* acts, const float* out, float* grad, float* work, float* loss, void* stream);
/* One Adam step (beta 0.9/0.999) on the fp32 master weights; refreshes the bf16 copy. */
int ipie_b200_mlp_adam(float* master, void* wbf, const float* grad, float* m, float* v, long long n, float lr, int t,
                       void* stream);
/* (x - mu) / sigma per feature column, in place. */
int ipie_b200_normalize_features(float* x, long long rows, int F, const float* mu, const float* sigma, void* stream);
/* 16 per-walker features (fp32, row-major (W,16)) from the exchange-free energy (W,3), the Coulomb
 * vector xv (W,X), overlaps, hybrid energies, Ghalf per spin (W,N_s,M), the trial's Ghalf (N_s,M),
 * the exchange gradient at the trial K_s (N_s,M) complex and, in the last column, lead[w] (e.g. the
 * exchange term over the leading Cholesky vectors; NULL: the weights); base (W,) f64 receives
 * the first-order change of the exchange term from its trial value, Re sum_s f_s K_s.(G_s - G_T,s)
 * (f_s = 1/2, or 1 for spin-aliased blocks: ghalfb == ghalfa, nb == na). */
int ipie_b200_cv_features(int W, int X, int na, int nb, int M, const void* energy, const void* xv, const void* ovlp,
                          const void* hybrid_energy, const void* ghalfa, const void* ghalfb, const void* ghalf_trial_a,
                          const void* ghalf_trial_b, const void* kmat_a, const void* kmat_b, const double* weight,
                          const double* lead, float* feat, double* base, void* stream);
/* dst[s] = src[idx[s]] for rows of `row` complex values. */
int ipie_b200_gather_walkers(const void* src, const int* idx, int S, long long row, void* dst, void* stream);
/* out[0..4] = [sum w (A - c), (W/S) sum_S w (y - c), sum w, sum w A, (W/S) sum_S w y]: the control-variate
 * estimate of the weighted energy numerator is out[0] - out[1] (A: exchange-free energy, c: prediction,
 * y: exact exchange term on the random subsample idx). */
int ipie_b200_cv_sums(int W, const double* weight, const void* energy_noexx, const float* pred, int S, const int* idx,
                      const double* y_s, double* out, void* stream);

/* ---- adjoint of the local energy w.r.t. the one-body Hamiltonian (no counterpart in ipie;
 * ipie's AD-AFQMC addon differentiates the same energy with torch autograd,
 * addons/adafqmc/estimators/estimator.py:4-23) ----
 * rdm[s] (M, M) complex = sum_w coeff[w] psi_s^* Ghalf_s^w, i.e. dL/dh1_s for upstream
 * gradients coeff of the per-walker e1b; with coeff = w / sum w, the mixed-estimator
 * one-body density matrix.  work: max(na,nb)*M complex. */
int ipie_b200_onebody_adjoint(int W, int M, int na, int nb, const void* ghalfa, const void* ghalfb,
                              const void* psia_conj, const void* psib_conj, const double* coeff, void* work, void* rdm,
                              void* stream);
/* Vector-Jacobian product of the local energy with respect to the half-rotated Green's
 * functions (no counterpart in ipie; its AD-AFQMC addon takes the same derivative with torch
 * autograd through addons/adafqmc/estimators/estimator.py:4-23):
 *   gbar_s[w] = ebar[w] * dE_w / dGhalf_s[w]   (holomorphic derivative, no conjugation)
 * for E of ipie_b200_local_energy_single_det_batch with the same operands (rhf = 1: the
 * doubled alpha-only energy, gbara only):
 *   dE/dG_s = f1 rH1_s + 2 fc sum_x X_x L_s,x - 2 fx sum_x (L_s,x G_s^T) L_s,x,
 *   X_x = sum_s L_s,x . G_s, L_s,x row x of rchol_s as (n_s, M).
 * ebar (W) complex; work: W*X complex; out: gbara (W,na,M), gbarb (W,nb,M) complex.
 * n_s * M <= 8192; FP64 on the CUDA cores (one CTA per walker and spin). */
int ipie_b200_local_energy_vjp(int rhf, const double* rchola, const double* rcholb, const void* rH1a,
                               const void* rH1b, const void* ghalfa, const void* ghalfb, int W, int X, int M, int na,
                               int nb, const void* ebar, void* work, void* gbara, void* gbarb, void* stream);
/* rH1 (N, M) complex = psi^H h1: the half-rotated one-body matrix for a given h1 (M, M) real
 * (trial_wavefunction/half_rotate.py:55-56). */
int ipie_b200_rotate_onebody(const void* psi_conj, const double* h1, int M, int N, void* rh1, void* stream);

/* ---- response through the walk: ipie's AD-AFQMC propagator in forward mode ----
 * Every walker carries its orbitals phi and their derivative dphi along the
 * coupling lambda of a one-body perturbation (h1 -> h1 + lambda V), stacked as
 * one (2M, N) block [phi; dphi] per walker (walker_stride = 2 M N complex, dphi
 * at phi + M N).  The orbital propagation runs ipie_b200_propagate_orbitals on
 * the block operators [[E, 0], [dE, E]] (E = expH1, dE its derivative) and
 * [[V, 0], [dV, V]] (ipie_b200_ad_block_vhs); the entries below do the rest.
 * replaces: addons/adafqmc/propagation/propagator.py:190-249 (propagate_walkers)
 *           with the derivative torch autograd takes of it in
 *           addons/adafqmc/qmc/adafqmc.py:300-344 (ad_block_gradient) */

/* O = phi^T psi_conj, Ghalf = O^-1 phi^T (W,N,M), log det O (W) and their
 * derivatives dGhalf = O^-1 dphi^T - (O^-1 dO) Ghalf, d log det O = tr(O^-1 dO).
 * N <= 32.  replaces: addons/adafqmc/trial_wavefunction/sdtrial.py:40-57
 * (calc_overlap, get_ghalf) and the torch.det of propagator.py:232. */
int ipie_b200_ad_greens_function(const void* phi, const void* dphi, long long walker_stride, int W, int M, int N,
                                 const void* psi_conj, void* ghalf, void* dghalf, void* logdet, void* dlogdet,
                                 unsigned int* status, void* stream);
/* xbar = -sqrt(dt) (i vbias - mf) scaled to |xbar| <= bound, xshifted = x - xbar
 * written (X, W), fb = sum_x x xbar - xbar^2 / 2, mfs = -sqrt(dt) sum_x xshifted mf,
 * and the derivatives of all of them from dvbias.  vbias, dvbias (W,X) complex,
 * x (W,X) double, mf (X) complex.  replaces: propagator.py:201-203 (force bias
 * bound), :219-220 (shifted fields), :235-238 (expfb, expmf exponents). */
int ipie_b200_ad_field_shift(const void* vbias, const void* dvbias, const double* x, const void* mf, int W, int X,
                             double sqrt_dt, double bound, void* xshifted, void* dxshifted, void* fb, void* dfb,
                             void* mfs, void* dmfs, void* stream);
/* w <- w |ratio exp(fb) exp(mfs) exp(c)| max(cos theta, 0), theta = arg(ratio
 * exp(mfs)), ratio = exp(2 (logdet_new - logdet_old)); then w <- min(w, 0.1
 * sum w); dweight follows (dc = derivative of c).  One CTA.
 * replaces: propagator.py:232-249 (weight update and cap). */
int ipie_b200_ad_update_weight(int W, const void* logdet_old, const void* dlogdet_old, const void* logdet_new,
                               const void* dlogdet_new, const void* fb, const void* dfb, const void* mfs,
                               const void* dmfs, double c, double dc, double* weight, double* dweight,
                               unsigned int* status, void* stream);
/* Modified Gram-Schmidt of each walker's phi (M, N) in place, the same column
 * operations applied to dphi.  replaces: addons/adafqmc/walkers/rhf_walkers.py:
 * 22-27 (reorthogonalize; every observable is invariant under phi -> phi T). */
int ipie_b200_ad_reortho(void* phi, void* dphi, long long walker_stride, int W, int M, int N, unsigned int* status,
                         void* stream);
/* out (W, 2M, 2M) complex = [[V, 0], [dV, V]] from V, dV (W, M, M) complex. */
int ipie_b200_ad_block_vhs(const void* vhs, const void* dvhs, int W, int M, void* out, void* stream);
/* out = a + s b over n complex entries (the Green's functions G +- s dG whose local energies
 * give the energy's derivative by polarisation: the local energy is quadratic in G). */
int ipie_b200_ad_axpy(const void* a, const void* b, double s, long long n, void* out, void* stream);
/* out[d] = in[src[d]], blocks of len complex entries (in != out): the stochastic
 * reconfiguration copy of the walkers' [phi; dphi].
 * replaces: addons/adafqmc/walkers/rhf_walkers.py:30-49 (the walker_states gather). */
int ipie_b200_ad_gather(const int* src, int W, long long len, const void* in, void* out, void* stream);

/* ---- particle-hole multi-determinant trial ----
 * Determinant by determinant (j), after the single-determinant Green's function
 * (ipie_b200_greens_function_single_det_batch with D_j's one-hot orbitals) and,
 * for energies, ipie_b200_local_energy_single_det_batch with D_j's half-rotated
 * integrals: acc_ovlp += c_j^* O_j, acc_energy += c_j^* O_j E_j (W,3) (may be
 * NULL), acc_g_s[occ_s[i], q] += c_j^* O_j ghalf_s[i, q] (full (W,M,M) Green's
 * functions, may be NULL).  occa (na) occb (nb) device ints: D_j's orbitals.
 * replaces: estimators/greens_function_multi_det.py:17-72 (greens_function_multi_det)
 *           and :1113 (greens_function_multi_det_wicks_opt), estimators/
 *           local_energy_batch.py:78-131 and local_energy_wicks.py:864 (energies). */
int ipie_b200_multidet_accumulate(int W, int M, int na, int nb, double coeff_re, double coeff_im, const int* occa,
                                  const int* occb, const void* ovlp, const void* energy, const void* ghalfa,
                                  const void* ghalfb, void* acc_ovlp, void* acc_energy, void* acc_ga, void* acc_gb,
                                  void* stream);
/* energy (W,3), ga, gb (W,M,M) (each may be NULL) divided by acc_ovlp (W): the
 * trial's local energies and Green's functions.  A zero total overlap sets status bit 1. */
int ipie_b200_multidet_finalize(int W, int M, const void* acc_ovlp, void* energy, void* ga, void* gb,
                                unsigned int* status, void* stream);

/* Split FP64 values into a TF32 head (round to nearest) and an FP32 remainder:
 * x ~= hi + lo, the operands of the 3-pass TF32 tensor-core products of the
 * mixed-precision form (lo may be NULL).  No counterpart in ipie. */
int ipie_b200_split_tf32(const double* x, float* hi, float* lo, long long n, void* stream);

/* Split FP64 values, scaled by a power of two, into FP16 head and remainder:
 * x * scale ~= hi + lo (IEEE binary16 arrays; lo may be NULL).  ~2^-22 relative
 * while |x * scale| lies in [2^-3, 65504].  No counterpart in ipie. */
int ipie_b200_split_f16(const double* x, void* hi, void* lo, long long n, double scale, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IPIE_B200_H */
