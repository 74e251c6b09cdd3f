"""numpy restatement of ipie's GHF walker step (CPU oracle).

TEST INFRASTRUCTURE ONLY: the checker of the GHF path, imported by ``tests/`` and nothing
in ``ipie_b200``.

ipie's ``GHFWalkers`` (``walkers/ghf_walkers.py:31-181``) carry one (2M, N) determinant per
walker, N = nalpha + nbeta, rows 0..M-1 the alpha and M..2M-1 the beta spin orbitals;
``SingleDetGHF`` (``trial_wavefunction/single_det_ghf.py:20-145``) holds the trial the same
way.  Restated here, each with its ipie citation:

* Green's function and overlap of the full (2M, N) determinants
  (``estimators/greens_function_single_det.py:44-61``, ``propagation/overlap.py:62-66``);
* force bias and mean-field shift from the spin-diagonal blocks ``Gaa + Gbb`` of the full G
  (``propagation/force_bias.py:155-183``, ``propagation/phaseless_base.py:175-196``);
* the propagation, which applies the one-body factors and exp(VHS) to ipie's ``phia`` and
  ``phib`` views only -- rows 0..M-1 x columns 0..nalpha-1 and rows M..2M-1 x columns
  nalpha..N-1 (``ghf_walkers.py:63-77``, ``phaseless_generic.py:35-58``,
  ``phaseless_base.py:274-280``); the off-diagonal spin blocks are left as they are;
* reorthogonalisation by a thin QR of the whole (2M, N) determinant (``ghf_walkers.py:124-151``);
* the local energy from the four spin blocks of G (``estimators/local_energy_sd.py:513-780``);
* with complex Cholesky vectors (ipie's ``GenericComplexChol``), the A/B fields of
  ``oracle/complex_chol_oracle.py`` in the force bias, mean-field shift, VHS and energy
  (``force_bias.py:186-213``, ``phaseless_base.py:219-239``, ``local_energy_sd.py:548-576,631-682,
  733-780``).

Walkers are ``afqmc_oracle.Walkers`` with ``phia`` holding the whole (W, 2M, N) determinant
and ``phib`` empty, so that population control (whose buffers hold ``phi``) and the weight
update are the UHF oracle's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg

from oracle import afqmc_oracle as O


@dataclass
class GHFSystem:
    nbasis: int  # spatial orbitals M
    nalpha: int
    nbeta: int
    h1e: np.ndarray
    chol: np.ndarray  # (M*M, X) float64
    ecore: float
    psi: np.ndarray  # (2M, N) trial
    dt: float = 0.005
    exp_nmax: int = 6
    chol_packed: np.ndarray = field(default=None)
    sym_idx: tuple = field(default=None)
    h1e_mod: np.ndarray = field(default=None)
    A: np.ndarray = field(default=None)
    B: np.ndarray = field(default=None)
    G: np.ndarray = field(default=None)
    mf_shift: np.ndarray = field(default=None)
    expH1: np.ndarray = field(default=None)

    @property
    def nchol(self):
        return self.chol.shape[-1]

    @property
    def complex_chol(self):
        return np.iscomplexobj(self.chol)

    @property
    def nfields(self):
        return 2 * self.nchol if self.complex_chol else self.nchol

    @property
    def nocc(self):
        return self.nalpha + self.nbeta

    def build(self):
        M = self.nbasis
        psi = np.asarray(self.psi)
        if np.iscomplexobj(psi) and np.sum(psi.imag.ravel() ** 2) <= 1e-8:
            psi = np.array(psi.real, dtype=np.float64)  # single_det_ghf.py:61-65
        self.psi = psi[:, : self.nocc]
        self.h1e_mod = O.construct_h1e_mod(self.chol, self.h1e)
        if self.complex_chol and not np.iscomplexobj(self.h1e):
            self.h1e_mod = self.h1e_mod.real.copy()  # generic.py:116-118
        self.sym_idx = np.triu_indices(M)
        self.G, _ = O.gab_mod(self.psi, self.psi)  # single_det_ghf.py:75
        if self.complex_chol:
            from oracle import complex_chol_oracle as C

            self.A, self.B = C.hermitian_parts(self.chol, M)
            g = (self.G[:M, :M] + self.G[M:, M:]).ravel()
            self.mf_shift = np.concatenate([1.0j * (self.A.T @ g), 1.0j * (self.B.T @ g)])
            self.expH1 = C.one_body_propagator_complex(self.h1e_mod, self.A, self.B, self.mf_shift, self.dt, M)
        else:
            self.chol_packed = O.pack_cholesky(self.chol, M)
            self.mf_shift = mean_field_shift_ghf(self.chol, self.G, M)
            self.expH1 = O.one_body_propagator(self.h1e_mod, self.chol, self.mf_shift, self.dt, M)
        return self

    def vhs(self, xshifted):
        if self.complex_chol:
            from oracle import complex_chol_oracle as C

            return C.construct_vhs_complex(self, xshifted)
        return O.construct_vhs(self, xshifted)

    def walkers(self, init, nwalkers):
        """``GHFWalkers(initial_walker, ...)`` (``ghf_walkers.py:79-113``) as oracle walkers."""
        w = O.Walkers.from_initial(np.asarray(init), self.nocc, nwalkers)
        w.phib = np.zeros((nwalkers, 2 * self.nbasis, 0), dtype=np.complex128)
        return w


def mean_field_shift_ghf(chol, G, M) -> np.ndarray:
    """``mf = 1j L^T Re(Gaa + Gbb) - L^T Im(Gaa + Gbb)``; ipie ``phaseless_base.py:175-196``."""
    g = (G[:M, :M] + G[M:, M:]).ravel()
    return 1.0j * (chol.T @ g.real) - chol.T @ g.imag


def greens_function_ghf(sys_: GHFSystem, w) -> np.ndarray:
    """``O = phi^T psi*``, ``Ghalf = O^-1 phi^T``, ``G = psi* Ghalf`` (2M, 2M), overlap with the
    walker's log_shift; ipie ``greens_function_single_det.py:44-61``.  Sets ``w.G`` and
    ``w.Ghalfa`` (W, N, 2M)."""
    phi = w.phia
    Om = np.einsum("wmi,mj->wij", phi, sys_.psi.conj(), optimize=True)
    w.Ghalfa = np.linalg.inv(Om) @ np.transpose(phi, (0, 2, 1))
    w.G = np.einsum("mi,wiq->wmq", sys_.psi.conj(), w.Ghalfa, optimize=True)
    s, l = np.linalg.slogdet(Om)
    return s * np.exp(l - w.log_shift)


def overlap_ghf(sys_: GHFSystem, w) -> np.ndarray:
    """ipie ``propagation/overlap.py:62-66``."""
    Om = np.einsum("wmi,mj->wij", w.phia, sys_.psi.conj(), optimize=True)
    s, l = np.linalg.slogdet(Om)
    return s * np.exp(l - w.log_shift)


def force_bias_ghf(sys_: GHFSystem, w) -> np.ndarray:
    """``vbias = L^T vec(Gaa + Gbb)`` (real L applied to Re and Im); ipie ``force_bias.py:155-183``."""
    M, W = sys_.nbasis, w.nwalkers
    gc = (w.G[:, :M, :M] + w.G[:, M:, M:]).reshape(W, -1)
    if sys_.complex_chol:
        return np.concatenate([gc @ sys_.A, gc @ sys_.B], axis=1)  # force_bias.py:186-213
    return gc.real @ sys_.chol + 1.0j * (gc.imag @ sys_.chol)


def local_energy_ghf(sys_: GHFSystem, w) -> np.ndarray:
    """(W, 3) ``[e1b + e2b, e1b, e2b]`` from the four spin blocks of G; ipie
    ``local_energy_sd.py:513-546,579-629,684-730``."""
    M, W = sys_.nbasis, w.nwalkers
    Gaa, Gbb = w.G[:, :M, :M], w.G[:, M:, M:]
    Gab, Gba = w.G[:, :M, M:], w.G[:, M:, :M]
    e1b = Gaa.reshape(W, -1) @ sys_.h1e[0].ravel() + Gbb.reshape(W, -1) @ sys_.h1e[1].ravel() + sys_.ecore
    gc = (Gaa + Gbb).reshape(W, -1)
    ops = (sys_.A, sys_.B) if sys_.complex_chol else (sys_.chol,)
    ecoul = np.zeros(W, dtype=np.complex128)
    exx = np.zeros(W, dtype=np.complex128)
    for K in ops:
        Xv = gc @ K
        ecoul += 0.5 * np.einsum("wx,wx->w", Xv, Xv)
        L = K.T.reshape(-1, M, M)
        for iw in range(W):
            for Gs, Gt, f in ((Gaa[iw], Gaa[iw], 1.0), (Gbb[iw], Gbb[iw], 1.0), (Gab[iw], Gba[iw], 2.0)):
                T1 = np.einsum("ji,xjk->xik", Gs, L, optimize=True)  # G^T K_x
                T2 = np.einsum("ji,xjk->xik", Gt, L, optimize=True)
                exx[iw] += f * np.einsum("xij,xji->", T1, T2, optimize=True)
    exx *= 0.5
    e2b = ecoul - exx
    out = np.zeros((W, 3), dtype=np.complex128)
    out[:, 0] = e1b + e2b
    out[:, 1] = e1b
    out[:, 2] = e2b
    return out


def _views(sys_, phi):
    M, na = sys_.nbasis, sys_.nalpha
    return phi[:, :M, :na], phi[:, M:, na:]


def _set_views(sys_, phi, pa, pb):
    M, na = sys_.nbasis, sys_.nalpha
    phi = phi.copy()
    phi[:, :M, :na] = pa
    phi[:, M:, na:] = pb
    return phi


def propagate_walkers_ghf(sys_: GHFSystem, w, eshift: float, xi: np.ndarray | None = None):
    """One phaseless step of GHF walkers; ipie ``phaseless_base.py:312-338`` with the GHF
    dispatches (the one-body and exp(VHS) act on the ``phia``/``phib`` views)."""
    ovlp = greens_function_ghf(sys_, w)
    pa, pb = _views(sys_, w.phia)
    pa = O.propagate_one_body(pa, sys_.expH1[0])
    if sys_.nbeta > 0:
        pb = O.propagate_one_body(pb, sys_.expH1[1])
    W, X = w.nwalkers, sys_.nfields
    sqrt_dt = math.sqrt(sys_.dt)
    vbias = force_bias_ghf(sys_, w)
    xbar = O.apply_bound_force_bias(-sqrt_dt * (1.0j * vbias - sys_.mf_shift), 1.0)
    if xi is None:
        xi = np.random.normal(0.0, 1.0, X * W).reshape(W, X)
    xshifted = xi - xbar
    cmf = -sqrt_dt * np.einsum("wx,x->w", xshifted, sys_.mf_shift)
    cfb = np.einsum("wx,wx->w", xi, xbar) - 0.5 * np.einsum("wx,wx->w", xbar, xbar)
    vhs = sys_.vhs(xshifted.T.copy())
    pa = O.apply_exponential(pa, vhs, sys_.exp_nmax)
    if sys_.nbeta > 0:
        pb = O.apply_exponential(pb, vhs, sys_.exp_nmax)
    pa = O.propagate_one_body(pa, sys_.expH1[0])
    if sys_.nbeta > 0:
        pb = O.propagate_one_body(pb, sys_.expH1[1])
    w.phia = _set_views(sys_, w.phia, pa, pb)
    ovlp_new = overlap_ghf(sys_, w)
    O.update_weight(sys_, w, ovlp, ovlp_new, cfb, cmf, eshift)


def reortho_ghf(sys_: GHFSystem, w) -> np.ndarray:
    """Thin QR of each (2M, N) determinant with ``diag(R) > 0``; ipie ``ghf_walkers.py:124-151``."""
    W = w.nwalkers
    detR = np.empty(W)
    for iw in range(W):
        q, r = scipy.linalg.qr(w.phia[iw], mode="economic")
        d = np.diag(r)
        w.phia[iw] = q @ np.diag(np.sign(d))
        detR[iw] = np.exp(np.sum(np.log(np.abs(d))) - w.detR_shift[iw])
        w.log_detR[iw] += np.log(detR[iw])
        w.detR[iw] = detR[iw]
        w.ovlp[iw] = w.ovlp[iw] / detR[iw]
    return detR


def ghf_from_uhf(psi_uhf: np.ndarray, nalpha: int, M: int) -> np.ndarray:
    """The block-diagonal (2M, N) determinant of a UHF one (``single_det_ghf.py:22-44``)."""
    N = psi_uhf.shape[1]
    out = np.zeros((2 * M, N), dtype=psi_uhf.dtype)
    out[:M, :nalpha] = psi_uhf[:, :nalpha]
    out[M:, nalpha:] = psi_uhf[:, nalpha:]
    return out
