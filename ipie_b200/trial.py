"""Single-determinant trial wavefunction on the device.

Mirror of ipie's ``SingleDet`` (``trial_wavefunction/single_det.py:30-211``):
constructor ``SingleDet(wavefunction, num_elec, num_basis)``, ``half_rotate``,
``calc_greens_function``, ``calc_overlap``, ``calc_force_bias`` and
``calculate_energy``.  The half-rotated integrals (``_rchola`` ...) are
computed once on the host and kept in HBM; every per-walker call goes to the
CUDA library.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg
import torch

from . import _lib
from ._lib import call, ptr, stream


def _gab_mod(A, B):
    """Trial density ``G = A* (B^T A*)^-1 B^T`` and its half-rotated form (ipie ``estimators/utils.py:99-132``)."""
    O = B.T @ A.conj()
    ghalf = scipy.linalg.inv(O) @ B.T
    return A.conj() @ ghalf, ghalf


class SingleDet:
    def __init__(self, wavefunction, num_elec, num_basis, handler=None, verbose=False, device="cuda"):
        psi = np.asarray(wavefunction)
        assert psi.ndim == 2
        self.nalpha, self.nbeta = num_elec
        self.nbasis = num_basis
        self.num_elec = num_elec
        self.verbose = verbose
        if np.iscomplexobj(psi) and np.sum(psi.imag.ravel() ** 2) <= 1e-8:
            psi = np.array(psi.real, dtype=np.float64)  # single_det.py:41-44
        self.psi = psi
        self.psi0a = np.ascontiguousarray(psi[:, : self.nalpha])
        self.psi0b = np.ascontiguousarray(psi[:, self.nalpha:])
        Ga, Gha = _gab_mod(self.psi0a, self.psi0a)
        if self.nbeta > 0:
            Gb, Ghb = _gab_mod(self.psi0b, self.psi0b)
        else:
            Gb, Ghb = np.zeros_like(Ga), np.zeros((0, num_basis), dtype=Gha.dtype)
        self.G = np.array([Ga, Gb])
        self.Ghalf = [Gha, Ghb]
        self.device = torch.device(device)
        self.psia_conj = torch.from_numpy(np.ascontiguousarray(self.psi0a.conj().astype(np.complex128))).to(self.device)
        self.psib_conj = torch.from_numpy(np.ascontiguousarray(self.psi0b.conj().astype(np.complex128))).to(self.device)
        self.half_rotated = False
        self.compute_trial_energy = False
        self.energy = None

    # ------------------------------------------------------------------ set-up
    def half_rotate(self, hamiltonian, comm=None):
        """``rH1_s = psi_s^H h1``, ``rchol_s[x, i*M+n] = sum_m psi*_mi L[m,n,x]``
        (ipie ``trial_wavefunction/half_rotate.py:11-116``)."""
        M, X = hamiltonian.nbasis, hamiltonian.nchol
        if getattr(hamiltonian, "complex_chol", False):
            return self._half_rotate_complex(hamiltonian)
        if np.iscomplexobj(self.psi):
            raise NotImplementedError("complex trial orbitals need a complex Cholesky Hamiltonian here")
        L = hamiltonian.chol.reshape(M, M, X)
        rH1a = np.einsum("pi,pq->iq", self.psi0a.conj(), hamiltonian.H1[0], optimize=True)
        rH1b = np.einsum("pi,pq->iq", self.psi0b.conj(), hamiltonian.H1[1], optimize=True)
        rchola = np.einsum("mi,mnx->xin", self.psi0a, L, optimize=True).reshape(X, -1)
        rcholb = np.einsum("mi,mnx->xin", self.psi0b, L, optimize=True).reshape(X, -1)
        dev = self.device
        self._rH1a = torch.from_numpy(np.ascontiguousarray(rH1a.astype(np.complex128))).to(dev)
        self._rchola = torch.from_numpy(np.ascontiguousarray(rchola)).to(dev)
        # identical spin blocks share one copy (the kernels then compute the block once)
        self.spin_symmetric = bool(self.nalpha == self.nbeta and np.array_equal(self.psi0a, self.psi0b)
                                   and np.array_equal(hamiltonian.H1[0], hamiltonian.H1[1]))
        if self.spin_symmetric:
            self._rH1b, self._rcholb = self._rH1a, self._rchola
            self.psib_conj = self.psia_conj
        else:
            self._rH1b = torch.from_numpy(np.ascontiguousarray(rH1b.astype(np.complex128))).to(dev)
            self._rcholb = torch.from_numpy(np.ascontiguousarray(rcholb)).to(dev)
        self.half_rotated = True

    def _half_rotate_complex(self, hamiltonian):
        """Complex-Cholesky branch of ``half_rotate_generic`` (``half_rotate.py:42-46,84-113``, stored as
        ``single_det.py:164-173``): L, ``Lbar = L^T*`` per vector, A and B, each half-rotated per spin.
        The device keeps what the kernels take: real and imaginary parts of rA, rB (force bias) and of
        rchol, rcholbar (Coulomb vectors), and for the exchange the eight real operands
        ``rchol_a +- rcholbar_b`` per spin (``ipie_b200_exchange_complex``)."""
        M, X = hamiltonian.nbasis, hamiltonian.nchol
        L = hamiltonian.chol.reshape(M, M, X)
        K = {"chol": L, "cholbar": L.transpose(1, 0, 2).conj(), "A": hamiltonian.A.reshape(M, M, X),
             "B": hamiltonian.B.reshape(M, M, X)}
        dev = self.device
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        rH1a = np.einsum("pi,pq->iq", self.psi0a.conj(), hamiltonian.H1[0], optimize=True)
        rH1b = np.einsum("pi,pq->iq", self.psi0b.conj(), hamiltonian.H1[1], optimize=True)
        self._rH1a = d(rH1a.astype(np.complex128))
        self._rH1b = d(rH1b.astype(np.complex128))
        self._cplx = {}
        for s_, psi in (("a", self.psi0a), ("b", self.psi0b)):
            r = {k: np.einsum("mi,mnx->xin", psi.conj(), v, optimize=True).reshape(X, -1) for k, v in K.items()}
            setattr(self, "_rchol" + s_, r["chol"])  # host copies, ipie's attribute names
            setattr(self, "_rcholbar" + s_, r["cholbar"])
            setattr(self, "_rA" + s_, r["A"])
            setattr(self, "_rB" + s_, r["B"])
            for k in ("chol", "cholbar", "A", "B"):
                self._cplx[k + s_] = (d(r[k].real), d(r[k].imag))
            R, S = r["chol"], r["cholbar"]
            pol = []
            for a, b in (("real", "real"), ("imag", "imag"), ("real", "imag"), ("imag", "real")):
                P, Q = getattr(R, a), getattr(S, b)
                pol += [P + Q, P - Q]
            self._cplx["pol" + s_] = d(np.stack(pol))
        self.spin_symmetric = False
        self.half_rotated = True

    def calculate_energy(self, system, hamiltonian):
        """Trial energy from the trial's own half-rotated densities (``single_det.py:65-86``)."""
        from .estimators import local_energy_of_density

        e = local_energy_of_density(hamiltonian, self, self.Ghalf[0], self.Ghalf[1])
        self.energy, self.e1b, self.e2b = e[0], e[1], e[2]
        return e

    # ---------------------------------------------------------------- kernels
    def calc_greens_function(self, walkers, build_full: bool = False):
        """Sets ``walkers.Ghalfa/b`` and returns the overlaps (W,) complex
        (ipie ``estimators/greens_function_single_det.py:106-154``)."""
        ovlp = torch.empty(walkers.nwalkers, dtype=torch.complex128, device=self.device)
        greens_function_into(walkers, self, ovlp)
        return ovlp

    def calc_overlap(self, walkers):
        """Walker-trial overlaps (ipie ``propagation/overlap.py:29-59``)."""
        ovlp = torch.empty(walkers.nwalkers, dtype=torch.complex128, device=self.device)
        overlap_into(walkers, self, ovlp)
        return ovlp

    def calc_force_bias(self, hamiltonian, walkers, mpi_handler=None):
        """``vbias`` (W, nfields) complex (ipie ``propagation/force_bias.py:79-121``; complex Cholesky
        ``:124-150``)."""
        vbias = torch.empty(walkers.nwalkers, hamiltonian.nfields, dtype=torch.complex128, device=self.device)
        force_bias_into(hamiltonian, walkers, self, vbias)
        return vbias


def greens_function_into(walkers, trial, ovlp_out):
    if getattr(trial, "multidet", False):
        # full Green's functions walkers.Ga/Gb of the determinant sum and its overlap
        ovlp_out.copy_(trial.calc_greens_function(walkers))
        return
    call(
        "ipie_b200_greens_function_single_det_batch",
        ptr(walkers.phia), ptr(walkers.phib), walkers.nwalkers, walkers.nbasis, walkers.nup, walkers.ndown,
        ptr(trial.psia_conj), ptr(trial.psib_conj), ptr(walkers.log_shift),
        ptr(walkers.Ghalfa), ptr(walkers.Ghalfb), ptr(ovlp_out), None, ptr(walkers.status), stream(),
    )


def overlap_into(walkers, trial, ovlp_out):
    if getattr(trial, "multidet", False):
        ovlp_out.copy_(trial.calc_overlap(walkers))
        return
    call(
        "ipie_b200_calc_overlap_single_det_uhf",
        ptr(walkers.phia), ptr(walkers.phib), walkers.nwalkers, walkers.nbasis, walkers.nup, walkers.ndown,
        ptr(trial.psia_conj), ptr(trial.psib_conj), ptr(walkers.log_shift), ptr(ovlp_out), ptr(walkers.status), stream(),
    )


def force_bias_into(hamiltonian, walkers, trial, vbias_out):
    if getattr(trial, "multidet", False):
        trial.calc_force_bias(hamiltonian, walkers, out=vbias_out)
        return
    if getattr(trial, "complex_rotated", False) and not getattr(hamiltonian, "complex_chol", False):
        # complex half-rotated Cholesky of a complex GHF trial: vbias = R . Ghalf
        re, im = trial._cplx["chola"]
        call("ipie_b200_force_bias_complex", ptr(re), ptr(im), ptr(walkers.Ghalfa), walkers.nwalkers,
             hamiltonian.nchol, walkers.nup * walkers.nbasis, ptr(vbias_out), hamiltonian.nchol, 0, 0, stream())
        return
    if getattr(hamiltonian, "complex_chol", False):
        # [rA . G ; rB . G]: per block the alpha term written, the beta term added
        W, X, M = walkers.nwalkers, hamiltonian.nchol, walkers.nbasis
        for xoff, name in ((0, "A"), (X, "B")):
            first = True
            for s_, g, n in (("a", walkers.Ghalfa, walkers.nup), ("b", walkers.Ghalfb, walkers.ndown)):
                if n == 0:
                    continue
                re, im = trial._cplx[name + s_]
                call("ipie_b200_force_bias_complex", ptr(re), ptr(im), ptr(g), W, X, n * M, ptr(vbias_out),
                     2 * X, xoff, 0 if first else 1, stream())
                first = False
        return
    call(
        "ipie_b200_construct_force_bias_batch_single_det",
        ptr(trial._rchola), ptr(trial._rcholb), ptr(walkers.Ghalfa), ptr(walkers.Ghalfb),
        walkers.nwalkers, hamiltonian.nchol, walkers.nbasis, walkers.nup, walkers.ndown, ptr(vbias_out), stream(),
    )
