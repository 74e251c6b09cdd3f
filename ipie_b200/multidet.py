"""Particle-hole multi-determinant trial (ipie's ``ParticleHole``) on the GPU.

Mirror of ipie's ``trial_wavefunction/particle_hole.py:31-160`` (the trial sum_j c_j |D_j> of
basis-orbital determinants given as ``(ci, occa, occb)``), with its Green's function and overlap
(``estimators/greens_function_multi_det.py:1113``, ``greens_function_multi_det_wicks_opt``) and
local energy (``estimators/local_energy_wicks.py:864``,
``local_energy_multi_det_trial_wicks_batch_opt``) under ipie's names.

ipie evaluates the sums over determinants with Wick's theorem from the reference determinant's
Green's function.  Here every determinant is a single determinant of one-hot orbitals, so the
library's batched single-determinant kernels give its overlap, half-rotated Green's function and
local energy for all walkers at once (its half-rotated integrals are rows of the Cholesky
vectors and of h1), and ``ipie_b200_multidet_accumulate`` adds c_j^* O_j times each into the
walkers' sums in the trial's order (``greens_function_multi_det.py:17-72`` and
``local_energy_batch.py:78-131`` state the same sums); the results equal ipie's Wick's-theorem
ones to rounding.  The cost is one single-determinant evaluation per determinant: a trial of a
few hundred determinants is fine, Wick's theorem's cost advantage at thousands is not built.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib, ptr, stream

C128 = torch.complex128
F64 = torch.float64


class ParticleHole:
    def __init__(self, wfn, nelec, nbasis, num_dets_for_props=100, num_dets_for_trial=-1, num_det_chunks=1,
                 use_active_space=True, verbose=False, device="cuda"):
        ci, occa, occb = wfn
        n = len(ci) if num_dets_for_trial is None or num_dets_for_trial < 0 else min(num_dets_for_trial, len(ci))
        self.coeffs = np.array(ci[:n], dtype=np.complex128)
        self.occa = np.array([np.asarray(o) for o in occa[:n]], dtype=np.int32).reshape(n, -1)
        self.occb = np.array([np.asarray(o) for o in occb[:n]], dtype=np.int32).reshape(n, -1)
        self.nelec = tuple(nelec)
        self.nalpha, self.nbeta = nelec
        self.nbasis = nbasis
        self.num_dets = n
        self.num_dets_for_props = min(n, num_dets_for_props) if num_dets_for_props > 0 else n
        self.verbose = verbose
        self.device = torch.device(device)
        I = np.eye(nbasis)
        self.psi0a = I[:, self.occa[0]].copy()
        self.psi0b = I[:, self.occb[0]].copy()
        self.psi0 = np.hstack([self.psi0a, self.psi0b])
        self.psi = self.psi0  # the walkers start from the reference determinant
        dev = self.device
        self.occa_dev = torch.from_numpy(self.occa).to(dev)
        self.occb_dev = torch.from_numpy(self.occb).to(dev)
        # conj(orbitals) of each determinant (one-hot columns), (ndets, M, n_s)
        oa = np.zeros((n, nbasis, self.nalpha), dtype=np.complex128)
        ob = np.zeros((n, nbasis, self.nbeta), dtype=np.complex128)
        for j in range(n):
            oa[j, self.occa[j], np.arange(self.nalpha)] = 1.0
            ob[j, self.occb[j], np.arange(self.nbeta)] = 1.0
        self.det_conj_a = torch.from_numpy(oa).to(dev)
        self.det_conj_b = torch.from_numpy(ob).to(dev)
        self.half_rotated = False
        self.spin_symmetric = False
        self.ghf = False
        self.multidet = True  # the propagator and estimators dispatch on it
        # spin-orbital occupations: alpha orbitals i, beta orbitals nbasis + i (particle_hole.py:96-97)
        self.spin_occs = [np.sort(np.concatenate([a, b + nbasis])) for a, b in zip(self.occa, self.occb)]
        self.G = compute_1rdm(self.coeffs, self.spin_occs, nbasis, self.num_dets_for_props)
        self._chol_t = None

    def build(self):
        """ipie builds its Wick's-theorem excitation tables here; the determinant sums need none."""

    def half_rotate(self, hamiltonian, comm=None):
        """Half-rotated integrals of every determinant: the rows occ_j of the Cholesky vectors and
        of h1 (ipie ``particle_hole.py:358-402``)."""
        if getattr(hamiltonian, "complex_chol", False):
            raise NotImplementedError("the particle-hole trial takes real Cholesky Hamiltonians")
        M, X = self.nbasis, hamiltonian.nchol
        L = np.asarray(hamiltonian.chol).reshape(M, M, X)
        h1 = np.asarray(hamiltonian.H1)
        dev = self.device
        ra = np.ascontiguousarray(np.stack([L[o].transpose(2, 0, 1).reshape(X, -1) for o in self.occa]))
        rb = np.ascontiguousarray(np.stack([L[o].transpose(2, 0, 1).reshape(X, -1) for o in self.occb]))
        self._rchola = torch.from_numpy(ra).to(dev)
        self._rcholb = torch.from_numpy(rb).to(dev)
        self._rH1a = torch.from_numpy(np.ascontiguousarray(h1[0][self.occa].astype(np.complex128))).to(dev)
        self._rH1b = torch.from_numpy(np.ascontiguousarray(h1[1][self.occb].astype(np.complex128))).to(dev)
        self.ecore = hamiltonian.ecore
        self.nchol = X
        self.half_rotated = True

    def calc_greens_function(self, walkers):
        return greens_function_multi_det_wicks_opt(walkers, self)

    def calc_overlap(self, walkers):
        return _sweep(walkers, self, want_g=False, energy_of=None)[0]

    def calc_force_bias(self, hamiltonian, walkers, mpi_handler=None, out=None):
        """vbias[w, x] = sum_pq L_x[p, q] (Ga + Gb)[w, p, q] from the walkers' full Green's functions
        (ipie ``propagation/force_bias.py:62-76``, ``construct_force_bias_batch_multi_det_trial``);
        the Cholesky vectors as rows (X, M^2) held once per trial."""
        if getattr(hamiltonian, "complex_chol", False):
            raise NotImplementedError("the particle-hole trial takes real Cholesky Hamiltonians")
        M, X, W = self.nbasis, hamiltonian.nchol, walkers.nwalkers
        if self._chol_t is None:
            L = np.asarray(hamiltonian.chol).reshape(M * M, X)
            self._chol_t = torch.from_numpy(np.ascontiguousarray(L.T)).to(self.device)
        if out is None:
            out = torch.empty(W, X, dtype=C128, device=walkers.device)
        ga, gb = walkers.Ga.contiguous(), walkers.Gb.contiguous()
        call("ipie_b200_construct_force_bias_batch_single_det", ptr(self._chol_t), ptr(self._chol_t), ptr(ga),
             ptr(gb), W, X, M, M, M, ptr(out), stream())
        return out


def _excitation_parity(from_orb, to_orb, di, dj):
    """True when aligning determinant dj to di (one orbital from_orb of dj replaced by to_orb of di,
    both sorted spin-orbital lists) is an odd permutation: the positions of the moved orbitals in
    their lists, each counted past the orbitals moved before it (ipie ``utils/from_dice.py:23-36``,
    ``get_perm``)."""
    n = 0
    for k, o in enumerate(from_orb):
        n += int(np.nonzero(dj == o)[0][0]) - k
    for k, o in enumerate(to_orb):
        n += int(np.nonzero(di == o)[0][0]) - k
    return n % 2 == 1


def compute_1rdm(coeffs, spin_occs, nbasis, ndets):
    """One-body density matrices (2, M, M) of the trial from its first ``ndets`` determinants
    (orthonormal basis-orbital determinants): the diagonal occupations weighted by |c_i|^2 and,
    for every pair differing by one orbital of one spin, the transition terms c_j^* c_i and their
    conjugates with the permutation sign, over sum |c_i|^2 (ipie ``particle_hole.py:458-506``,
    ``compute_1rdm``; the mean-field shift and the one-body propagator use it)."""
    c = np.asarray(coeffs[:ndets], dtype=np.complex128)
    P = np.zeros((2, nbasis, nbasis), dtype=np.complex128)
    for i in range(ndets):
        di = spin_occs[i]
        for o in di:
            P[int(o) // nbasis, int(o) % nbasis, int(o) % nbasis] += np.conj(c[i]) * c[i]
        si = set(int(o) for o in di)
        for j in range(i + 1, ndets):
            dj = spin_occs[j]
            sj = set(int(o) for o in dj)
            frm, to = sorted(sj - si), sorted(si - sj)
            if len(frm) != 1:
                continue
            phase = -1.0 if _excitation_parity(frm, to, di, dj) else 1.0
            (ii, s_i), (aa, s_a) = (frm[0] % nbasis, frm[0] // nbasis), (to[0] % nbasis, to[0] // nbasis)
            if s_i == s_a:
                P[s_i, aa, ii] += np.conj(c[j]) * c[i] * phase
                P[s_i, ii, aa] += c[j] * np.conj(c[i]) * phase
    return P / np.sum(np.conj(c) * c)


def _workspace(walkers, trial, energy):
    W, M, na, nb = walkers.nwalkers, trial.nbasis, trial.nalpha, trial.nbeta
    ws = getattr(walkers, "_multidet_ws", None)
    if ws is None or ws["W"] != W:
        dev = walkers.device
        ws = {"W": W,
              "ga": torch.empty(W, na, M, dtype=C128, device=dev), "gb": torch.empty(W, max(nb, 1), M, dtype=C128, device=dev),
              "ovlp": torch.empty(W, dtype=C128, device=dev), "e": torch.empty(W, 3, dtype=C128, device=dev),
              "zero_shift": torch.zeros(W, dtype=F64, device=dev), "work": None}
        walkers._multidet_ws = ws
    if energy and ws["work"] is None:
        X = trial.nchol
        rows = sum(max(lib().ipie_b200_exchange_rows(W, X, M, n), 0) for n in (na, nb) if n > 0)
        ws["work"] = torch.empty(W * X + rows * W, dtype=C128, device=walkers.device)
    return ws


def _sweep(walkers, trial, want_g, energy_of):
    """Accumulate the determinant sums; returns (total overlap (W,), energy (W, 3) or None)."""
    W, M, na, nb = walkers.nwalkers, trial.nbasis, trial.nalpha, trial.nbeta
    ws = _workspace(walkers, trial, energy_of is not None)
    dev = walkers.device
    acc_ovlp = torch.zeros(W, dtype=C128, device=dev)
    acc_e = torch.zeros(W, 3, dtype=C128, device=dev) if energy_of is not None else None
    if want_g:
        walkers.Ga = torch.zeros(W, M, M, dtype=C128, device=dev)
        walkers.Gb = torch.zeros(W, M, M, dtype=C128, device=dev)
    for j in range(trial.num_dets):
        c = complex(trial.coeffs[j])
        call("ipie_b200_greens_function_single_det_batch", ptr(walkers.phia), ptr(walkers.phib), W, M, na, nb,
             ptr(trial.det_conj_a[j]), ptr(trial.det_conj_b[j]), ptr(ws["zero_shift"]), ptr(ws["ga"]), ptr(ws["gb"]),
             ptr(ws["ovlp"]), None, ptr(walkers.status), stream())
        if energy_of is not None:
            call("ipie_b200_local_energy_single_det_batch", 0, ptr(trial._rchola[j]), ptr(trial._rcholb[j]),
                 ptr(trial._rH1a[j]), ptr(trial._rH1b[j]), trial.ecore, ptr(ws["ga"]), ptr(ws["gb"]), W, trial.nchol,
                 M, na, nb, ptr(ws["work"]), ptr(ws["e"]), ptr(walkers.status), stream())
        call("ipie_b200_multidet_accumulate", W, M, na, nb, c.real, c.imag, ptr(trial.occa_dev[j]),
             ptr(trial.occb_dev[j]), ptr(ws["ovlp"]), ptr(ws["e"]) if energy_of is not None else None, ptr(ws["ga"]),
             ptr(ws["gb"]), ptr(acc_ovlp), ptr(acc_e), ptr(walkers.Ga) if want_g else None,
             ptr(walkers.Gb) if want_g else None, stream())
        if j == 0 and want_g:
            # ipie keeps the reference determinant's half-rotated Green's functions on the walkers
            walkers.Ghalfa = ws["ga"].clone()
            walkers.Ghalfb = ws["gb"].clone()
    if want_g or acc_e is not None:
        call("ipie_b200_multidet_finalize", W, M, ptr(acc_ovlp), ptr(acc_e), ptr(walkers.Ga) if want_g else None,
             ptr(walkers.Gb) if want_g else None, ptr(walkers.status), stream())
    return acc_ovlp, acc_e


def greens_function_multi_det_wicks_opt(walker_batch, trial, build_full=False):
    """Total overlaps sum_j c_j^* O_j (returned) and the walkers' full Green's functions ``Ga``, ``Gb``
    (W, M, M) (ipie ``estimators/greens_function_multi_det.py:1113``)."""
    ovlp, _ = _sweep(walker_batch, trial, want_g=True, energy_of=None)
    return ovlp


def local_energy_multi_det_trial_wicks_batch_opt(system, ham, walkers, trial, max_mem=2.0):
    """(W, 3) complex [E, E1, E2] of a particle-hole trial (ipie ``estimators/local_energy_wicks.py:864``)."""
    if not trial.half_rotated:
        trial.half_rotate(ham)
    _, energy = _sweep(walkers, trial, want_g=False, energy_of=ham)
    return energy


local_energy_multi_det_trial_batch = local_energy_multi_det_trial_wicks_batch_opt
greens_function_multi_det = greens_function_multi_det_wicks_opt
