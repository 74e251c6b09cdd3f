"""GHF walkers and trial (ipie's ``GHFWalkers`` and ``SingleDetGHF``) on the device.

A GHF determinant is one (2M, N) matrix, N = nalpha + nbeta electrons, rows 0..M-1 the
alpha and M..2M-1 the beta spin orbitals (``walkers/ghf_walkers.py:31-181``,
``trial_wavefunction/single_det_ghf.py:20-145``).  On the device it is a single-determinant
block of 2M "orbitals" and N electrons, so the Green's function, overlap, reorthogonalisation,
population control and estimator kernels of the UHF path run on it unchanged with
``nbasis = 2M``, ``nup = N``, ``ndown = 0``.  What the spin structure changes:

* the trial is half-rotated over both spin blocks: ``R_x = [psi_a^H L_x | psi_b^H L_x]``
  (N, 2M) and ``rH1 = [psi_a^H h1_a | psi_b^H h1_b]``, so that ``R . Ghalf`` is ipie's
  ``L^T vec(Gaa + Gbb)`` (force bias, Coulomb vectors), ``Ghalf . rH1`` its one-body energy and
  ``1/2 sum_x tr((R_x Ghalf^T)^2)`` its exchange ``1/2 sum_x tr(Taa^2) + tr(Tbb^2) + 2 tr(Tab Tba)``
  (``estimators/local_energy_sd.py:579-629``);
* the propagation acts on ipie's ``phia``/``phib`` views only -- rows 0..M-1 x columns
  0..nalpha-1 and rows M..2M-1 x columns nalpha..N-1 -- which ``ipie_b200_ghf_blocks`` copies
  out and back (``phaseless_generic.py:35-58``, ``phaseless_base.py:274-280``).

A complex trial makes R complex; its products then run on the complex-operand kernels of the
complex-Cholesky path.  With complex Cholesky vectors (ipie's ``GenericComplexChol``) the trial
is rotated for the A and B fields, ``RA`` and ``RB``: the force bias is ``[RA . Ghalf ; RB . Ghalf]``
and the energy runs over the 2X rows ``[RA ; RB]`` (``local_energy_sd.py:548-576,631-682``).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg
import torch

from .trial import SingleDet
from .walkers import UHFWalkers


def _gab_mod(A, B):
    O = B.T @ A.conj()
    ghalf = scipy.linalg.inv(O) @ B.T
    return A.conj() @ ghalf, ghalf


class SingleDetGHF(SingleDet):
    """``SingleDetGHF(wavefunction (2M, N), (nalpha, nbeta), M)`` or ``SingleDetGHF(uhf_trial)``."""

    ghf = True

    def __init__(self, wavefunction, num_elec=None, num_basis=None, handler=None, verbose=False, device="cuda"):
        if isinstance(wavefunction, SingleDet):
            uhf = wavefunction
            M, na, nb = uhf.nbasis, uhf.nalpha, uhf.nbeta
            psi = np.zeros((2 * M, na + nb), dtype=np.result_type(uhf.psi0a, uhf.psi0b))
            psi[:M, :na] = uhf.psi0a
            psi[M:, na:] = uhf.psi0b
            num_elec, num_basis, device = (na, nb), M, uhf.device
        else:
            psi = np.asarray(wavefunction)
            if psi.ndim != 2 or psi.shape[0] != 2 * num_basis:
                raise AssertionError("GHF wavefunction must be (2 * num_basis, N)")
        if np.iscomplexobj(psi) and np.sum(psi.imag.ravel() ** 2) <= 1e-8:
            psi = np.array(psi.real, dtype=np.float64)  # single_det_ghf.py:61-65
        self.nalpha, self.nbeta = num_elec
        self.num_elec = tuple(num_elec)
        self.nelec = self.num_elec
        self.nbasis = num_basis
        self.nocc = self.nalpha + self.nbeta
        self.verbose = verbose
        self.psi = psi[:, : self.nocc]
        self.psi0 = self.psi
        self.psi0a = self.psi[:num_basis]
        self.psi0b = self.psi[num_basis:]
        self.Gfull, gh = _gab_mod(self.psi, self.psi)  # single_det_ghf.py:75
        self.G = self.Gfull
        self.Ghalf = [gh, np.zeros((0, 2 * num_basis), dtype=gh.dtype)]
        self.device = torch.device(device)
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.psia_conj = d(self.psi.conj().astype(np.complex128))
        self.psib_conj = d(np.zeros((2 * num_basis, 0), dtype=np.complex128))
        self.half_rotated = False
        self.complex_rotated = False
        self.spin_symmetric = False
        self.compute_trial_energy = False
        self.energy = None

    def half_rotate(self, hamiltonian, comm=None):
        """``R`` and ``rH1`` over both spin blocks (see the module docstring); ipie keeps the full
        Green's function for GHF instead (``single_det_ghf.py:114-121``), with the same products."""
        M, X = hamiltonian.nbasis, hamiltonian.nchol
        if M != self.nbasis:
            raise AssertionError("Hamiltonian and trial basis sizes differ")
        pa, pb = self.psi[:M].conj(), self.psi[M:].conj()

        def rotate(K):  # [psi_a^H K_x | psi_b^H K_x] as (X, N * 2M)
            K = K.reshape(M, M, X)
            return np.concatenate([np.einsum("pn,pqx->xnq", pa, K, optimize=True),
                                   np.einsum("pn,pqx->xnq", pb, K, optimize=True)], axis=2).reshape(X, -1)

        H1 = hamiltonian.H1
        rH1 = np.concatenate([pa.T @ H1[0], pb.T @ H1[1]], axis=1)
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self._rH1a = d(rH1.astype(np.complex128))
        self._rH1b = d(np.zeros((0, 2 * M), dtype=np.complex128))
        if getattr(hamiltonian, "complex_chol", False):
            # A and B fields: force bias [RA . G ; RB . G], energy over the 2X rows [RA ; RB]
            RA, RB = rotate(hamiltonian.A), rotate(hamiltonian.B)
            R = np.concatenate([RA, RB], axis=0)
            self._cplx = {"Aa": (d(RA.real), d(RA.imag)), "Ba": (d(RB.real), d(RB.imag))}
        else:
            R = rotate(hamiltonian.chol)
            self._cplx = {}
        self._R = R
        self._cplx_rows = R.shape[0]
        self.complex_rotated = bool(np.iscomplexobj(R) and np.abs(R.imag).max() > 0)
        if self.complex_rotated:
            re, im = d(R.real), d(R.imag)
            pol = []
            for a, b in (("real", "real"), ("imag", "imag"), ("real", "imag"), ("imag", "real")):
                P, Q = getattr(R, a), getattr(R, b)
                pol += [P + Q, P - Q]
            self._cplx.update({"chola": (re, im), "cholbara": (re, im), "pola": d(np.stack(pol))})
            self._rchola = self._rcholb = None
        else:
            self._rchola = d(np.asarray(R.real, dtype=np.float64))
            self._rcholb = self._rchola
        self.half_rotated = True

    def calculate_energy(self, system, hamiltonian):
        """Trial energy from its own Green's function (``single_det_ghf.py:91-112``)."""
        from .estimators import _local_energy

        w = GHFWalkers(self.psi, self.nalpha, self.nbeta, self.nbasis, 1, device=self.device)
        w.build(self)
        e = _local_energy(hamiltonian, w, self, rhf=False)[0].cpu().numpy()
        self.energy, self.e1b, self.e2b = e[0], e[1], e[2]
        return e


class GHFWalkers(UHFWalkers):
    """``GHFWalkers(initial_walker (2M, N), nup, ndown, nbasis, nwalkers)`` or
    ``GHFWalkers.from_uhf(uhf_walkers)`` (``walkers/ghf_walkers.py:31-113``).

    ``phi`` (W, 2M, N) is the walkers' determinant; the kernel-facing sizes are those of one
    2M-orbital spin block (``nbasis = 2M``, ``nup = N``, ``ndown = 0``); ipie's sizes are
    ``nalpha``, ``nbeta`` and ``nbasis_spatial``."""

    ghf = True

    def __init__(self, initial_walker, nup, ndown, nbasis, nwalkers, mpi_handler=None, verbose=False, device="cuda"):
        init = np.asarray(initial_walker)
        if init.ndim != 2 or init.shape[0] != 2 * nbasis or init.shape[1] < nup + ndown:
            raise AssertionError("GHF initial walker must be (2 * nbasis, nup + ndown)")
        super().__init__(init[:, : nup + ndown], nup + ndown, 0, 2 * nbasis, nwalkers, mpi_handler, verbose, device)
        self.nalpha, self.nbeta, self.nbasis_spatial = nup, ndown, nbasis
        self.buff_names = self.buff_names[:-2] + ["phi"]

    @classmethod
    def from_uhf(cls, walkers):
        """Block-diagonal GHF walkers from UHF ones (``ghf_walkers.py:33-61``)."""
        M, na, nb = walkers.nbasis, walkers.nup, walkers.ndown
        out = cls(np.zeros((2 * M, na + nb)), na, nb, M, walkers.nwalkers, device=walkers.device)
        phi = torch.zeros(walkers.nwalkers, 2 * M, na + nb, dtype=walkers.phia.dtype, device=walkers.device)
        phi[:, :M, :na] = walkers.phia
        phi[:, M:, na:] = walkers.phib
        out.phi = phi.contiguous()
        for n in ("weight", "unscaled_weight", "phase", "ovlp", "hybrid_energy", "log_shift", "detR", "detR_shift",
                  "log_detR"):
            getattr(out, n).copy_(getattr(walkers, n))
        return out

    @property
    def phi(self):
        return self.phia

    @phi.setter
    def phi(self, value):
        self.phia = value

    @property
    def Ghalf(self):
        return self.Ghalfa
