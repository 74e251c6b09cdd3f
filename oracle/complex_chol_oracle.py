"""numpy restatement of ipie's walker step for a complex Cholesky Hamiltonian (CPU oracle).

TEST INFRASTRUCTURE ONLY: the checker of the complex-Cholesky kernels, imported by
``tests/`` and nothing in ``ipie_b200``.

ipie's ``GenericComplexChol`` (``hamiltonians/generic.py:100-150``) keeps the complex
Cholesky vectors L (M*M, X) and their Hermitian combinations
``A_x = (L_x + L_x^H) / 2``, ``B_x = i (L_x - L_x^H) / 2``; the auxiliary fields double
(``nfields = 2X``: the first X couple to A, the rest to B).  What changes against the real
case (``oracle/afqmc_oracle.py``), each restated below with its ipie citation:

* half rotation of L, of ``Lbar = L^T*`` (per x) and of A and B (``half_rotate.py:42-46,84-113``,
  stored by ``single_det.py:164-173``);
* the mean-field shift and one-body propagator from A and B (``phaseless_base.py:78-106,
  199-218``);
* the force bias ``[rA . G ; rB . G]`` (``propagation/force_bias.py:124-150``);
* ``VHS = i sqrt(dt) (A xs[:X] + B xs[X:])``, a general complex (W, M, M)
  (``phaseless_generic.py:99-111``);
* the local energy with ``ecoul = 1/2 X1 . X2`` (X1 from L, X2 from Lbar) and
  ``exx = 1/2 sum_x sum_ij T1_ij T2_ji`` (``estimators/local_energy_sd.py:205-262,307-355,
  406-460``).

Everything else -- Green's function, overlap, exponential, one-body application, weights,
reortho, population control, the driver -- is the real case's code, reached through the
``System`` hooks (``nfields``, ``vbias``, ``vhs``, ``local_energy``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg

from oracle import afqmc_oracle as O


def hermitian_parts(chol: np.ndarray, M: int):
    """``A_x = (L_x + L_x^H)/2``, ``B_x = i (L_x - L_x^H)/2`` as (M*M, X); ipie ``generic.py:120-133``."""
    X = chol.shape[-1]
    L = chol.reshape(M, M, X)
    LH = L.transpose(1, 0, 2).conj()
    A = 0.5 * (L + LH)
    B = 0.5j * (L - LH)
    return A.reshape(M * M, X), B.reshape(M * M, X)


def half_rotate_complex(psia, psib, chol, A, B, h1e):
    """``rH1_s``, and ``r*_s[x, i*M + n] = sum_m psi*_mi K[m, n, x]`` for K in (L, Lbar, A, B),
    ``Lbar[m, n, x] = conj(L[n, m, x])``; ipie ``half_rotate.py:11-116`` (complex branch)."""
    M = psia.shape[0]
    X = chol.shape[-1]
    L = chol.reshape(M, M, X)
    Lbar = L.transpose(1, 0, 2).conj()
    out = {}
    out["rH1a"] = np.einsum("pi,pq->iq", psia.conj(), h1e[0], optimize=True)
    out["rH1b"] = np.einsum("pi,pq->iq", psib.conj(), h1e[1], optimize=True)
    for name, K in (("rchol", L), ("rcholbar", Lbar), ("rA", A.reshape(M, M, X)), ("rB", B.reshape(M, M, X))):
        out[name + "a"] = np.einsum("mi,mnx->xin", psia.conj(), K, optimize=True).reshape(X, -1)
        out[name + "b"] = np.einsum("mi,mnx->xin", psib.conj(), K, optimize=True).reshape(X, -1)
    return out


def mean_field_shift_complex(A, B, G) -> np.ndarray:
    """``mf[:X] = i A^T vec(G_a + G_b)``, ``mf[X:] = i B^T vec(G_a + G_b)``; ipie ``phaseless_base.py:199-218``."""
    g = (G[0] + G[1]).ravel()
    return np.concatenate([1.0j * (A.T @ g), 1.0j * (B.T @ g)])


def one_body_propagator_complex(h1e_mod, A, B, mf, dt, M):
    """``expH1_s = expm(-dt/2 (h1e_mod_s - i (A mf[:X] + B mf[X:])))``; ipie ``phaseless_base.py:78-106``."""
    X = A.shape[-1]
    shift = 1.0j * np.einsum("mx,x->m", A, mf[:X]).reshape(M, M)
    shift = shift + 1.0j * np.einsum("mx,x->m", B, mf[X:]).reshape(M, M)
    H1 = h1e_mod - np.array([shift, shift])
    return np.array([scipy.linalg.expm(-0.5 * dt * H1[0]), scipy.linalg.expm(-0.5 * dt * H1[1])])


def force_bias_complex(sys_, w) -> np.ndarray:
    """``vbias[w, :X] = rA_a . Ga_w + rA_b . Gb_w``, ``vbias[w, X:]`` with rB; ipie ``force_bias.py:124-150``."""
    W = w.nwalkers
    Ga = w.Ghalfa.reshape(W, -1)
    Gb = w.Ghalfb.reshape(W, -1)
    va = sys_.rAa @ Ga.T + sys_.rAb @ Gb.T
    vb = sys_.rBa @ Ga.T + sys_.rBb @ Gb.T
    return np.concatenate([va, vb], axis=0).T.copy()


def construct_vhs_complex(sys_, xshifted: np.ndarray) -> np.ndarray:
    """``VHS = i sqrt(dt) (A . xs[:X] + B . xs[X:])`` reshaped (W, M, M); ipie ``phaseless_generic.py:99-111``.
    ``xshifted`` is (2X, W)."""
    M, X = sys_.nbasis, sys_.nchol
    W = xshifted.shape[-1]
    v = (1.0j * math.sqrt(sys_.dt)) * (sys_.A @ xshifted[:X] + sys_.B @ xshifted[X:])
    return v.T.reshape(W, M, M).copy()


def exx_kernel_complex(rchol, rcholbar, Ghalf) -> np.ndarray:
    """``exx_w = 1/2 sum_x sum_ij T1_ij T2_ji``, ``T1 = rchol_x . G^T``, ``T2 = rcholbar_x . G^T``;
    ipie ``local_energy_sd.py:307-355``."""
    W, N, M = Ghalf.shape
    X = rchol.shape[0]
    r1 = rchol.reshape(X * N, M)
    r2 = rcholbar.reshape(X * N, M)
    exx = np.zeros(W, dtype=np.complex128)
    for iw in range(W):
        T1 = (r1 @ Ghalf[iw].T).reshape(X, N, N)
        T2 = (r2 @ Ghalf[iw].T).reshape(X, N, N)
        exx[iw] = np.sum(T1 * np.transpose(T2, (0, 2, 1)))
    return 0.5 * exx


def ecoul_kernel_complex(sys_, Ghalfa, Ghalfb) -> np.ndarray:
    """``ecoul_w = 1/2 X1_w . X2_w`` (no conjugation), X1 from rchol, X2 from rcholbar;
    ipie ``local_energy_sd.py:205-262``."""
    W = Ghalfa.shape[0]
    Ga = Ghalfa.reshape(W, -1)
    Gb = Ghalfb.reshape(W, -1)
    X1 = Ga @ sys_.rchola.T + Gb @ sys_.rcholb.T
    X2 = Ga @ sys_.rcholbara.T + Gb @ sys_.rcholbarb.T
    return 0.5 * np.einsum("wx,wx->w", X1, X2)


def local_energy_complex(sys_, w) -> np.ndarray:
    """(W, 3) ``[e1b + e2b, e1b, e2b]``; ipie ``local_energy_sd.py:406-460``."""
    W = w.nwalkers
    e1b = w.Ghalfa.reshape(W, -1) @ sys_.rH1a.ravel()
    e1b = e1b + w.Ghalfb.reshape(W, -1) @ sys_.rH1b.ravel()
    e1b = e1b + sys_.ecore
    ecoul = ecoul_kernel_complex(sys_, w.Ghalfa, w.Ghalfb)
    exx = exx_kernel_complex(sys_.rchola, sys_.rcholbara, w.Ghalfa)
    exx = exx + exx_kernel_complex(sys_.rcholb, sys_.rcholbarb, w.Ghalfb)
    e2b = ecoul - exx
    out = np.zeros((W, 3), dtype=np.complex128)
    out[:, 0] = e1b + e2b
    out[:, 1] = e1b
    out[:, 2] = e2b
    return out


@dataclass
class ComplexSystem(O.System):
    """``GenericComplexChol`` + ``SingleDet`` + ``PhaselessBase.build`` for a complex (M*M, X) Cholesky."""

    A: np.ndarray = field(default=None)
    B: np.ndarray = field(default=None)
    rcholbara: np.ndarray = field(default=None)
    rcholbarb: np.ndarray = field(default=None)
    rAa: np.ndarray = field(default=None)
    rAb: np.ndarray = field(default=None)
    rBa: np.ndarray = field(default=None)
    rBb: np.ndarray = field(default=None)

    def build(self):
        M = self.nbasis
        psi = self.psi
        if np.iscomplexobj(psi) and np.sum(psi.imag.ravel() ** 2) <= 1e-8:
            psi = np.array(psi.real, dtype=np.float64)
        self.psi = psi
        self.chol = np.asarray(self.chol, dtype=np.complex128)
        self.psi0a = np.ascontiguousarray(psi[:, : self.nup])
        self.psi0b = np.ascontiguousarray(psi[:, self.nup:])
        # ipie allocates h1e_mod with H1's dtype (generic.py:116-118): for a real H1 the imaginary
        # (antisymmetric) part of 1/2 L L^H is dropped
        self.h1e_mod = O.construct_h1e_mod(self.chol, self.h1e)
        if not np.iscomplexobj(self.h1e):
            self.h1e_mod = self.h1e_mod.real.copy()
        self.A, self.B = hermitian_parts(self.chol, M)
        self.G, _ = O.trial_density(psi, self.nup, self.ndown)
        r = half_rotate_complex(self.psi0a, self.psi0b, self.chol, self.A, self.B, self.h1e)
        self.rH1a, self.rH1b = r["rH1a"], r["rH1b"]
        self.rchola, self.rcholb = r["rchola"], r["rcholb"]
        self.rcholbara, self.rcholbarb = r["rcholbara"], r["rcholbarb"]
        self.rAa, self.rAb, self.rBa, self.rBb = r["rAa"], r["rAb"], r["rBa"], r["rBb"]
        self.mf_shift = mean_field_shift_complex(self.A, self.B, self.G)
        self.expH1 = one_body_propagator_complex(self.h1e_mod, self.A, self.B, self.mf_shift, self.dt, M)
        return self

    @property
    def nfields(self):
        return 2 * self.nchol

    def vbias(self, w):
        return force_bias_complex(self, w)

    def vhs(self, xshifted):
        return construct_vhs_complex(self, xshifted)

    def local_energy(self, w):
        return local_energy_complex(self, w)
