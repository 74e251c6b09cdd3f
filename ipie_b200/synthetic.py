"""Seeded synthetic ab-initio Hamiltonians used by the benchmarks and tests.

The generator follows the workload definitions the walker-step benchmarks are
quoted on (there is no public dataset for this path):

* ``h1`` real symmetric: diagonal ``linspace(-2, 1, M)`` plus symmetric
  off-diagonal entries drawn ``N(0, 0.05)`` (upper triangle drawn, mirrored);
* Cholesky tensor ``L[g, p, q]`` symmetric in ``p, q``: upper-triangle entries
  ``N(0, 1)`` mirrored, scaled by ``0.3 * exp(-g / decay)``;
* ``ecore = 5.0``;
* RHF trial: the lowest ``N`` eigenvectors of ``F = h1 + sum_g L_g tr(L_g D)``
  with ``D`` the density of the lowest ``N`` eigenvectors of ``h1``
  (``trial_density="hartree"``), or of ``h1`` alone (``"h1"``);
* UHF trial: the RHF orbitals rotated per spin by ``expm(0.05 A_s)``,
  ``A_s`` antisymmetric with ``N(0, 1)`` entries.

ipie's array layout is produced directly: ``chol`` is (M*M, X) with
``chol[p*M + q, g] = L[g, p, q]`` and ``h1e`` is (2, M, M).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.linalg


@dataclass
class SyntheticSystem:
    nbasis: int
    nup: int
    ndown: int
    nchol: int
    h1e: np.ndarray  # (2, M, M)
    chol: np.ndarray  # (M*M, X)
    ecore: float
    psi: np.ndarray  # (M, nup + ndown) trial orbitals
    init: np.ndarray  # (M, nup + ndown) initial walker


def _sym_normal(rng, shape_lead, M, scale):
    a = rng.normal(0.0, 1.0, size=shape_lead + (M, M))
    up = np.triu(a)
    return (up + np.swapaxes(np.triu(a, 1), -1, -2)) * scale


def generate(
    nbasis: int,
    nocc,
    nchol: int,
    decay: float,
    seed: int = 7,
    uhf: bool = False,
    trial_density: str = "hartree",
    chol_scale="literal",
) -> SyntheticSystem:
    """Build one seeded system; ``chol_scale`` is a number, ``"literal"`` or ``"stable"``.

    ``"literal"`` is the 0.3 amplitude of the workload definitions.  At that
    amplitude the auxiliary-field operator grows like ``sqrt(decay * M)``: its
    2-norm per step is 0.71 at M=26 and 5.6 at M=200, where the order-6
    Taylor series no longer converges and ``expm(-dt/2 H1)`` has norm ~4e3, and
    every walk collapses (total weight -> 0) within ~100 steps even at M=26.
    ``"stable"`` keeps every other part of the recipe and sets the amplitude to
    ``0.1 * sqrt(30 * 26 / (decay * M))``, which pins that norm near 0.24 for
    every size (the M=26 walk then survives thousands of steps).
    """
    if chol_scale == "literal":
        chol_scale = 0.3
    elif chol_scale == "stable":
        chol_scale = 0.1 * np.sqrt(30.0 * 26.0 / (decay * nbasis))
    rng = np.random.default_rng(seed)
    na, nb = (nocc, nocc) if np.isscalar(nocc) else tuple(nocc)
    M, X, N = nbasis, nchol, na
    off = rng.normal(0.0, 0.05, size=(M, M))
    off = np.triu(off, 1)
    h1 = np.diag(np.linspace(-2.0, 1.0, M)) + off + off.T
    g = np.arange(X, dtype=np.float64)
    L = _sym_normal(rng, (X,), M, 1.0) * (chol_scale * np.exp(-g / decay))[:, None, None]
    chol = np.ascontiguousarray(L.reshape(X, M * M).T)
    e, c = np.linalg.eigh(h1)
    C0 = c[:, :N]
    if trial_density == "hartree":
        D = C0 @ C0.T
        J = np.einsum("gpq,g->pq", L, np.einsum("gpq,pq->g", L, D))
        _, c = np.linalg.eigh(h1 + J)
    elif trial_density != "h1":
        raise ValueError(f"unknown trial_density {trial_density!r}")
    if uhf:
        A = rng.normal(0.0, 1.0, size=(2, M, M))
        A = A - np.swapaxes(A, -1, -2)
        Ca = scipy.linalg.expm(0.05 * A[0]) @ c[:, :na]
        Cb = scipy.linalg.expm(0.05 * A[1]) @ c[:, :nb]
        psi = np.hstack([Ca, Cb])
    else:
        if na != nb:
            raise ValueError("an RHF trial needs nup == ndown")
        psi = np.hstack([c[:, :na], c[:, :nb]])
    return SyntheticSystem(
        nbasis=M,
        nup=na,
        ndown=nb,
        nchol=X,
        h1e=np.array([h1, h1]),
        chol=chol,
        ecore=5.0,
        psi=psi,
        init=psi.copy(),
    )


def generate_complex(nbasis: int, nocc, nchol: int, decay: float, seed: int = 7, uhf: bool = False,
                     imag: float = 0.3, chol_scale="stable") -> SyntheticSystem:
    """A complex-Cholesky system (ipie's ``GenericComplexChol`` input): the real system of
    :func:`generate` with an imaginary part ``i * imag * K_x`` added to every Cholesky vector,
    K_x a general (non-symmetric) N(0, 1) matrix under the same amplitude and decay, so that
    both Hermitian parts A and B are non-zero; trial and initial walker as :func:`generate`."""
    base = generate(nbasis, nocc, nchol, decay, seed=seed, uhf=uhf, chol_scale=chol_scale)
    M, X = nbasis, nchol
    if chol_scale == "literal":
        chol_scale = 0.3
    elif chol_scale == "stable":
        chol_scale = 0.1 * np.sqrt(30.0 * 26.0 / (decay * nbasis))
    rng = np.random.default_rng(seed + 1000)
    g = np.arange(X, dtype=np.float64)
    K = rng.normal(0.0, 1.0, size=(X, M, M)) * (imag * chol_scale * np.exp(-g / decay))[:, None, None]
    chol = base.chol + 1.0j * np.ascontiguousarray(K.reshape(X, M * M).T)
    return SyntheticSystem(nbasis=M, nup=base.nup, ndown=base.ndown, nchol=X, h1e=base.h1e,
                           chol=np.ascontiguousarray(chol), ecore=base.ecore, psi=base.psi, init=base.init)


# Named workloads: (nbasis, nocc, nchol, decay, walkers, steps, uhf)
WORKLOADS = {
    "c0_rhf_m26": dict(nbasis=26, nocc=5, nchol=120, decay=30.0, walkers=64, steps=200, uhf=False),
    "c1_uhf_m108": dict(nbasis=108, nocc=15, nchol=600, decay=100.0, walkers=640, steps=500, uhf=True),
    "c2_rhf_m200": dict(nbasis=200, nocc=32, nchol=1600, decay=200.0, walkers=2048, steps=1000, uhf=False),
    "c4_rhf_m76": dict(nbasis=76, nocc=10, nchol=400, decay=30.0, walkers=512, steps=300, uhf=False),
}


def workload(name: str, seed: int = 7, **kw) -> SyntheticSystem:
    p = WORKLOADS[name]
    return generate(p["nbasis"], p["nocc"], p["nchol"], p["decay"], seed=seed, uhf=p["uhf"], **kw)
