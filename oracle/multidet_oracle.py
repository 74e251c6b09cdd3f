"""CPU restatement of ipie's particle-hole multi-determinant trial: overlap, Green's function and
local energy as sums over the determinants.

Test infrastructure: the checker of ``ipie_b200.multidet``, never part of the product path.

ipie's trial |Psi_T> = sum_j c_j |D_j>, every D_j a determinant of basis orbitals (occupation
lists ``occa[j]``, ``occb[j]``; ``trial_wavefunction/particle_hole.py:31-160``).  For a walker phi
(``estimators/greens_function_multi_det.py:17-72`` ``greens_function_multi_det`` and
``estimators/local_energy_batch.py:78-131`` ``local_energy_multi_det_trial_batch``):

    O_j = <D_j|phi> = det(D_ja^H phi_a) det(D_jb^H phi_b),
    G_s = sum_j c_j^* O_j G_j,s / sum_j c_j^* O_j,   G_j,s = [phi_s (D_js^H phi_s)^-1 D_js^H]^T,
    E_L = sum_j c_j^* O_j E_L(G_j) / sum_j c_j^* O_j

with E_L(G_j) the single-determinant local energy (``estimators/local_energy.py`` ``local_energy_G``:
ecore + sum h1 G + 1/2 sum_x [(L_x . (Ga + Gb))^2 - tr(L_x Ga L_x Ga) - tr(L_x Gb L_x Gb)]).
ipie's Wick's-theorem routines (``greens_function_multi_det_wicks_opt``,
``local_energy_wicks.py:864``) evaluate the same sums from the reference determinant's G.
"""
from __future__ import annotations

import numpy as np


def det_green(phi, occ):
    """(overlap, G (M, M)) of one spin block phi (M, N) against the determinant of basis orbitals occ."""
    O = phi[occ, :]  # D^H phi with D = I[:, occ]
    sign, lab = np.linalg.slogdet(O)
    ovlp = sign * np.exp(lab)
    G = np.zeros((phi.shape[0], phi.shape[0]), dtype=np.complex128)
    # [phi O^-1 D^H]^T: row occ[i] of G is row i of (phi O^-1)^T
    G[occ, :] = (phi @ np.linalg.inv(O)).T
    return ovlp, G


def local_energy_G(h1e, chol, ecore, Ga, Gb):
    """Single-determinant local energy from full Green's functions; chol (M*M, X)."""
    M = Ga.shape[0]
    L = chol.T.reshape(-1, M, M)
    e1 = np.sum(h1e[0] * Ga) + np.sum(h1e[1] * Gb)
    Xa = np.einsum("xpq,pq->x", L, Ga)
    Xb = np.einsum("xpq,pq->x", L, Gb)
    ej = 0.5 * np.sum((Xa + Xb) ** 2)
    Ta = np.einsum("xpr,qr->xpq", L, Ga)
    Tb = np.einsum("xpr,qr->xpq", L, Gb)
    ek = 0.5 * (np.einsum("xpq,xqp->", Ta, Ta) + np.einsum("xpq,xqp->", Tb, Tb))
    e2 = ej - ek
    return np.array([ecore + e1 + e2, ecore + e1, e2])


def multi_det(ci, occa, occb, phia, phib, h1e=None, chol=None, ecore=0.0):
    """(total overlap (W,), Ga, Gb (W, M, M), energy (W, 3) or None)."""
    W, M = phia.shape[0], phia.shape[1]
    tot = np.zeros(W, dtype=np.complex128)
    Ga = np.zeros((W, M, M), dtype=np.complex128)
    Gb = np.zeros((W, M, M), dtype=np.complex128)
    en = np.zeros((W, 3), dtype=np.complex128) if h1e is not None else None
    for w in range(W):
        for c, oa, ob in zip(ci, occa, occb):
            oa_, ga = det_green(phia[w], np.asarray(oa))
            ob_, gb = det_green(phib[w], np.asarray(ob))
            wt = np.conj(c) * oa_ * ob_
            tot[w] += wt
            Ga[w] += wt * ga
            Gb[w] += wt * gb
            if en is not None:
                en[w] += wt * local_energy_G(h1e, chol, ecore, ga, gb)
        Ga[w] /= tot[w]
        Gb[w] /= tot[w]
        if en is not None:
            en[w] /= tot[w]
    return tot, Ga, Gb, en
