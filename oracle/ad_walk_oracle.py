"""CPU restatement of ipie's AD-AFQMC block walk with its derivative along a one-body coupling.

Test infrastructure: the checker of ``ipie_b200.adwalk``, never part of the product path.

ipie differentiates the block energy of its AD propagator with torch autograd
(``addons/adafqmc/qmc/adafqmc.py:222-344``, ``ad_block`` and ``ad_block_gradient``).  This
module runs the same walk in numpy and carries the forward-mode derivative along lambda
(h1 -> h1 + lambda V in both h1e and h1e_mod, ``addons/adafqmc/hamiltonians/hamiltonian.py:
116-128``) with explicit formulas, step by step:

* the Hamiltonian rotated into the trial's orbitals (``rot_ham_with_orbs``, ``:94-113``), the
  trial the identity's first N columns (``ad_block``, ``adafqmc.py:232-233``), the trial's own
  orbital tangent zero (no orbital relaxation);
* ``Propagator.__init__`` (``propagation/propagator.py:160-175``): mean-field shift, expH1 and its
  Frechet derivative along V, the trial energy estimate and its derivative 2 sum_i V_ii;
* ``propagate_walkers`` (``:190-249``): Green's function, bounded force bias, one-body, VHS and
  Taylor-6, one-body, (det ratio)^2 importance function, projection 1/2 (|cos| + cos), the
  0.1 total-weight cap;
* ``propagate_block`` (``:251-283``): QR every ``stabilize_freq`` steps, the block energy and
  the detached energy estimate, stochastic reconfiguration (``walkers/rhf_walkers.py:30-49``)
  every ``pop_control_freq`` steps, which resets the weights (and their derivative) to the mean.

Fields and reconfiguration uniforms are given (ipie draws them from torch's generator).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg


class ADSystem:
    def __init__(self, h1, chol, ecore, V, C, nocc, dt=0.005):
        """h1 (M, M), chol (X, M, M), V (M, M) in the atomic basis; C (M, M) the trial's orbitals."""
        self.M, self.N, self.X = h1.shape[0], nocc, chol.shape[0]
        self.dt, self.ecore = dt, float(ecore)
        self.h1 = C.T @ h1 @ C
        self.chol = np.einsum("qi,aij,jp->aqp", C.T, chol, C)
        self.V = C.T @ V @ C
        M, N = self.M, self.N
        self.psi = np.eye(M)[:, :N]
        G = self.psi @ self.psi.T
        self.h1e_mod = self.h1 - 0.5 * np.einsum("apr,arq->pq", self.chol, self.chol)
        self.mf = 2j * np.einsum("pij,ij->p", self.chol, G)
        h1e_mf = self.h1e_mod + np.einsum("p,pij->ij", self.mf.imag, self.chol)
        A = -0.5 * dt * h1e_mf
        B = -0.5 * dt * self.V
        big = scipy.linalg.expm(np.block([[A, B], [np.zeros_like(A), A]]))
        self.expH1, self.dexpH1 = big[:M, :M], big[:M, M:]
        self.rh1 = self.h1[:N, :]
        self.drh1 = self.V[:N, :]
        self.rchol = self.chol[:, :N, :]
        iu = np.triu_indices(M)
        self.packed = self.chol[:, iu[0], iu[1]]
        self.iu = iu
        self.e_trial = self.local_energy(self.psi[None].astype(complex))[0].real
        self.de_trial = 2.0 * np.trace(self.V[:N, :N])
        self.h0shift = self.ecore - 0.5 * float(np.dot(self.mf.imag, self.mf.imag))

    # ---------------------------------------------------------------- pieces
    def greens(self, phi, dphi):
        O = np.einsum("mi,wmj->wij", self.psi.conj(), phi)
        dO = np.einsum("mi,wmj->wij", self.psi.conj(), dphi)
        Oi = np.linalg.inv(O)
        G = phi @ Oi
        dG = (dphi - G @ dO) @ Oi
        sgn, lab = np.linalg.slogdet(O)
        logdet = lab + 1j * np.angle(sgn)
        dlogdet = np.einsum("wii->w", Oi @ dO)
        return G, dG, logdet, dlogdet

    def local_energy(self, G, dG=None, drh1=None):
        """e = ecore + 2 rh1.G + 1/2 (EJ - EX) (``estimators/estimator.py:4-23``) and, given dG, its
        derivative (with the coupling's rh1 derivative drh1)."""
        X = 2 * np.einsum("pij,aji->ap", self.rchol, G)
        T = np.einsum("gip,apj->agij", self.rchol, G)
        e = self.ecore + 2 * np.einsum("ij,aji->a", self.rh1, G) + 0.5 * (
            np.einsum("ap,ap->a", X, X) - 2 * np.einsum("agij,agji->a", T, T))
        if dG is None:
            return e
        dX = 2 * np.einsum("pij,aji->ap", self.rchol, dG)
        dT = np.einsum("gip,apj->agij", self.rchol, dG)
        de = 2 * np.einsum("ij,aji->a", self.rh1, dG) + 0.5 * (
            2 * np.einsum("ap,ap->a", X, dX) - 4 * np.einsum("agij,agji->a", T, dT))
        if drh1 is not None:
            de = de + 2 * np.einsum("ij,aji->a", drh1, G)
        return e, de

    def vhs(self, xs):
        M = self.M
        packed = 1j * np.sqrt(self.dt) * (xs.real @ self.packed + 1j * (xs.imag @ self.packed))
        V = np.empty((xs.shape[0], M, M), dtype=complex)
        V[:, self.iu[0], self.iu[1]] = packed
        V[:, self.iu[1], self.iu[0]] = packed
        return V

    # ---------------------------------------------------------------- one step
    def step(self, phi, dphi, w, dw, x, e_est, de_est):
        dt, sqdt = self.dt, np.sqrt(self.dt)
        G, dG, ld0, dld0 = self.greens(phi, dphi)
        vb = 2 * np.einsum("pij,aji->ap", self.rchol, G)
        dvb = 2 * np.einsum("pij,aji->ap", self.rchol, dG)
        xb = -sqdt * (1j * vb - self.mf)
        dxb = -sqdt * 1j * dvb
        a = np.abs(xb)
        big = a > 1.0
        re = (xb.real * dxb.real + xb.imag * dxb.imag) / np.where(big, a ** 3, 1.0)
        dxb = np.where(big, dxb / np.where(big, a, 1.0) - xb * re, dxb)
        xb = np.where(big, xb / np.where(big, a, 1.0), xb)
        E, dE = self.expH1, self.dexpH1
        dphi = np.einsum("pq,wqr->wpr", dE, phi) + np.einsum("pq,wqr->wpr", E, dphi)
        phi = np.einsum("pq,wqr->wpr", E, phi)
        xs = x - xb
        dxs = -dxb
        Vh, dVh = self.vhs(xs), self.vhs(dxs)
        T, dT = phi.copy(), dphi.copy()
        for n in range(1, 7):
            dT = (dVh @ T + Vh @ dT) / n
            T = (Vh @ T) / n
            phi = phi + T
            dphi = dphi + dT
        dphi = np.einsum("pq,wqr->wpr", dE, phi) + np.einsum("pq,wqr->wpr", E, dphi)
        phi = np.einsum("pq,wqr->wpr", E, phi)
        _, _, ld1, dld1 = self.greens(phi, dphi)
        lr, dlr = 2 * (ld1 - ld0), 2 * (dld1 - dld0)
        fb = np.einsum("wi,wi->w", x, xb) - 0.5 * np.einsum("wi,wi->w", xb, xb)
        dfb = np.einsum("wi,wi->w", x, dxb) - np.einsum("wi,wi->w", xb, dxb)
        mfs = -sqdt * (xs @ self.mf)
        dmfs = -sqdt * (dxs @ self.mf)
        c, dc = dt * (e_est - self.h0shift), dt * de_est
        mod = np.exp(lr.real + fb.real + mfs.real + c)
        dmod = dlr.real + dfb.real + dmfs.real + dc
        theta = lr.imag + mfs.imag
        dtheta = dlr.imag + dmfs.imag
        proj = 0.5 * (np.abs(np.cos(theta)) + np.cos(theta))
        factor = mod * proj
        dfactor = mod * dmod * proj + np.where(np.cos(theta) > 0, -mod * np.sin(theta) * dtheta, 0.0)
        w, dw = w * factor, dw * factor + w * dfactor
        bound, dbound = 0.1 * w.sum(), 0.1 * dw.sum()
        cap = ~(w < bound)
        w = np.where(cap, bound, w)
        dw = np.where(cap, dbound, dw)
        return phi, dphi, w, dw

    # ---------------------------------------------------------------- the block
    def ad_block(self, phi, w, draws, zetas, steps_per_block=10, ad_block_size=30, stabilize_freq=5,
                 pop_control_freq=5, sr_indices=None, e_est_blocks=None):
        """E, dE/dlambda, total weight W and dW/dlambda of one AD block (``adafqmc.py:222-298``).

        ``sr_indices`` (a list) receives the reconfiguration choices; given as a list of arrays it
        replays them instead of choosing (common population-control choices).  ``e_est_blocks``
        replaces the energy estimate taken after each propagation block (ipie detaches it, so its
        dependence on lambda is not part of the derivative; a finite difference holds it fixed)."""
        dphi = np.zeros_like(phi)
        dw = np.zeros_like(w)
        e_est, de_est = self.e_trial, self.de_trial
        nb = ad_block_size // steps_per_block
        etots, detots, tw, dtw = [], [], [], []
        k = 0
        isr = 0
        replay = sr_indices is not None and len(sr_indices) > 0 and not isinstance(sr_indices[0], list)
        record = [] if not replay else None
        for ib in range(nb):
            for i in range(steps_per_block):
                j = ib * steps_per_block + i
                if j % stabilize_freq == stabilize_freq - 1:
                    # QR in ipie; any phi -> phi T leaves every observable unchanged
                    for a in range(phi.shape[0]):
                        q, r = np.linalg.qr(phi[a])
                        dphi[a] = np.linalg.solve(r.T, dphi[a].T).T
                        phi[a] = q
                phi, dphi, w, dw = self.step(phi, dphi, w, dw, draws[k], e_est, de_est)
                k += 1
                if i == steps_per_block - 1:
                    G, dG, _, _ = self.greens(phi, dphi)
                    e, de = self.local_energy(G, dG, self.drh1)
                    S, dS = w.sum(), dw.sum()
                    et = (np.sum(w * e) / S).real
                    det = ((np.sum(dw * e + w * de) / S) - np.sum(w * e) * dS / S ** 2).real
                    etots.append(et)
                    detots.append(det)
                    tw.append(S)
                    dtw.append(dS)
                    e_est, de_est = (et if e_est_blocks is None else e_est_blocks[ib]), 0.0
                if j % pop_control_freq == pop_control_freq - 1:
                    if replay:
                        idx = sr_indices[isr]
                    else:
                        idx = self.sr_indices(w, zetas[isr])
                        record.append(idx)
                    isr += 1
                    wn = w / w.sum() * w.size
                    avg = np.cumsum(wn)[-1] / w.size
                    phi, dphi = phi[idx].copy(), dphi[idx].copy()
                    w = np.full_like(w, avg)
                    dw = np.zeros_like(dw)
        if sr_indices is not None and not replay:
            sr_indices.extend(record)
        etots, detots, tw, dtw = map(np.array, (etots, detots, tw, dtw))
        self.last_block_energies = etots
        W = tw.sum()
        dW = dtw.sum()
        E = np.sum(etots * tw) / W
        dEd = (np.sum(detots * tw + etots * dtw) / W) - np.sum(etots * tw) * dW / W ** 2
        return E, dEd, W, dW, phi, w

    @staticmethod
    def sr_indices(w, zeta):
        """ipie's stochastic reconfiguration choice (``walkers/rhf_walkers.py:30-49``)."""
        W = w.size
        wn = w / w.sum() * W
        cum = np.cumsum(wn)
        total = cum[-1]
        z = total * (np.arange(W) + zeta) / W
        idx = np.searchsorted(cum, z, side="left")
        return np.where(idx < W, idx, 0)
