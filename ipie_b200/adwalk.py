"""Response of an AFQMC block energy to a one-body coupling, differentiated through the walk.

Mirror of ipie's AD-AFQMC block (``addons/adafqmc/qmc/adafqmc.py:222-344``: ``ad_block`` and
``ad_block_gradient``): the Hamiltonian h1 + lambda V is rotated into the trial's orbitals
(``hamiltonians/hamiltonian.py:94-128``), an RHF walk runs ipie's AD propagator
(``propagation/propagator.py:160-283``: (det ratio)^2 importance function, 1/2 (|cos| + cos)
projection, 0.1 total-weight cap, QR every ``stabilize_freq`` steps, block energies, stochastic
reconfiguration every ``pop_control_freq`` steps) and the block energy is differentiated along
lambda with the auxiliary fields and the reconfiguration choices held fixed -- the derivative
ipie takes with torch autograd.  The trial's orbital tangent is zero (no orbital relaxation).

Here the derivative is carried forward with the walk: every walker holds [phi; dphi] as one
(2M, N) block and its weight's derivative, the orbital propagation is the library's fused
one-body . Taylor-6 . one-body kernel on the block operators [[E, 0], [dE, E]] and
[[V, 0], [dV, V]], and ``ipie_b200_ad_*`` kernels do the Green's function, fields, weights,
Gram-Schmidt and reconfiguration copies with their derivatives.  For one coupling this costs
about two walks and stores no trajectory.  :class:`BlockEnergyResponse` puts the result behind
a ``torch.autograd.Function``: its backward returns grad_output x dE/dlambda.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg
import torch

from ._lib import call, lib, ptr, stream
from .hamiltonian import Generic

C128 = torch.complex128
F64 = torch.float64


class ADWalk:
    def __init__(self, h1, chol, ecore, V, C, nocc, nwalkers, dt=0.005, device="cuda"):
        """h1 (M, M) real, chol (X, M, M), V (M, M) symmetric, all in the atomic basis; C (M, M) the
        trial's orbitals (its first ``nocc`` columns occupied)."""
        dev = torch.device(device)
        self.dev = dev
        h1 = np.asarray(h1, dtype=np.float64)
        chol = np.asarray(chol, dtype=np.float64)
        V = np.asarray(V, dtype=np.float64)
        C = np.asarray(C, dtype=np.float64)
        M, N, X = h1.shape[0], nocc, chol.shape[0]
        self.M, self.N, self.X, self.W = M, N, X, nwalkers
        self.dt, self.sqrt_dt, self.ecore = dt, math.sqrt(dt), float(ecore)
        # rotate into the trial's orbitals (set-up, host)
        h1r = C.T @ h1 @ C
        Lr = np.einsum("qi,aij,jp->aqp", C.T, chol, C)
        Vr = C.T @ V @ C
        self.ham = Generic(np.array([h1r, h1r]), np.ascontiguousarray(Lr.reshape(X, M * M).T), ecore)
        psi = np.eye(M)[:, :N]
        G = psi @ psi.T
        h1e_mod = self.ham.h1e_mod[0]
        self.mf = 2j * np.einsum("pij,ij->p", Lr, G)
        A = -0.5 * dt * (h1e_mod + np.einsum("p,pij->ij", self.mf.imag, Lr))
        B = -0.5 * dt * Vr
        big = scipy.linalg.expm(np.block([[A, B], [np.zeros_like(A), A]]))
        E, dE = big[:M, :M], big[:M, M:]
        # the block one-body operator [[E, 0], [dE, E]], rows padded to an even length
        self.lda = 2 * M + ((2 * M) & 1)
        eb = np.zeros((2 * M, self.lda))
        eb[:M, :M] = E
        eb[M:, :M] = dE
        eb[M:, M:2 * M] = E
        self.eblk = torch.from_numpy(eb).to(dev)
        self.psi_conj = torch.from_numpy(np.ascontiguousarray(psi.astype(np.complex128))).to(dev)
        self.rchol = torch.from_numpy(np.ascontiguousarray(Lr[:, :N, :].reshape(X, N * M))).to(dev)
        rh1 = h1r[:N, :].astype(np.complex128)
        drh1 = Vr[:N, :].astype(np.complex128)
        self.rh1 = torch.from_numpy(np.ascontiguousarray(rh1)).to(dev)
        self.rh1_p = torch.from_numpy(np.ascontiguousarray(rh1 + drh1)).to(dev)
        self.rh1_m = torch.from_numpy(np.ascontiguousarray(rh1 - drh1)).to(dev)
        self.mf_dev = torch.from_numpy(self.mf.astype(np.complex128)).to(dev)
        self._buffers()
        # the trial's energy (the first energy estimate) and its derivative 2 sum_i V_ii
        gt = torch.from_numpy(np.ascontiguousarray(psi.T.astype(np.complex128))[None]).to(dev)
        self.e_trial = float(self._energies(gt, self.rh1, 1)[0].real)
        self.de_trial = 2.0 * float(np.trace(Vr[:N, :N]))
        self.h0shift = self.ecore - 0.5 * float(np.dot(self.mf.imag, self.mf.imag))

    def _buffers(self):
        W, M, N, X, dev = self.W, self.M, self.N, self.X, self.dev
        self.state = torch.zeros(W, 2 * M, N, dtype=C128, device=dev)
        self.state_tmp = torch.zeros_like(self.state)
        self.weight = torch.zeros(W, dtype=F64, device=dev)
        self.dweight = torch.zeros(W, dtype=F64, device=dev)
        self.g = torch.empty(W, N, M, dtype=C128, device=dev)
        self.dg = torch.empty_like(self.g)
        self.g2 = torch.empty_like(self.g)
        self.ld = [torch.empty(W, dtype=C128, device=dev) for _ in range(4)]  # logdet/dlogdet old, new
        self.vbias = torch.empty(W, X, dtype=C128, device=dev)
        self.dvbias = torch.empty_like(self.vbias)
        self.xs = torch.empty(X, W, dtype=C128, device=dev)
        self.dxs = torch.empty_like(self.xs)
        self.sums = [torch.empty(W, dtype=C128, device=dev) for _ in range(4)]  # fb, dfb, mfs, dmfs
        self.vhs = torch.empty(W, M, M, dtype=C128, device=dev)
        self.dvhs = torch.empty_like(self.vhs)
        self.vblk = torch.empty(W, 2 * M, 2 * M, dtype=C128, device=dev)
        self.x = torch.empty(W, X, dtype=F64, device=dev)
        self.src = torch.empty(W, dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        rows = lib().ipie_b200_exchange_rows(W, X, M, N)
        self.work = torch.empty(W * X + 2 * rows * W, dtype=C128, device=dev)

    # ------------------------------------------------------------------ pieces
    def _energies(self, g, rh1, W):
        """Local energies (W,) of half-rotated Green's functions g (W, N, M) (RHF, spin-doubled)."""
        X, M, N = self.X, self.M, self.N
        rows = lib().ipie_b200_exchange_rows(W, X, M, N)
        work = self.work if W == self.W else torch.empty(W * X + 2 * rows * W, dtype=C128, device=self.dev)
        out = torch.empty(W, 3, dtype=C128, device=self.dev)
        call("ipie_b200_local_energy_single_det_batch", 1, ptr(self.rchol), ptr(self.rchol), ptr(rh1), ptr(rh1),
             self.ecore, ptr(g), ptr(g), W, X, M, N, N, ptr(work), ptr(out), ptr(self.status), stream())
        return out[:, 0]

    def _gf(self, which):
        M, N = self.M, self.N
        lo, dlo = self.ld[2 * which], self.ld[2 * which + 1]
        st = self.state
        call("ipie_b200_ad_greens_function", ptr(st), ctypes_offset(st, M * N), 2 * M * N, self.W, M, N,
             ptr(self.psi_conj), ptr(self.g), ptr(self.dg), ptr(lo), ptr(dlo), ptr(self.status), stream())

    def _force_bias(self, g, out):
        call("ipie_b200_construct_force_bias_batch_single_det", ptr(self.rchol), ptr(self.rchol), ptr(g), ptr(g),
             self.W, self.X, self.M, self.N, self.N, ptr(out), stream())

    def step(self, x, e_est, de_est):
        """One step of ipie's AD propagator (``propagator.py:190-249``) with the derivatives."""
        W, M, N, X = self.W, self.M, self.N, self.X
        self._gf(0)
        self._force_bias(self.g, self.vbias)
        self._force_bias(self.dg, self.dvbias)
        self.x.copy_(x, non_blocking=True)
        fb, dfb, mfs, dmfs = self.sums
        call("ipie_b200_ad_field_shift", ptr(self.vbias), ptr(self.dvbias), ptr(self.x), ptr(self.mf_dev), W, X,
             self.sqrt_dt, 1.0, ptr(self.xs), ptr(self.dxs), ptr(fb), ptr(dfb), ptr(mfs), ptr(dmfs), stream())
        h = self.ham
        for xs, out in ((self.xs, self.vhs), (self.dxs, self.dvhs)):
            call("ipie_b200_construct_vhs", ptr(h.chol_packed), ptr(h.sym_idx_i), ptr(h.sym_idx_j), M, X, ptr(xs), W,
                 self.sqrt_dt, ptr(out), stream())
        call("ipie_b200_ad_block_vhs", ptr(self.vhs), ptr(self.dvhs), W, M, ptr(self.vblk), stream())
        call("ipie_b200_propagate_orbitals", ptr(self.vblk), ptr(self.eblk), self.lda, ptr(self.state),
             ptr(self.state_tmp), W, 2 * M, N, 6, 1, 1, stream())
        self.state, self.state_tmp = self.state_tmp, self.state
        self._gf(1)
        c = self.dt * (e_est - self.h0shift)
        dc = self.dt * de_est
        call("ipie_b200_ad_update_weight", W, ptr(self.ld[0]), ptr(self.ld[1]), ptr(self.ld[2]), ptr(self.ld[3]),
             ptr(fb), ptr(dfb), ptr(mfs), ptr(dmfs), c, dc, ptr(self.weight), ptr(self.dweight), ptr(self.status),
             stream())

    def block_energy(self):
        """(E, dE, sum w, sum dw) of the current walkers; self.g / self.dg hold their Green's function."""
        e = self._energies(self.g, self.rh1, self.W)
        call("ipie_b200_ad_axpy", ptr(self.g), ptr(self.dg), 1.0, self.g.numel(), ptr(self.g2), stream())
        ep = self._energies(self.g2, self.rh1, self.W)
        call("ipie_b200_ad_axpy", ptr(self.g), ptr(self.dg), -1.0, self.g.numel(), ptr(self.g2), stream())
        em = self._energies(self.g2, self.rh1, self.W)
        e1p = self._energies(self.g, self.rh1_p, self.W)
        e1m = self._energies(self.g, self.rh1_m, self.W)
        # the local energy is quadratic in G and linear in rh1: both differences are exact
        e, ep, em, e1p, e1m = (t.cpu().numpy() for t in (e, ep, em, e1p, e1m))
        de = 0.5 * (ep - em) + 0.5 * (e1p - e1m)
        w, dw = self.weight.cpu().numpy(), self.dweight.cpu().numpy()
        S, dS = w.sum(), dw.sum()
        E = float((np.sum(w * e) / S).real)
        dE = float(((np.sum(dw * e + w * de) / S) - np.sum(w * e) * dS / S ** 2).real)
        return E, dE, float(S), float(dS)

    def reortho(self):
        M, N = self.M, self.N
        call("ipie_b200_ad_reortho", ptr(self.state), ctypes_offset(self.state, M * N), 2 * M * N, self.W, M, N,
             ptr(self.status), stream())

    def reconfigure(self, idx):
        """ipie's stochastic reconfiguration copy (``rhf_walkers.py:30-49``): walker d <- idx[d];
        every weight becomes the mean of the rescaled weights (its derivative zero)."""
        w = self.weight.cpu().numpy()
        wn = w / w.sum() * w.size
        avg = np.cumsum(wn)[-1] / w.size
        self.src.copy_(torch.from_numpy(np.asarray(idx, dtype=np.int32)))
        M, N = self.M, self.N
        call("ipie_b200_ad_gather", ptr(self.src), self.W, 2 * M * N, ptr(self.state), ptr(self.state_tmp), stream())
        self.state, self.state_tmp = self.state_tmp, self.state
        self.weight.fill_(avg)
        self.dweight.zero_()

    @staticmethod
    def sr_indices(w, zeta):
        """The reconfiguration choice of ``rhf_walkers.py:30-49`` from weights and one uniform."""
        W = w.size
        wn = w / w.sum() * W
        cum = np.cumsum(wn)
        z = cum[-1] * (np.arange(W) + zeta) / W
        idx = np.searchsorted(cum, z, side="left")
        return np.where(idx < W, idx, 0)

    # ------------------------------------------------------------------ the block
    def ad_block(self, phi0, w0, draws, zetas, steps_per_block=10, ad_block_size=30, stabilize_freq=5,
                 pop_control_freq=5, sr_indices=None, e_est_blocks=None):
        """(E, dE/dlambda, W, dW/dlambda, phi, w) of one AD block (``adafqmc.py:222-298``).

        ``draws``: (steps, W, X) fields (host); ``zetas``: reconfiguration uniforms.  ``sr_indices`` (a
        list) receives the reconfiguration choices, or replays them when it holds arrays;
        ``e_est_blocks`` replaces the (detached) energy estimates taken after each block."""
        M, N = self.M, self.N
        init = np.zeros((self.W, 2 * M, N), dtype=np.complex128)
        init[:, :M] = phi0
        self.state.copy_(torch.from_numpy(init))
        self.weight.copy_(torch.from_numpy(np.asarray(w0, dtype=np.float64)))
        self.dweight.zero_()
        self.status.zero_()
        replay = sr_indices is not None and len(sr_indices) > 0
        record = None if (sr_indices is None or replay) else sr_indices
        e_est, de_est = self.e_trial, self.de_trial
        nb = ad_block_size // steps_per_block
        pinned = torch.empty(self.W, self.X, dtype=F64).pin_memory()
        out = []
        k = isr = 0
        for ib in range(nb):
            for i in range(steps_per_block):
                j = ib * steps_per_block + i
                if j % stabilize_freq == stabilize_freq - 1:
                    self.reortho()
                torch.cuda.current_stream().synchronize()  # the pinned field buffer is free again
                pinned.numpy()[...] = draws[k]
                self.step(pinned, e_est, de_est)
                k += 1
                if i == steps_per_block - 1:
                    blk = self.block_energy()
                    out.append(blk)
                    e_est, de_est = (blk[0] if e_est_blocks is None else e_est_blocks[ib]), 0.0
                if j % pop_control_freq == pop_control_freq - 1:
                    if replay:
                        idx = sr_indices[isr]
                    else:
                        idx = self.sr_indices(self.weight.cpu().numpy(), zetas[isr])
                        if record is not None:
                            record.append(idx)
                    isr += 1
                    self.reconfigure(idx)
        self.check_status()
        et, det, tw, dtw = (np.array(v) for v in zip(*out))
        self.last_block_energies = et
        Wt, dWt = tw.sum(), dtw.sum()
        E = float(np.sum(et * tw) / Wt)
        dE = float((np.sum(det * tw + et * dtw) / Wt) - np.sum(et * tw) * dWt / Wt ** 2)
        phi = self.state[:, :M].cpu().numpy()
        return E, dE, float(Wt), float(dWt), phi, self.weight.cpu().numpy()

    def check_status(self):
        s = int(self.status.item())
        if s:
            self.status.zero_()
            raise FloatingPointError(f"AD walk reported status bits {s:#x}")


def ctypes_offset(t, elements):
    """Device pointer ``elements`` complex entries into a contiguous complex128 tensor."""
    import ctypes

    return ctypes.c_void_p(t.data_ptr() + 16 * int(elements))


class BlockEnergyResponse(torch.autograd.Function):
    """E(lambda) of an AD block at lambda = 0 with its hand-written derivative: ``forward(lam, walk,
    args)`` runs :meth:`ADWalk.ad_block` (``args``: its keyword arguments) and returns the block
    energy as a 0-d tensor; ``backward`` returns grad_output x dE/dlambda for ``lam``.  The walk
    was built for the coupling's direction V; lam itself must be zero (the expansion point)."""

    @staticmethod
    def forward(ctx, lam, walk, args):
        if float(lam) != 0.0:
            raise ValueError("the walk is expanded at lambda = 0; build it with h1 + lambda V to move the point")
        E, dE, *_ = walk.ad_block(**args)
        ctx.dE = dE
        return torch.tensor(E, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_output):
        return grad_output * ctx.dE, None, None
