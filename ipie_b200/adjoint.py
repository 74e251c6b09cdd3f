"""Hand-written adjoint of the local energy with respect to the one-body Hamiltonian.

``OneBodyLocalEnergy`` is a ``torch.autograd.Function``: its forward returns
every walker's local energy (real part) for a given one-body matrix ``h1``
(2, M, M) with the walkers held fixed, and its backward is the library's
adjoint kernel (``ipie_b200_onebody_adjoint``):

    dE_w/dh1_s[p, q] = Re G_s^w[p, q],   G_s^w = psi_s^* Ghalf_s^w,

so any scalar built from the energies differentiates through it with
autograd, e.g. the response dE/dlambda of ``h1 + lambda V`` and the
mixed-estimator one-body density matrix (upstream gradient w_w / sum w).
ipie's AD-AFQMC addon obtains the same derivative by autograd through its
torch local energy (``addons/adafqmc/estimators/estimator.py:4-23``).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib, ptr, stream

C128, F64 = torch.complex128, torch.float64


class LocalEnergyState:
    """Fixed walkers and the h1-independent part of their local energies."""

    def __init__(self, hamiltonian, trial, walkers, energy):
        self.ham, self.trial, self.walkers = hamiltonian, trial, walkers
        W, M = walkers.nwalkers, hamiltonian.nbasis
        dev = walkers.device
        # two-body part is independent of h1: E = e1b(h1) + ecore + e2b
        self.e2b = energy[:, 2].contiguous()
        self.rh1a = torch.empty(walkers.nup, M, dtype=C128, device=dev)
        self.rh1b = torch.empty(max(walkers.ndown, 1), M, dtype=C128, device=dev)
        self.e1 = torch.empty(W, 3, dtype=C128, device=dev)
        self.zero_xv = torch.zeros(W, 1, dtype=C128, device=dev)
        self.work = torch.empty(max(walkers.nup, walkers.ndown, 1) * M, dtype=C128, device=dev)


class OneBodyLocalEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, h1, state):
        w, trial, ham = state.walkers, state.trial, state.ham
        W, M = w.nwalkers, ham.nbasis
        h1 = h1.detach().to(F64).contiguous()
        call("ipie_b200_rotate_onebody", ptr(trial.psia_conj), ptr(h1[0]), M, w.nup, ptr(state.rh1a), stream())
        gb = None
        if w.ndown > 0:
            call("ipie_b200_rotate_onebody", ptr(trial.psib_conj), ptr(h1[1]), M, w.ndown, ptr(state.rh1b), stream())
            gb = w.Ghalfb
        # e1b only: no Coulomb vector (X = 1 zero column), no exchange rows, no ecore
        call("ipie_b200_energy_combine", W, 1, M, w.nup, w.ndown, ptr(w.Ghalfa), ptr(gb), ptr(state.rh1a),
             ptr(state.rh1b), 0.0, ptr(state.zero_xv), None, 0, 1.0, 0.0, 0.0, ptr(state.e1), ptr(w.status), stream())
        ctx.state = state
        return (state.e1[:, 1] + state.e2b).real + ham.ecore

    @staticmethod
    def backward(ctx, grad_e):
        state = ctx.state
        w, trial, ham = state.walkers, state.trial, state.ham
        M = ham.nbasis
        g = grad_e.detach().to(F64).contiguous()
        rdm = torch.empty(2, M, M, dtype=C128, device=w.device)
        call("ipie_b200_onebody_adjoint", w.nwalkers, M, w.nup, w.ndown, ptr(w.Ghalfa), ptr(w.Ghalfb),
             ptr(trial.psia_conj), ptr(trial.psib_conj), ptr(g), ptr(state.work), ptr(rdm), stream())
        return rdm.real.contiguous(), None


def local_energy_state(hamiltonian, trial, walkers):
    """Green's functions and full local energies of the current walkers (FP64 kernels)."""
    from .estimators import local_energy_single_det_uhf_batch

    trial.calc_greens_function(walkers)
    e = local_energy_single_det_uhf_batch(None, hamiltonian, walkers, trial)
    return LocalEnergyState(hamiltonian, trial, walkers, e)


def mixed_one_rdm(hamiltonian, trial, walkers):
    """Mixed-estimator one-body density matrix (2, M, M) real, as the gradient of the weighted energy."""
    state = local_energy_state(hamiltonian, trial, walkers)
    h1 = torch.from_numpy(np.ascontiguousarray(hamiltonian.H1)).to(walkers.device).requires_grad_(True)
    e = OneBodyLocalEnergy.apply(h1, state)
    wt = walkers.weight
    (e * wt).sum().div(wt.sum()).backward()
    return h1.grad


def energy_response(hamiltonian, trial, walkers, V):
    """dE/dlambda of the weighted mixed energy for h1 -> h1 + lambda V at fixed walkers, and the energy."""
    state = local_energy_state(hamiltonian, trial, walkers)
    lam = torch.zeros((), dtype=F64, device=walkers.device, requires_grad=True)
    h1 = torch.from_numpy(np.ascontiguousarray(hamiltonian.H1)).to(walkers.device)
    Vd = torch.as_tensor(V, dtype=F64, device=walkers.device)
    if Vd.dim() == 2:
        Vd = torch.stack([Vd, Vd])
    e = OneBodyLocalEnergy.apply(h1 + lam * Vd, state)
    wt = walkers.weight
    E = (e * wt).sum() / wt.sum()
    E.backward()
    return float(lam.grad.item()), float(E.item())


class LocalEnergyGreens(torch.autograd.Function):
    """Per-walker local energies (W,) complex as a function of the half-rotated Green's functions
    ``ghalfa`` (W, na, M) and ``ghalfb`` (W, nb, M) at fixed Hamiltonian and trial; the backward is
    the library's vector-Jacobian product (``ipie_b200_local_energy_vjp``).  ``rhf`` selects the
    doubled alpha-only energy (``ghalfb`` then gets no gradient).

    The energy is holomorphic in G, so for an upstream gradient g_w PyTorch's convention asks for
    g_w conj(dE_w/dG): the kernel's ebar * dE/dG is taken with ebar = conj(g) and conjugated back.
    ipie's AD-AFQMC addon differentiates the same energy with autograd through its torch
    implementation (``addons/adafqmc/estimators/estimator.py:4-23``)."""

    @staticmethod
    def forward(ctx, ghalfa, ghalfb, hamiltonian, trial, rhf=False):
        ga, gb = ghalfa.detach().contiguous(), ghalfb.detach().contiguous()
        W, na, M = ga.shape
        nb = gb.shape[1]
        X = hamiltonian.nchol
        dev = ga.device
        rows = lib().ipie_b200_exchange_rows(W, X, M, na)
        if not rhf and nb > 0:
            rows += lib().ipie_b200_exchange_rows(W, X, M, nb)
        work = torch.empty(W * X + rows * W, dtype=C128, device=dev)
        energy = torch.empty(W, 3, dtype=C128, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        call("ipie_b200_local_energy_single_det_batch", int(rhf), ptr(trial._rchola), ptr(trial._rcholb),
             ptr(trial._rH1a), ptr(trial._rH1b), hamiltonian.ecore, ptr(ga), ptr(gb), W, X, M, na, nb, ptr(work),
             ptr(energy), ptr(status), stream())
        ctx.save_for_backward(ga, gb)
        ctx.ham, ctx.trial, ctx.rhf = hamiltonian, trial, rhf
        return energy[:, 0].clone()

    @staticmethod
    def backward(ctx, grad_e):
        ga, gb = ctx.saved_tensors
        ham, trial, rhf = ctx.ham, ctx.trial, ctx.rhf
        W, na, M = ga.shape
        nb = gb.shape[1]
        X = ham.nchol
        ebar = grad_e.detach().to(C128).conj().resolve_conj().contiguous()
        work = torch.empty(W * X, dtype=C128, device=ga.device)
        gbara = torch.empty_like(ga)
        gbarb = torch.empty_like(gb) if not rhf and nb > 0 else gbara
        call("ipie_b200_local_energy_vjp", int(rhf), ptr(trial._rchola), ptr(trial._rcholb), ptr(trial._rH1a),
             ptr(trial._rH1b), ptr(ga), ptr(gb), W, X, M, na, nb, ptr(ebar), ptr(work), ptr(gbara), ptr(gbarb),
             stream())
        ga_grad = gbara.conj()
        gb_grad = None if (rhf or nb == 0) else gbarb.conj()
        return ga_grad, gb_grad, None, None, None
