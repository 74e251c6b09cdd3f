"""Local energy and the energy estimator on the device.

Mirrors ipie's ``local_energy_single_det_uhf_batch`` / ``_rhf_batch`` /
``local_energy_single_det_batch_gpu`` (``estimators/local_energy_sd.py``),
``local_energy_batch`` (``estimators/local_energy_batch.py:36-75``) and
``EnergyEstimator`` (``estimators/energy.py:133-181``).  The exchange term
runs in the fused kernel (the intermediate T is never stored).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, lib, ptr, stream

C128 = torch.complex128


def _energy_work(walkers, hamiltonian, rhf):
    W, X, M = walkers.nwalkers, hamiltonian.nchol, walkers.nbasis
    rows = lib().ipie_b200_exchange_rows(W, X, M, walkers.nup)
    if not rhf and walkers.ndown > 0:
        rows += lib().ipie_b200_exchange_rows(W, X, M, walkers.ndown)
    need = W * X + rows * W
    buf = getattr(walkers, "_energy_work", None)
    if buf is None or buf.numel() < need:
        buf = torch.empty(need, dtype=C128, device=walkers.device)
        walkers._energy_work = buf
    return buf


def _local_energy_complex(hamiltonian, walkers, trial):
    """Complex-Cholesky UHF local energy (ipie ``local_energy_sd.py:406-460``): X1 = sum_s rchol_s . G_s and
    X2 = sum_s rcholbar_s . G_s give ecoul = X1 . X2 / 2, the exchange 1/2 sum_x tr(T1 T2) per spin runs as
    eight real exchange passes (polarisation), and the combine adds the one-body term."""
    # rows of the rotated operands: X, or 2X for a GHF trial with complex Cholesky vectors ([RA ; RB])
    W, X, M = walkers.nwalkers, getattr(trial, "_cplx_rows", hamiltonian.nchol), walkers.nbasis
    rows = max(lib().ipie_b200_exchange_rows(W, X, M, n) for n in (walkers.nup, walkers.ndown) if n > 0)
    need = 2 * W * X + rows * W + W
    buf = getattr(walkers, "_energy_work_cplx", None)
    if buf is None or buf.numel() < need:
        buf = torch.empty(need, dtype=C128, device=walkers.device)
        walkers._energy_work_cplx = buf
    x1, x2 = buf[: W * X], buf[W * X: 2 * W * X]
    part, exx = buf[2 * W * X: 2 * W * X + rows * W], buf[2 * W * X + rows * W: need]
    exx.zero_()
    for xv, name in ((x1, "chol"), (x2, "cholbar")):
        xv.zero_()
        for s_, g, n in (("a", walkers.Ghalfa, walkers.nup), ("b", walkers.Ghalfb, walkers.ndown)):
            if n == 0:
                continue
            re, im = trial._cplx[name + s_]
            call("ipie_b200_force_bias_complex", ptr(re), ptr(im), ptr(g), W, X, n * M, ptr(xv), X, 0, 1, stream())
    for s_, g, n in (("a", walkers.Ghalfa, walkers.nup), ("b", walkers.Ghalfb, walkers.ndown)):
        if n == 0:
            continue
        call("ipie_b200_exchange_complex", ptr(trial._cplx["pol" + s_]), ptr(g), W, X, M, n, ptr(part), ptr(exx), 1,
             stream())
    energy = torch.empty(W, 3, dtype=C128, device=walkers.device)
    call("ipie_b200_energy_complex", ptr(walkers.Ghalfa), ptr(walkers.Ghalfb), W, walkers.nup * M,
         walkers.ndown * M, ptr(trial._rH1a), ptr(trial._rH1b), hamiltonian.ecore, ptr(x1), ptr(x2), X, ptr(exx),
         ptr(energy), stream())
    return energy


def _local_energy(hamiltonian, walkers, trial, rhf):
    if not trial.half_rotated:
        raise RuntimeError("trial.half_rotate(hamiltonian) must run before computing local energies")
    if getattr(hamiltonian, "complex_chol", False) or getattr(trial, "complex_rotated", False):
        return _local_energy_complex(hamiltonian, walkers, trial)
    W = walkers.nwalkers
    work = _energy_work(walkers, hamiltonian, rhf)
    energy = torch.empty(W, 3, dtype=C128, device=walkers.device)
    call("ipie_b200_local_energy_single_det_batch", int(rhf), ptr(trial._rchola), ptr(trial._rcholb),
         ptr(trial._rH1a), ptr(trial._rH1b), hamiltonian.ecore, ptr(walkers.Ghalfa), ptr(walkers.Ghalfb), W,
         hamiltonian.nchol, walkers.nbasis, walkers.nup, walkers.ndown, ptr(work), ptr(energy),
         ptr(walkers.status), stream())
    return energy


def _mixed_energy_operands(trial, hamiltonian):
    """Padded FP16 head/remainder copies of the half-rotated Cholesky with their power-of-two
    scale, (hi, lo, scale) per spin (built once per trial)."""
    if getattr(trial, "_rpad", None) is not None:
        return trial._rpad
    X, M = hamiltonian.nchol, hamiltonian.nbasis
    Mp = (M + 7) // 8 * 8
    out = []
    for r, n in ((trial._rchola, trial.nalpha), (trial._rcholb, trial.nbeta)):
        if out and r is trial._rchola:
            out.append(out[0])
            continue
        NP = 8 if n <= 8 else 16 if n <= 16 else 32
        # head and remainder in one allocation: the products load both tiles with one copy
        hilo = torch.empty(2, X * NP * Mp, dtype=torch.float16, device=trial.device)
        hi, lo = hilo[0], hilo[1]
        scale = 1.0
        if n > 0:
            rmax = float(r.abs().max().item()) or 1.0
            scale = 2.0 ** (14 - int(np.ceil(np.log2(rmax))))
            call("ipie_b200_rchol_pad_split", ptr(r), X, n, M, scale, ptr(hi), ptr(lo), stream())
        out.append((hi, lo, scale))
    trial._rpad = out
    return out


def exchange_reference(trial, hamiltonian):
    """Trial Ghalf_s, the exchange gradient K_s there and raw_s = sum_x tr(T_s T_s) (FP64, once per trial).

    The mixed energy expands the exchange around the trial so that only the
    deviation G - G_T passes through the tensor cores.
    """
    ref = getattr(trial, "_exchange_ref", None)
    if ref is not None:
        return ref
    from .control_variate import exchange_gradient

    dev = trial.device
    X, M = hamiltonian.nchol, hamiltonian.nbasis
    gts, ks = [], []
    raw = torch.zeros(2, dtype=C128, device=dev)
    for s_, (gh, rchol, n) in enumerate(((trial.Ghalf[0], trial._rchola, trial.nalpha),
                                          (trial.Ghalf[1], trial._rcholb, trial.nbeta))):
        if n == 0:
            gts.append(None)
            ks.append(None)
            continue
        if s_ == 1 and rchol is trial._rchola and np.array_equal(np.asarray(gh), np.asarray(trial.Ghalf[0])):
            gts.append(gts[0])
            ks.append(ks[0])
            raw[1] = raw[0]
            continue
        g = torch.from_numpy(np.ascontiguousarray(np.asarray(gh).astype(np.complex128))).to(dev)
        gts.append(g)
        ks.append(exchange_gradient(rchol, g))
        rows = lib().ipie_b200_exchange_rows(1, X, M, n)
        part = torch.empty(rows, dtype=C128, device=dev)
        call("ipie_b200_exchange", ptr(rchol), ptr(g), 1, X, M, n, ptr(part), stream())
        raw[s_] = part.sum()
    trial._exchange_ref = (gts, ks, raw)
    return trial._exchange_ref


def local_energy_mixed(system, hamiltonian, walkers, trial, rhf=False, reference=True):
    """Mixed-precision local energy: the exchange as 3-pass TF32 tensor-core products
    (around the trial when ``reference``), Coulomb and one-body in FP64."""
    W, X, M = walkers.nwalkers, hamiltonian.nchol, hamiltonian.nbasis
    (ra_hi, ra_lo, ra_s), (rb_hi, rb_lo, rb_s) = _mixed_energy_operands(trial, hamiltonian)
    rows = 2
    for n in (walkers.nup, walkers.ndown):
        NP = 8 if n <= 8 else 16 if n <= 16 else 32
        rows += (X * NP + 127) // 128
    need = W * X + rows * W
    buf = getattr(walkers, "_energy_work_mixed", None)
    if buf is None or buf.numel() < need:
        buf = torch.empty(need, dtype=C128, device=walkers.device)
        walkers._energy_work_mixed = buf
        walkers._energy_gwork = torch.empty(2 * W * 2 * 32 * M, dtype=torch.float32, device=walkers.device)
    energy = torch.empty(W, 3, dtype=C128, device=walkers.device)
    gts, ks, raw = exchange_reference(trial, hamiltonian) if reference else ((None, None), (None, None), None)
    call("ipie_b200_local_energy_mixed", int(rhf), ptr(trial._rchola), ptr(trial._rcholb), ptr(ra_hi), ptr(ra_lo),
         ra_s, ptr(rb_hi), ptr(rb_lo), rb_s, ptr(trial._rH1a),
         ptr(trial._rH1b), hamiltonian.ecore, ptr(walkers.Ghalfa), ptr(walkers.Ghalfb), ptr(gts[0]), ptr(gts[1]),
         ptr(ks[0]), ptr(ks[1]), ptr(raw), W, X, M, walkers.nup,
         walkers.ndown, ptr(walkers._energy_gwork), ptr(buf), ptr(energy), ptr(walkers.status), stream())
    return energy


def local_energy_single_det_uhf_batch(system, hamiltonian, walkers, trial):
    """(W, 3) complex ``[e1b + e2b, e1b, e2b]`` (ipie ``local_energy_sd.py:358-403``)."""
    return _local_energy(hamiltonian, walkers, trial, rhf=False)


def local_energy_single_det_batch_gpu(system, hamiltonian, walkers, trial, max_mem=2.0):
    """ipie's GPU entry point (``local_energy_sd.py:987-1080``); same arithmetic as the UHF batch."""
    return _local_energy(hamiltonian, walkers, trial, rhf=False)


def local_energy_single_det_rhf_batch(system, hamiltonian, walkers, trial):
    """RHF form: spin-alpha only, doubled (ipie ``local_energy_sd.py:106-155``)."""
    return _local_energy(hamiltonian, walkers, trial, rhf=True)


def local_energy_batch(system, hamiltonian, walkers, trial):
    """Dispatch as ipie's ``local_energy_batch`` (``local_energy_batch.py:36-75``)."""
    if getattr(trial, "multidet", False):
        from .multidet import local_energy_multi_det_trial_wicks_batch_opt

        return local_energy_multi_det_trial_wicks_batch_opt(system, hamiltonian, walkers, trial)
    if walkers.rhf:
        return local_energy_single_det_rhf_batch(system, hamiltonian, walkers, trial)
    return local_energy_single_det_uhf_batch(system, hamiltonian, walkers, trial)


local_energy = local_energy_batch


class _OneWalker:
    """A one-walker view holding given half-rotated densities (for trial energies)."""

    def __init__(self, Ghalfa, Ghalfb, nbasis, device):
        self.nwalkers = 1
        self.nbasis = nbasis
        self.nup = Ghalfa.shape[0]
        self.ndown = Ghalfb.shape[0]
        self.device = device
        self.Ghalfa = torch.from_numpy(np.ascontiguousarray(Ghalfa[None].astype(np.complex128))).to(device)
        self.Ghalfb = torch.from_numpy(np.ascontiguousarray(Ghalfb[None].astype(np.complex128))).to(device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.rhf = False


def local_energy_of_density(hamiltonian, trial, Ghalfa, Ghalfb):
    """Local energy of one pair of half-rotated densities (e.g. the trial's own); complex (3,)."""
    w = _OneWalker(np.asarray(Ghalfa), np.asarray(Ghalfb), hamiltonian.nbasis, trial.device)
    return _local_energy(hamiltonian, w, trial, rhf=False)[0].cpu().numpy()


class EnergyEstimator:
    """Weighted energy sums of a block (ipie ``estimators/energy.py:133-181``)."""

    names = ["ENumer", "EDenom", "ETotal", "E1Body", "E2Body"]

    def __init__(self, system=None, ham=None, trial=None, filename=None, precision="fp64"):
        self.precision = precision
        self._data = {k: 0.0j for k in self.names}
        self._sums = None
        self.print_to_stdout = True
        self.ascii_filename = filename

    def compute_estimator(self, system=None, walkers=None, hamiltonian=None, trial=None):
        # ipie recomputes the Green's function here; it is skipped while the cached one is current
        if getattr(trial, "multidet", False) and self.precision == "mixed":
            raise NotImplementedError("the particle-hole trial's energy runs in FP64 (precision='fp64')")
        if not walkers.gf_current(trial):
            trial.calc_greens_function(walkers)
        if self.precision == "mixed" and not getattr(hamiltonian, "complex_chol", False) and not getattr(walkers, "ghf", False):
            energy = local_energy_mixed(system, hamiltonian, walkers, trial, rhf=walkers.rhf)
        else:
            energy = local_energy_batch(system, hamiltonian, walkers, trial)
        if self._sums is None:
            self._sums = torch.zeros(7, dtype=C128, device=walkers.device)
        call("ipie_b200_walker_sums", walkers.nwalkers, ptr(walkers.weight), None, None, ptr(energy), ptr(self._sums),
             0, stream())
        s = self._sums.cpu().numpy()
        self._data["ENumer"] = s[3].real
        self._data["EDenom"] = s[4].real
        self._data["E1Body"] = s[5].real
        self._data["E2Body"] = s[6].real
        self._data["ETotal"] = 0.0j
        self.energies = energy
        return self.data

    @property
    def data(self):
        return np.array([self._data[k] for k in self.names], dtype=np.complex128)

    def __getitem__(self, k):
        return self._data[k]

    def post_reduce_hook(self, data):
        data[2] = data[0] / data[1]
        data[3] = data[3] / data[1]
        data[4] = data[4] / data[1]
