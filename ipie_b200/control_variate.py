"""Learned control variate for the exchange energy (no counterpart in ipie).

The exchange term dominates the cost of a local-energy evaluation
(O(W X N^2 M)).  Each walker's exchange term is predicted as

    c_w = b_w + MLP(f_w),

b_w the exact exchange term over the leading X/``lead_fraction`` Cholesky
vectors (the half-rotated vectors are ordered by decreasing weight, so these
carry most of it, at 1/``lead_fraction`` of the exact cost), and a small MLP
(16 -> 256 -> 256 -> 1, SiLU, bf16 weights, FP32 accumulation) learning the
remaining tail from cheap per-walker features (one-body and Coulomb energies,
Coulomb vector norms, overlap phase and magnitude, hybrid energy,
Green's-function norms, the first-order change of the exchange from its trial
value K_s.(G_s - G_T,s), b_w itself; see ``ipie_b200_cv_features``).  The
block estimate stays unbiased: the exact exchange is evaluated on a uniform
random subsample S of the walkers and

    sum_w w_w E_w  ~=  sum_w w_w (A_w - c_w)  -  (W/|S|) sum_{s in S} w_s (y_s - c_s)

with A_w the exchange-free energy, c_w the prediction and y_s the exact
exchange term.  The expectation over S equals the exact sum for any c, so a
poor network only costs variance; the exact kernel remains the reference.

Training runs entirely on the GPU through the library's own forward,
backward and Adam kernels (``ipie_b200_mlp_*``).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import call, lib, ptr, stream

F32, F64, C128 = torch.float32, torch.float64, torch.complex128
NFEAT = 16


def _param_count(F, H):
    return F * H + H + H * H + H + H + 1


class ExchangeControlVariate:
    """MLP predictor of the per-walker exchange term, trained on the GPU."""

    def __init__(self, hidden=256, device="cuda", seed=0):
        self.F, self.H = NFEAT, hidden
        self.device = torch.device(device)
        n = _param_count(self.F, self.H)
        self.n = n
        rng = np.random.default_rng(seed)
        theta = np.zeros(n, dtype=np.float32)
        o = 0
        for fan_in, fan_out in ((self.F, self.H), (self.H, self.H), (self.H, 1)):
            lim = math.sqrt(6.0 / (fan_in + fan_out))
            theta[o:o + fan_in * fan_out] = rng.uniform(-lim, lim, fan_in * fan_out)
            o += fan_in * fan_out + fan_out  # biases start at zero
        dev = self.device
        self.master = torch.from_numpy(theta).to(dev)
        self.wbf = self.master.to(torch.bfloat16)
        self.grad = torch.zeros(n, dtype=F32, device=dev)
        self.m = torch.zeros(n, dtype=F32, device=dev)
        self.v = torch.zeros(n, dtype=F32, device=dev)
        self.t = 0
        self.mu = torch.zeros(self.F, dtype=F32, device=dev)
        self.sigma = torch.ones(self.F, dtype=F32, device=dev)
        self.y_mean = 0.0
        self.y_scale = 1.0
        self.trained = False

    def clone(self):
        """An independent copy (weights, optimiser state and normalisation)."""
        import copy

        new = copy.copy(self)
        for name in ("master", "wbf", "grad", "m", "v", "mu", "sigma"):
            setattr(new, name, getattr(self, name).clone())
        new._rbuf_key = None
        return new

    # ------------------------------------------------------------ training
    def fit(self, feats, y, base=None, epochs=60, batch=4096, lr=2e-3, holdout=0.1, seed=0):
        """Train on (features, exchange term) pairs; returns the train/holdout MSE history (normalised units).

        ``feats``: (n, 16) float32 CUDA tensor of raw features; ``y``: (n,) float64/32 targets;
        ``base``: (n,) float64 linear term the network is added to (the network learns y - base).
        """
        n = feats.shape[0]
        if base is not None:
            y = y.double() - base.double()
        fm = feats.double().mean(0)
        fs = feats.double().std(0)
        fs = torch.where(fs > 0, fs, torch.ones_like(fs))
        self.mu.copy_(fm.float())
        self.sigma.copy_(fs.float())
        yd = y.double()
        self.y_mean = float(yd.mean())
        self.y_scale = float(yd.std()) or 1.0
        x = feats.float().contiguous().clone()
        call("ipie_b200_normalize_features", ptr(x), n, self.F, ptr(self.mu), ptr(self.sigma), stream())
        yt = ((yd - self.y_mean) / self.y_scale).float().contiguous()
        gen = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(n, generator=gen).to(self.device)
        nho = int(n * holdout)
        ho, tr = perm[:nho], perm[nho:]
        xh, yh = x[ho].contiguous(), yt[ho].contiguous()
        acts = torch.empty(4 * batch * self.H, dtype=F32, device=self.device)
        work = torch.empty(batch + 2 * batch * self.H, dtype=F32, device=self.device)
        out = torch.empty(batch, dtype=F32, device=self.device)
        loss = torch.zeros(1, dtype=F32, device=self.device)
        history = []
        for ep in range(epochs):
            order = tr[torch.randperm(tr.numel(), generator=gen).to(self.device)]
            loss.zero_()
            nb = 0
            for b0 in range(0, order.numel() - batch + 1, batch):
                idx = order[b0:b0 + batch]
                xb, yb = x[idx].contiguous(), yt[idx].contiguous()
                self._step(xb, yb, batch, acts, work, out, loss, lr)
                nb += 1
            tr_loss = float(loss.item()) / max(nb, 1)
            history.append((tr_loss, self.mse(xh, yh)))
        self.trained = True
        return history

    def _step(self, xb, yb, B, acts, work, out, loss, lr):
        call("ipie_b200_mlp_forward", ptr(xb), B, self.F, self.H, ptr(self.wbf), ptr(self.master), ptr(acts), ptr(out),
             stream())
        call("ipie_b200_mlp_backward", ptr(xb), ptr(yb), B, self.F, self.H, ptr(self.wbf), ptr(acts), ptr(out),
             ptr(self.grad), ptr(work), ptr(loss), stream())
        self.t += 1
        call("ipie_b200_mlp_adam", ptr(self.master), ptr(self.wbf), ptr(self.grad), ptr(self.m), ptr(self.v), self.n,
             float(lr), self.t, stream())

    def refine(self, feats, y, base, steps=4, batch=1024, lr=5e-4, seed=0):
        """A few Adam steps on new (features, exchange term, linear term) pairs, keeping the feature
        and target normalisation of :meth:`fit` (the online refit of the estimator)."""
        n = feats.shape[0]
        B = min(batch, n)
        x = feats.float().contiguous().clone()
        call("ipie_b200_normalize_features", ptr(x), n, self.F, ptr(self.mu), ptr(self.sigma), stream())
        yt = (((y.double() - base.double()) - self.y_mean) / self.y_scale).float().contiguous()
        key = ("refine", B)
        if getattr(self, "_rbuf_key", None) != key:
            self._rbuf = (torch.empty(4 * B * self.H, dtype=F32, device=self.device),
                          torch.empty(B + 2 * B * self.H, dtype=F32, device=self.device),
                          torch.empty(B, dtype=F32, device=self.device),
                          torch.zeros(1, dtype=F32, device=self.device))
            self._rbuf_key = key
        acts, work, out, loss = self._rbuf
        gen = torch.Generator(device="cpu").manual_seed(seed)
        for _ in range(steps):
            idx = torch.randperm(n, generator=gen)[:B].to(self.device, non_blocking=True)
            self._step(x[idx].contiguous(), yt[idx].contiguous(), B, acts, work, out, loss, lr)

    def mse(self, x_norm, y_norm):
        pred = self.forward_normalised(x_norm)
        return float(((pred - y_norm) ** 2).mean().item())

    def forward_normalised(self, x_norm):
        B = x_norm.shape[0]
        acts = torch.empty(4 * B * self.H, dtype=F32, device=self.device)
        out = torch.empty(B, dtype=F32, device=self.device)
        call("ipie_b200_mlp_forward", ptr(x_norm.contiguous()), B, self.F, self.H, ptr(self.wbf), ptr(self.master),
             ptr(acts), ptr(out), stream())
        return out

    def predict(self, feats, base=None):
        """Exchange-term prediction (fp32, physical units) for raw features (W, 16) and the linear term."""
        x = feats.float().contiguous().clone()
        call("ipie_b200_normalize_features", ptr(x), x.shape[0], self.F, ptr(self.mu), ptr(self.sigma), stream())
        out = self.forward_normalised(x)
        # physical units: c = base + mean + scale * out (a tiny elementwise map; kept as torch plumbing)
        c = out.double() * self.y_scale + self.y_mean
        if base is not None:
            c = c + base
        return c.float().contiguous()


# ----------------------------------------------------------------------------
# energy pieces used by the estimator and by training-data generation
# ----------------------------------------------------------------------------
def exchange_gradient(rchol, ghalf_trial):
    """K = d raw / d Ghalf at the trial, (N, M) complex, for raw = sum_x sum_ij T^x_ij T^x_ji.

    T^x_ij = sum_m L_x[i, m] G[j, m] with L_x the half-rotated Cholesky vector
    (rows of ``rchol`` (X, N*M)); dT^x_ab/dG[j, m] = delta_bj L_x[a, m] gives
    K[j, m] = 2 sum_x sum_a T^x_ja L_x[a, m] (holomorphic, no conjugation).  Done once per
    trial with two library GEMMs (torch plumbing; the per-walker contraction is a kernel).
    """
    N, M = ghalf_trial.shape
    L = rchol.reshape(-1, N, M).to(torch.complex128)
    T = torch.einsum("xim,jm->xij", L, ghalf_trial.to(torch.complex128))
    return (2.0 * torch.einsum("xja,xam->jm", T, L)).contiguous()


class EnergyParts:
    """Exchange-free energies, Coulomb vectors, exact exchange terms and features of a walker batch."""

    def __init__(self, hamiltonian, trial, walkers, lead_fraction=8, precision="fp64"):
        """``precision="mixed"``: exchange terms as 3-pass TF32 tensor-core products (the exact
        subsample expanded around the trial, as the mixed local energy does)."""
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision {precision!r}: 'fp64' or 'mixed'")
        if getattr(hamiltonian, "complex_chol", False):
            raise NotImplementedError("the energy control variate takes real Cholesky Hamiltonians")
        self.ham, self.trial = hamiltonian, trial
        self.precision = precision
        self.n_lead = max(1, hamiltonian.nchol // lead_fraction)
        W, X, M = walkers.nwalkers, hamiltonian.nchol, hamiltonian.nbasis
        dev = walkers.device
        self.xv = torch.empty(W, X, dtype=C128, device=dev)
        self.energy_noexx = torch.empty(W, 3, dtype=C128, device=dev)
        self.feat = torch.empty(W, NFEAT, dtype=F32, device=dev)
        self.base = torch.empty(W, dtype=F64, device=dev)  # exchange term over the leading vectors
        self.linear = torch.empty(W, dtype=F64, device=dev)  # first-order change from the trial value
        self.exx = torch.empty(W, dtype=C128, device=dev)
        from .estimators import exchange_reference

        self.ghalf_trial, self.kmat, self.raw_trial = exchange_reference(trial, hamiltonian)

    def compute(self, walkers, with_features=True):
        """Green's functions, exchange-free energy and features for every walker."""
        from .trial import force_bias_into

        ham, trial = self.ham, self.trial
        W, X, M = walkers.nwalkers, ham.nchol, ham.nbasis
        if not walkers.gf_current(trial):
            trial.calc_greens_function(walkers)
        force_bias_into(ham, walkers, trial, self.xv)  # Coulomb vector X_a + X_b
        rhf = bool(walkers.rhf)
        f1, fc = (2.0, 2.0) if rhf else (1.0, 0.5)
        gb = None if (rhf or walkers.ndown == 0) else walkers.Ghalfb
        call("ipie_b200_energy_combine", W, X, M, walkers.nup, walkers.ndown, ptr(walkers.Ghalfa), ptr(gb),
             ptr(trial._rH1a), ptr(trial._rH1b), ham.ecore, ptr(self.xv), None, 0, f1, fc, 0.0,
             ptr(self.energy_noexx), ptr(walkers.status), stream())
        if with_features:
            self.base.copy_(self.exchange_term(walkers, nchol=self.n_lead))
            call("ipie_b200_cv_features", W, X, walkers.nup, walkers.ndown, M, ptr(self.energy_noexx), ptr(self.xv),
                 ptr(walkers.ovlp), ptr(walkers.hybrid_energy), ptr(walkers.Ghalfa), ptr(walkers.Ghalfb),
                 ptr(self.ghalf_trial[0]), ptr(self.ghalf_trial[1]), ptr(self.kmat[0]), ptr(self.kmat[1]),
                 ptr(walkers.weight), ptr(self.base), ptr(self.feat), ptr(self.linear), stream())

    def exchange_term(self, walkers, idx=None, nchol=None):
        """Exact exchange term y = 1/2 Re(raw_a + raw_b) (W,) or on the subsample ``idx``; float64.

        ``nchol`` restricts the sum to the leading Cholesky vectors (rows of the half-rotated
        Cholesky are contiguous per vector, so the leading block is a prefix)."""
        ham = self.ham
        X, M = (nchol or ham.nchol), ham.nbasis
        S = walkers.nwalkers if idx is None else int(idx.numel())
        total = torch.zeros(S, dtype=F64, device=walkers.device)
        blocks = [(self.trial._rchola, walkers.Ghalfa, walkers.nup, 1.0 if walkers.spin_alias else 0.5)]
        if walkers.ndown > 0 and not walkers.spin_alias:
            blocks.append((self.trial._rcholb, walkers.Ghalfb, walkers.ndown, 0.5))
        if self.precision == "mixed":
            from .estimators import _mixed_energy_operands

            ops = _mixed_energy_operands(self.trial, ham)
        for s_, (rchol, gh, n, fac) in enumerate(blocks):
            if idx is not None:
                sub = torch.empty(S, n, M, dtype=C128, device=walkers.device)
                call("ipie_b200_gather_walkers", ptr(gh), ptr(idx), S, n * M, ptr(sub), stream())
            else:
                sub = gh
            if self.precision == "mixed":
                hi, lo, rs = ops[s_]
                NP = 8 if n <= 8 else 16 if n <= 16 else 32
                rows = (X * NP + 127) // 128 + 1
                part = torch.empty(rows * S, dtype=C128, device=walkers.device)
                gwork = torch.empty(2 * S * 2 * 32 * M, dtype=F32, device=walkers.device)
                exx = torch.empty(S, dtype=C128, device=walkers.device)
                ref = nchol is None  # the trial reference belongs to the full Cholesky sum
                call("ipie_b200_exchange_mixed", ptr(hi), ptr(lo), rs, ptr(sub),
                     ptr(self.ghalf_trial[s_]) if ref else None, ptr(self.kmat[s_]) if ref else None,
                     ptr(self.raw_trial[s_:s_ + 1]) if ref else None, S, X, M, n, ptr(gwork), ptr(part), ptr(exx),
                     ptr(walkers.status), stream())
                total += fac * exx.real
            else:
                rows = lib().ipie_b200_exchange_rows(S, X, M, n)
                part = torch.empty(rows * S, dtype=C128, device=walkers.device)
                call("ipie_b200_exchange", ptr(rchol), ptr(sub), S, X, M, n, ptr(part), stream())
                total += fac * part.view(rows, S).sum(0).real
        return total


class ControlVariateEnergyEstimator:
    """Block energy with the learned control variate and a uniform 1/``fraction`` exact subsample."""

    names = ["ENumer", "EDenom", "ETotal", "E1Body", "E2Body"]

    def __init__(self, cv, fraction=8, seed=11, precision="fp64", refit=True, buffer_blocks=8, refit_steps=2,
                 refit_lr=5e-4):
        """``refit``: after every block, the network takes ``refit_steps`` Adam steps on the exact
        subsamples of the last ``buffer_blocks`` blocks (this block's included), so that it follows
        walkers that drift away from its training data.  The prediction used for a block comes from
        a network that has seen earlier blocks only, so the estimate stays unbiased."""
        self.cv = cv
        self.fraction = fraction
        self.precision = precision
        self.rng = np.random.default_rng(seed)
        self.parts = None
        self._out = None
        self.last = {}
        self.refit, self.buffer_blocks, self.refit_steps, self.refit_lr = refit, buffer_blocks, refit_steps, refit_lr
        self._buffer = []
        self._calls = 0

    def compute_estimator(self, system=None, walkers=None, hamiltonian=None, trial=None):
        W = walkers.nwalkers
        S = max(1, W // self.fraction)
        if self.parts is None:
            self.parts = EnergyParts(hamiltonian, trial, walkers, precision=self.precision)
            self._out = torch.zeros(5, dtype=F64, device=walkers.device)
            self._idx_host = torch.empty(S, dtype=torch.int32).pin_memory()
            self._idx = torch.empty(S, dtype=torch.int32, device=walkers.device)
        p = self.parts
        p.compute(walkers)
        pred = self.cv.predict(p.feat, p.base)
        self._idx_host.numpy()[...] = np.sort(self.rng.choice(W, S, replace=False))
        self._idx.copy_(self._idx_host, non_blocking=True)
        idx = self._idx
        y_s = p.exchange_term(walkers, idx)
        call("ipie_b200_cv_sums", W, ptr(walkers.weight), ptr(p.energy_noexx), ptr(pred), S, ptr(idx), ptr(y_s),
             ptr(self._out), stream())
        o = self._out.cpu().numpy()
        if self.refit:
            il = idx.long()
            self._buffer.append((p.feat[il].clone(), y_s.clone(), p.base[il].clone()))
            self._buffer = self._buffer[-self.buffer_blocks:]
            f = torch.cat([b[0] for b in self._buffer])
            y = torch.cat([b[1] for b in self._buffer])
            b = torch.cat([b[2] for b in self._buffer])
            self._calls += 1
            self.cv.refine(f, y, b, steps=self.refit_steps, lr=self.refit_lr, seed=self._calls)
        numer = o[0] - o[1]
        self.last = {"cv": numer, "plain_subsample": o[3] - o[4], "denom": o[2]}
        self._data = np.array([numer, o[2], 0.0, 0.0, 0.0], dtype=np.complex128)
        return self.data

    @property
    def data(self):
        return self._data

    def post_reduce_hook(self, data):
        data[2] = data[0] / data[1]


def generate_training_data(afqmc, steps=100, first_step=1):
    """(features, exact exchange term, linear term) for every walker at each of ``steps`` driver steps.

    Runs the walk forward with the plain method (the AFQMC object's own
    propagator); returns float32 features (steps*W, 16), float64 targets and
    float64 linear terms.
    """
    w = afqmc.walkers
    parts = EnergyParts(afqmc.hamiltonian, afqmc.trial, w)
    feats, ys, bases = [], [], []
    for step in range(first_step, first_step + steps):
        afqmc.step(step)
        parts.compute(w)
        ys.append(parts.exchange_term(w))
        feats.append(parts.feat.clone())
        bases.append(parts.base.clone())
    return torch.cat(feats), torch.cat(ys), torch.cat(bases)


def subsample_variances(cv, parts, walkers, fraction=8, trials=64, seed=3):
    """Spread of the subsampled exchange estimate over random subsamples: with no control variate,
    with the full one (leading-vector term + network) and with the leading-vector term alone (the
    method without the network).

    Returns (std_without, std_with, exact, std_linear) for the weighted exchange sum of the current
    walkers.
    """
    parts.compute(walkers)
    y = parts.exchange_term(walkers)
    wt = walkers.weight.double()
    exact = float((wt * y).sum().item())
    pred = cv.predict(parts.feat, parts.base).double()
    lin = parts.base.double()
    full_c = float((wt * pred).sum().item())
    full_l = float((wt * lin).sum().item())
    rng = np.random.default_rng(seed)
    W = walkers.nwalkers
    S = max(1, W // fraction)
    plain, with_cv, with_lin = [], [], []
    for _ in range(trials):
        idx = torch.from_numpy(rng.choice(W, S, replace=False)).to(walkers.device)
        f = W / S
        plain.append(f * float((wt[idx] * y[idx]).sum().item()))
        with_cv.append(full_c + f * float((wt[idx] * (y[idx] - pred[idx])).sum().item()))
        with_lin.append(full_l + f * float((wt[idx] * (y[idx] - lin[idx])).sum().item()))
    return float(np.std(plain)), float(np.std(with_cv)), exact, float(np.std(with_lin))


def cv_estimator_error(cv, parts, walkers, fraction=8, trials=64, seed=5):
    """Error the subsampled estimate adds to the block energy of the current walkers, in mEh.

    Over ``trials`` random subsamples: the spread of (estimate - exact) / sum w with the
    control variate and without it (plain subsample), and the mean difference with its
    standard error (zero within it: the estimator is unbiased).
    """
    sd_plain, sd_cv, exact, sd_lin = subsample_variances(cv, parts, walkers, fraction=fraction, trials=trials,
                                                         seed=seed)
    y = parts.exchange_term(walkers)
    wt = walkers.weight.double()
    pred = cv.predict(parts.feat, parts.base).double()
    full_c = float((wt * pred).sum().item())
    rng = np.random.default_rng(seed + 1)
    W = walkers.nwalkers
    S = max(1, W // fraction)
    diffs = []
    for _ in range(trials):
        idx = torch.from_numpy(rng.choice(W, S, replace=False)).to(walkers.device)
        est = full_c + (W / S) * float((wt[idx] * (y[idx] - pred[idx])).sum().item())
        diffs.append(est - exact)
    wsum = float(wt.sum().item())
    d = np.asarray(diffs) / wsum * 1e3
    return {"noise_mEh": float(d.std()), "plain_subsample_noise_mEh": sd_plain / wsum * 1e3,
            "linear_term_only_noise_mEh": sd_lin / wsum * 1e3,
            "mean_diff_mEh": float(d.mean()), "mean_diff_stderr_mEh": float(d.std() / np.sqrt(trials)),
            "fraction": fraction, "trials": trials}
