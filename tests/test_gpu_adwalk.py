"""Response of the block energy through the walk (``ipie_b200.adwalk``) against ipie's AD-AFQMC
(torch autograd of ``ad_block``, same draws) and against central differences on the
nbasis-76 workload (M=76, 10+10 electrons, X=400, 512 walkers, 300 steps)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from ipie_b200 import synthetic  # noqa: E402
from tests._systems import checksum, load  # noqa: E402

pytestmark = pytest.mark.gpu


def test_ad_block_matches_ipie_autograd():
    from ipie_b200.adwalk import ADWalk

    f = load("ad_walk_m14.npz")
    s = synthetic.generate(14, (3, 3), 36, decay=30.0, seed=21, uhf=False, chol_scale="stable")
    np.testing.assert_allclose(checksum(s.chol), f["chol_checksum"], rtol=1e-13)
    L = s.chol.T.reshape(s.nchol, s.nbasis, s.nbasis)
    walk = ADWalk(s.h1e[0], L, s.ecore, f["V"], f["C"], s.nup, nwalkers=8)
    E, dE, W, dW, phi, w = walk.ad_block(f["phi0"], f["w0"], f["draws"], f["zetas"])
    assert abs(E - f["energy"]) <= 1e-10 * abs(f["energy"])
    assert abs(W - f["total_weight"]) <= 1e-10 * abs(f["total_weight"])
    assert abs(dE - f["dE_dlambda"]) <= 1e-9 * abs(f["dE_dlambda"])
    assert abs(dW - f["dW_dlambda"]) <= 1e-9 * abs(f["dW_dlambda"])
    np.testing.assert_allclose(w, f["final_weight"], rtol=1e-12)
    g = phi @ np.linalg.inv(phi[:, : s.nup, :])
    gr = f["final_phi"] @ np.linalg.inv(f["final_phi"][:, : s.nup, :])
    assert np.max(np.abs(g - gr)) <= 1e-10 * np.max(np.abs(gr))


def test_block_energy_response_autograd_function():
    from ipie_b200.adwalk import ADWalk, BlockEnergyResponse

    f = load("ad_walk_m14.npz")
    s = synthetic.generate(14, (3, 3), 36, decay=30.0, seed=21, uhf=False, chol_scale="stable")
    L = s.chol.T.reshape(s.nchol, s.nbasis, s.nbasis)
    walk = ADWalk(s.h1e[0], L, s.ecore, f["V"], f["C"], s.nup, nwalkers=8)
    lam = torch.zeros((), dtype=torch.float64, requires_grad=True)
    E = BlockEnergyResponse.apply(lam, walk, dict(phi0=f["phi0"], w0=f["w0"], draws=f["draws"], zetas=f["zetas"]))
    E.backward()
    assert abs(float(lam.grad) - f["dE_dlambda"]) <= 1e-9 * abs(f["dE_dlambda"])


class _Fields:
    """N(0, 1) fields of step k from a generator keyed by (seed, k): common to every run."""

    def __init__(self, seed, W, X):
        self.seed, self.W, self.X = seed, W, X

    def __getitem__(self, k):
        return np.random.default_rng([self.seed, k]).standard_normal((self.W, self.X))


def test_ad_block_central_difference_nbasis76():
    """dE/dlambda and dW/dlambda through 300 steps of 512 walkers against (f(+h) - f(-h)) / 2h,
    h = 1e-4, with common fields, common reconfiguration choices and the same detached energy
    estimates (the quantities ipie's derivative holds fixed)."""
    from ipie_b200.adwalk import ADWalk

    s = synthetic.workload("c4_rhf_m76", chol_scale="stable")
    M, N, X = s.nbasis, s.nup, s.nchol
    rng = np.random.default_rng(76)
    V = rng.normal(0.0, 0.1, size=(M, M))
    V = np.triu(V) + np.triu(V, 1).T
    q, _ = np.linalg.qr(np.hstack([s.psi[:, :N], rng.normal(size=(M, M - N))]))
    C = np.hstack([s.psi[:, :N], q[:, N:]])
    L = s.chol.T.reshape(X, M, M)
    W, steps, block = 512, 300, 25
    fields = _Fields(4, W, X)
    zetas = rng.uniform(size=steps // 5)
    phi0 = np.repeat(np.eye(M)[None, :, :N], W, axis=0).astype(np.complex128)
    w0 = np.ones(W)
    kw = dict(steps_per_block=block, ad_block_size=steps, stabilize_freq=5, pop_control_freq=5)
    walk = ADWalk(s.h1e[0], L, s.ecore, V, C, N, nwalkers=W)
    chosen = []
    E0, dE, W0, dW, _, _ = walk.ad_block(phi0, w0, fields, zetas, sr_indices=chosen, **kw)
    e_blocks = walk.last_block_energies
    assert len(chosen) == steps // 5 and np.isfinite(E0)
    h = 1e-4
    res = []
    for sign in (1, -1):
        wk = ADWalk(s.h1e[0] + sign * h * V, L, s.ecore, V, C, N, nwalkers=W)
        res.append(wk.ad_block(phi0, w0, fields, zetas, sr_indices=list(chosen), e_est_blocks=e_blocks, **kw))
        del wk
    fd_e = (res[0][0] - res[1][0]) / (2 * h)
    fd_w = (res[0][2] - res[1][2]) / (2 * h)
    assert abs(fd_e - dE) <= 1e-5 * max(abs(dE), 1e-2), (fd_e, dE)
    assert abs(fd_w - dW) <= 1e-5 * max(abs(dW), 1e-2 * abs(W0)), (fd_w, dW)
