"""Particle-hole multi-determinant trial on the GPU against ipie's Wick's-theorem Green's function,
overlap and local energy (``greens_function_multi_det_wicks_opt``,
``local_energy_multi_det_trial_wicks_batch_opt``), and against the oracle on another trial."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from ipie_b200 import synthetic  # noqa: E402
from tests._systems import load  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _objects(s, wfn, phia, phib):
    from ipie_b200 import Generic, UHFWalkers
    from ipie_b200.multidet import ParticleHole

    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = ParticleHole(wfn, (s.nup, s.ndown), s.nbasis)
    trial.build()
    trial.half_rotate(ham)
    W = phia.shape[0]
    walkers = UHFWalkers(trial.psi, s.nup, s.ndown, s.nbasis, W)
    walkers.phia = torch.from_numpy(np.ascontiguousarray(phia)).cuda()
    walkers.phib = torch.from_numpy(np.ascontiguousarray(phib)).cuda()
    return ham, trial, walkers


def test_multidet_matches_ipie_wicks():
    from ipie_b200.multidet import greens_function_multi_det_wicks_opt, local_energy_multi_det_trial_wicks_batch_opt

    f = load("multidet_m14.npz")
    s = synthetic.generate(14, (4, 3), 42, decay=30.0, seed=31, uhf=True, chol_scale="stable")
    ham, trial, walkers = _objects(s, (f["ci"], list(f["occa"]), list(f["occb"])), f["phia"], f["phib"])
    ovlp = greens_function_multi_det_wicks_opt(walkers, trial)
    energy = local_energy_multi_det_trial_wicks_batch_opt(None, ham, walkers, trial)
    torch.cuda.synchronize()
    walkers.check_status()
    assert rel(ovlp, f["ovlp"]) < TOL
    assert rel(walkers.Ga, f["Ga"]) < TOL
    assert rel(walkers.Gb, f["Gb"]) < TOL
    assert rel(energy, f["energy"]) < TOL
    # the overlap alone
    assert rel(trial.calc_overlap(walkers), f["ovlp"]) < TOL


def test_multidet_matches_oracle_larger():
    """M = 30, 6+5 electrons, 120 determinants with up to 5 holes per spin, 16 walkers."""
    import itertools

    from ipie_b200.multidet import greens_function_multi_det_wicks_opt, local_energy_multi_det_trial_wicks_batch_opt
    from oracle.multidet_oracle import multi_det

    s = synthetic.generate(30, (6, 5), 90, decay=30.0, seed=41, uhf=True, chol_scale="stable")
    M, na, nb = s.nbasis, s.nup, s.ndown
    rng = np.random.default_rng(42)
    occa = [np.arange(na)] + [np.sort(rng.choice(M, na, replace=False)) for _ in range(119)]
    occb = [np.arange(nb)] + [np.sort(rng.choice(M, nb, replace=False)) for _ in range(119)]
    ci = rng.normal(size=120) + 1j * rng.normal(size=120)
    W = 16
    base = np.eye(M)[:, :na], np.eye(M)[:, :nb]
    phia = base[0][None] + 0.3 * (rng.normal(size=(W, M, na)) + 1j * rng.normal(size=(W, M, na)))
    phib = base[1][None] + 0.3 * (rng.normal(size=(W, M, nb)) + 1j * rng.normal(size=(W, M, nb)))
    ham, trial, walkers = _objects(s, (ci, occa, occb), phia, phib)
    ovlp = greens_function_multi_det_wicks_opt(walkers, trial)
    energy = local_energy_multi_det_trial_wicks_batch_opt(None, ham, walkers, trial)
    tot, Ga, Gb, en = multi_det(ci, occa, occb, phia, phib, s.h1e, s.chol, s.ecore)
    assert rel(ovlp, tot) < TOL
    assert rel(walkers.Ga, Ga) < TOL
    assert rel(walkers.Gb, Gb) < TOL
    assert rel(energy, en) < TOL
    del itertools
