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


def test_multidet_propagation_matches_ipie():
    """Four phaseless steps with the particle-hole trial (ipie ``PhaselessGeneric.propagate_walkers``
    with the trial's Green's function, overlap and full-G force bias; numpy's draws seeded per
    step): the trial's 1-RDM and mean-field shift, every step's weights, overlaps and orbitals, and
    the final local energies against ipie's run (``tests/golden/multidet_prop_m14.npz``)."""
    from ipie_b200 import Generic, UHFWalkers
    from ipie_b200.estimators import local_energy_batch
    from ipie_b200.multidet import ParticleHole
    from ipie_b200.propagation import PhaselessGeneric

    f = load("multidet_prop_m14.npz")
    g = load("multidet_m14.npz")  # the same trial and starting walker
    s = synthetic.generate(14, (4, 3), 42, decay=30.0, seed=31, uhf=True, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = ParticleHole((g["ci"], list(g["occa"]), list(g["occb"])), (s.nup, s.ndown), s.nbasis)
    trial.build()
    trial.half_rotate(ham)
    assert np.max(np.abs(trial.G - f["G"])) < 1e-12
    W = f["weight0"].shape[0]
    walkers = UHFWalkers(g["init"], s.nup, s.ndown, s.nbasis, W)
    walkers.build(trial)
    assert rel(walkers.ovlp, f["ovlp_init"]) < TOL
    prop = PhaselessGeneric(0.005, rng="numpy")
    prop.build(ham, trial, walkers)
    assert np.max(np.abs(prop.mf_shift - f["mf_shift"])) < 1e-12 * np.max(np.abs(f["mf_shift"]))
    for step in range(4):
        np.random.seed(400 + step)
        prop.propagate_walkers(walkers, ham, trial, -3.0 if step else 0.0)
        torch.cuda.synchronize()
        walkers.check_status()
        assert rel(walkers.weight, f[f"weight{step}"]) < TOL
        assert rel(walkers.ovlp, f[f"ovlp{step}"]) < TOL
        assert rel(walkers.phia, f[f"phia{step}"]) < TOL
        assert rel(walkers.phib, f[f"phib{step}"]) < TOL
    energy = local_energy_batch(None, ham, walkers, trial)
    assert rel(energy, f["energy"]) < TOL


def test_multidet_afqmc_run_matches_ipie():
    """``AFQMC.build(...).run()`` with the particle-hole trial from given walkers (the perturbed
    reference; 2 blocks of 10 steps, 10 walkers, reortho and pair-branch population control every 5
    steps) against ipie's own run: block estimates and final walkers
    (``tests/golden/multidet_run_m14.npz``)."""
    from ipie_b200 import AFQMC, Generic, UHFWalkers
    from ipie_b200.multidet import ParticleHole

    f = load("multidet_run_m14.npz")
    g = load("multidet_m14.npz")
    s = synthetic.generate(14, (4, 3), 42, decay=30.0, seed=31, uhf=True, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = ParticleHole((g["ci"], list(g["occa"]), list(g["occb"])), (s.nup, s.ndown), s.nbasis)
    trial.build()
    trial.half_rotate(ham)
    walkers = UHFWalkers(g["init"], s.nup, s.ndown, s.nbasis, 10)
    walkers.build(trial)
    afqmc = AFQMC.build((s.nup, s.ndown), ham, trial, walkers=walkers, num_walkers=10, seed=5,
                        num_steps_per_block=10, num_blocks=2, timestep=0.005, stabilize_freq=5, pop_control_freq=5,
                        verbose=False)
    blocks = afqmc.run()
    ref = f["blocks"].real
    # rows: Weight, WeightFactor, HybridEnergy, ENumer, EDenom, ETotal, E1Body, E2Body
    assert blocks.shape == ref.shape
    for col in (0, 1, 3, 4, 5, 6, 7):
        assert rel(blocks[:, col], ref[:, col]) < TOL, col
    assert np.max(np.abs(blocks[:, 2] - ref[:, 2])) <= TOL * np.max(np.abs(ref[:, 5]))
    w = afqmc.walkers
    assert rel(w.weight, f["weight"]) < TOL
    assert rel(w.unscaled_weight, f["unscaled_weight"]) < TOL
    assert rel(w.ovlp, f["ovlp"]) < TOL
    assert rel(w.hybrid_energy, f["hybrid_energy"]) < TOL
    assert rel(w.phia, f["phia"]) < TOL
    assert rel(w.phib, f["phib"]) < TOL
