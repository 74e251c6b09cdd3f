"""Parity of the complex-Cholesky walker step (ipie's ``GenericComplexChol`` path) with ipie's
outputs and with the CPU oracle.

``complex_uhf_m20.npz`` holds ipie's own set-up, kernel outputs and a three-step walk
(``tests/golden/make_golden.py``); the larger cases, a complex trial among them, compare with
``oracle/complex_chol_oracle.py`` on identical numpy draws.  Tolerances as for the real FP64
form: 1e-12 for single contractions, 1e-10 for weights, overlaps, orbitals and energies after
steps.  Every call goes through the C ABI (``libipie_b200.so``).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import afqmc_oracle as O  # noqa: E402
from oracle.complex_chol_oracle import ComplexSystem  # noqa: E402
from tests._systems import load  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def complex_system(M=20, nelec=(4, 3), X=60, seed=3, complex_trial=False):
    from ipie_b200 import synthetic

    s = synthetic.generate_complex(M, nelec, X, decay=30.0, seed=seed, uhf=True)
    if complex_trial:
        # a unitary rotation among the occupied orbitals of each spin with complex phases
        rng = np.random.default_rng(seed + 77)
        psi = s.psi.astype(np.complex128)
        na = s.nup
        for lo, hi in ((0, na), (na, psi.shape[1])):
            n = hi - lo
            q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
            psi[:, lo:hi] = psi[:, lo:hi] @ q
        s.psi = psi
        s.init = psi.copy()
    return s


def oracle_of(s, dt=0.005):
    return ComplexSystem(nbasis=s.nbasis, nup=s.nup, ndown=s.ndown, h1e=s.h1e, chol=s.chol, ecore=s.ecore,
                         psi=s.psi, dt=dt).build()


def gpu_objects(s, W, dt=0.005):
    from ipie_b200 import Generic, SingleDet, UHFWalkers
    from ipie_b200.hamiltonian import GenericComplexChol
    from ipie_b200.propagation import PhaselessGeneric

    ham = Generic(s.h1e, s.chol, s.ecore)
    assert isinstance(ham, GenericComplexChol) and ham.nfields == 2 * s.nchol
    trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis)
    trial.half_rotate(ham)
    walkers = UHFWalkers(s.init, s.nup, s.ndown, s.nbasis, W)
    walkers.build(trial)
    prop = PhaselessGeneric(dt)
    prop.build(ham, trial, walkers)
    return ham, trial, walkers, prop


def test_complex_kernels_match_ipie():
    from ipie_b200.estimators import local_energy_single_det_uhf_batch

    f = load("complex_uhf_m20.npz")
    s = complex_system()
    W = f["phia_in"].shape[0]
    ham, trial, walkers, prop = gpu_objects(s, W)
    assert rel(ham.h1e_mod, f["h1e_mod"]) < 1e-13
    for k in ("rchola", "rcholb", "rcholbara", "rcholbarb", "rAa", "rAb", "rBa", "rBb", "rH1a", "rH1b"):
        assert rel(getattr(trial, "_" + k), f[k]) < 1e-13, k
    assert rel(prop.mf_shift, f["mf_shift"]) < 1e-12
    assert rel(prop.expH1, f["expH1"]) < 1e-12
    walkers.phia = dev(f["phia_in"])
    walkers.phib = dev(f["phib_in"])
    ovlp = trial.calc_greens_function(walkers)
    assert rel(ovlp, f["ovlp"]) < 1e-11
    assert rel(walkers.Ghalfa, f["Ghalfa"]) < 1e-11
    assert rel(walkers.Ghalfb, f["Ghalfb"]) < 1e-11
    vbias = trial.calc_force_bias(ham, walkers)
    assert vbias.shape == (W, 2 * s.nchol)
    assert rel(vbias, f["vbias"]) < 1e-12
    vhs = prop.construct_VHS(ham, dev(f["xshifted"]))
    assert rel(vhs, f["VHS"]) < 1e-13
    e = local_energy_single_det_uhf_batch(None, ham, walkers, trial)
    assert rel(e, f["energy_uhf"]) < 1e-11
    walkers.check_status()


@pytest.mark.parametrize("fused", [True, False])
def test_complex_steps_match_ipie(fused):
    """Three steps from ipie's perturbed walkers with numpy's stream seeded as ipie's walk was."""
    f = load("complex_uhf_m20.npz")
    s = complex_system()
    W = f["phia_in"].shape[0]
    ham, trial, walkers, prop = gpu_objects(s, W)
    prop.fused = fused
    walkers.phia = dev(f["phia_in"])
    walkers.phib = dev(f["phib_in"])
    walkers.ovlp = trial.calc_greens_function(walkers)
    np.random.seed(21)
    for step in range(3):
        prop.propagate_walkers(walkers, ham, trial, -7.0 if step else 0.0)
    assert rel(walkers.weight, f["walk_weight"]) < TOL
    assert rel(walkers.ovlp, f["walk_ovlp"]) < TOL
    assert rel(walkers.phia, f["walk_phia"]) < TOL
    assert rel(walkers.phib, f["walk_phib"]) < TOL
    assert rel(walkers.hybrid_energy, f["walk_hybrid_energy"]) < TOL
    walkers.check_status()


@pytest.mark.parametrize("M,nelec,X,W,complex_trial", [(26, (5, 3), 120, 16, False), (26, (5, 5), 90, 8, True),
                                                       (40, (8, 6), 160, 12, True)])
def test_complex_step_and_energy_match_oracle(M, nelec, X, W, complex_trial):
    from ipie_b200.estimators import local_energy_single_det_uhf_batch

    s = complex_system(M, nelec, X, seed=4, complex_trial=complex_trial)
    S = oracle_of(s)
    ham, trial, walkers, prop = gpu_objects(s, W)
    assert rel(prop.expH1, S.expH1) < 1e-12
    rng = np.random.default_rng(9)
    pa = s.init[:, : s.nup][None] + 0.15 * (rng.normal(size=(W, M, s.nup)) + 1j * rng.normal(size=(W, M, s.nup)))
    pb = s.init[:, s.nup:][None] + 0.15 * (rng.normal(size=(W, M, s.ndown)) + 1j * rng.normal(size=(W, M, s.ndown)))
    walkers.phia, walkers.phib = dev(pa), dev(pb)
    ow = O.Walkers.from_initial(s.init, s.nup, W)
    ow.phia, ow.phib = pa.copy(), pb.copy()
    walkers.ovlp = trial.calc_greens_function(walkers)
    ow.ovlp = O.greens_function(S, ow)
    assert rel(walkers.ovlp, ow.ovlp) < 1e-11
    assert rel(trial.calc_force_bias(ham, walkers), S.vbias(ow)) < 1e-12
    e_gpu = local_energy_single_det_uhf_batch(None, ham, walkers, trial)
    assert rel(e_gpu, S.local_energy(ow)) < 1e-11
    for step in range(3):
        np.random.seed(200 + step)
        prop.propagate_walkers(walkers, ham, trial, 0.0 if step == 0 else -2.0)
        np.random.seed(200 + step)
        O.propagate_walkers(S, ow, 0.0 if step == 0 else -2.0)
        if step == 1:
            walkers.reortho()
            O.reortho(S, ow)
    assert rel(walkers.weight, ow.weight) < TOL
    assert rel(walkers.ovlp, ow.ovlp) < TOL
    assert rel(walkers.hybrid_energy, ow.hybrid_energy) < TOL
    assert rel(walkers.phia, ow.phia) < TOL
    assert rel(walkers.phib, ow.phib) < TOL
    trial.calc_greens_function(walkers)
    O.greens_function(S, ow)
    assert rel(local_energy_single_det_uhf_batch(None, ham, walkers, trial), S.local_energy(ow)) < TOL
    walkers.check_status()


def test_complex_afqmc_run_matches_oracle():
    """``AFQMC.build(...).run()`` on a complex Cholesky Hamiltonian against the oracle's driver."""
    from ipie_b200 import AFQMC, Generic, SingleDet

    s = complex_system(20, (4, 3), 60, seed=3)
    S = oracle_of(s)
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis)
    trial.half_rotate(ham)
    W, nb = 10, 2
    afqmc = AFQMC.build((s.nup, s.ndown), ham, trial, num_walkers=W, seed=5, num_steps_per_block=25, num_blocks=nb,
                        timestep=0.005, stabilize_freq=5, pop_control_freq=5, verbose=False)
    blocks = afqmc.run()
    ow = O.Walkers.from_initial(S.psi, S.nup, W)
    ref = O.run_afqmc(S, ow, num_blocks=nb, seed=5)
    cols = ("Weight", "WeightFactor", "HybridEnergy", "ENumer", "EDenom", "ETotal", "E1Body", "E2Body")
    ref = np.array([[r[c] for c in cols] for r in ref])
    assert blocks.shape == ref.shape
    for col in (0, 1, 3, 4, 5, 6, 7):
        assert rel(blocks[:, col], ref[:, col]) < TOL, cols[col]
    w = afqmc.walkers
    assert rel(w.weight, ow.weight) < TOL
    assert rel(w.phia, ow.phia) < TOL
    assert rel(w.phib, ow.phib) < TOL


def test_complex_mixed_form_refuses():
    from ipie_b200.propagation import PhaselessGeneric

    s = complex_system()
    ham, trial, walkers, _ = gpu_objects(s, 4)
    prop = PhaselessGeneric(0.005, precision="mixed")
    with pytest.raises(NotImplementedError):
        prop.build(ham, trial, walkers)
