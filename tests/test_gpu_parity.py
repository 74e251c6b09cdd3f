"""Parity of the CUDA walker step with ipie's outputs and with the CPU oracle.

Tolerance: 1e-10 relative (max-abs error over max-abs value) in weights,
overlaps and local energies, the bar for the plain FP64 form; kernels that are
a single contraction are held to 1e-12.  Every call goes through the C ABI
(``libipie_b200.so``).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import afqmc_oracle as O  # noqa: E402
from tests._systems import RUN_PARAMS, compare_walkers, fixture_system, load, oracle_system  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_objects(s, nwalkers, dt=0.005, rng="numpy"):
    from ipie_b200 import Generic, SingleDet, UHFWalkers
    from ipie_b200.propagation import PhaselessGeneric

    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis)
    trial.half_rotate(ham)
    walkers = UHFWalkers(s.init, s.nup, s.ndown, s.nbasis, nwalkers)
    walkers.build(trial)
    prop = PhaselessGeneric(dt, rng=rng)
    prop.build(ham, trial, walkers)
    return ham, trial, walkers, prop


KERNEL_FIXTURES = ["kernels_rhf_m26.npz", "kernels_uhf_m30.npz"]


@pytest.mark.parametrize("name", KERNEL_FIXTURES)
def test_kernels_match_ipie(name):
    from ipie_b200.estimators import local_energy_single_det_rhf_batch, local_energy_single_det_uhf_batch

    f = load(name)
    s = fixture_system(name)
    W = f["phia_in"].shape[0]
    ham, trial, walkers, prop = gpu_objects(s, W)
    assert rel(prop.mf_shift, f["mf_shift"]) < 1e-12
    assert rel(prop.expH1, f["expH1"]) < 1e-12
    assert rel(trial._rchola, f["rchola"]) < 1e-13
    walkers.phia = dev(f["phia_in"])
    walkers.phib = dev(f["phib_in"])
    ovlp = trial.calc_greens_function(walkers)
    assert rel(ovlp, f["ovlp"]) < 1e-11
    assert rel(walkers.Ghalfa, f["Ghalfa"]) < 1e-11
    assert rel(walkers.Ghalfb, f["Ghalfb"]) < 1e-11
    vbias = trial.calc_force_bias(ham, walkers)
    assert rel(vbias, f["vbias"]) < 1e-12
    vhs = prop.construct_VHS(ham, dev(f["xshifted"]))
    assert rel(vhs, f["VHS"]) < 1e-13
    out = torch.empty_like(walkers.phia)
    work = torch.empty(2 * walkers.phia.numel(), dtype=torch.complex128, device="cuda")
    from ipie_b200._lib import call, ptr, stream

    vhs_d = dev(f["VHS"])
    call("ipie_b200_apply_exponential_batch", ptr(vhs_d), ptr(walkers.phia), ptr(out), ptr(work), W,
         s.nbasis, s.nup, 6, stream())
    assert rel(out, f["phia_exp"]) < 1e-13
    call("ipie_b200_propagate_one_body", ptr(prop.expH1_dev[0]), int(prop.expH1_complex), ptr(walkers.phia), ptr(out),
         W, s.nbasis, s.nup, stream())
    assert rel(out, f["phia_onebody"]) < 1e-13
    assert rel(trial.calc_overlap(walkers), f["ovlp_overlap"]) < 1e-11
    e = local_energy_single_det_uhf_batch(None, ham, walkers, trial)
    assert rel(e, f["energy_uhf"]) < 1e-11
    if "energy_rhf" in f:
        e = local_energy_single_det_rhf_batch(None, ham, walkers, trial)
        assert rel(e, f["energy_rhf"]) < 1e-11
    walkers.ovlp = ovlp.clone()
    detR = walkers.reortho()
    assert rel(walkers.phia, f["reortho_phia"]) < 1e-11
    assert rel(walkers.phib, f["reortho_phib"]) < 1e-11
    assert rel(detR, f["reortho_detR"]) < 1e-12
    assert rel(walkers.ovlp, f["reortho_ovlp"]) < 1e-11
    walkers.check_status()


@pytest.mark.parametrize("name", sorted(RUN_PARAMS))
def test_afqmc_run_matches_ipie(name):
    """``AFQMC.build(...).run()`` against ipie's own run: block energies and final walkers."""
    from ipie_b200 import AFQMC, Generic, SingleDet

    f = load(name)
    p = RUN_PARAMS[name]
    s = fixture_system(name)
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis)
    trial.half_rotate(ham)
    afqmc = AFQMC.build((s.nup, s.ndown), ham, trial, num_walkers=p["nwalkers"], seed=p["seed"],
                        num_steps_per_block=p["steps"], num_blocks=p["num_blocks"], timestep=0.005, stabilize_freq=5,
                        pop_control_freq=5, verbose=False)
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
    compare_walkers(rel, w.phia.cpu().numpy(), w.phib.cpu().numpy(), f, TOL)
    if "energy" in f:
        # local energies of the final walkers (ipie's estimator call on them)
        from ipie_b200.estimators import local_energy_single_det_uhf_batch

        trial.calc_greens_function(w)
        e = local_energy_single_det_uhf_batch(None, ham, w, trial)
        assert rel(e, f["energy"]) < TOL


def test_known_answer_pair_branch():
    """ipie ``walkers/tests/test_population_control.py:30-81`` on the CUDA path."""
    from ipie_b200 import Generic, PopController, SingleDet, UHFWalkers
    from ipie_b200.propagation import PhaselessGeneric

    f = load("known_answers.npz")
    M = f["pb_h1e"].shape[-1]
    ham = Generic(f["pb_h1e"], f["pb_chol"], 0.0)
    trial = SingleDet(f["pb_psi"], (5, 5), M)
    trial.half_rotate(ham)
    walkers = UHFWalkers(f["pb_init"], 5, 5, M, 10)
    walkers.build(trial)
    np.random.seed(7)
    prop = PhaselessGeneric(0.005)
    prop.build(ham, trial, walkers)
    pc = PopController(10, 10)
    eshift = complex(f["pb_eshift"]).real
    for _ in range(10):
        prop.propagate_walkers(walkers, ham, trial, eshift)
        walkers.reortho()
        pc.pop_control(walkers)
        trial.calc_greens_function(walkers)
    wt = walkers.weight.cpu().numpy()
    assert wt[0] == pytest.approx(0.2571750688329709, rel=1e-9)
    assert wt[1] == pytest.approx(1.0843219322894988, rel=1e-9)
    assert wt[2] == pytest.approx(0.8338283613093604, rel=1e-9)
    assert complex(walkers.phia[9, 0, 0].item()) == pytest.approx(-0.0005573508035052743 + 0.12432250308987346j,
                                                                 rel=1e-9)


def _known_answer_walk_gpu(method):
    """ipie's ``build_test_case_handlers_mpi`` loop (``utils/testing.py:465-528``) on the CUDA path."""
    from ipie_b200 import Generic, PopController, SingleDet, UHFWalkers
    from ipie_b200.propagation import PhaselessGeneric

    f = load("known_answers.npz")
    M = f["pb_h1e"].shape[-1]
    ham = Generic(f["pb_h1e"], f["pb_chol"], 0.0)
    trial = SingleDet(f["pb_psi"], (5, 5), M)
    trial.half_rotate(ham)
    walkers = UHFWalkers(f["pb_init"], 5, 5, M, 10)
    walkers.build(trial)
    np.random.seed(7)
    prop = PhaselessGeneric(0.005)
    prop.build(ham, trial, walkers)
    pc = PopController(10, 10, pop_control_method=method, reconfiguration_freq=3)
    eshift = complex(f["pb_eshift"]).real
    for _ in range(10):
        prop.propagate_walkers(walkers, ham, trial, eshift)
        walkers.reortho()
        pc.pop_control(walkers)
        trial.calc_greens_function(walkers)
    walkers.check_status()
    return walkers


def test_known_answer_comb():
    """ipie ``walkers/tests/test_population_control.py:84-142`` (comb) on the CUDA path."""
    walkers = _known_answer_walk_gpu("comb")
    assert complex(walkers.phia[9, 0, 0].item()) == pytest.approx(-0.0597200851442905 - 0.002353281222663805j,
                                                                 rel=1e-9)
    f = load("pop_control.npz")
    assert rel(walkers.weight, f["comb_weight"]) < 1e-12
    assert rel(walkers.unscaled_weight, f["comb_unscaled_weight"]) < 1e-9
    assert rel(walkers.phia, f["comb_phia"]) < 1e-9
    assert rel(walkers.phib, f["comb_phib"]) < 1e-9


def test_stochastic_reconfiguration_matches_ipie():
    """ipie's stochastic reconfiguration every 3rd call (``walkers/pop_controller.py:432-475``)."""
    walkers = _known_answer_walk_gpu("stochastic_reconfiguration")
    f = load("pop_control.npz")
    assert rel(walkers.weight, f["sr_weight"]) < 1e-9
    assert rel(walkers.unscaled_weight, f["sr_unscaled_weight"]) < 1e-9
    assert rel(walkers.phia, f["sr_phia"]) < 1e-9
    assert rel(walkers.phib, f["sr_phib"]) < 1e-9
    # the particle-hole trial of ipie's builder scales every overlap by its determinant coefficient
    ratio = walkers.ovlp.cpu().numpy() / f["sr_ovlp"]
    assert np.max(np.abs(ratio - ratio[0])) < 1e-9 * abs(ratio[0])


def test_known_answer_local_energy():
    """ipie ``estimators/tests/test_generic.py:51-69`` on the CUDA path."""
    from ipie_b200 import Generic, SingleDet

    f = load("known_answers.npz")
    M = f["le_h1e"].shape[-1]
    ham = Generic(f["le_h1e"], f["le_chol"], float(f["le_ecore"]))
    trial = SingleDet(f["le_psi"], (4, 2), M)
    trial.half_rotate(ham)
    e = trial.calculate_energy(None, ham)
    assert e[0].real == pytest.approx(20.6826247016273, rel=1e-11)
    assert e[1].real == pytest.approx(23.0173528796140, rel=1e-11)
    assert e[2].real == pytest.approx(-2.3347281779866, rel=1e-11)


def test_known_answer_energy_estimator():
    """ipie ``estimators/tests/test_estimators.py:27-41`` on the CUDA path."""
    from ipie_b200 import EnergyEstimator, Generic, SingleDet, UHFWalkers

    f = load("known_answers.npz")
    ham = Generic(f["ee_h1e"], f["ee_chol"], 0.0)
    trial = SingleDet(f["ee_psi"], (8, 8), 10)
    trial.half_rotated = True
    trial._rchola, trial._rcholb = dev(f["ee_rchola"]), dev(f["ee_rcholb"])
    trial._rH1a = dev(f["ee_rH1a"].astype(np.complex128))
    trial._rH1b = dev(f["ee_rH1b"].astype(np.complex128))
    walkers = UHFWalkers(f["ee_psi"], 8, 8, 10, 10)
    walkers.phia, walkers.phib = dev(f["ee_phia"]), dev(f["ee_phib"])
    est = EnergyEstimator()
    est.compute_estimator(None, walkers, ham, trial)
    assert est["ENumer"] == pytest.approx(-754.0373585215561, rel=1e-11)
    d = est.data.copy()
    est.post_reduce_hook(d)
    assert d[2].real == pytest.approx(-75.40373585215562, rel=1e-11)


# --------------------------------------------------------------------------
# Against the oracle at other shapes (odd sizes, ndown = 0, one walker, N = 32)
# --------------------------------------------------------------------------
SHAPES = [
    # (M, (na, nb), X, W, uhf)
    (17, (3, 2), 41, 5, True),
    (26, (5, 5), 120, 1, False),
    (21, (4, 0), 33, 7, True),
    (48, (1, 1), 64, 33, True),
    (70, (32, 32), 150, 6, False),
    (108, (15, 15), 600, 24, True),
]


def _walker_pert(s, W, seed):
    rng = np.random.default_rng(seed)
    pa = s.init[:, : s.nup][None] + 0.15 * (rng.normal(size=(W, s.nbasis, s.nup)) + 1j * rng.normal(size=(W, s.nbasis, s.nup)))
    pb = s.init[:, s.nup:][None] + 0.15 * (rng.normal(size=(W, s.nbasis, s.ndown)) + 1j * rng.normal(size=(W, s.nbasis, s.ndown)))
    return pa, pb


@pytest.mark.parametrize("M,nelec,X,W,uhf", SHAPES)
def test_step_and_energy_match_oracle(M, nelec, X, W, uhf):
    from ipie_b200 import synthetic
    from ipie_b200.estimators import local_energy_single_det_uhf_batch

    s = synthetic.generate(M, nelec, X, decay=30.0, seed=3, uhf=uhf, chol_scale="stable")
    S = oracle_system(s)
    ham, trial, walkers, prop = gpu_objects(s, W)
    pa, pb = _walker_pert(s, W, 5)
    walkers.phia, walkers.phib = dev(pa), dev(pb)
    ow = O.Walkers.from_initial(s.init, s.nup, W)
    ow.phia, ow.phib = pa.copy(), pb.copy()
    # energies
    trial.calc_greens_function(walkers)
    O.greens_function(S, ow)
    e_gpu = local_energy_single_det_uhf_batch(None, ham, walkers, trial)
    e_ref = O.local_energy_single_det_uhf_batch(S, ow)
    assert rel(e_gpu, e_ref) < TOL
    # three full steps with identical draws, reortho after the second
    ow.ovlp = O.greens_function(S, ow)
    walkers.ovlp = trial.calc_greens_function(walkers)
    for step in range(3):
        np.random.seed(100 + step)
        prop.propagate_walkers(walkers, ham, trial, 0.0 if step == 0 else -1.5)
        np.random.seed(100 + step)
        O.propagate_walkers(S, ow, 0.0 if step == 0 else -1.5)
        if step == 1:
            walkers.reortho()
            O.reortho(S, ow)
    assert rel(walkers.weight, ow.weight) < TOL
    assert rel(walkers.ovlp, ow.ovlp) < TOL
    assert rel(walkers.hybrid_energy, ow.hybrid_energy) < TOL
    assert rel(walkers.phia, ow.phia) < TOL
    if s.ndown:
        assert rel(walkers.phib, ow.phib) < TOL
    walkers.check_status()


def test_device_rng_moments():
    """Device normal draws: mean 0, variance 1, no repeats across counter blocks."""
    from ipie_b200._lib import call, ptr, stream

    n = 1 << 22
    a = torch.empty(n, dtype=torch.float64, device="cuda")
    b = torch.empty(n, dtype=torch.float64, device="cuda")
    call("ipie_b200_normal_fill", ptr(a), n, 1234, 0, stream())
    call("ipie_b200_normal_fill", ptr(b), n, 1234, 1, stream())
    x = a.cpu().numpy()
    assert abs(x.mean()) < 5.0 / np.sqrt(n)
    assert abs(x.var() - 1.0) < 5.0 * np.sqrt(2.0 / n)
    assert abs(np.mean(x ** 4) - 3.0) < 0.02
    assert not np.allclose(x[:100], b.cpu().numpy()[:100])


@pytest.mark.parametrize("M,N,pre,post", [(26, 5, 1, 1), (21, 4, 1, 0), (33, 7, 0, 1), (64, 16, 0, 0), (200, 32, 1, 1)])
def test_fused_orbital_update_matches_oracle(M, N, pre, post):
    """``ipie_b200_propagate_orbitals`` = one-body, exp(VHS) (order 6), one-body; odd M exercises padding."""
    from ipie_b200 import synthetic
    from ipie_b200._lib import call, ptr, stream

    s = synthetic.generate(M, (N, N), 3 * M, decay=30.0, seed=4, uhf=True, chol_scale="stable")
    S = oracle_system(s)
    ham, trial, walkers, prop = gpu_objects(s, 3)
    W = 3
    pa, _ = _walker_pert(s, W, 8)
    xs = np.random.default_rng(2).normal(size=(s.nchol, W)) + 0.2j * np.random.default_rng(3).normal(size=(s.nchol, W))
    vhs = O.construct_vhs(S, xs)
    ref = pa.copy()
    if pre:
        ref = O.propagate_one_body(ref, S.expH1[0])
    ref = O.apply_exponential(ref, vhs, 6)
    if post:
        ref = O.propagate_one_body(ref, S.expH1[0])
    out = torch.empty(W, M, N, dtype=torch.complex128, device="cuda")
    vhs_d, pa_d = dev(vhs), dev(pa)  # keep the inputs alive until the kernel has run
    call("ipie_b200_propagate_orbitals", ptr(vhs_d), ptr(prop.expH1_pad[0]), prop.lda_e, ptr(pa_d), ptr(out),
         W, M, N, 6, pre, post, stream())
    assert rel(out, ref) < 1e-13


def test_spin_alias_equals_two_blocks_and_oracle():
    """RHF walkers computed once per block (aliased) vs both blocks propagated, vs the oracle."""
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic

    s = synthetic.generate(30, (6, 6), 90, decay=30.0, seed=11, uhf=False, chol_scale="stable")
    runs = {}
    for alias in (True, False):
        ham = Generic(s.h1e, s.chol, s.ecore)
        trial = SingleDet(s.psi, (6, 6), 30)
        trial.half_rotate(ham)
        af = AFQMC.build((6, 6), ham, trial, num_walkers=10, seed=3, num_steps_per_block=25, num_blocks=2,
                         verbose=False, spin_alias="auto" if alias else False)
        assert af.walkers.spin_alias is alias
        runs[alias] = (af.run(), af.walkers.weight.cpu().numpy(), af.walkers.phia.cpu().numpy(),
                       af.walkers.phib.cpu().numpy())
    a, b = runs[True], runs[False]
    assert rel(a[0], b[0]) < 1e-12
    assert rel(a[1], b[1]) < 1e-12
    assert rel(a[2], b[2]) < 1e-12
    assert rel(a[3], b[3]) < 1e-12
    S = oracle_system(s)
    ow = O.Walkers.from_initial(s.init, 6, 10)
    ow.ovlp = O.greens_function(S, ow)
    blocks = O.run_afqmc(S, ow, num_blocks=2, seed=3)
    et = np.array([blk["ETotal"] for blk in blocks])
    assert rel(a[0][:, 5], et) < TOL
    assert rel(a[1], ow.weight) < TOL


def test_unfused_step_path_matches_oracle():
    """The per-stage launches (one-body, Taylor terms, one-body) used when the fused kernel does not apply."""
    from ipie_b200 import synthetic

    s = synthetic.generate(26, (5, 3), 60, decay=30.0, seed=6, uhf=True, chol_scale="stable")
    S = oracle_system(s)
    ham, trial, walkers, prop = gpu_objects(s, 4)
    prop.fused = False
    ow = O.Walkers.from_initial(s.init, s.nup, 4)
    ow.ovlp = O.greens_function(S, ow)
    walkers.ovlp = trial.calc_greens_function(walkers)
    for step in range(2):
        np.random.seed(31 + step)
        prop.propagate_walkers(walkers, ham, trial, 0.0)
        np.random.seed(31 + step)
        O.propagate_walkers(S, ow, 0.0)
    assert rel(walkers.weight, ow.weight) < TOL
    assert rel(walkers.phia, ow.phia) < TOL
    assert rel(walkers.phib, ow.phib) < TOL


def test_cached_green_function_stays_current():
    """The step reuses the Green's function computed at the end of the previous one; after
    propagation, reortho and pair branch it must equal a fresh computation."""
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic

    s = synthetic.generate(30, (6, 4), 90, decay=30.0, seed=12, uhf=True, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (6, 4), 30)
    trial.half_rotate(ham)
    af = AFQMC.build((6, 4), ham, trial, num_walkers=12, seed=4, num_steps_per_block=25, num_blocks=1, verbose=False)
    af.setup_run()
    for step in range(1, 11):  # includes reortho (every 5) and pair branch (every 5)
        af.step(step)
        w = af.walkers
        assert w.gf_current(trial)
        ga, gb, ov = w.Ghalfa.clone(), w.Ghalfb.clone(), w.ovlp.clone()
        fresh = trial.calc_greens_function(w)
        assert rel(ga, w.Ghalfa) < 1e-12
        assert rel(gb, w.Ghalfb) < 1e-12
        assert rel(ov, fresh) < 1e-12
    w.phia = w.phia.clone()
    assert not w.gf_current(trial)


def test_host_fields_prefetch_matches_numpy_draws():
    """``rng="host"`` (each step's array uploaded on a copy stream during the previous step) walks
    exactly as ``rng="numpy"`` fed the same draws."""
    from ipie_b200 import synthetic
    from ipie_b200.propagation import PhaselessGeneric

    s = synthetic.generate(26, (5, 3), 60, decay=30.0, seed=6, uhf=True, chol_scale="stable")
    W, nsteps = 12, 6
    ham, trial, w1, p1 = gpu_objects(s, W)
    _, _, w2, _ = gpu_objects(s, W)
    p2 = PhaselessGeneric(0.005, rng="host")
    p2.build(ham, trial, w2)
    np.random.seed(77)
    draws = [np.random.normal(0.0, 1.0, ham.nfields * W).reshape(W, ham.nfields) for _ in range(nsteps)]
    p2.host_fields = iter([torch.from_numpy(d.copy()).pin_memory() for d in draws])
    np.random.seed(77)
    for step in range(nsteps):
        p1.propagate_walkers(w1, ham, trial, 0.0 if step == 0 else -1.0)
        p2.propagate_walkers(w2, ham, trial, 0.0 if step == 0 else -1.0)
    torch.cuda.synchronize()
    assert torch.equal(w1.weight, w2.weight)
    assert torch.equal(w1.phia, w2.phia)
    assert torch.equal(w1.ovlp, w2.ovlp)


def test_host_fields_new_iterator_drops_prefetch():
    """Replacing ``propagator.host_fields`` part-way through an iterator: the array prefetched from
    the old iterator is dropped and the next step takes the new iterator's first array."""
    from ipie_b200 import synthetic
    from ipie_b200.propagation import PhaselessGeneric

    s = synthetic.generate(26, (5, 3), 60, decay=30.0, seed=6, uhf=True, chol_scale="stable")
    W, k, nsteps = 12, 3, 7
    ham, trial, w1, p1 = gpu_objects(s, W)
    _, _, w2, _ = gpu_objects(s, W)
    p2 = PhaselessGeneric(0.005, rng="host")
    p2.build(ham, trial, w2)
    np.random.seed(91)
    draws = [np.random.normal(0.0, 1.0, ham.nfields * W).reshape(W, ham.nfields) for _ in range(nsteps)]
    pinned = [torch.from_numpy(d.copy()).pin_memory() for d in draws]
    # the first iterator holds k steps' arrays plus two that are never used
    stale = [torch.from_numpy(np.full_like(draws[0], 3.0)).pin_memory() for _ in range(2)]
    p2.host_fields = iter(pinned[:k] + stale)
    np.random.seed(91)
    for step in range(nsteps):
        if step == k:
            p2.host_fields = iter(pinned[k:])
        p1.propagate_walkers(w1, ham, trial, 0.0 if step == 0 else -1.0)
        p2.propagate_walkers(w2, ham, trial, 0.0 if step == 0 else -1.0)
    torch.cuda.synchronize()
    assert torch.equal(w1.weight, w2.weight)
    assert torch.equal(w1.phia, w2.phia)
    assert torch.equal(w1.ovlp, w2.ovlp)
