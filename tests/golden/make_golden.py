"""Generate the golden fixtures in this directory by running ipie itself.

Run from the repository root with ipie's source tree available:

    python tests/golden/make_golden.py /path/to/ipie-checkout [ad|pop|complex|ghf]

ipie needs ``plum`` and ``h5py``, which are absent here; the small stand-ins in
``_ref_shims/`` are put first on ``sys.path``.  mpi4py is absent, so ipie
selects its single-process ``FakeComm``.  Everything runs ipie's numpy (CPU)
path.  Fixtures are small ``.npz`` files: inputs that cannot be regenerated
from ``ipie_b200.synthetic`` plus ipie's outputs.  Synthetic inputs are
regenerated in the tests and checked against the stored checksums.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IPIE_SRC", "")
sys.path.insert(0, os.path.join(HERE, "_ref_shims"))
sys.path.insert(0, REF)
sys.path.insert(0, ROOT)

import h5py  # noqa: E402  (the in-memory shim)

from ipie.estimators.greens_function_single_det import greens_function_single_det  # noqa: E402
from ipie.estimators.local_energy_sd import (  # noqa: E402
    local_energy_single_det_rhf_batch,
    local_energy_single_det_uhf_batch,
)
from ipie.hamiltonians.generic import Generic as HamGeneric  # noqa: E402
from ipie.propagation.operations import apply_exponential, propagate_one_body  # noqa: E402
from ipie.propagation.overlap import calc_overlap_single_det_uhf  # noqa: E402
from ipie.propagation.phaseless_generic import PhaselessGeneric  # noqa: E402
from ipie.qmc.afqmc import AFQMC  # noqa: E402
from ipie.systems.generic import Generic  # noqa: E402
from ipie.trial_wavefunction.single_det import SingleDet  # noqa: E402
from ipie.utils.mpi import MPIHandler  # noqa: E402
from ipie.walkers.walkers_dispatch import UHFWalkersTrial  # noqa: E402

from ipie_b200 import synthetic  # noqa: E402


def checksum(a):
    a = np.ascontiguousarray(a)
    return np.array([a.real.sum(), (a.real ** 2).sum(), np.abs(a).max()])


def build(sysw, nwalkers, dt=0.005):
    ham = HamGeneric(h1e=sysw.h1e.copy(), chol=sysw.chol.copy(), ecore=sysw.ecore)
    trial = SingleDet(sysw.psi.copy(), (sysw.nup, sysw.ndown), sysw.nbasis)
    trial.half_rotate(ham)
    walkers = UHFWalkersTrial(trial, sysw.init.copy(), sysw.nup, sysw.ndown, sysw.nbasis, nwalkers, MPIHandler())
    walkers.build(trial)
    prop = PhaselessGeneric(dt)
    prop.build(ham, trial, walkers, MPIHandler())
    return ham, trial, walkers, prop


def kernels_fixture(name, sysw, nwalkers, seed):
    """Per-kernel inputs and ipie outputs on perturbed walkers."""
    ham, trial, walkers, prop = build(sysw, nwalkers)
    rng = np.random.default_rng(seed)
    M, na, nb, X = sysw.nbasis, sysw.nup, sysw.ndown, sysw.nchol
    W = nwalkers
    pa = walkers.phia + 0.2 * (rng.normal(size=(W, M, na)) + 1j * rng.normal(size=(W, M, na)))
    pb = walkers.phib + 0.2 * (rng.normal(size=(W, M, nb)) + 1j * rng.normal(size=(W, M, nb)))
    walkers.phia = pa.copy()
    walkers.phib = pb.copy()
    out = dict(phia_in=pa, phib_in=pb)
    out["ovlp"] = greens_function_single_det(walkers, trial)
    out["Ghalfa"] = walkers.Ghalfa.copy()
    out["Ghalfb"] = walkers.Ghalfb.copy()
    out["vbias"] = trial.calc_force_bias(ham, walkers, MPIHandler())
    xs = rng.normal(size=(X, W)) + 0.3j * rng.normal(size=(X, W))
    out["xshifted"] = xs
    vhs = prop.construct_VHS(ham, xs.copy())
    out["VHS"] = vhs
    phia_exp = pa.copy()
    for iw in range(W):
        phia_exp[iw] = apply_exponential(phia_exp[iw], vhs[iw], 6)
    out["phia_exp"] = phia_exp
    out["phia_onebody"] = propagate_one_body(pa.copy(), prop.expH1[0])
    out["phib_onebody"] = propagate_one_body(pb.copy(), prop.expH1[1])
    out["ovlp_overlap"] = calc_overlap_single_det_uhf(walkers, trial)
    system = Generic((sysw.nup, sysw.ndown))
    out["energy_uhf"] = local_energy_single_det_uhf_batch(system, ham, walkers, trial)
    if sysw.nup == sysw.ndown:
        walkers.rhf = True
        out["energy_rhf"] = local_energy_single_det_rhf_batch(system, ham, walkers, trial)
        walkers.Ghalfa = out["Ghalfa"].copy()
        walkers.rhf = False
    walkers.ovlp = out["ovlp"].copy()
    detR = walkers.reortho()
    out["reortho_phia"] = walkers.phia.copy()
    out["reortho_phib"] = walkers.phib.copy()
    out["reortho_ovlp"] = walkers.ovlp.copy()
    out["reortho_detR"] = np.array(detR)
    out["mf_shift"] = prop.mf_shift
    out["expH1"] = prop.expH1
    out["rchola"] = trial._rchola
    out["rcholb"] = trial._rcholb
    out["rH1a"] = trial._rH1a
    out["rH1b"] = trial._rH1b
    out["h1e_mod"] = ham.h1e_mod
    out["chol_checksum"] = checksum(sysw.chol)
    out["psi_checksum"] = checksum(sysw.psi)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name)


def run_fixture(name, sysw, nwalkers, num_blocks, seed, snap_steps=(), steps_per_block=25, keep_walkers=None):
    """ipie's own AFQMC.build(...).run() end to end; block estimates + final walker state.

    ``keep_walkers``: store the orbitals of that many leading walkers only (plus checksums of all
    of them) and ipie's local energies of the final walkers, for batches too large to commit."""
    ham = HamGeneric(h1e=sysw.h1e.copy(), chol=sysw.chol.copy(), ecore=sysw.ecore)
    trial = SingleDet(sysw.psi.copy(), (sysw.nup, sysw.ndown), sysw.nbasis)
    trial.half_rotate(ham)
    afqmc = AFQMC.build(
        (sysw.nup, sysw.ndown),
        ham,
        trial,
        num_walkers=nwalkers,
        seed=seed,
        num_steps_per_block=steps_per_block,
        num_blocks=num_blocks,
        timestep=0.005,
        stabilize_freq=5,
        pop_control_freq=5,
        verbose=False,
    )
    h5py.FILES.clear()
    afqmc.run(estimator_filename="golden_run.h5", verbose=False)
    store = h5py.FILES["golden_run.h5"]
    data = store["block_size_1/data/000000000"][: num_blocks + 1]
    w = afqmc.walkers
    out = dict(
        blocks=data,
        weight=np.array(w.weight),
        unscaled_weight=np.array(w.unscaled_weight),
        ovlp=np.array(w.ovlp),
        hybrid_energy=np.array(w.hybrid_energy),
        phia=np.array(w.phia)[:keep_walkers],
        phib=np.array(w.phib)[:keep_walkers],
        total_weight=np.array(afqmc.pcontrol.total_weight),
        chol_checksum=checksum(sysw.chol),
        psi_checksum=checksum(sysw.psi),
    )
    if keep_walkers is not None:
        out["phia_checksum"] = checksum(np.array(w.phia))
        out["phib_checksum"] = checksum(np.array(w.phib))
        # ipie's local energies of the final walkers (the estimator's own call path)
        greens_function_single_det(w, trial)
        out["energy"] = local_energy_single_det_uhf_batch(Generic((sysw.nup, sysw.ndown)), ham, w, trial)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, "ETotal per block", data[:, 3].real if data.shape[1] > 3 else data)


def known_answer_inputs(name):
    """Inputs of three of ipie's own known-answer unit tests.

    * ``walkers/tests/test_population_control.py:30-81`` (pair branch),
    * ``estimators/tests/test_generic.py:51-69`` (local energy of a trial),
    * ``estimators/tests/test_estimators.py:27-41`` (energy estimator).
    The constants those tests assert are restated in the fixture tests.
    """
    from ipie.utils.misc import dotdict
    from ipie.utils.testing import (
        build_test_case_handlers_mpi,
        gen_random_test_instances,
        generate_hamiltonian,
        get_random_nomsd,
    )
    from ipie.utils.testing import build_random_trial

    out = {}
    # (a) pair branch: capture the builder's inputs by replaying its RNG use.
    nelec, nmo, nwalkers, nsteps = (5, 5), 10, 10, 10
    np.random.seed(7)
    h1e, chol, _, _ = generate_hamiltonian(nmo, nelec, cplx=False)
    trial, init = build_random_trial(nelec, nmo, num_dets=1, wfn_type="opt", trial_type="phmsd", complex_trial=True)
    ham = HamGeneric(h1e=np.array([h1e, h1e]), chol=chol.reshape((-1, nmo ** 2)).T.copy(), ecore=0)
    trial.half_rotate(ham)
    trial.calculate_energy(Generic(nelec), ham)
    out["pb_h1e"] = np.array([h1e, h1e])
    out["pb_chol"] = chol.reshape((-1, nmo ** 2)).T.copy()
    out["pb_psi"] = np.hstack([trial.psi0a, trial.psi0b])
    out["pb_init"] = init
    out["pb_eshift"] = np.array(trial.energy)
    qmc = dotdict({"dt": 0.005, "nstblz": 5, "nwalkers": nwalkers, "batched": True, "hybrid": True,
                   "num_steps": nsteps, "population_control": "pair_branch"})
    d = build_test_case_handlers_mpi(nelec, nmo, MPIHandler(), num_dets=1, complex_trial=True, options=qmc, seed=7)
    out["pb_weight"] = np.array(d.walkers.weight)
    out["pb_unscaled_weight"] = np.array(d.walkers.unscaled_weight)
    out["pb_phia"] = np.array(d.walkers.phia)
    out["pb_phib"] = np.array(d.walkers.phib)
    # (b) local energy of a random real single determinant.
    np.random.seed(7)
    nmo, nelec = 24, (4, 2)
    h1e, chol, enuc, _ = generate_hamiltonian(nmo, nelec, cplx=False)
    _, wfn = get_random_nomsd(nelec[0], nelec[1], nmo, ndet=1, cplx=False)
    out["le_h1e"] = np.array([h1e, h1e])
    out["le_chol"] = chol.reshape((-1, nmo * nmo)).T.copy()
    out["le_ecore"] = np.array(enuc)
    out["le_psi"] = wfn[0]
    # (c) energy estimator on random half-rotated integrals.
    system, ham, walkers, trial = gen_random_test_instances(10, 8, 30, 10)
    out["ee_psi"] = trial.psi
    out["ee_phia"] = np.array(walkers.phia)
    out["ee_phib"] = np.array(walkers.phib)
    out["ee_rchola"] = trial._rchola
    out["ee_rcholb"] = trial._rcholb
    out["ee_rH1a"] = trial._rH1a
    out["ee_rH1b"] = trial._rH1b
    out["ee_h1e"] = ham.H1
    out["ee_chol"] = ham.chol
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name)


def ad_fixture(name):
    """Derivative of RHF local energies w.r.t. a one-body coupling, by ipie's AD-AFQMC addon.

    ``addons/adafqmc/estimators/estimator.py:4-23`` (get_local_energy) and
    ``addons/adafqmc/trial_wavefunction/sdtrial.py`` (half rotation, Ghalf), with
    torch autograd through h1 -> h1 + lambda V at lambda = 0 and fixed walkers.
    """
    import torch
    from types import SimpleNamespace

    from ipie.addons.adafqmc.estimators.estimator import get_local_energy
    from ipie.addons.adafqmc.trial_wavefunction.sdtrial import SDTrial

    sysw = synthetic.generate(30, (6, 6), 90, decay=30.0, seed=13, uhf=False, chol_scale="stable")
    M, N, X = sysw.nbasis, sysw.nup, sysw.nchol
    rng = np.random.default_rng(14)
    V = rng.normal(0.0, 0.1, size=(M, M))
    V = np.triu(V) + np.triu(V, 1).T
    W = 8
    phi = sysw.psi[:, :N][None] + 0.15 * (rng.normal(size=(W, M, N)) + 1j * rng.normal(size=(W, M, N)))
    weights = rng.uniform(0.5, 1.5, size=W)
    chol = torch.from_numpy(sysw.chol.T.reshape(X, M, M).copy())
    lam = torch.zeros((), dtype=torch.float64, requires_grad=True)
    h1 = torch.from_numpy(sysw.h1e[0].copy()) + lam * torch.from_numpy(V)
    trial = SDTrial(torch.from_numpy(sysw.psi[:, :N].copy()), N)
    trial.half_rot(SimpleNamespace(h1e=h1, chol=chol))
    ghalf = trial.get_ghalf(SimpleNamespace(walker_states=torch.from_numpy(phi)))
    e = get_local_energy(trial.rh1, ghalf, trial.rchol, sysw.ecore)
    wt = torch.from_numpy(weights)
    E = (wt * e.real).sum() / wt.sum()
    E.backward()
    dE_total = float(lam.grad)
    dE_walker = []
    for iw in range(W):
        lam2 = torch.zeros((), dtype=torch.float64, requires_grad=True)
        h1w = torch.from_numpy(sysw.h1e[0].copy()) + lam2 * torch.from_numpy(V)
        t2 = SDTrial(torch.from_numpy(sysw.psi[:, :N].copy()), N)
        t2.half_rot(SimpleNamespace(h1e=h1w, chol=chol))
        ew = get_local_energy(t2.rh1, ghalf.detach(), t2.rchol, sysw.ecore)[iw].real
        ew.backward()
        dE_walker.append(float(lam2.grad))
    out = dict(V=V, phi=phi, weights=weights, energy=e.detach().numpy(), dE_dlambda=np.array(dE_total),
               dE_walker=np.array(dE_walker), E=np.array(float(E)), chol_checksum=checksum(sysw.chol),
               psi_checksum=checksum(sysw.psi))
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, "dE/dlambda", dE_total)


def pop_control_fixture(name):
    """ipie's comb (``walkers/tests/test_population_control.py:84-142``) and stochastic
    reconfiguration (no ipie test; reconfiguration every 3rd call) on the known-answer
    builder's system (the pair-branch inputs of ``known_answers.npz``)."""
    from ipie.utils.misc import dotdict
    from ipie.utils.testing import build_test_case_handlers_mpi

    out = {}
    for key, method in (("comb", "comb"), ("sr", "stochastic_reconfiguration")):
        qmc = dotdict({"dt": 0.005, "nstblz": 5, "nwalkers": 10, "batched": True, "hybrid": True,
                       "num_steps": 10, "population_control": method, "reconfiguration_freq": 3})
        d = build_test_case_handlers_mpi((5, 5), 10, MPIHandler(), num_dets=1, complex_trial=True, options=qmc,
                                         seed=7)
        out[f"{key}_weight"] = np.array(d.walkers.weight)
        out[f"{key}_unscaled_weight"] = np.array(d.walkers.unscaled_weight)
        out[f"{key}_phia"] = np.array(d.walkers.phia)
        out[f"{key}_phib"] = np.array(d.walkers.phib)
        out[f"{key}_ovlp"] = np.array(d.walkers.ovlp)
    print("comb phia[9][0,0]", out["comb_phia"][9][0, 0])
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name)


def complex_fixture(name, sysw, nwalkers, seed, nsteps=3):
    """ipie's complex-Cholesky path (``GenericComplexChol``): per-kernel outputs on perturbed
    walkers, then ``nsteps`` of ``PhaselessGeneric.propagate_walkers`` with numpy's global
    stream seeded (the fields are drawn as ipie draws them)."""
    ham, trial, walkers, prop = build(sysw, nwalkers)
    rng = np.random.default_rng(seed)
    M, na, nb, X = sysw.nbasis, sysw.nup, sysw.ndown, sysw.nchol
    W = nwalkers
    pa = walkers.phia + 0.2 * (rng.normal(size=(W, M, na)) + 1j * rng.normal(size=(W, M, na)))
    pb = walkers.phib + 0.2 * (rng.normal(size=(W, M, nb)) + 1j * rng.normal(size=(W, M, nb)))
    walkers.phia = pa.copy()
    walkers.phib = pb.copy()
    out = dict(phia_in=pa, phib_in=pb)
    out["ovlp"] = greens_function_single_det(walkers, trial)
    out["Ghalfa"] = walkers.Ghalfa.copy()
    out["Ghalfb"] = walkers.Ghalfb.copy()
    out["vbias"] = trial.calc_force_bias(ham, walkers, MPIHandler())
    xs = rng.normal(size=(2 * X, W)) + 0.3j * rng.normal(size=(2 * X, W))
    out["xshifted"] = xs
    out["VHS"] = prop.construct_VHS(ham, xs.copy())
    system = Generic((sysw.nup, sysw.ndown))
    out["energy_uhf"] = local_energy_single_det_uhf_batch(system, ham, walkers, trial)
    out["mf_shift"] = prop.mf_shift
    out["expH1"] = prop.expH1
    out["h1e_mod"] = ham.h1e_mod
    for k in ("rchola", "rcholb", "rcholbara", "rcholbarb", "rAa", "rAb", "rBa", "rBb", "rH1a", "rH1b"):
        out[k] = getattr(trial, "_" + k)
    # a short walk from the perturbed walkers with ipie's own draws
    walkers.ovlp = out["ovlp"].copy()
    np.random.seed(seed)
    for step in range(nsteps):
        prop.propagate_walkers(walkers, ham, trial, -7.0 if step else 0.0)
    out["walk_weight"] = np.array(walkers.weight)
    out["walk_ovlp"] = np.array(walkers.ovlp)
    out["walk_phia"] = np.array(walkers.phia)
    out["walk_phib"] = np.array(walkers.phib)
    out["walk_hybrid_energy"] = np.array(walkers.hybrid_energy)
    out["chol_checksum"] = checksum(sysw.chol)
    out["psi_checksum"] = checksum(sysw.psi)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name)


def ghf_fixture(name, sysw, nwalkers, seed, nsteps=3):
    """ipie's GHF path (``SingleDetGHF``, ``GHFWalkers``): case "b" (block) builds the trial and
    walkers from UHF ones, case "m" (mixed) a complex spin-mixed determinant; each with per-kernel
    outputs on perturbed walkers (all four spin blocks perturbed), a 3-step walk with ipie's own
    draws and a reorthogonalisation."""
    from ipie.estimators.energy import local_energy
    from ipie.trial_wavefunction.single_det_ghf import SingleDetGHF
    from ipie.walkers.ghf_walkers import GHFWalkers

    M, na, nb = sysw.nbasis, sysw.nup, sysw.ndown
    N = na + nb
    W = nwalkers
    rng = np.random.default_rng(seed)
    out = {}
    # case "c": the spin-mixed trial with a complex Cholesky Hamiltonian (imaginary parts added
    # to the same vectors as synthetic.generate_complex does)
    crng = np.random.default_rng(seed + 500)
    K = crng.normal(size=sysw.chol.shape) * 0.3 * np.abs(sysw.chol).max()
    cchol = sysw.chol + 1.0j * K
    out["c_chol_imag"] = K
    for case in ("b", "m", "c"):
        ham = HamGeneric(h1e=sysw.h1e.copy(), chol=(cchol if case == "c" else sysw.chol).copy(), ecore=sysw.ecore)
        uhf = SingleDet(sysw.psi.copy(), (na, nb), M)
        if case != "c":
            uhf.half_rotate(ham)
        if case == "b":
            trial = SingleDetGHF(uhf)
            uw = UHFWalkersTrial(uhf, sysw.init.copy(), na, nb, M, W, MPIHandler())
            uw.build(uhf)
            walkers = GHFWalkers(uw)
        else:
            import scipy.linalg

            base = np.zeros((2 * M, N))
            base[:M, :na] = sysw.psi[:, :na]
            base[M:, na:] = sysw.psi[:, na:]
            A = rng.normal(size=(2 * M, 2 * M)) + 1j * rng.normal(size=(2 * M, 2 * M))
            U = scipy.linalg.expm(0.08 * (A - A.conj().T))
            psi = U @ base
            if case == "m":
                out["m_psi"] = psi
            else:
                psi = out["m_psi"]
            trial = SingleDetGHF(psi.copy(), (na, nb), M)
            walkers = GHFWalkers(psi.copy(), na, nb, M, W, MPIHandler())
        walkers.build(trial)
        prop = PhaselessGeneric(0.005)
        prop.build(ham, trial, walkers, MPIHandler())
        phi = walkers.phi + 0.15 * (rng.normal(size=walkers.phi.shape) + 1j * rng.normal(size=walkers.phi.shape))
        walkers.phi = phi.copy()
        out[case + "_phi_in"] = phi
        out[case + "_ovlp"] = trial.calc_greens_function(walkers)
        out[case + "_G"] = walkers.G.copy()
        out[case + "_vbias"] = trial.calc_force_bias(ham, walkers, MPIHandler())
        out[case + "_energy"] = local_energy(Generic((na, nb)), ham, walkers, trial)
        out[case + "_mf_shift"] = prop.mf_shift
        out[case + "_expH1"] = prop.expH1
        walkers.ovlp = out[case + "_ovlp"].copy()
        np.random.seed(seed + {"b": 1, "m": 2, "c": 3}[case])
        for step in range(nsteps):
            prop.propagate_walkers(walkers, ham, trial, -3.0 if step else 0.0)
        out[case + "_walk_weight"] = np.array(walkers.weight)
        out[case + "_walk_ovlp"] = np.array(walkers.ovlp)
        out[case + "_walk_phi"] = np.array(walkers.phi)
        out[case + "_walk_hybrid_energy"] = np.array(walkers.hybrid_energy)
        out[case + "_reortho_detR"] = np.array(walkers.reortho())
        out[case + "_reortho_phi"] = np.array(walkers.phi)
        out[case + "_reortho_ovlp"] = np.array(walkers.ovlp)
    out["chol_checksum"] = checksum(sysw.chol)
    out["psi_checksum"] = checksum(sysw.psi)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name)


def ad_walk_fixture(name):
    """ipie's AD-AFQMC block derivative through the walk (``addons/adafqmc/qmc/adafqmc.py:222-344``,
    ``ad_block`` and ``ad_block_gradient``) on a small RHF system, with the trial's orbital tangent
    set to zero (no orbital relaxation), FakeComm, and torch's draws recorded: the auxiliary
    fields of every step (``propagation/propagator.py:219``) and the stochastic-reconfiguration
    uniforms (``walkers/rhf_walkers.py:41``)."""
    import torch

    from ipie.addons.adafqmc.hamiltonians.hamiltonian import HamObs
    from ipie.addons.adafqmc.qmc.adafqmc import ADAFQMC
    from ipie.addons.adafqmc.walkers.rhf_walkers import Walkers
    from ipie.qmc.comm import FakeComm

    class TrialwithTangent(torch.autograd.Function):
        # the trial passes through unchanged; its derivative is the given tangent
        # (ipie addons/adafqmc/utils/miscellaneous.py:162-175; that module imports pyscf)
        @staticmethod
        def forward(ctx, coupling, trial, tangent):
            ctx.save_for_backward(tangent)
            return trial

        @staticmethod
        def backward(ctx, grad_output):
            (tangent,) = ctx.saved_tensors
            return tangent * grad_output, None, None

    sysw = synthetic.generate(14, (3, 3), 36, decay=30.0, seed=21, uhf=False, chol_scale="stable")
    M, N, X = sysw.nbasis, sysw.nup, sysw.nchol
    rng = np.random.default_rng(22)
    V = rng.normal(0.0, 0.1, size=(M, M))
    V = np.triu(V) + np.triu(V, 1).T
    # the trial's full orbital set: its N occupied orbitals completed to an orthonormal basis
    q, _ = np.linalg.qr(np.hstack([sysw.psi[:, :N], rng.normal(size=(M, M - N))]))
    C = np.hstack([sysw.psi[:, :N], q[:, N:]])
    L = sysw.chol.T.reshape(X, M, M)
    hamobs = HamObs(N, M, torch.from_numpy(sysw.h1e[0].copy()), torch.from_numpy(L.copy()),
                    torch.tensor(sysw.ecore, dtype=torch.float64), observable=(torch.from_numpy(V.copy()), torch.tensor(0.0, dtype=torch.float64)),
                    obs_type="dipole")
    W = 8
    phi0 = np.eye(M)[:, :N][None] + 0.1 * (rng.normal(size=(W, M, N)) + 1j * rng.normal(size=(W, M, N)))
    w0 = rng.uniform(0.5, 1.5, size=W)
    walkers = Walkers(W, torch.from_numpy(phi0.copy()), torch.from_numpy(w0.copy()))
    af = ADAFQMC.build(FakeComm(), lambda c, t, g: TrialwithTangent.apply(c, t, g), num_walkers_per_process=W,
                       num_steps_per_block=10, ad_block_size=30, num_ad_blocks=1, timestep=0.005,
                       stabilize_freq=5, pop_control_freq=5, seed=3)
    draws, zetas = [], []
    randn0, rand0 = torch.randn, torch.rand

    def randn(*a, **k):
        x = randn0(*a, **k)
        draws.append(x.numpy().copy())
        return x

    def rand(*a, **k):
        z = rand0(*a, **k)
        zetas.append(float(z.item()))
        return z

    torch.manual_seed(5)
    torch.randn, torch.rand = randn, rand
    try:
        out_w, e, obs, blkwts, wtsgrad = af.ad_block_gradient(hamobs, walkers, torch.from_numpy(C.copy()),
                                                             torch.zeros(M, M, dtype=torch.float64))
    finally:
        torch.randn, torch.rand = randn0, rand0
    out = dict(V=V, C=C, phi0=phi0, w0=w0, draws=np.array(draws), zetas=np.array(zetas),
               energy=np.array(float(e)), dE_dlambda=np.array(float(obs[0])), total_weight=np.array(float(blkwts)),
               dW_dlambda=np.array(float(wtsgrad[0])), final_phi=out_w.walker_states.numpy(),
               final_weight=out_w.walker_weights.numpy(), chol_checksum=checksum(sysw.chol),
               psi_checksum=checksum(sysw.psi))
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, "E", float(e), "dE/dlambda", float(obs[0]), "W", float(blkwts), "dW", float(wtsgrad[0]))


def multidet_fixture(name):
    """ipie's particle-hole multi-determinant trial: the Wick's-theorem Green's function and overlap
    (``estimators/greens_function_multi_det.py:1113``, ``greens_function_multi_det_wicks_opt``) and
    local energy (``estimators/local_energy_wicks.py:864``,
    ``local_energy_multi_det_trial_wicks_batch_opt``) on perturbed walkers, with ipie's naive
    per-determinant path (``ParticleHoleNaive``, ``greens_function_multi_det``,
    ``local_energy_batch.py:78`` ``local_energy_multi_det_trial_batch``) as a cross-check."""

    from ipie.estimators.greens_function_multi_det import (
        greens_function_multi_det,
        greens_function_multi_det_wicks_opt,
    )
    from ipie.estimators.local_energy_batch import local_energy_multi_det_trial_batch
    from ipie.estimators.local_energy_wicks import local_energy_multi_det_trial_wicks_batch_opt
    from ipie.trial_wavefunction.particle_hole import ParticleHoleNaive, ParticleHoleNonChunked

    sysw, wfn, init, rng = _multidet_system()
    M, na, nb = sysw.nbasis, sysw.nup, sysw.ndown
    ci, occa, occb = wfn
    ham = HamGeneric(h1e=sysw.h1e.copy(), chol=sysw.chol.copy(), ecore=sysw.ecore)
    system = Generic((na, nb))
    W = 6
    out = dict(ci=ci, occa=np.array(occa), occb=np.array(occb), init=init)
    results = {}
    for key, cls in (("opt", ParticleHoleNonChunked), ("naive", ParticleHoleNaive)):
        trial = cls(wfn, (na, nb), M)
        trial.build()
        trial.half_rotate(ham)
        walkers = UHFWalkersTrial(trial, init.copy(), na, nb, M, W, MPIHandler())
        walkers.build(trial)
        prng = np.random.default_rng(33)
        walkers.phia = walkers.phia + 0.2 * (prng.normal(size=walkers.phia.shape) + 1j * prng.normal(size=walkers.phia.shape))
        walkers.phib = walkers.phib + 0.2 * (prng.normal(size=walkers.phib.shape) + 1j * prng.normal(size=walkers.phib.shape))
        if key == "opt":
            ovlp = greens_function_multi_det_wicks_opt(walkers, trial)
            # the energy normalises by walkers.ovlp, which a propagation step would have set
            walkers.ovlp = ovlp
            energy = local_energy_multi_det_trial_wicks_batch_opt(system, ham, walkers, trial)
            out["phia"], out["phib"] = np.array(walkers.phia), np.array(walkers.phib)
        else:
            ovlp = greens_function_multi_det(walkers, trial)
            energy = local_energy_multi_det_trial_batch(system, ham, walkers, trial)
        results[key] = (np.array(ovlp), np.array(walkers.Ga), np.array(walkers.Gb), np.array(energy))
    for a, b in zip(results["opt"], results["naive"]):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))
    out["ovlp"], out["Ga"], out["Gb"], out["energy"] = results["opt"]
    out["chol_checksum"] = checksum(sysw.chol)
    out["psi_checksum"] = checksum(sysw.psi)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, "energies", out["energy"][:, 0])


def _multidet_system():
    """The synthetic system, particle-hole trial (reference + 59 random excited determinants) and
    starting walker of the multi-determinant fixtures."""
    import itertools

    sysw = synthetic.generate(14, (4, 3), 42, decay=30.0, seed=31, uhf=True, chol_scale="stable")
    M, na, nb = sysw.nbasis, sysw.nup, sysw.ndown
    rng = np.random.default_rng(32)
    # the reference (lowest orbitals) and a random selection of excited determinants up to four
    # holes per spin, ordered by excitation level as ipie's inputs usually are
    oa = [tuple(range(na))] + [c for c in itertools.combinations(range(M), na) if c != tuple(range(na))]
    ob = [tuple(range(nb))] + [c for c in itertools.combinations(range(M), nb) if c != tuple(range(nb))]
    pick_a = [0] + list(rng.choice(np.arange(1, len(oa)), 59))
    pick_b = [0] + list(rng.choice(np.arange(1, len(ob)), 59))
    occa = [np.array(oa[i]) for i in pick_a]
    occb = [np.array(ob[i]) for i in pick_b]
    ci = rng.normal(size=60) + 1j * rng.normal(size=60)
    ci[0] = 3.0
    ci /= np.linalg.norm(ci)
    order = np.argsort([-abs(c) for c in ci], kind="stable")
    ci, occa, occb = ci[order], [occa[i] for i in order], [occb[i] for i in order]
    init = np.hstack([np.eye(M)[:, :na], np.eye(M)[:, :nb]]) + 0.3 * rng.normal(size=(M, na + nb))
    return sysw, (ci, occa, occb), init, rng


def multidet_run_fixture(name, nwalkers=10, num_blocks=2, steps=10, seed=5):
    """ipie's own ``AFQMC.build(...).run()`` with the particle-hole trial (Wick's-theorem Green's
    function, overlap and force bias, reortho and pair-branch population control every 5 steps) from
    given walkers (the perturbed reference): block estimates and final walkers."""
    from ipie.trial_wavefunction.particle_hole import ParticleHoleNonChunked

    sysw, wfn, init, _ = _multidet_system()
    M, na, nb = sysw.nbasis, sysw.nup, sysw.ndown
    ham = HamGeneric(h1e=sysw.h1e.copy(), chol=sysw.chol.copy(), ecore=sysw.ecore)
    trial = ParticleHoleNonChunked(wfn, (na, nb), M)
    trial.build()
    trial.half_rotate(ham)
    # walkers started from the perturbed reference (every determinant of the trial overlaps them)
    walkers = UHFWalkersTrial(trial, init.copy(), na, nb, M, nwalkers, MPIHandler())
    walkers.build(trial)
    afqmc = AFQMC.build((na, nb), ham, trial, walkers=walkers, num_walkers=nwalkers, seed=seed,
                        num_steps_per_block=steps, num_blocks=num_blocks, timestep=0.005, stabilize_freq=5,
                        pop_control_freq=5, verbose=False)
    h5py.FILES.clear()
    afqmc.run(estimator_filename="golden_run.h5", verbose=False)
    data = h5py.FILES["golden_run.h5"]["block_size_1/data/000000000"][: num_blocks + 1]
    w = afqmc.walkers
    out = dict(blocks=data, weight=np.array(w.weight), unscaled_weight=np.array(w.unscaled_weight),
               ovlp=np.array(w.ovlp), hybrid_energy=np.array(w.hybrid_energy), phia=np.array(w.phia),
               phib=np.array(w.phib), chol_checksum=checksum(sysw.chol))
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, "ETotal per block", data[:, 5].real)


def multidet_prop_fixture(name, nsteps=4):
    """Phaseless propagation with ipie's particle-hole trial (``PhaselessGeneric.propagate_walkers``,
    ``propagation/phaseless_base.py:312-338``, with the trial's Wick's-theorem Green's function,
    overlap and full-G force bias, ``propagation/force_bias.py:62-76``), the trial's 1-RDM
    (``particle_hole.py:458-506``) and mean-field shift, numpy's global draws seeded per step; then
    the local energy of the final walkers."""
    from ipie.estimators.greens_function_multi_det import greens_function_multi_det_wicks_opt
    from ipie.estimators.local_energy_wicks import local_energy_multi_det_trial_wicks_batch_opt
    from ipie.trial_wavefunction.particle_hole import ParticleHoleNonChunked

    sysw, wfn, init, _ = _multidet_system()
    M, na, nb = sysw.nbasis, sysw.nup, sysw.ndown
    ham = HamGeneric(h1e=sysw.h1e.copy(), chol=sysw.chol.copy(), ecore=sysw.ecore)
    system = Generic((na, nb))
    W = 8
    trial = ParticleHoleNonChunked(wfn, (na, nb), M)
    trial.build()
    trial.half_rotate(ham)
    walkers = UHFWalkersTrial(trial, init.copy(), na, nb, M, W, MPIHandler())
    walkers.build(trial)
    prop = PhaselessGeneric(0.005)
    prop.build(ham, trial, walkers, MPIHandler())
    out = dict(G=np.array(trial.G), mf_shift=np.array(prop.mf_shift), ovlp_init=np.array(walkers.ovlp))
    for step in range(nsteps):
        np.random.seed(400 + step)
        prop.propagate_walkers(walkers, ham, trial, -3.0 if step else 0.0)
        out[f"weight{step}"] = np.array(walkers.weight)
        out[f"ovlp{step}"] = np.array(walkers.ovlp)
        out[f"phia{step}"] = np.array(walkers.phia)
        out[f"phib{step}"] = np.array(walkers.phib)
    ovlp = greens_function_multi_det_wicks_opt(walkers, trial)
    walkers.ovlp = ovlp
    out["energy"] = np.array(local_energy_multi_det_trial_wicks_batch_opt(system, ham, walkers, trial))
    out["chol_checksum"] = checksum(sysw.chol)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, "weights", out[f"weight{nsteps - 1}"], "energies", out["energy"][:, 0])


def analysis_fixture(name):
    """ipie's autocorrelation reblocking (``analysis/autocorr.py:54-105``) on seeded series:
    white noise and AR(1) series with correlation 0.5 and 0.9, of several lengths."""
    from ipie.analysis.autocorr import reblock_by_autocorr

    rng = np.random.default_rng(2024)
    out = {}
    cases = []
    for n in (40, 257, 1000):
        for phi in (0.0, 0.5, 0.9):
            e = rng.normal(size=n)
            y = np.empty(n)
            y[0] = e[0]
            for i in range(1, n):
                y[i] = phi * y[i - 1] + e[i]
            y = -150.0 + 1e-3 * y
            df = reblock_by_autocorr(y)
            key = f"n{n}_phi{int(phi * 10)}"
            cases.append(key)
            out[key + "_y"] = y
            out[key + "_ref"] = np.array([df["ETotal_ac"].values[0], df["ETotal_error_ac"].values[0],
                                          df["ETotal_nsamp_ac"].values[0], df["ac"].values[0]], dtype=np.float64)
    out["cases"] = np.array(cases)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name)


def config_fixtures():
    """Parity runs at the workload sizes themselves (the stable Cholesky amplitude).

    * RHF M=26, 5+5 electrons, X=120, 64 walkers, 3 blocks of 25 steps with reortho and pair
      branch every 5 steps (ipie's AFQMC.run, seed 7);
    * UHF M=108, 15+15 electrons, X=600, 640 walkers, one block of 10 steps with its energy
      evaluation (ipie's AFQMC.run, seed 7)."""
    c0 = synthetic.workload("c0_rhf_m26", chol_scale="stable")
    run_fixture("run_c0_rhf_m26_w64.npz", c0, nwalkers=64, num_blocks=3, seed=7)
    c1 = synthetic.workload("c1_uhf_m108", chol_scale="stable")
    run_fixture("run_c1_uhf_m108_w640.npz", c1, nwalkers=640, num_blocks=1, seed=7, steps_per_block=10,
                keep_walkers=4)


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "multidet_prop":
        multidet_prop_fixture("multidet_prop_m14.npz")
        multidet_run_fixture("multidet_run_m14.npz")
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "multidet":
        multidet_fixture("multidet_m14.npz")
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "adwalk":
        ad_walk_fixture("ad_walk_m14.npz")
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "analysis":
        analysis_fixture("reblock_autocorr.npz")
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "configs":
        config_fixtures()
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "ghf":
        ghf = synthetic.generate(14, (4, 3), 40, decay=30.0, seed=8, uhf=True, chol_scale="stable")
        ghf_fixture("ghf_m14.npz", ghf, nwalkers=5, seed=31)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "complex":
        cplx = synthetic.generate_complex(20, (4, 3), 60, decay=30.0, seed=3, uhf=True)
        complex_fixture("complex_uhf_m20.npz", cplx, nwalkers=5, seed=21)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "ad":
        ad_fixture("ad_onebody_m30.npz")
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "pop":
        pop_control_fixture("pop_control.npz")
        sys.exit(0)
    c0 = synthetic.workload("c0_rhf_m26")
    kernels_fixture("kernels_rhf_m26.npz", c0, nwalkers=8, seed=11)
    uhf = synthetic.generate(30, (6, 4), 90, decay=30.0, seed=5, uhf=True)
    kernels_fixture("kernels_uhf_m30.npz", uhf, nwalkers=6, seed=12)
    c0s = synthetic.workload("c0_rhf_m26", chol_scale="stable")
    run_fixture("run_rhf_m26.npz", c0s, nwalkers=16, num_blocks=3, seed=7)
    gentle = synthetic.generate(30, (6, 4), 90, decay=30.0, seed=5, uhf=True, chol_scale=0.1)
    run_fixture("run_uhf_m30.npz", gentle, nwalkers=12, num_blocks=3, seed=9)
    known_answer_inputs("known_answers.npz")
    pop_control_fixture("pop_control.npz")
    ad_fixture("ad_onebody_m30.npz")
    cplx = synthetic.generate_complex(20, (4, 3), 60, decay=30.0, seed=3, uhf=True)
    complex_fixture("complex_uhf_m20.npz", cplx, nwalkers=5, seed=21)
    ghf = synthetic.generate(14, (4, 3), 40, decay=30.0, seed=8, uhf=True, chol_scale="stable")
    ghf_fixture("ghf_m14.npz", ghf, nwalkers=5, seed=31)
