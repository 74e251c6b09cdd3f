"""Parity of the GHF walker step (``SingleDetGHF``, ``GHFWalkers``) with ipie's outputs.

``ghf_m14.npz`` holds ipie's own results for a block-diagonal trial built from a UHF one
(case "b"), a complex spin-mixed trial (case "m") and that trial with complex Cholesky vectors
(case "c"): Green's function, force bias and local
energy of perturbed walkers, a 3-step walk with ipie's draws and a reorthogonalisation
(``tests/golden/make_golden.py``).  Tolerances as for the FP64 UHF form.  Every call goes
through the C ABI.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import ghf_oracle as G  # noqa: E402
from tests._systems import load  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ghf_objects(case, f, W):
    from ipie_b200 import Generic, SingleDet, synthetic
    from ipie_b200.ghf import GHFWalkers, SingleDetGHF
    from ipie_b200.propagation import PhaselessGeneric

    s = synthetic.generate(14, (4, 3), 40, decay=30.0, seed=8, uhf=True, chol_scale="stable")
    ham = Generic(s.h1e, s.chol + 1.0j * f["c_chol_imag"] if case == "c" else s.chol, s.ecore)
    if case == "b":
        trial = SingleDetGHF(SingleDet(s.psi, (s.nup, s.ndown), s.nbasis))
        init = G.ghf_from_uhf(s.init, s.nup, s.nbasis)
    else:
        trial = SingleDetGHF(f["m_psi"], (s.nup, s.ndown), s.nbasis)
        init = f["m_psi"]
    trial.half_rotate(ham)
    walkers = GHFWalkers(init, s.nup, s.ndown, s.nbasis, W)
    walkers.build(trial)
    prop = PhaselessGeneric(0.005)
    prop.build(ham, trial, walkers)
    return s, ham, trial, walkers, prop


@pytest.mark.parametrize("case,fused", [("b", True), ("b", False), ("m", True), ("m", False), ("c", False)])
def test_ghf_step_matches_ipie(case, fused):
    from ipie_b200.estimators import local_energy_batch

    f = load("ghf_m14.npz")
    W = f[case + "_phi_in"].shape[0]
    s, ham, trial, walkers, prop = ghf_objects(case, f, W)
    prop.fused = fused
    assert trial.complex_rotated == (case in ("m", "c"))
    assert rel(prop.mf_shift, f[case + "_mf_shift"]) < 1e-12
    assert rel(prop.expH1, f[case + "_expH1"]) < 1e-12
    walkers.phi = dev(f[case + "_phi_in"])
    ovlp = trial.calc_greens_function(walkers)
    assert rel(ovlp, f[case + "_ovlp"]) < 1e-11
    Gfull = np.einsum("mi,wiq->wmq", trial.psi.conj(), walkers.Ghalf.cpu().numpy())
    assert rel(Gfull, f[case + "_G"]) < 1e-11
    assert rel(trial.calc_force_bias(ham, walkers), f[case + "_vbias"]) < 1e-12
    assert rel(local_energy_batch(None, ham, walkers, trial), f[case + "_energy"]) < 1e-11
    walkers.ovlp = ovlp.clone()
    np.random.seed(31 + {"b": 1, "m": 2, "c": 3}[case])
    for step in range(3):
        prop.propagate_walkers(walkers, ham, trial, -3.0 if step else 0.0)
    assert rel(walkers.weight, f[case + "_walk_weight"]) < TOL
    assert rel(walkers.ovlp, f[case + "_walk_ovlp"]) < TOL
    assert rel(walkers.phi, f[case + "_walk_phi"]) < TOL
    assert rel(walkers.hybrid_energy, f[case + "_walk_hybrid_energy"]) < TOL
    detR = walkers.reortho()
    assert rel(detR, f[case + "_reortho_detR"]) < 1e-12
    assert rel(walkers.phi, f[case + "_reortho_phi"]) < TOL
    assert rel(walkers.ovlp, f[case + "_reortho_ovlp"]) < TOL
    walkers.check_status()


def test_ghf_afqmc_block0_is_the_trial_energy():
    """``AFQMC.build`` with a GHF trial starts GHF walkers from it: block 0 is the trial energy
    (the oracle's GHF local energy of the trial determinant); later blocks stay finite."""
    from ipie_b200 import AFQMC

    f = load("ghf_m14.npz")
    s, ham, trial, _, _ = ghf_objects("m", f, 2)
    af = AFQMC.build((s.nup, s.ndown), ham, trial, num_walkers=8, seed=3, num_steps_per_block=10, num_blocks=2,
                     timestep=0.005, verbose=False)
    blocks = af.run()
    S = G.GHFSystem(nbasis=s.nbasis, nalpha=s.nup, nbeta=s.ndown, h1e=s.h1e, chol=s.chol, ecore=s.ecore,
                    psi=f["m_psi"]).build()
    w = S.walkers(S.psi, 1)
    G.greens_function_ghf(S, w)
    e = G.local_energy_ghf(S, w)[0].real
    np.testing.assert_allclose(blocks[0, 5:8], e, rtol=0, atol=1e-11)
    assert np.all(np.isfinite(blocks))
