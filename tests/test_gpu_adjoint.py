"""Hand-written adjoint of the local energy w.r.t. the one-body Hamiltonian.

Checked against central finite differences (lambda = +-1e-4, same walkers)
and against ipie's AD-AFQMC addon (torch autograd through its local energy),
whose derivatives are stored in ``tests/golden/ad_onebody_m30.npz``.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tests._systems import checksum, load  # noqa: E402
from tests.test_gpu_parity import _walker_pert, dev, gpu_objects, rel  # noqa: E402

pytestmark = pytest.mark.gpu


def _ad_system():
    from ipie_b200 import synthetic

    return synthetic.generate(30, (6, 6), 90, decay=30.0, seed=13, uhf=False, chol_scale="stable")


def test_adjoint_matches_central_differences():
    from ipie_b200.adjoint import OneBodyLocalEnergy, energy_response, local_energy_state
    from ipie_b200 import synthetic

    s = synthetic.generate(40, (7, 5), 120, decay=30.0, seed=8, uhf=True, chol_scale="stable")
    ham, trial, walkers, prop = gpu_objects(s, 12)
    pa, pb = _walker_pert(s, 12, 9)
    walkers.phia, walkers.phib = dev(pa), dev(pb)
    walkers.weight = dev(np.random.default_rng(1).uniform(0.5, 1.5, 12))
    V = np.random.default_rng(2).normal(0, 0.1, (40, 40))
    V = V + V.T
    dE, E0 = energy_response(ham, trial, walkers, V)
    state = local_energy_state(ham, trial, walkers)
    h1 = torch.from_numpy(ham.H1.copy()).cuda()
    Vd = torch.from_numpy(np.stack([V, V])).cuda()
    wt = walkers.weight
    eps = 1e-4
    ep = (OneBodyLocalEnergy.apply(h1 + eps * Vd, state) * wt).sum() / wt.sum()
    em = (OneBodyLocalEnergy.apply(h1 - eps * Vd, state) * wt).sum() / wt.sum()
    fd = float((ep - em).item()) / (2 * eps)
    assert abs(dE - fd) < 1e-7 * max(1.0, abs(fd))


def test_adjoint_matches_ipie_ad_afqmc():
    from ipie_b200.adjoint import OneBodyLocalEnergy, energy_response, local_energy_state

    f = load("ad_onebody_m30.npz")
    s = _ad_system()
    np.testing.assert_allclose(checksum(s.chol), f["chol_checksum"], rtol=1e-13)
    phi = f["phi"]
    W = phi.shape[0]
    ham, trial, walkers, prop = gpu_objects(s, W)
    walkers.phia = dev(phi)
    walkers.phib = dev(phi.copy())
    walkers.weight = dev(f["weights"])
    dE, E = energy_response(ham, trial, walkers, f["V"])
    assert abs(E - float(f["E"])) < 1e-10 * abs(float(f["E"]))
    assert abs(dE - float(f["dE_dlambda"])) < 1e-10 * max(1.0, abs(float(f["dE_dlambda"])))
    # per-walker derivatives: unit upstream gradient on each walker
    state = local_energy_state(ham, trial, walkers)
    for iw in range(W):
        lam = torch.zeros((), dtype=torch.float64, device="cuda", requires_grad=True)
        h1 = torch.from_numpy(ham.H1.copy()).cuda() + lam * torch.from_numpy(np.stack([f["V"], f["V"]])).cuda()
        OneBodyLocalEnergy.apply(h1, state)[iw].backward()
        assert abs(float(lam.grad) - f["dE_walker"][iw]) < 1e-10 * max(1.0, abs(f["dE_walker"][iw]))


def test_mixed_one_rdm_properties():
    """The mixed 1-RDM from the adjoint: trace = electrons per spin; equals the trial density for trial walkers."""
    from ipie_b200.adjoint import mixed_one_rdm

    s = _ad_system()
    ham, trial, walkers, prop = gpu_objects(s, 5)
    rdm = mixed_one_rdm(ham, trial, walkers).cpu().numpy()
    assert abs(np.trace(rdm[0]) - 6) < 1e-10 and abs(np.trace(rdm[1]) - 6) < 1e-10
    np.testing.assert_allclose(rdm[0], trial.G[0].real, atol=1e-10)


def test_adjoint_response_on_walked_c4_walkers():
    """The adjoint-property workload (M=76, 10+10 electrons, X=400, 512 walkers, V entries N(0, 0.1)):
    after 25 steps of the walk, dE/dlambda from the adjoint equals the contraction of the mixed
    1-RDM with V and central differences (lambda = +-1e-4) of the production energy estimator."""
    from ipie_b200 import AFQMC, EnergyEstimator, Generic, SingleDet, synthetic
    from ipie_b200.adjoint import energy_response, mixed_one_rdm

    s = synthetic.workload("c4_rhf_m76", chol_scale="stable")
    M = s.nbasis
    A = np.random.default_rng(4).normal(0.0, 0.1, (M, M))
    V = 0.5 * (A + A.T)
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (s.nup, s.ndown), M)
    trial.half_rotate(ham)
    af = AFQMC.build((s.nup, s.ndown), ham, trial, num_walkers=512, seed=3, num_steps_per_block=25, num_blocks=1,
                     verbose=False, rng="device")
    af.setup_run()
    for step in range(1, 26):
        af.step(step)
    w = af.walkers
    dE, E0 = energy_response(ham, trial, w, V)
    rdm = mixed_one_rdm(ham, trial, w).cpu().numpy()
    assert abs(np.sum(rdm[0] * V) + np.sum(rdm[1] * V) - dE) < 1e-10 * max(1.0, abs(dE))
    eps = 1e-4
    energies = []
    for sign in (1.0, -1.0):
        h1 = s.h1e + sign * eps * np.stack([V, V])
        ham_s = Generic(h1, s.chol, s.ecore)
        trial_s = SingleDet(s.psi, (s.nup, s.ndown), M)
        trial_s.half_rotate(ham_s)
        d = EnergyEstimator().compute_estimator(None, w, ham_s, trial_s)
        energies.append((d[0] / d[1]).real)
    fd = (energies[0] - energies[1]) / (2 * eps)
    assert abs(fd - dE) < 1e-7 * max(1.0, abs(dE))
    w.check_status()


def _torch_energy(ham, trial, ga, gb, rhf):
    """Plain torch FP64 restatement of the single-determinant local energy (ipie
    ``estimators/local_energy_sd.py:358-403``, and ``:106-155`` for the doubled RHF form) from the
    half-rotated operands, differentiated by torch autograd."""
    W, na, M = ga.shape
    nb = gb.shape[1]
    X = ham.nchol
    La = trial._rchola.reshape(X, na, M).to(torch.complex128)
    ea = torch.einsum("ip,wip->w", trial._rH1a, ga)
    Xa = torch.einsum("xip,wip->wx", La, ga)
    Ta = torch.einsum("xip,wjp->wxij", La, ga)
    kxa = torch.einsum("wxij,wxji->w", Ta, Ta)
    if rhf:
        return ham.ecore + 2 * ea + 2 * (Xa * Xa).sum(1) - kxa
    Lb = trial._rcholb.reshape(X, nb, M).to(torch.complex128)
    eb = torch.einsum("ip,wip->w", trial._rH1b, gb)
    Xb = torch.einsum("xip,wip->wx", Lb, gb)
    Tb = torch.einsum("xip,wjp->wxij", Lb, gb)
    kxb = torch.einsum("wxij,wxji->w", Tb, Tb)
    return ham.ecore + ea + eb + 0.5 * ((Xa + Xb) ** 2).sum(1) - 0.5 * (kxa + kxb)


@pytest.mark.parametrize("uhf,na,nb,rhf,alias", [(True, 7, 5, False, False), (False, 6, 6, True, False),
                                                 (False, 6, 6, False, True)])
def test_local_energy_vjp_matches_autograd(uhf, na, nb, rhf, alias):
    """ipie_b200_local_energy_vjp (through LocalEnergyGreens) against torch autograd through the FP64
    restatement: energies and the gradient of a complex-weighted loss w.r.t. both Green's
    functions (UHF; the doubled RHF form; UHF with one tensor passed for both spins)."""
    from ipie_b200 import synthetic
    from ipie_b200.adjoint import LocalEnergyGreens

    s = synthetic.generate(40, (na, nb), 120, decay=30.0, seed=21, uhf=uhf, chol_scale="stable")
    W = 6
    ham, trial, walkers, prop = gpu_objects(s, W)
    rng = np.random.default_rng(5)

    def rand_g(n):
        return torch.from_numpy(rng.normal(0, 0.3, (W, n, 40)) + 1j * rng.normal(0, 0.3, (W, n, 40))).cuda()

    ga0 = rand_g(na)
    gb0 = ga0 if alias else rand_g(nb)
    c = torch.from_numpy(rng.normal(size=W) + 1j * rng.normal(size=W)).cuda()

    def loss(e):
        return (c * e).real.sum() + 0.3 * (c.conj() * e).imag.sum()

    ga = ga0.clone().requires_grad_(True)
    gb = ga if alias else gb0.clone().requires_grad_(True)
    e = LocalEnergyGreens.apply(ga, gb, ham, trial, rhf)
    loss(e).backward()
    ra = ga0.clone().requires_grad_(True)
    rb = ra if alias else gb0.clone().requires_grad_(True)
    e_ref = _torch_energy(ham, trial, ra, rb, rhf)
    loss(e_ref).backward()
    assert rel(e.detach(), e_ref.detach()) < 1e-11
    assert rel(ga.grad, ra.grad) < 1e-10
    if not rhf and not alias:
        assert rel(gb.grad, rb.grad) < 1e-10


def test_local_energy_vjp_central_difference():
    """One directional derivative of the summed energy against a central difference (+-1e-5)."""
    from ipie_b200 import synthetic
    from ipie_b200.adjoint import LocalEnergyGreens

    s = synthetic.generate(30, (5, 4), 90, decay=30.0, seed=4, uhf=True, chol_scale="stable")
    W = 3
    ham, trial, walkers, prop = gpu_objects(s, W)
    rng = np.random.default_rng(8)
    ga0 = torch.from_numpy(rng.normal(0, 0.3, (W, 5, 30)) + 1j * rng.normal(0, 0.3, (W, 5, 30))).cuda()
    gb0 = torch.from_numpy(rng.normal(0, 0.3, (W, 4, 30)) + 1j * rng.normal(0, 0.3, (W, 4, 30))).cuda()
    da = torch.from_numpy(rng.normal(size=(W, 5, 30))).cuda().to(torch.complex128)
    db = torch.from_numpy(rng.normal(size=(W, 4, 30))).cuda().to(torch.complex128)
    ga = ga0.clone().requires_grad_(True)
    gb = gb0.clone().requires_grad_(True)
    LocalEnergyGreens.apply(ga, gb, ham, trial, False).real.sum().backward()
    # torch's gradient of a real loss w.r.t. complex z is dL/dRe z + i dL/dIm z: along a real
    # direction d the derivative is Re(conj(grad) . d)
    ad = float((ga.grad.conj() * da).real.sum() + (gb.grad.conj() * db).real.sum())
    h = 1e-5
    ep = LocalEnergyGreens.apply(ga0 + h * da, gb0 + h * db, ham, trial, False).real.sum()
    em = LocalEnergyGreens.apply(ga0 - h * da, gb0 - h * db, ham, trial, False).real.sum()
    fd = float(ep - em) / (2 * h)
    assert abs(ad - fd) < 1e-6 * max(1.0, abs(fd))
