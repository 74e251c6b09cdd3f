"""Pin the GHF oracle (ipie's ``GHFWalkers`` / ``SingleDetGHF`` path) against ipie's own outputs.

``tests/golden/ghf_m14.npz`` was written by ``tests/golden/make_golden.py ... ghf`` running
ipie's numpy path on ``synthetic.generate(14, (4, 3), 40, decay=30, seed=8, uhf=True,
chol_scale="stable")``: case "b" with the trial and walkers built from UHF ones (block
diagonal), case "m" with a complex spin-mixed determinant, case "c" that determinant with
complex Cholesky vectors; per-kernel outputs on perturbed
walkers, a 3-step walk with ipie's draws and a reorthogonalisation.  CPU only.
"""
import numpy as np
import pytest

from oracle import afqmc_oracle as O
from oracle import ghf_oracle as G
from tests._systems import checksum, load


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def ghf_system(case, f=None):
    from ipie_b200 import synthetic

    s = synthetic.generate(14, (4, 3), 40, decay=30.0, seed=8, uhf=True, chol_scale="stable")
    psi = G.ghf_from_uhf(s.psi, s.nup, s.nbasis) if case == "b" else f["m_psi"]
    chol = s.chol + 1.0j * f["c_chol_imag"] if case == "c" else s.chol
    S = G.GHFSystem(nbasis=s.nbasis, nalpha=s.nup, nbeta=s.ndown, h1e=s.h1e, chol=chol, ecore=s.ecore,
                    psi=psi).build()
    init = G.ghf_from_uhf(s.init, s.nup, s.nbasis) if case == "b" else f["m_psi"]
    return s, S, init


def test_ghf_fixture_inputs_regenerate():
    f = load("ghf_m14.npz")
    s, _, _ = ghf_system("b", f)
    np.testing.assert_allclose(checksum(s.chol), f["chol_checksum"], rtol=1e-13)
    np.testing.assert_allclose(checksum(s.psi), f["psi_checksum"], rtol=1e-13)


@pytest.mark.parametrize("case", ["b", "m", "c"])
def test_ghf_oracle_matches_ipie(case):
    f = load("ghf_m14.npz")
    _, S, init = ghf_system(case, f)
    assert rel(S.mf_shift, f[case + "_mf_shift"]) < 1e-12
    assert rel(S.expH1, f[case + "_expH1"]) < 1e-12
    phi = f[case + "_phi_in"]
    W = phi.shape[0]
    w = S.walkers(init, W)
    w.phia = phi.copy()
    ovlp = G.greens_function_ghf(S, w)
    assert rel(ovlp, f[case + "_ovlp"]) < 1e-11
    assert rel(w.G, f[case + "_G"]) < 1e-11
    assert rel(G.force_bias_ghf(S, w), f[case + "_vbias"]) < 1e-12
    assert rel(G.local_energy_ghf(S, w), f[case + "_energy"]) < 1e-11
    w.ovlp = ovlp.copy()
    np.random.seed(31 + {"b": 1, "m": 2, "c": 3}[case])
    for step in range(3):
        G.propagate_walkers_ghf(S, w, -3.0 if step else 0.0)
    assert rel(w.weight, f[case + "_walk_weight"]) < 1e-10
    assert rel(w.ovlp, f[case + "_walk_ovlp"]) < 1e-10
    assert rel(w.phia, f[case + "_walk_phi"]) < 1e-10
    assert rel(w.hybrid_energy, f[case + "_walk_hybrid_energy"]) < 1e-10
    detR = G.reortho_ghf(S, w)
    assert rel(detR, f[case + "_reortho_detR"]) < 1e-12
    assert rel(w.phia, f[case + "_reortho_phi"]) < 1e-10
    assert rel(w.ovlp, f[case + "_reortho_ovlp"]) < 1e-10
