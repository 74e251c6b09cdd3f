"""Pin the complex-Cholesky oracle (ipie's ``GenericComplexChol`` path) against ipie's own outputs.

``tests/golden/complex_uhf_m20.npz`` was written by ``tests/golden/make_golden.py ... complex``
running ipie's numpy path on ``synthetic.generate_complex(20, (4, 3), 60, decay=30, seed=3,
uhf=True)``: set-up integrals, per-kernel outputs on perturbed walkers and three propagation
steps with ipie's own field draws.  CPU only.
"""
import numpy as np

from oracle import afqmc_oracle as O
from oracle.complex_chol_oracle import ComplexSystem
from tests._systems import checksum, load


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _system():
    from ipie_b200 import synthetic

    s = synthetic.generate_complex(20, (4, 3), 60, decay=30.0, seed=3, uhf=True)
    return s, ComplexSystem(nbasis=s.nbasis, nup=s.nup, ndown=s.ndown, h1e=s.h1e, chol=s.chol, ecore=s.ecore,
                            psi=s.psi).build()


def test_complex_fixture_inputs_regenerate():
    f = load("complex_uhf_m20.npz")
    s, _ = _system()
    np.testing.assert_allclose(checksum(s.chol), f["chol_checksum"], rtol=1e-13)
    np.testing.assert_allclose(checksum(s.psi), f["psi_checksum"], rtol=1e-13)


def test_complex_oracle_setup_matches_ipie():
    f = load("complex_uhf_m20.npz")
    _, S = _system()
    assert rel(S.h1e_mod, f["h1e_mod"]) < 1e-13
    for k in ("rchola", "rcholb", "rcholbara", "rcholbarb", "rAa", "rAb", "rBa", "rBb", "rH1a", "rH1b"):
        assert rel(getattr(S, k), f[k]) < 1e-13, k
    assert rel(S.mf_shift, f["mf_shift"]) < 1e-12
    assert rel(S.expH1, f["expH1"]) < 1e-12


def test_complex_oracle_kernels_match_ipie():
    f = load("complex_uhf_m20.npz")
    _, S = _system()
    W = f["phia_in"].shape[0]
    w = O.Walkers.from_initial(S.psi, S.nup, W)
    w.phia = f["phia_in"].copy()
    w.phib = f["phib_in"].copy()
    ovlp = O.greens_function(S, w)
    assert rel(ovlp, f["ovlp"]) < 1e-11
    assert rel(w.Ghalfa, f["Ghalfa"]) < 1e-11
    assert rel(S.vbias(w), f["vbias"]) < 1e-12
    assert rel(S.vhs(f["xshifted"]), f["VHS"]) < 1e-13
    assert rel(S.local_energy(w), f["energy_uhf"]) < 1e-11


def test_complex_oracle_steps_match_ipie():
    """Three steps of the oracle with numpy's global stream seeded as ipie's run was."""
    f = load("complex_uhf_m20.npz")
    _, S = _system()
    W = f["phia_in"].shape[0]
    w = O.Walkers.from_initial(S.psi, S.nup, W)
    w.phia = f["phia_in"].copy()
    w.phib = f["phib_in"].copy()
    w.ovlp = f["ovlp"].copy()
    np.random.seed(21)
    for step in range(3):
        O.propagate_walkers(S, w, -7.0 if step else 0.0)
    assert rel(w.weight, f["walk_weight"]) < 1e-10
    assert rel(w.ovlp, f["walk_ovlp"]) < 1e-10
    assert rel(w.phia, f["walk_phia"]) < 1e-10
    assert rel(w.phib, f["walk_phib"]) < 1e-10
    assert rel(w.hybrid_energy, f["walk_hybrid_energy"]) < 1e-10
