"""The multi-determinant oracle (sums over determinants) against ipie's Wick's-theorem Green's
function and local energy (CPU)."""
import numpy as np

from ipie_b200 import synthetic
from oracle.multidet_oracle import multi_det
from tests._systems import checksum, load


def test_multidet_oracle_matches_ipie_wicks():
    f = load("multidet_m14.npz")
    s = synthetic.generate(14, (4, 3), 42, decay=30.0, seed=31, uhf=True, chol_scale="stable")
    np.testing.assert_allclose(checksum(s.chol), f["chol_checksum"], rtol=1e-13)
    tot, Ga, Gb, en = multi_det(f["ci"], f["occa"], f["occb"], f["phia"], f["phib"], s.h1e, s.chol, s.ecore)
    for got, ref in ((tot, f["ovlp"]), (Ga, f["Ga"]), (Gb, f["Gb"]), (en, f["energy"])):
        assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_trial_1rdm_matches_ipie():
    """The particle-hole trial's 1-RDM (single excitations between its determinants with their
    permutation signs, ipie ``particle_hole.py:458-506``) from the host helper the trial uses, against
    ipie's ``trial.G`` in ``tests/golden/multidet_prop_m14.npz``; its trace is the electron count."""
    from ipie_b200.multidet import compute_1rdm

    f = load("multidet_prop_m14.npz")
    g = load("multidet_m14.npz")
    M = g["init"].shape[0]
    occs = [np.sort(np.concatenate([a, b + M])) for a, b in zip(g["occa"], g["occb"])]
    P = compute_1rdm(g["ci"], occs, M, len(g["ci"]))
    assert np.max(np.abs(P - f["G"])) < 1e-13
    assert abs(np.trace(P[0]) + np.trace(P[1]) - (g["occa"].shape[1] + g["occb"].shape[1])) < 1e-12
