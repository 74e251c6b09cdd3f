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
