"""Reblocking of block-energy series (CPU): ipie's autocorrelation reblocking reproduced on its
own outputs, and the Flyvbjerg-Petersen levels on series with known errors."""
import math

import numpy as np

from ipie_b200 import analysis
from tests._systems import load


def test_reblock_by_autocorr_matches_ipie():
    f = load("reblock_autocorr.npz")
    for key in f["cases"]:
        y, ref = f[f"{key}_y"], f[f"{key}_ref"]
        got = analysis.reblock_by_autocorr(y)
        assert abs(got["mean"] - ref[0]) <= 1e-13 * abs(ref[0]), key
        assert abs(got["error"] - ref[1]) <= 1e-12 * ref[1], key
        assert got["nsamp"] == int(ref[2]) and got["block"] == int(ref[3]), key


def test_blocking_levels_halve_and_average():
    y = np.arange(11, dtype=np.float64)
    levels = analysis.reblock(y)
    assert [lv[0] for lv in levels] == [1, 2, 4, 8][: len(levels)]
    assert [lv[1] for lv in levels] == [11, 5, 2]
    assert levels[0][2] == 5.0
    assert math.isclose(levels[0][3], y.std(ddof=1) / math.sqrt(11))
    assert levels[1][2] == np.mean([0.5, 2.5, 4.5, 6.5, 8.5])


def test_reblock_mixed_white_noise_and_ar1():
    rng = np.random.default_rng(5)
    # white noise: the error is the plain standard error (level 0 qualifies)
    y = rng.normal(size=4096)
    r = analysis.reblock_mixed(y)
    assert r["converged"]
    assert abs(r["error"] - y.std(ddof=1) / 64.0) < 0.15 * r["error"]
    # AR(1) with phi = 0.8: the true error of the mean is sqrt((1+phi)/(1-phi)) = 3 times the naive one
    n, phi = 2 ** 16, 0.8
    e = rng.normal(size=n)
    z = np.empty(n)
    z[0] = e[0] / math.sqrt(1 - phi * phi)
    for i in range(1, n):
        z[i] = phi * z[i - 1] + e[i]
    r = analysis.reblock_mixed(z)
    naive = z.std(ddof=1) / math.sqrt(n)
    assert r["converged"] and r["block"] > 1
    assert 2.5 < r["error"] / naive < 3.5
    # blocks of ceil(tau) samples (ipie's choice) are still slightly correlated: a little below 3
    assert 2.0 < r["error_ac"] / naive < 3.5
