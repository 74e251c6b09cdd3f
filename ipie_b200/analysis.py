"""Error bars of block-energy series: ipie's reblocking analysis, restated.

ipie's ``analysis/blocking.py:133`` (``reblock_mixed``) reblocks each estimator column with
pyblock's Flyvbjerg-Petersen blocking (pyblock is an optional dependency of ipie, not pinned in
its requirements and absent here) and adds the autocorrelation-time reblocking of
``analysis/autocorr.py:54-105`` (``reblock_by_autocorr``) on ``ETotal``.  Both are restated here
on plain numpy arrays:

* :func:`reblock` -- Flyvbjerg & Petersen, J. Chem. Phys. 91, 461 (1989): repeatedly average
  neighbouring pairs; at each level the standard error of the mean and its own error; the
  optimal level is the first whose block length B satisfies B^3 > 2 n (s_B / s_0)^4 (Lee, Needs
  & Drummond, Phys. Rev. B 84, 245117 (2011), the criterion pyblock applies);
* :func:`reblock_by_autocorr` -- ipie's integrated autocorrelation time (FFT autocorrelation,
  Goodman-Weare automatic window with c = 5), blocks of ceil(tau) samples, the last block
  taking the remainder;
* :func:`reblock_mixed` -- both on one series, as ipie's ``reblock_mixed`` reports them.
"""
from __future__ import annotations

import math

import numpy as np


def _next_pow_two(n: int) -> int:
    p = 1
    while p < n:
        p <<= 1
    return p


def autocorrelation(y) -> np.ndarray:
    """Normalised autocorrelation function of a series by FFT (ipie ``autocorr.py:13-29``)."""
    y = np.atleast_1d(np.asarray(y, dtype=np.float64))
    if y.ndim != 1:
        raise ValueError("autocorrelation takes a 1-d series")
    n = _next_pow_two(len(y))
    f = np.fft.fft(y - y.mean(), n=2 * n)
    acf = np.fft.ifft(f * np.conjugate(f))[: len(y)].real
    return acf / acf[0] if acf[0] != 0 else acf


def integrated_time(y, c: float = 5.0) -> float:
    """Integrated autocorrelation time with the Goodman-Weare window: the first lag m with
    m >= c tau(m), tau(m) = 2 sum_{k<=m} rho_k - 1 (ipie ``autocorr.py:32-44``)."""
    taus = 2.0 * np.cumsum(autocorrelation(y)) - 1.0
    inside = np.arange(len(taus)) < c * taus
    window = int(np.argmin(inside)) if inside.any() else len(taus) - 1
    return float(taus[window])


def reblock_by_autocorr(y) -> dict:
    """Mean and error from blocks of ceil(tau) samples (ipie ``autocorr.py:54-105``): the block
    length comes from the whole series, the last block takes what is left over, and the error is
    the population standard deviation of the block means over sqrt(number of blocks)."""
    y = np.asarray(y, dtype=np.float64)
    block = max(1, int(math.ceil(integrated_time(y))))
    nblocks = max(1, len(y) // block)
    means = [y[i * block:(i + 1) * block].mean() if i < nblocks - 1 else y[i * block:].mean()
             for i in range(nblocks)]
    means = np.array(means)
    return {"mean": float(means.mean()), "error": float(means.std() / math.sqrt(nblocks)),
            "nsamp": nblocks, "block": block}


def reblock(y) -> list:
    """Flyvbjerg-Petersen levels: for block length 2^k, (block length, number of blocks, mean,
    standard error, error of the standard error).  A level needs at least two blocks."""
    y = np.asarray(y, dtype=np.float64)
    levels = []
    k = 0
    while len(y) >= 2:
        n = len(y)
        var = y.var(ddof=1)
        sem = math.sqrt(var / n)
        levels.append((2 ** k, n, float(y.mean()), sem, sem / math.sqrt(2.0 * (n - 1))))
        if n % 2:
            y = y[:-1]  # the unpaired last sample is dropped from the next level
        y = 0.5 * (y[0::2] + y[1::2])
        k += 1
    return levels


def optimal_level(levels, ndata: int):
    """Index of the first level with B^3 > 2 ndata (sem_B / sem_0)^4, or None when no level
    qualifies (too few samples for a converged error)."""
    if not levels:
        return None
    s0 = levels[0][3]
    for i, (B, _, _, sem, _) in enumerate(levels):
        ratio = sem / s0 if s0 > 0 else 1.0
        if B ** 3 > 2.0 * ndata * ratio ** 4:
            return i
    return None


def reblock_mixed(y) -> dict:
    """The two error estimates ipie's ``reblock_mixed`` reports for ``ETotal``: the blocking
    analysis at the optimal level (``error``, ``error_error``, ``block``; ``converged`` False when
    no level qualifies, in which case the largest-block level with at least 4 blocks stands in)
    and the autocorrelation reblocking (``error_ac``, ``block_ac``)."""
    y = np.asarray(y, dtype=np.float64)
    if len(y) < 2:
        raise ValueError("reblocking needs at least two samples")
    levels = reblock(y)
    opt = optimal_level(levels, len(y))
    converged = opt is not None
    if opt is None:
        usable = [i for i, lv in enumerate(levels) if lv[1] >= 4] or [0]
        opt = usable[-1]
    B, n, mean, sem, sem_err = levels[opt]
    ac = reblock_by_autocorr(y)
    return {"mean": float(y.mean()), "error": sem, "error_error": sem_err, "block": B, "nblocks": n,
            "converged": converged, "error_ac": ac["error"], "block_ac": ac["block"], "n": len(y)}
