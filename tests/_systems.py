"""Shared builders for the tests: synthetic systems and fixture loading."""
import os

import numpy as np

from ipie_b200 import synthetic
from oracle import afqmc_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def checksum(a):
    a = np.ascontiguousarray(a)
    return np.array([a.real.sum(), (a.real ** 2).sum(), np.abs(a).max()])


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def fixture_system(name):
    """The synthetic system a golden fixture was generated from."""
    if name == "kernels_rhf_m26.npz":
        s = synthetic.workload("c0_rhf_m26")
    elif name == "kernels_uhf_m30.npz":
        s = synthetic.generate(30, (6, 4), 90, decay=30.0, seed=5, uhf=True)
    elif name == "run_rhf_m26.npz":
        s = synthetic.workload("c0_rhf_m26", chol_scale="stable")
    elif name == "run_uhf_m30.npz":
        s = synthetic.generate(30, (6, 4), 90, decay=30.0, seed=5, uhf=True, chol_scale=0.1)
    else:
        raise KeyError(name)
    return s


def oracle_system(s, dt=0.005):
    return O.System(s.nbasis, s.nup, s.ndown, s.h1e, s.chol, s.ecore, s.psi, dt=dt).build()


RUN_PARAMS = {
    "run_rhf_m26.npz": dict(nwalkers=16, num_blocks=3, seed=7),
    "run_uhf_m30.npz": dict(nwalkers=12, num_blocks=3, seed=9),
}
