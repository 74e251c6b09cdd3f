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
    elif name == "run_c0_rhf_m26_w64.npz":
        s = synthetic.workload("c0_rhf_m26", chol_scale="stable")
    elif name == "run_c1_uhf_m108_w640.npz":
        s = synthetic.workload("c1_uhf_m108", chol_scale="stable")
    else:
        raise KeyError(name)
    return s


def oracle_system(s, dt=0.005):
    return O.System(s.nbasis, s.nup, s.ndown, s.h1e, s.chol, s.ecore, s.psi, dt=dt).build()


RUN_PARAMS = {
    "run_rhf_m26.npz": dict(nwalkers=16, num_blocks=3, seed=7, steps=25),
    "run_uhf_m30.npz": dict(nwalkers=12, num_blocks=3, seed=9, steps=25),
    # the workloads' own sizes: the small RHF workload (M=26, 64 walkers, 3 blocks with pop control)
    # and the UHF one (M=108, 15+15, X=600, 640 walkers, one 10-step block and its energy)
    "run_c0_rhf_m26_w64.npz": dict(nwalkers=64, num_blocks=3, seed=7, steps=25),
    "run_c1_uhf_m108_w640.npz": dict(nwalkers=640, num_blocks=1, seed=7, steps=10),
}


def compare_walkers(rel, w_phia, w_phib, f, tol):
    """Final orbitals against a run fixture: all of them, or the stored leading walkers plus the
    checksums of all of them (large batches)."""
    n = f["phia"].shape[0]
    assert rel(np.asarray(w_phia)[:n], f["phia"]) < tol
    assert rel(np.asarray(w_phib)[:n], f["phib"]) < tol
    for key, phi in (("phia_checksum", w_phia), ("phib_checksum", w_phib)):
        if key in f:
            c, ref = checksum(np.asarray(phi)), f[key]
            assert abs(c[0] - ref[0]) <= tol * np.asarray(phi).size * ref[2], key
            assert abs(c[1] - ref[1]) <= tol * ref[1], key
            assert abs(c[2] - ref[2]) <= tol * ref[2], key
