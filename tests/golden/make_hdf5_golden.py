"""Golden fixture for the HDF5 readers: ipie's neon cc-pVDZ integration input.

Run from the repository root with ipie's source tree available:

    python tests/golden/make_hdf5_golden.py /path/to/ipie-checkout

ipie's integration test ``qmc/tests/reference_data/neon_cc-pvdz_rhf`` ships its
input (``afqmc.h5``: a QMCPACK dense Hamiltonian, M=10, X=27, and a NOMSD
UHF-layout single determinant, 5+5 electrons) and ipie's recorded output
(``reference.json``).  Block 0 of that output is the mixed estimate over walkers
that all equal the initial determinant, so it depends on the file's contents only
(not on the 4 MPI ranks or their random streams of the later blocks).  This script
reads the file with ``ipie_b200.io`` (``from_qmcpack_dense``,
``read_qmcpack_wfn_hdf``), checks that the oracle's local energy of those arrays
reproduces ipie's block-0 ``ETotal``, ``E1Body`` and ``E2Body``, and stores the
arrays and the recorded values in ``neon_qmcpack.npz``.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ipie_b200 import io  # noqa: E402
from oracle import afqmc_oracle as O  # noqa: E402


def main(ref):
    d = os.path.join(ref, "ipie", "qmc", "tests", "reference_data", "neon_cc-pvdz_rhf")
    fname = os.path.join(d, "afqmc.h5")
    hcore, chol, enuc, nmo, na, nb = io.from_qmcpack_dense(fname)
    (coeffs, wfn), psi0, nelec = io.read_qmcpack_wfn_hdf(fname, get_nelec=True)
    assert len(coeffs) == 1 and nelec == (na, nb)
    with open(os.path.join(d, "reference.json")) as fh:
        rec = json.load(fh)
    S = O.System(nmo, na, nb, np.array([hcore, hcore]), chol, float(enuc), wfn[0]).build()
    w = O.Walkers.from_initial(psi0, na, 1)
    O.greens_function(S, w)
    e = O.local_energy_single_det_uhf_batch(S, w)[0].real
    block0 = np.array([rec["ETotal"][0], rec["E1Body"][0], rec["E2Body"][0]])
    err = np.abs(e - block0).max()
    print("oracle block-0 energies", e, "recorded", block0, "max diff", err)
    assert err < 1e-12, err
    with open(fname, "rb") as fh:
        sha = hashlib.sha256(fh.read()).hexdigest()
    np.savez_compressed(os.path.join(HERE, "neon_qmcpack.npz"), hcore=hcore, chol=chol, enuc=enuc,
                        nelec=np.array(nelec), psi=wfn[0], psi0=psi0, coeffs=coeffs, block0=block0,
                        file_sha256=np.array(sha))
    print("wrote neon_qmcpack.npz")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IPIE_SRC", ""))
