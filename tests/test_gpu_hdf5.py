"""``AFQMC.build_from_hdf5`` and the estimator file on the GPU, on ipie's neon cc-pVDZ input.

The Hamiltonian and trial of ``tests/golden/neon_qmcpack.npz`` (read from ipie's own
integration input, see ``make_hdf5_golden.py``) are written in the QMCPACK layouts, the
driver is built from those files, and the run is compared with ipie's recorded block-0
energies and with the oracle's driver on the same draws (1e-10).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import afqmc_oracle as O  # noqa: E402
from tests._systems import load  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_build_from_hdf5_neon_matches_ipie_block0_and_oracle(tmp_path):
    from ipie_b200 import AFQMC, io

    f = load("neon_qmcpack.npz")
    na, nb = (int(x) for x in f["nelec"])
    M = f["hcore"].shape[0]
    ham_f, wfn_f, est_f = str(tmp_path / "ham.h5"), str(tmp_path / "wfn.h5"), str(tmp_path / "estimates.0.h5")
    io.write_qmcpack_dense(f["hcore"], f["chol"], (na, nb), M, enuc=float(f["enuc"]), filename=ham_f)
    io.write_qmcpack_wfn(wfn_f, (f["coeffs"], f["psi"].astype(np.complex128)), "uhf", (na, nb), M)
    W, nblocks = 16, 3
    afqmc = AFQMC.build_from_hdf5((na, nb), ham_f, wfn_f, num_walkers=W, seed=7, num_steps_per_block=10,
                                  num_blocks=nblocks, timestep=0.005, stabilize_freq=5, pop_control_freq=5,
                                  verbose=False)
    blocks = afqmc.run(estimator_filename=est_f)
    # rows: Weight, WeightFactor, HybridEnergy, ENumer, EDenom, ETotal, E1Body, E2Body
    np.testing.assert_allclose(blocks[0, 5:8], f["block0"], rtol=0, atol=1e-11)
    psi = np.real(f["psi"])
    S = O.System(M, na, nb, np.array([f["hcore"], f["hcore"]]), f["chol"], float(f["enuc"]), psi).build()
    ow = O.Walkers.from_initial(psi, na, W)
    ref = O.run_afqmc(S, ow, num_blocks=nblocks, num_steps_per_block=10, stabilize_freq=5, pop_control_freq=5,
                      seed=7)
    cols = ("Weight", "WeightFactor", "HybridEnergy", "ENumer", "EDenom", "ETotal", "E1Body", "E2Body")
    ref = np.array([[r[c] for c in cols] for r in ref])
    for col in (0, 1, 3, 4, 5, 6, 7):
        assert rel(blocks[:, col], ref[:, col]) < TOL, cols[col]
    w = afqmc.walkers
    assert rel(w.weight, ow.weight) < TOL
    assert rel(w.phia, ow.phia) < TOL
    assert rel(w.phib, ow.phib) < TOL
    df = io.extract_observable(est_f, "energy")
    assert len(df) == nblocks + 1
    np.testing.assert_allclose(df["ETotal"].values, blocks[:, 5], rtol=0, atol=0)
    np.testing.assert_allclose(df["Weight"].values, blocks[:, 0], rtol=0, atol=0)
