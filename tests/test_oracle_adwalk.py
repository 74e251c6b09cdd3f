"""The AD-walk oracle (ipie's AD-AFQMC block with its derivative along a one-body coupling, in
numpy) against ipie's own torch-autograd result on the same draws (CPU)."""
import numpy as np

from ipie_b200 import synthetic
from oracle.ad_walk_oracle import ADSystem
from tests._systems import checksum, load


def ad_fixture_system():
    f = load("ad_walk_m14.npz")
    s = synthetic.generate(14, (3, 3), 36, decay=30.0, seed=21, uhf=False, chol_scale="stable")
    np.testing.assert_allclose(checksum(s.chol), f["chol_checksum"], rtol=1e-13)
    L = s.chol.T.reshape(s.nchol, s.nbasis, s.nbasis)
    S = ADSystem(s.h1e[0], L, s.ecore, f["V"], f["C"], s.nup)
    return f, s, S


def test_ad_walk_oracle_matches_ipie_autograd():
    f, s, S = ad_fixture_system()
    E, dE, W, dW, phi, w = S.ad_block(f["phi0"].copy(), f["w0"].copy(), f["draws"], f["zetas"])
    assert abs(E - f["energy"]) <= 1e-11 * abs(f["energy"])
    assert abs(W - f["total_weight"]) <= 1e-11 * abs(f["total_weight"])
    assert abs(dE - f["dE_dlambda"]) <= 1e-9 * abs(f["dE_dlambda"])
    assert abs(dW - f["dW_dlambda"]) <= 1e-9 * abs(f["dW_dlambda"])
    np.testing.assert_allclose(w, f["final_weight"], rtol=1e-12)
    # final orbitals up to the column gauge of the QR: compare Ghalf = phi (psi^H phi)^-1
    g = phi @ np.linalg.inv(phi[:, : s.nup, :])
    gr = f["final_phi"] @ np.linalg.inv(f["final_phi"][:, : s.nup, :])
    assert np.max(np.abs(g - gr)) <= 1e-10 * np.max(np.abs(gr))


def test_ad_walk_oracle_central_difference():
    """The forward-mode derivative against (E(+h) - E(-h)) / 2h with the same draws, the same
    reconfiguration choices and the same (detached) energy estimates (h = 1e-4)."""
    f, s, S = ad_fixture_system()
    chosen = []
    E0, dE, _, dW, _, _ = S.ad_block(f["phi0"].copy(), f["w0"].copy(), f["draws"], f["zetas"], sr_indices=chosen)
    L = s.chol.T.reshape(s.nchol, s.nbasis, s.nbasis)
    h = 1e-4
    res = []
    for sign in (1, -1):
        Sh = ADSystem(s.h1e[0] + sign * h * f["V"], L, s.ecore, f["V"], f["C"], s.nup)
        res.append(Sh.ad_block(f["phi0"].copy(), f["w0"].copy(), f["draws"], f["zetas"], sr_indices=list(chosen),
                               e_est_blocks=S.last_block_energies))
    fd_e = (res[0][0] - res[1][0]) / (2 * h)
    fd_w = (res[0][2] - res[1][2]) / (2 * h)
    assert abs(fd_e - dE) <= 1e-6 * max(abs(dE), 1e-3)
    assert abs(fd_w - dW) <= 1e-6 * max(abs(dW), 1e-3)
