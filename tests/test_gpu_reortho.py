"""Reorthogonalisation through the C ABI (`ipie_b200_reortho`) on well- and ill-conditioned
orbitals, against numpy's Householder QR with the sign fix ipie applies (positive diag R).

Blocks of at most 32 orbitals run Cholesky QR, whose error grows like cond(phi)^2 eps; a block
whose R diagonal spreads gets a second pass, so the result stays orthonormal to rounding and
matches the Householder factors to ~cond(phi) eps, as a backward-stable QR does.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _orbitals(W, M, N, cond, seed):
    """W blocks phi = U diag(s) V^H with singular values spread log-uniformly over [1/cond, 1]."""
    rng = np.random.default_rng(seed)
    out = np.empty((W, M, N), dtype=np.complex128)
    for w in range(W):
        u = np.linalg.qr(rng.normal(size=(M, N)) + 1j * rng.normal(size=(M, N)))[0]
        v = np.linalg.qr(rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N)))[0]
        s = np.logspace(0.0, -np.log10(cond), N)
        out[w] = (u * s) @ v.conj().T
    return out


def _householder(phi):
    q, r = np.linalg.qr(phi)
    d = np.diag(r)
    ph = d / np.abs(d)
    return q * ph, np.sum(np.log(np.abs(d)))


@pytest.mark.parametrize("M,N,cond,tol", [(200, 32, 1.5, 1e-12), (40, 8, 1e4, 1e-10), (60, 16, 1e6, 1e-8)])
def test_reortho_matches_householder(M, N, cond, tol):
    from ipie_b200._lib import call, ptr, stream

    W = 6
    phi0 = _orbitals(W, M, N, cond, seed=int(cond) % 97 + N)
    phi = torch.from_numpy(phi0).cuda()
    shift = torch.zeros(W, dtype=torch.float64, device="cuda")
    detR = torch.empty(W, dtype=torch.float64, device="cuda")
    logd = torch.zeros(W, dtype=torch.float64, device="cuda")
    ovlp = torch.ones(W, dtype=torch.complex128, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    # one spin block (phib aliases phia with no beta electrons)
    call("ipie_b200_reortho", ptr(phi), ptr(phi), W, M, N, 0, ptr(shift), ptr(detR), ptr(logd), ptr(ovlp),
         ptr(status), stream())
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    q = phi.cpu().numpy()
    for w in range(W):
        qh, logdet = _householder(phi0[w])
        assert np.abs(q[w].conj().T @ q[w] - np.eye(N)).max() < 1e-13
        assert np.abs(q[w] - qh).max() < tol
        assert abs(np.log(detR[w].item()) - logdet) < 1e-10 * max(1.0, abs(logdet))
        assert abs(logd[w].item() - logdet) < 1e-10 * max(1.0, abs(logdet))
        assert abs(ovlp[w].item() - np.exp(-logdet)) < 1e-10 * abs(np.exp(-logdet))
