"""Host-side logic of the drop-in that runs without a GPU."""
import numpy as np
import pytest

from ipie_b200 import synthetic
from ipie_b200.pop_control import pair_branch_table
from oracle import afqmc_oracle as O


@pytest.mark.parametrize("seed", range(5))
def test_pair_branch_table_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    w = np.abs(rng.lognormal(0.0, 1.2, size=64))
    w[rng.integers(0, 64, 5)] = 0.0
    d1 = np.random.default_rng(seed + 100).random(64)
    d2 = d1.copy()
    it1, it2 = iter(d1), iter(d2)
    a = pair_branch_table(w, 4.0, 0.1, rand=lambda: next(it1))
    b = O.pair_branch_table(w, 4.0, 0.1, rand=lambda: next(it2))
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_pair_branch_conserves_pair_weight_and_counts():
    w = np.array([0.05, 0.5, 5.0, 1.0, 0.08, 6.0, 1.1, 0.9])
    neww, st = pair_branch_table(w, 4.0, 0.1, rand=lambda: 0.3)
    assert (st == 2).sum() == (st == 0).sum()
    assert np.isclose(neww.sum(), w.sum() - (w[st == 0].sum() + w[st == 2].sum()) + neww[st == 2].sum())


def test_synthetic_generator_shapes_and_symmetry():
    s = synthetic.generate(12, (3, 2), 20, decay=10.0, seed=1, uhf=True)
    L = s.chol.T.reshape(20, 12, 12)
    assert np.allclose(L, np.swapaxes(L, 1, 2))
    assert np.allclose(s.h1e[0], s.h1e[0].T)
    assert np.allclose(np.diag(s.h1e[0]), np.linspace(-2, 1, 12))
    assert s.psi.shape == (12, 5)
    # orthonormal occupied orbitals per spin
    assert np.allclose(s.psi[:, :3].T @ s.psi[:, :3], np.eye(3))


def test_stable_scale_pins_field_operator_norm():
    """The stable amplitude keeps |VHS|_2 ~ 0.24 across sizes (literal 0.3 grows like sqrt(decay*M))."""
    norms = []
    for M, X, d in ((26, 120, 30.0), (60, 240, 60.0)):
        s = synthetic.generate(M, 4, X, decay=d, seed=2, chol_scale="stable")
        S = O.System(s.nbasis, s.nup, s.ndown, s.h1e, s.chol, s.ecore, s.psi).build()
        xs = np.random.default_rng(0).normal(size=(X, 3)).astype(complex)
        norms.append(np.mean([np.linalg.norm(v, 2) for v in O.construct_vhs(S, xs)]))
    assert 0.15 < norms[0] < 0.35 and 0.15 < norms[1] < 0.35


def test_exchange_gradient_is_the_derivative_of_the_oracle_exchange():
    """K = d raw / d Ghalf (raw = 2 * oracle exx): central differences are exact for the quadratic."""
    torch = pytest.importorskip("torch")
    from ipie_b200.control_variate import exchange_gradient

    rng = np.random.default_rng(4)
    X, N, M = 12, 3, 7
    rchol = rng.normal(size=(X, N * M))
    g = rng.normal(size=(N, M)) + 1j * rng.normal(size=(N, M))
    d = rng.normal(size=(N, M)) + 1j * rng.normal(size=(N, M))
    K = exchange_gradient(torch.from_numpy(rchol), torch.from_numpy(g)).numpy()
    eps = 0.37
    raw = lambda G: 2.0 * O.exx_kernel(rchol.reshape(X, N, M), G[None])[0]  # noqa: E731
    fd = (raw(g + eps * d) - raw(g - eps * d)) / (2 * eps)
    assert abs(fd - np.sum(K * d)) < 1e-10 * abs(fd)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_comb_and_reconfiguration_tables_match_oracle(seed):
    """Host decisions of comb and stochastic reconfiguration equal the oracle's ipie restatement."""
    from ipie_b200.pop_control import comb_parent_counts, reconfiguration_sources

    rng = np.random.default_rng(seed)
    w = rng.exponential(size=37) * (rng.random(37) < 0.9)
    r = rng.random()
    assert np.array_equal(comb_parent_counts(w, 37, r), O.comb_parent_counts(w, 37, r))
    # the oracle's walker-level restatement on dummy walkers carrying their index
    ow = O.Walkers.from_initial(np.eye(4, 2), 1, 37)
    ow.weight = w.copy()
    ow.phia = np.arange(37, dtype=np.complex128)[:, None, None] * np.ones((37, 4, 1))
    ix = O.stochastic_reconfiguration(ow, rand=lambda: r)
    src, mean_w = reconfiguration_sources(np.abs(w), r)
    assert np.array_equal(src, ix)
    assert np.allclose(ow.phia[:, 0, 0].real, src)
    assert np.all(ow.weight == mean_w)


@pytest.mark.parametrize("M", [1, 7, 26, 30, 108, 200])
def test_tiled_packing_covers_the_upper_triangle_once(M):
    from ipie_b200.hamiltonian import tiled_triu_indices

    i, j = tiled_triu_indices(M)
    assert len(i) == M * (M + 1) // 2
    pairs = set(zip(i.tolist(), j.tolist()))
    assert len(pairs) == len(i)
    assert all(a <= b < M for a, b in pairs)


def test_complex_cholesky_host_setup_matches_ipie():
    """``Generic`` picks the complex-Cholesky class for complex vectors; its h1e_mod, the trial's
    half rotations, the mean-field shift and the one-body propagator (all host set-up) equal ipie's."""
    from ipie_b200 import SingleDet
    from ipie_b200.hamiltonian import GenericComplexChol
    from ipie_b200.propagation import construct_mean_field_shift, construct_one_body_propagator
    from tests._systems import load

    f = load("complex_uhf_m20.npz")
    s = synthetic.generate_complex(20, (4, 3), 60, decay=30.0, seed=3, uhf=True)
    ham = GenericComplexChol(s.h1e, s.chol, s.ecore, device="cpu")
    assert ham.complex_chol and ham.nfields == 2 * s.nchol
    np.testing.assert_allclose(ham.h1e_mod, f["h1e_mod"], rtol=0, atol=1e-13 * np.abs(f["h1e_mod"]).max())
    trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis, device="cpu")
    trial.half_rotate(ham)
    for k in ("rchola", "rcholb", "rcholbara", "rcholbarb", "rAa", "rAb", "rBa", "rBb"):
        ref = f[k]
        assert np.max(np.abs(getattr(trial, "_" + k) - ref)) <= 1e-13 * np.abs(ref).max(), k
    for k in ("rH1a", "rH1b"):
        ref = f[k]
        assert np.max(np.abs(getattr(trial, "_" + k).numpy() - ref)) <= 1e-13 * np.abs(ref).max(), k
    # the device operands: C = [A | B] parts and the polarised exchange stacks
    C = ham.c_re.numpy() + 1j * ham.c_im.numpy()
    assert np.array_equal(C[:, : s.nchol], ham.A) and np.array_equal(C[:, s.nchol:], ham.B)
    pol = trial._cplx["pola"].numpy()
    R, S = f["rchola"], f["rcholbara"]
    np.testing.assert_allclose(pol[4], R.real + S.imag, atol=1e-13)
    np.testing.assert_allclose(pol[7], R.imag - S.real, atol=1e-13)
    mf = construct_mean_field_shift(ham, trial)
    assert np.max(np.abs(mf - f["mf_shift"])) <= 1e-12 * np.abs(f["mf_shift"]).max()
    expH1 = construct_one_body_propagator(ham, mf, 0.005)
    assert np.max(np.abs(expH1 - f["expH1"])) <= 1e-12


@pytest.mark.parametrize("case", ["b", "m", "c"])
def test_ghf_half_rotation_reproduces_the_four_block_energy(case):
    """The GHF trial's half rotation over both spin blocks (R = [psi_a^H K | psi_b^H K], rH1) gives
    the force bias, one-body energy, Coulomb and exchange of ipie's full-G GHF formulas (the oracle):
    the identities the device path relies on, checked in numpy on perturbed walkers."""
    from ipie_b200.ghf import SingleDetGHF
    from ipie_b200.hamiltonian import Generic
    from oracle import ghf_oracle as G
    from tests._systems import load

    f = load("ghf_m14.npz")
    s = synthetic.generate(14, (4, 3), 40, decay=30.0, seed=8, uhf=True, chol_scale="stable")
    chol = s.chol + 1.0j * f["c_chol_imag"] if case == "c" else s.chol
    psi = G.ghf_from_uhf(s.psi, s.nup, s.nbasis) if case == "b" else f["m_psi"]
    from ipie_b200.hamiltonian import GenericComplexChol, GenericRealChol

    ham = (GenericComplexChol if case == "c" else GenericRealChol)(s.h1e, chol, s.ecore, device="cpu")
    trial = SingleDetGHF(psi, (s.nup, s.ndown), s.nbasis, device="cpu")
    trial.half_rotate(ham)
    S = G.GHFSystem(nbasis=s.nbasis, nalpha=s.nup, nbeta=s.ndown, h1e=s.h1e, chol=chol, ecore=s.ecore, psi=psi).build()
    w = S.walkers(psi, 5)
    w.phia = f[case + "_phi_in"].copy()
    G.greens_function_ghf(S, w)
    gh = w.Ghalfa.reshape(5, -1)  # (W, N * 2M)
    R = trial._R
    X = s.nchol
    vb = gh @ R.T
    ref_vb = G.force_bias_ghf(S, w)
    assert np.max(np.abs(vb - ref_vb)) <= 1e-12 * np.abs(ref_vb).max()
    rH1 = trial._rH1a.numpy().ravel()
    e1 = gh @ rH1 + s.ecore
    ecoul = 0.5 * np.einsum("wx,wx->w", vb, vb)
    N, M2 = s.nup + s.ndown, 2 * s.nbasis
    T = np.einsum("xnk,wmk->wxnm", R.reshape(R.shape[0], N, M2), w.Ghalfa, optimize=True)
    exx = 0.5 * np.einsum("wxnm,wxmn->w", T, T, optimize=True)
    ref = G.local_energy_ghf(S, w)
    assert np.max(np.abs(e1 - ref[:, 1])) <= 1e-12 * np.abs(ref[:, 1]).max()
    assert np.max(np.abs(ecoul - exx - ref[:, 2])) <= 1e-11 * np.abs(ref[:, 2]).max()
    assert R.shape[0] == (2 * X if case == "c" else X)


def test_pair_branch_pairs_replay():
    """The pairs recorded by the pairing walk, applied to the same weights, give the walk's own
    result; applied to perturbed weights they branch the same walkers."""
    from ipie_b200.pop_control import apply_pairs, pair_branch_table

    rng = np.random.default_rng(3)
    absw = np.exp(rng.normal(0.0, 1.5, size=300))
    absw *= absw.size / absw.sum()
    draws = rng.uniform(size=300)
    it = iter(draws)
    pairs = []
    neww, status = pair_branch_table(absw, 4.0, 0.1, lambda: next(it), pairs=pairs)
    assert len(pairs) > 10
    w2, s2 = apply_pairs(absw, pairs)
    assert np.array_equal(s2, status)
    assert np.array_equal(w2, neww)
    w3, s3 = apply_pairs(absw * (1 + 1e-9 * rng.normal(size=absw.size)), pairs)
    assert np.array_equal(s3, status)
    assert np.allclose(w3, neww, rtol=1e-8)
