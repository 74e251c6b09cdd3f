"""HDF5 readers and writers (``ipie_b200.h5lite``, ``ipie_b200.io``), CPU only.

The reader is pinned by ``tests/golden/neon_qmcpack.npz``: arrays read from ipie's neon
cc-pVDZ integration input (a file written by the HDF5 library) whose block-0 energies equal
ipie's recorded ones (``make_hdf5_golden.py`` asserts that when it writes the fixture; the
test below recomputes them).  The writer is checked by round trips through the reader in
every layout ipie uses.
"""
import numpy as np
import pytest

from ipie_b200 import h5lite, io
from oracle import afqmc_oracle as O
from tests._systems import load


def test_h5lite_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    tree = {
        "f8": rng.normal(size=(7, 5)),
        "f4": rng.normal(size=(3, 4, 2)).astype(np.float32),
        "i8": rng.integers(-10**12, 10**12, size=11),
        "i4": rng.integers(-1000, 1000, size=(2, 3)).astype(np.int32),
        "u2": rng.integers(0, 60000, size=9).astype(np.uint16),
        "c16": rng.normal(size=(4, 6)) + 1j * rng.normal(size=(4, 6)),
        "scalar_f": np.float64(3.25),
        "scalar_i": np.int64(-7),
        "text": np.bytes_(b"ENumer EDenom"),
        "names": np.array([b"Weight", b"WeightFactor", b"HybridEnergy"]),
        "empty": np.zeros((0, 3)),
        "flag": np.array([True, False]),
        "grp": {"a": np.arange(6.0), "sub": {"b": np.arange(4, dtype=np.int32)}, "empty_grp": {}},
    }
    tree.update({f"many_{i:03d}": np.full(i + 1, float(i)) for i in range(40)})
    p = tmp_path / "t.h5"
    h5lite.write_file(p, tree)
    with h5lite.File(p) as f:
        assert sorted(f.keys()) == sorted(tree.keys())
        for k in ("f8", "f4", "i8", "i4", "u2", "c16", "names"):
            v = f[k][()]
            assert v.dtype == tree[k].dtype and v.shape == tree[k].shape, k
            np.testing.assert_array_equal(v, tree[k])
        assert f["scalar_f"][()] == 3.25 and f["scalar_i"][()] == -7
        assert f["text"][()] == b"ENumer EDenom"
        assert f["empty"][()].shape == (0, 3)
        np.testing.assert_array_equal(f["flag"][()].astype(bool), [True, False])
        np.testing.assert_array_equal(f["grp/sub/b"][:], np.arange(4))
        np.testing.assert_array_equal(f["grp"]["a"][1:3], [1.0, 2.0])
        assert f["grp/empty_grp"].keys() == []
        assert "grp/sub" in f and "grp/missing" not in f
        for i in range(40):
            np.testing.assert_array_equal(f[f"many_{i:03d}"][()], np.full(i + 1, float(i)))
        with pytest.raises(KeyError):
            f["nope"]


def test_h5lite_rejects_other_files(tmp_path):
    p = tmp_path / "x.h5"
    p.write_bytes(b"not an hdf5 file" * 10)
    with pytest.raises(OSError):
        h5lite.File(p)


def test_native_hamiltonian_and_wavefunctions(tmp_path):
    rng = np.random.default_rng(1)
    M, X = 6, 9
    h = rng.normal(size=(M, M))
    h = h + h.T
    L = rng.normal(size=(X, M, M))
    io.write_hamiltonian(h, L, 1.5, filename=str(tmp_path / "ham.h5"))
    h2, L2, e0 = io.read_hamiltonian(str(tmp_path / "ham.h5"))
    np.testing.assert_array_equal(h2, h)
    np.testing.assert_array_equal(L2, L)
    assert e0 == 1.5
    # read_integrals: the native layout's chol comes back as (M, M, X) with chol[n, m, x] = LXmn[x, m, n]
    h3, chol, e3 = io.read_integrals(str(tmp_path / "ham.h5"))
    np.testing.assert_array_equal(chol, L.T.reshape(M, M, X))
    psi = rng.normal(size=(M, 3))
    io.write_wavefunction(psi, filename=str(tmp_path / "rhf.h5"))
    assert io.determine_wavefunction_type(str(tmp_path / "rhf.h5")) == "single_determinant"
    wfn, phi0 = io.read_wavefunction(str(tmp_path / "rhf.h5"))
    np.testing.assert_array_equal(wfn[0], psi)
    np.testing.assert_array_equal(wfn[1], psi)
    pa, pb = psi, rng.normal(size=(M, 2)) + 1j * rng.normal(size=(M, 2))
    io.write_wavefunction([pa, pb], filename=str(tmp_path / "uhf.h5"))
    wfn, phi0 = io.read_single_det_wavefunction(str(tmp_path / "uhf.h5"))
    np.testing.assert_array_equal(wfn[1], pb)
    np.testing.assert_array_equal(phi0[1], pb)
    ci = np.array([0.9, -0.3 + 0.1j])
    occa, occb = np.array([[0, 1, 2], [0, 1, 3]]), np.array([[0, 1], [0, 2]])
    io.write_wavefunction((ci, occa, occb), filename=str(tmp_path / "ph.h5"))
    assert io.determine_wavefunction_type(str(tmp_path / "ph.h5")) == "particle_hole"
    (c2, a2, b2), _ = io.read_wavefunction(str(tmp_path / "ph.h5"))
    np.testing.assert_array_equal(c2, ci)
    np.testing.assert_array_equal(b2, occb)
    io.write_wavefunction((ci, [np.stack([pa, pa]), np.stack([pb, pb])]), filename=str(tmp_path / "noci.h5"))
    assert io.determine_wavefunction_type(str(tmp_path / "noci.h5")) == "noci"
    (c3, (a3, b3)), _ = io.read_wavefunction(str(tmp_path / "noci.h5"))
    np.testing.assert_array_equal(b3[1], pb)


@pytest.mark.parametrize("real", [True, False])
def test_qmcpack_layouts_round_trip(tmp_path, real):
    rng = np.random.default_rng(2)
    M, X, na, nb = 7, 12, 3, 2
    h = rng.normal(size=(M, M))
    h = h + h.T
    chol = rng.normal(size=(M * M, X))
    chol[np.abs(chol) < 0.3] = 0.0
    if not real:
        h = h + 1j * (rng.normal(size=(M, M)) - rng.normal(size=(M, M)).T) * 0.0
        chol = chol + 0.2j * rng.normal(size=(M * M, X))
    dense = str(tmp_path / "dense.h5")
    io.write_qmcpack_dense(h, chol, (na, nb), M, enuc=2.5, filename=dense, real_chol=real)
    h2, c2, e2, nmo, a2, b2 = io.from_qmcpack_dense(dense)
    np.testing.assert_array_equal(h2, h)
    np.testing.assert_array_equal(c2, chol)
    assert (e2, nmo, a2, b2) == (2.5, M, na, nb)
    sparse = str(tmp_path / "sparse.h5")
    io.write_qmcpack_sparse(h, chol, (na, nb), M, enuc=2.5, filename=sparse, real_chol=real)
    h3, c3, e3, *_ = io.from_qmcpack_sparse(sparse)
    np.testing.assert_allclose(c3.toarray(), chol, rtol=0, atol=0)
    np.testing.assert_allclose(h3, h, rtol=0, atol=0)
    with pytest.raises(KeyError):
        io.from_qmcpack_sparse(dense)
    # read_integrals tries sparse, then dense
    for fname in (sparse, dense):
        _, c4, e4 = io.read_integrals(fname)
        np.testing.assert_allclose(np.asarray(c4).reshape(M * M, X), chol, rtol=0, atol=0)


@pytest.mark.parametrize("uhf", [False, True])
def test_qmcpack_wavefunction_round_trip(tmp_path, uhf):
    rng = np.random.default_rng(3)
    M, na, nb = 8, 3, 3 if not uhf else 2
    psi = np.linalg.qr(rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M)))[0]
    wfn = np.hstack([psi[:, :na], psi[:, :nb] if not uhf else psi[:, na:na + nb]])
    f = str(tmp_path / "wfn.h5")
    io.write_qmcpack_wfn(f, (np.array([1.0 + 0j]), wfn.copy()), "uhf" if uhf else "rhf", (na, nb), M)
    (coeffs, w2), psi0, nelec = io.read_qmcpack_wfn_hdf(f, get_nelec=True)
    assert nelec == (na, nb)
    np.testing.assert_allclose(w2[0], wfn, rtol=0, atol=1e-15)
    np.testing.assert_allclose(psi0, wfn, rtol=0, atol=1e-15)
    assert io.determine_wavefunction_type(f) == "qmcpack"
    # particle-hole layout
    occa, occb = np.array([[0, 1, 2]]), np.array([[0, 1, 2]])
    f2 = str(tmp_path / "ph.h5")
    io.write_qmcpack_wfn(f2, (np.array([1.0 + 0j]), occa, occb), "uhf", (3, 3), M,
                         init=[wfn[:, :na], wfn[:, :na]])
    (c, a, b), psi0 = io.read_qmcpack_wfn_hdf(f2)
    np.testing.assert_array_equal(a, occa)
    np.testing.assert_array_equal(b, occb)


def test_neon_qmcpack_input_pins_the_reader(tmp_path):
    """The arrays that h5lite read from ipie's neon input give ipie's recorded block-0
    energies; written back in the QMCPACK layouts and read again they are unchanged."""
    f = load("neon_qmcpack.npz")
    na, nb = (int(x) for x in f["nelec"])
    M = f["hcore"].shape[0]
    S = O.System(M, na, nb, np.array([f["hcore"], f["hcore"]]), f["chol"], float(f["enuc"]), f["psi"]).build()
    w = O.Walkers.from_initial(f["psi0"], na, 1)
    O.greens_function(S, w)
    e = O.local_energy_single_det_uhf_batch(S, w)[0].real
    np.testing.assert_allclose(e, f["block0"], rtol=0, atol=1e-12)
    ham_f, wfn_f = str(tmp_path / "ham.h5"), str(tmp_path / "wfn.h5")
    io.write_qmcpack_dense(f["hcore"], f["chol"], (na, nb), M, enuc=float(f["enuc"]), filename=ham_f)
    io.write_qmcpack_wfn(wfn_f, (f["coeffs"], f["psi"].astype(np.complex128)), "uhf", (na, nb), M)
    h, chol, ecore = io.read_integrals(ham_f)
    np.testing.assert_array_equal(chol, f["chol"])
    trial = io.get_trial_wavefunction((na, nb), M, wfn_f, device="cpu")
    assert trial.nelec == (na, nb)
    np.testing.assert_allclose(trial.psi, f["psi"], rtol=0, atol=1e-15)
    ham = io.get_hamiltonian(ham_f, device="cpu")
    assert ham.nbasis == M and ham.nchol == f["chol"].shape[1] and ham.ecore == float(f["enuc"])


def test_estimator_file_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    rows = rng.normal(size=(7, 8))
    p = str(tmp_path / "estimates.0.h5")
    io.write_estimates(p, rows, metadata='{"qmc": {"dt": 0.005}}', buffer_size=4)
    df = io.extract_observable(p, "energy")
    assert list(df.columns) == ["Weight", "WeightFactor", "HybridEnergy", "ENumer", "EDenom", "ETotal", "E1Body",
                                "E2Body"]
    # ipie's extraction sums the per-chunk last-row indices (3 + 2): the layout is kept as is
    np.testing.assert_array_equal(df.values, rows[:6])
    with h5lite.File(p) as f:
        assert f["metadata"][()] == b'{"qmc": {"dt": 0.005}}'
        assert f["block_size_1/offset/energy"][()] == 3
        assert sorted(f["block_size_1/data"].keys()) == ["000000000", "000000001"]


def _chunked_file(path, arr, chunk, deflate):
    """A file holding one 2-D float64 dataset in chunked layout (version-1 B-tree of type 1), the
    chunks optionally deflate-compressed: built by hand from the format specification so the
    reader's chunk path is exercised without h5py."""
    import struct
    import zlib

    from ipie_b200.h5lite import _Writer, _dtype_msg, _message, _object_header, SIGNATURE

    w = _Writer(leaf_k=4)
    w.alloc(96)
    rows, cols = arr.shape
    cr, cc = chunk
    keys = []
    for r0 in range(0, rows, cr):
        for c0 in range(0, cols, cc):
            blk = np.zeros((cr, cc))
            sub = arr[r0:r0 + cr, c0:c0 + cc]
            blk[: sub.shape[0], : sub.shape[1]] = sub
            raw = blk.astype("<f8").tobytes()
            if deflate:
                raw = zlib.compress(raw)
            a = w.alloc(len(raw))
            w.put(a, raw)
            keys.append((len(raw), r0, c0, a))
    ksize = 8 + 8 * 3
    node = w.alloc(24 + len(keys) * (ksize + 8) + ksize)
    body = b""
    for size, r0, c0, a in keys:
        body += struct.pack("<IIQQQ", size, 0, r0, c0, 0) + struct.pack("<Q", a)
    body += struct.pack("<IIQQQ", 0, 0, rows, cols, 0)
    w.put(node, b"TREE" + struct.pack("<BBH", 1, 0, len(keys)) + b"\xff" * 16 + body)
    space = struct.pack("<BBBB", 2, 2, 0, 1) + struct.pack("<QQ", rows, cols)
    layout = struct.pack("<BBBQ", 3, 2, 3, node) + struct.pack("<III", cr, cc, 8)
    msgs = [_message(0x0001, space), _message(0x0003, _dtype_msg(np.dtype("<f8")), 1), _message(0x0008, layout)]
    if deflate:
        msgs.append(_message(0x000B, struct.pack("<BB6xHHHH", 1, 1, 1, 0, 1, 1) + struct.pack("<I4x", 6)))
    hdr = _object_header(msgs)
    oh = w.alloc(len(hdr))
    w.put(oh, hdr)
    names = b"\0" * 8 + b"data\0\0\0\0"
    hd = w.alloc(len(names))
    w.put(hd, names)
    heap = w.alloc(32)
    w.put(heap, b"HEAP" + struct.pack("<B3xQ", 0, len(names)) + b"\xff" * 8 + struct.pack("<Q", hd))
    snod = w.alloc(8 + 8 * 40)
    w.put(snod, b"SNOD" + struct.pack("<BBH", 1, 0, 1) + struct.pack("<QQII16x", 8, oh, 0, 0))
    bt = w.alloc(24 + 33 * 8 + 32 * 8)
    w.put(bt, b"TREE" + struct.pack("<BBH", 0, 0, 1) + b"\xff" * 16 + struct.pack("<QQQ", 0, snod, 8))
    ghdr = _object_header([_message(0x0011, struct.pack("<QQ", bt, heap))])
    root = w.alloc(len(ghdr))
    w.put(root, ghdr)
    sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0)
    sb += struct.pack("<Q", 0) + b"\xff" * 8 + struct.pack("<Q", len(w.buf)) + b"\xff" * 8
    sb += struct.pack("<QQII", 0, root, 1, 0) + struct.pack("<QQ", bt, heap)
    w.put(0, sb)
    with open(path, "wb") as fh:
        fh.write(bytes(w.buf))


@pytest.mark.parametrize("deflate", [False, True])
def test_h5lite_reads_chunked_datasets(tmp_path, deflate):
    arr = np.random.default_rng(5).normal(size=(13, 10))
    p = tmp_path / "chunked.h5"
    _chunked_file(p, arr, (4, 3), deflate)
    with h5lite.File(p) as f:
        d = f["data"]
        assert d.shape == (13, 10)
        np.testing.assert_array_equal(d[()], arr)
