"""Hamiltonian and wavefunction files in ipie's HDF5 layouts, through :mod:`ipie_b200.h5lite`.

Same functions, file layouts and return values as ipie's ``utils/io.py``: the
native layout (``hcore``, ``LXmn``, ``e0``; ``psi_T_alpha`` ...), QMCPACK's
dense and sparse Hamiltonians (``Hamiltonian/...``) and its NOMSD / PHMSD
wavefunctions (``Wavefunction/...``).  The set-up helpers ``read_integrals``
(``hamiltonians/generic.py:160-178``), ``get_hamiltonian``
(``hamiltonians/utils.py:28-97``) and ``get_trial_wavefunction``
(``trial_wavefunction/utils.py:17-93``) build this package's device objects from
such files; single-determinant trials only (the walker step takes one
determinant).
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np
import scipy.sparse

from .h5lite import File, write_file


# ---------------------------------------------------------------- native layout (utils/io.py:31-191)
def write_hamiltonian(hcore: np.ndarray, LXmn: np.ndarray, e0: float, filename: str = "hamiltonian.h5") -> None:
    """``hcore`` (M, M), ``LXmn`` (naux, M, M), ``e0``; ipie ``utils/io.py:31-43``."""
    if hcore.ndim != 2:
        raise AssertionError(f"hcore must be a 2-d (M, M) array, got {hcore.ndim} dimensions")
    nmo = hcore.shape[0]
    naux = LXmn.size // (nmo * nmo)
    if LXmn.ndim != 3:
        raise AssertionError(f"LXmn must be a 3-d (naux, M, M) array, got {LXmn.ndim} dimensions")
    if LXmn.shape[0] != naux:
        raise AssertionError(f"LXmn has {LXmn.shape[0]} Cholesky vectors along axis 0, its size implies {naux}")
    write_file(filename, {"hcore": np.asarray(hcore), "LXmn": np.asarray(LXmn), "e0": np.float64(e0)})


def read_hamiltonian(filename: str) -> Tuple[np.ndarray, np.ndarray, float]:
    """ipie ``utils/io.py:46-57``."""
    with File(filename) as f:
        hcore = np.array(f["hcore"][()])
        LXmn = np.array(f["LXmn"][()])
        e0 = float(f["e0"][()])
    if hcore.ndim != 2:
        raise AssertionError(f"hcore must be a 2-d (M, M) array, got {hcore.ndim} dimensions")
    nmo = hcore.shape[0]
    naux = LXmn.size // (nmo * nmo)
    if LXmn.ndim != 3 or LXmn.shape[0] != naux:
        raise AssertionError(f"LXmn of shape {LXmn.shape} is not (naux, M, M) with M = {nmo}")
    return hcore, LXmn, e0


def write_wavefunction(wfn, filename: str = "wavefunction.h5", phi0=None) -> None:
    """Single determinant (array or [psia, psib]), particle-hole (ci, occa, occb) or NOCI
    (ci, [psia, psib]); ipie ``utils/io.py:60-74``."""
    if isinstance(wfn, (np.ndarray, list)):
        write_single_det_wavefunction(wfn, filename, phi0=phi0)
    elif len(wfn) == 3:
        write_particle_hole_wavefunction(wfn, filename, phi0=phi0)
    elif len(wfn) == 2:
        write_noci_wavefunction(wfn, filename, phi0=phi0)
    else:
        raise RuntimeError("wavefunction is neither an array/list, a (ci, occa, occb) triple nor a (ci, [psia, psib]) pair")


def write_single_det_wavefunction(wfn, filename: str, phi0=None) -> None:
    """ipie ``utils/io.py:108-128``: UHF as psi_T_alpha/beta (+ phi0_*), RHF as psi_T_alpha only."""
    if isinstance(wfn, list) or np.asarray(wfn).ndim == 3:
        if len(wfn) != 2:
            raise AssertionError("a UHF wavefunction is a pair [psia, psib]")
        tree = {"psi_T_alpha": np.asarray(wfn[0]), "psi_T_beta": np.asarray(wfn[1])}
        init = wfn if phi0 is None else phi0
        tree["phi0_alpha"] = np.asarray(init[0])
        tree["phi0_beta"] = np.asarray(init[1])
    else:
        wfn = np.asarray(wfn)
        if wfn.ndim != 2:
            raise AssertionError("an RHF wavefunction is one (M, N) array")
        tree = {"psi_T_alpha": wfn, "phi0_alpha": wfn if phi0 is None else np.asarray(phi0[0])}
    write_file(filename, tree)


def write_particle_hole_wavefunction(wfn: tuple, filename: str, phi0=None) -> None:
    """ipie ``utils/io.py:131-138``."""
    if len(wfn) != 3:
        raise AssertionError("a particle-hole wavefunction is the triple (ci, occa, occb)")
    write_file(filename, {"ci_coeffs": np.asarray(wfn[0]), "occ_alpha": np.asarray(wfn[1]),
                          "occ_beta": np.asarray(wfn[2])})


def write_noci_wavefunction(wfn: tuple, filename: str, phi0=None) -> None:
    """ipie ``utils/io.py:141-155``."""
    ci, (pa, pb) = wfn
    tree = {"ci_coeffs": np.asarray(ci), "psi_T_alpha": np.asarray(pa), "psi_T_beta": np.asarray(pb)}
    tree["phi0_alpha"] = np.asarray(pa[0] if phi0 is None else phi0[0])
    tree["phi0_beta"] = np.asarray(pb[0] if phi0 is None else phi0[1])
    write_file(filename, tree)


def read_particle_hole_wavefunction(filename: str):
    """ipie ``utils/io.py:158-165``."""
    with File(filename) as f:
        return (np.array(f["ci_coeffs"][()]), np.array(f["occ_alpha"][()]), np.array(f["occ_beta"][()])), None


def read_noci_wavefunction(filename: str):
    """ipie ``utils/io.py:168-175``."""
    with File(filename) as f:
        return (np.array(f["ci_coeffs"][()]), [np.array(f["psi_T_alpha"][()]), np.array(f["psi_T_beta"][()])]), None


def read_single_det_wavefunction(filename: str) -> Tuple[List[np.ndarray], List[np.ndarray]]:
    """ipie ``utils/io.py:178-190``: an RHF file returns the alpha orbitals for both spins."""
    with File(filename) as f:
        psia = np.array(f["psi_T_alpha"][()])
        phi0a = np.array(f["phi0_alpha"][()])
        if "psi_T_beta" in f:
            return [psia, np.array(f["psi_T_beta"][()])], [phi0a, np.array(f["phi0_beta"][()])]
    return [psia, psia], [phi0a, phi0a]


def read_wavefunction(filename: str):
    """ipie ``utils/io.py:77-89``: particle-hole, then NOCI, then single determinant."""
    for reader in (read_particle_hole_wavefunction, read_noci_wavefunction):
        try:
            return reader(filename)
        except KeyError:
            pass
    try:
        return read_single_det_wavefunction(filename)
    except Exception as exc:
        raise RuntimeError(f"{filename}: no wavefunction layout recognised") from exc


def determine_wavefunction_type(filename: str) -> str:
    """ipie ``utils/io.py:92-105``."""
    with File(filename) as f:
        keys = f.keys()
    if "occ_alpha" in keys:
        return "particle_hole"
    if "ci_coeffs" in keys:
        return "noci"
    if "psi_T_alpha" in keys:
        return "single_determinant"
    if "Wavefunction" in keys:
        return "qmcpack"
    raise RuntimeError(f"{filename}: no wavefunction datasets found")


# ---------------------------------------------------------------- QMCPACK layouts (utils/io.py:273-717)
def to_qmcpack_complex(array: np.ndarray) -> np.ndarray:
    """Complex array as float64 with a trailing (re, im) axis; ipie ``utils/io.py:525-527``."""
    array = np.ascontiguousarray(array, dtype=np.complex128)
    return array.view(np.float64).reshape(array.shape + (2,))


def from_qmcpack_complex(data: np.ndarray, shape) -> np.ndarray:
    """ipie ``utils/io.py:713-714``."""
    return np.ascontiguousarray(data).view(np.complex128).ravel().reshape(shape)


def from_qmcpack_dense(filename):
    """(hcore, chol (M*M, X), enuc, nmo, nalpha, nbeta); complex when stored with a (re, im) axis;
    ipie ``utils/io.py:530-546``."""
    with File(filename) as f:
        enuc = f["Hamiltonian/Energies"][()][0]
        dims = f["Hamiltonian/dims"][()]
        nmo = int(dims[3])
        hcore = np.array(f["Hamiltonian/hcore"][()])
        chol = np.array(f["Hamiltonian/DenseFactorized/L"][()])
        if hcore.ndim == 3 and hcore.shape[-1] == 2:
            hcore = from_qmcpack_complex(hcore, (nmo, nmo))
            chol = from_qmcpack_complex(chol, (nmo * nmo, -1))
        return hcore, chol, enuc, nmo, int(dims[4]), int(dims[5])


def from_qmcpack_sparse(filename):
    """(hcore, chol as scipy CSR (M*M, X), enuc, nmo, nalpha, nbeta); ipie ``utils/io.py:549-595``."""
    with File(filename) as f:
        enuc = f["Hamiltonian/Energies"][()][0]
        dims = f["Hamiltonian/dims"][()]
        nmo = int(dims[3])
        real_ints = False
        if "Hamiltonian/hcore" in f:
            hcore = np.array(f["Hamiltonian/hcore"][()])
            if hcore.ndim == 3 and hcore.shape[-1] == 2:
                hcore = hcore.view(np.complex128).reshape(nmo, nmo)
            else:
                real_ints = True
        else:
            # old sparse format: lower triangle of H1 with (row, col) pairs
            vals = np.array(f["Hamiltonian/H1"][()]).view(np.complex128).ravel()
            idx = f["Hamiltonian/H1_indx"][()]
            h = scipy.sparse.csr_matrix((vals, (idx[::2], idx[1::2]))).toarray()
            hcore = np.tril(h, -1) + np.tril(h, 0).conj().T
        block_sizes = f["Hamiltonian/Factorized/block_sizes"][()]
        nchol = int(dims[7])
        nval = int(np.sum(block_sizes))
        vals = np.zeros(nval, dtype=np.float64 if real_ints else np.complex128)
        row = np.zeros(nval, dtype=np.int32)
        col = np.zeros(nval, dtype=np.int32)
        s = 0
        for ic, bs in enumerate(block_sizes):
            bs = int(bs)
            ix = f[f"Hamiltonian/Factorized/index_{ic}"][()]
            row[s:s + bs] = ix[::2]
            col[s:s + bs] = ix[1::2]
            v = np.array(f[f"Hamiltonian/Factorized/vals_{ic}"][()])
            vals[s:s + bs] = np.real(v).ravel() if real_ints else v.view(np.complex128).ravel()
            s += bs
        chol = scipy.sparse.csr_matrix((vals, (row, col)), shape=(nmo * nmo, nchol))
        return hcore, chol, enuc, nmo, int(dims[4]), int(dims[5])


def write_qmcpack_dense(hcore, chol, nelec, nmo, enuc=0.0, filename="hamiltonian.h5", real_chol=True, verbose=False,
                        ortho=None):
    """ipie ``utils/io.py:598-621``."""
    if chol.ndim != 2 or chol.shape[0] != nmo * nmo:
        raise AssertionError("chol must be (nmo*nmo, nchol)")
    ham = {"Energies": np.array([enuc, 0.0]),
           "dims": np.array([0, 0, 0, nmo, nelec[0], nelec[1], 0, chol.shape[-1]], dtype=np.int64)}
    if real_chol:
        ham["hcore"] = np.real(hcore)
        ham["DenseFactorized"] = {"L": np.real(chol)}
    else:
        ham["hcore"] = to_qmcpack_complex(hcore)
        ham["DenseFactorized"] = {"L": to_qmcpack_complex(chol)}
    if ortho is not None:
        ham["X"] = np.asarray(ortho)
    write_file(filename, {"Hamiltonian": ham})


def to_sparse(vals, offset=0, cutoff=1e-8):
    """(row, col) pairs and values of the entries above ``cutoff``; ipie ``utils/io.py:717-724``."""
    nz = np.where(np.abs(vals) > cutoff)
    ix = np.empty(nz[0].size + nz[1].size, dtype=np.int32)
    ix[0::2] = nz[0]
    ix[1::2] = nz[1]
    return ix, np.array(vals[nz], dtype=np.complex128)


def write_qmcpack_sparse(hcore, chol, nelec, nmo, enuc=0.0, filename="hamiltonian.h5", real_chol=False,
                         verbose=False, cutoff=1e-16, ortho=None):
    """ipie ``utils/io.py:624-675`` (one integral block)."""
    ham = {"Energies": np.array([enuc, 0.0])}
    ham["hcore"] = np.asarray(hcore) if real_chol else to_qmcpack_complex(hcore)
    if ortho is not None:
        ham["X"] = np.asarray(ortho)
    ix, vals = to_sparse(chol, cutoff=cutoff)
    ham["Factorized"] = {"block_sizes": np.array([len(vals)]), "index_0": np.array(ix),
                         "vals_0": np.real(vals) if real_chol else to_qmcpack_complex(vals)}
    na, nb = nelec
    ham["dims"] = np.array([0, len(vals), 1, nmo, na, nb, 0, chol.shape[-1]], dtype=np.int64)
    ham["occups"] = np.array(list(range(na)) + [i + nmo for i in range(nb)])
    write_file(filename, {"Hamiltonian": ham})


def _nomsd_single(psi_h: scipy.sparse.csr_matrix) -> dict:
    """One NOMSD component, stored as the CSR matrix of A^H (ipie ``utils/io.py:458-476``)."""
    return {"dims": np.array([psi_h.shape[0], psi_h.shape[1], psi_h.nnz], dtype=np.int32),
            "data_": to_qmcpack_complex(psi_h.data), "jdata_": psi_h.indices.astype(np.int32),
            "pointers_begin_": psi_h.indptr[:-1].astype(np.int32),
            "pointers_end_": psi_h.indptr[1:].astype(np.int32)}


def write_qmcpack_wfn(filename, wfn, walker_type, nelec, norb, init=None, mode="w"):
    """NOMSD ``(coeffs, psi)`` or PHMSD ``(coeffs, occa, occb)`` under ``Wavefunction/``;
    ipie ``utils/io.py:367-411`` (``mode="w"``: a new file)."""
    na, nb = nelec
    if len(wfn) == 3:
        coeffs, occa, occb = wfn
        grp = {"occs": np.hstack([np.asarray(occa), np.asarray(occb) + norb]).ravel()}
        wt = 2
        if init is not None:
            grp["Psi0_alpha"] = to_qmcpack_complex(init[0])
            grp["Psi0_beta"] = to_qmcpack_complex(init[1])
        name = "PHMSD"
    elif len(wfn) == 2:
        coeffs, psi = wfn
        wt = {"ghf": 3, "uhf": 2}.get(walker_type, 1)
        uhf = walker_type == "uhf"
        psi = np.array(psi, dtype=np.complex128)
        psi[np.abs(psi) < 1e-8] = 0.0
        if psi.ndim == 2:
            psi = psi[None]
        grp = {}
        if init is not None:
            grp["Psi0_alpha"] = to_qmcpack_complex(init[0])
            grp["Psi0_beta"] = to_qmcpack_complex(init[1])
        else:
            grp["Psi0_alpha"] = to_qmcpack_complex(psi[0, :, :na])
            if uhf:
                grp["Psi0_beta"] = to_qmcpack_complex(psi[0, :, na:])
        for idet, w in enumerate(psi):
            ix = 2 * idet if uhf else idet
            grp[f"PsiT_{ix:d}"] = _nomsd_single(scipy.sparse.csr_matrix(w[:, :na].conj().T))
            if uhf:
                grp[f"PsiT_{2 * idet + 1:d}"] = _nomsd_single(scipy.sparse.csr_matrix(w[:, na:].conj().T))
        name = "NOMSD"
    else:
        raise RuntimeError("wavefunction to write is neither particle-hole (ci, occa, occb) nor NOCI (ci, determinants)")
    coeffs = np.asarray(coeffs)
    grp["ci_coeffs"] = to_qmcpack_complex(coeffs)
    grp["dims"] = np.array([norb, na, nb, wt, len(coeffs)], dtype=np.int32)
    if mode != "w":
        raise NotImplementedError("h5lite writes whole files: mode='w' only")
    write_file(filename, {"Wavefunction": {name: grp}})


def orbs_from_dset(dset) -> np.ndarray:
    """The CSR matrix of A^H in a NOMSD component, returned as A; ipie ``utils/io.py:509-522``."""
    dims = dset["dims"][()]
    nnz = int(dims[2])
    data = from_qmcpack_complex(dset["data_"][()], (nnz,))
    indptr = np.zeros(int(dims[0]) + 1)
    indptr[:-1] = dset["pointers_begin_"][()]
    indptr[-1] = dset["pointers_end_"][()][-1]
    m = scipy.sparse.csr_matrix((data, dset["jdata_"][()], indptr), shape=(int(dims[0]), int(dims[1])))
    return m.toarray().conj().T.copy()


def read_qmcpack_nomsd_hdf5(wgroup, nelec=None):
    """((coeffs, wfn (ndet, M, na+nb)), psi0); ipie ``utils/io.py:297-332``."""
    dims = wgroup["dims"][()]
    nmo, na, nb = int(dims[0]), int(dims[1]), int(dims[2])
    if nelec is not None:
        assert na == nelec[0] and nb == nelec[1], f"file holds {na}+{nb} electrons, the caller asked for {nelec[0]}+{nelec[1]}"
    uhf = int(dims[3]) == 2
    nci = int(dims[4])
    coeffs = from_qmcpack_complex(wgroup["ci_coeffs"][()], (nci,))
    psi0 = np.zeros((nmo, na + nb), dtype=np.complex128)
    psi0a = from_qmcpack_complex(wgroup["Psi0_alpha"][()], (nmo, na))
    psi0[:, :na] = psi0a
    psi0[:, na:] = from_qmcpack_complex(wgroup["Psi0_beta"][()], (nmo, nb)) if uhf else psi0a[:, :nb]
    wfn = np.zeros((nci, nmo, na + nb), dtype=np.complex128)
    for idet in range(nci):
        pa = orbs_from_dset(wgroup[f"PsiT_{2 * idet if uhf else idet:d}"])
        wfn[idet, :, :na] = pa
        wfn[idet, :, na:] = orbs_from_dset(wgroup[f"PsiT_{2 * idet + 1:d}"]) if uhf else pa[:, :nb]
    return (coeffs, wfn), psi0


def read_qmcpack_phmsd_hdf5(wgroup, nelec=None):
    """((coeffs, occa, occb), psi0); ipie ``utils/io.py:335-364``."""
    dims = wgroup["dims"][()]
    nmo, na, nb = int(dims[0]), int(dims[1]), int(dims[2])
    uhf = int(dims[3]) == 2
    nci = int(dims[4])
    coeffs = from_qmcpack_complex(wgroup["ci_coeffs"][()], (nci,))
    occs = wgroup["occs"][()].reshape((nci, na + nb))
    psi0 = np.zeros((nmo, na + nb), dtype=np.complex128)
    psi0a = from_qmcpack_complex(wgroup["Psi0_alpha"][()], (nmo, na))
    psi0[:, :na] = psi0a
    psi0[:, na:] = from_qmcpack_complex(wgroup["Psi0_beta"][()], (nmo, nb)) if uhf else psi0a
    return (coeffs, occs[:, :na], occs[:, na:] - nmo), psi0


def read_qmcpack_wfn_hdf(filename, nelec=None, get_nelec=False):
    """ipie ``utils/io.py:273-294``."""
    with File(filename) as f:
        if "Wavefunction/NOMSD" in f:
            g = f["Wavefunction/NOMSD"]
            wfn, psi0 = read_qmcpack_nomsd_hdf5(g, nelec=nelec)
        elif "Wavefunction/PHMSD" in f:
            g = f["Wavefunction/PHMSD"]
            wfn, psi0 = read_qmcpack_phmsd_hdf5(g, nelec=nelec)
        else:
            raise KeyError("no Wavefunction/NOMSD or Wavefunction/PHMSD group in the file")
        dims = g["dims"][()]
    if get_nelec:
        return wfn, psi0, (int(dims[1]), int(dims[2]))
    return wfn, psi0


# ---------------------------------------------------------------- set-up from files
def read_integrals(integral_file):
    """(h1e (M, M), chol (M, M, X) or (M*M, X), ecore): QMCPACK sparse, QMCPACK dense, then the
    native layout, as ipie ``hamiltonians/generic.py:160-178``."""
    try:
        h1e, schol, ecore, *_ = from_qmcpack_sparse(integral_file)
        return h1e, schol.toarray(), ecore
    except KeyError:
        pass
    try:
        h1e, chol, ecore, *_ = from_qmcpack_dense(integral_file)
        return h1e, chol, ecore
    except KeyError:
        pass
    h1e, chol, ecore = read_hamiltonian(integral_file)
    naux, nbsf = chol.shape[0], chol.shape[-1]
    return h1e, chol.T.reshape((nbsf, nbsf, naux)), ecore


def get_hamiltonian(filename, scomm=None, verbose=False, pack_chol=True, device="cuda"):
    """:class:`ipie_b200.Generic` from an integral file (ipie ``hamiltonians/utils.py:28-97``, one process)."""
    from .hamiltonian import GenericComplexChol, GenericRealChol

    hcore, chol, ecore = read_integrals(filename)
    M = hcore.shape[-1]
    chol = np.asarray(chol).reshape(M * M, -1)
    h1e = np.array([hcore, hcore])
    if chol.dtype == np.complex128:
        return GenericComplexChol(h1e, chol, ecore, device=device, verbose=verbose)
    return GenericRealChol(h1e, chol, ecore, device=device, verbose=verbose)


def get_trial_wavefunction(num_elec, nbasis, wfn_file, ndets=-1, ndets_props=100, ndet_chunks=1, verbose=False,
                           device="cuda"):
    """:class:`ipie_b200.SingleDet` from a wavefunction file (ipie ``trial_wavefunction/utils.py:17-93``;
    ``trial.nelec`` holds the electron counts read).  Multi-determinant files raise ``NotImplementedError``."""
    from .trial import SingleDet

    kind = determine_wavefunction_type(wfn_file)
    trial = None
    if kind == "single_determinant":
        wfn, _ = read_single_det_wavefunction(wfn_file)
        nelec = (wfn[0].shape[-1], wfn[1].shape[-1])
        if wfn[0].shape[0] != nbasis:
            raise AssertionError("wavefunction basis size differs from the Hamiltonian's")
        trial = SingleDet(np.hstack(wfn), nelec, nbasis, device=device)
    elif kind == "qmcpack":
        wfn, _, nelec = read_qmcpack_wfn_hdf(wfn_file, get_nelec=True)
        if len(wfn) == 2 and len(wfn[0]) == 1:
            psi = wfn[1][0]
            trial = SingleDet(psi, nelec, psi.shape[0], device=device)
    if trial is None:
        raise NotImplementedError(f"{kind} trial wavefunctions with several determinants")
    trial.nelec = tuple(int(n) for n in nelec)
    return trial


# ---------------------------------------------------------------- estimator output (estimators/handler.py:149-242)
ESTIMATOR_BUFFER_SIZE = 1000  # rows per data chunk, ipie config.py:87
WALKER_HEADER = ("Weight", "WeightFactor", "HybridEnergy")
ENERGY_NAMES = ("ENumer", "EDenom", "ETotal", "E1Body", "E2Body")


def write_estimates(filename, rows, metadata="{}", buffer_size=ESTIMATOR_BUFFER_SIZE):
    """Block estimates in the layout of ipie's ``EstimatorHandler`` / ``H5EstimatorHelper``
    (``estimators/handler.py:149-242``, ``estimators/utils.py:46-96``): ``metadata`` (the run's
    JSON), and under ``block_size_1/`` the walker-property header, the energy estimator's shape,
    size, scalar flag, names and offset, and the rows ``[Weight, WeightFactor, HybridEnergy,
    ENumer, EDenom, ETotal, E1Body, E2Body]`` (complex) in chunks of ``buffer_size`` rows
    (``data/000000000`` ...) with ``max_block/<chunk>`` = the last row written in that chunk."""
    rows = np.asarray(rows, dtype=np.complex128).reshape(-1, len(WALKER_HEADER) + len(ENERGY_NAMES))
    data, max_block = {}, {}
    for c in range(max(1, -(-len(rows) // buffer_size))):
        part = rows[c * buffer_size:(c + 1) * buffer_size]
        chunk = np.zeros((buffer_size, rows.shape[1]), dtype=np.complex128)
        chunk[:len(part)] = part
        data[f"{c:09d}"] = chunk
        max_block[f"{c:09d}"] = np.int64(max(len(part) - 1, 0))
    nw = len(WALKER_HEADER)
    block = {
        "num_walker_props": np.int64(nw),
        "walker_prop_header": np.array([h.encode() for h in WALKER_HEADER]),
        "shape": {"energy": np.array([len(ENERGY_NAMES)], dtype=np.int64)},
        "size": {"energy": np.int64(len(ENERGY_NAMES))},
        "scalar": {"energy": np.int64(1)},
        "names": {"energy": np.bytes_(" ".join(ENERGY_NAMES).encode())},
        "offset": {"energy": np.int64(nw)},
        "data": data,
        "max_block": max_block,
    }
    write_file(filename, {"metadata": np.bytes_(metadata.encode()), "block_size_1": block})


def extract_observable(filename, name="energy", block_idx=1):
    """Block rows of one observable as a DataFrame (walker header + the observable's names);
    ipie ``analysis/extraction.py:10-68`` (scalar observables)."""
    import pandas as pd

    grp = f"block_size_{block_idx}"
    with File(filename) as f:
        data = np.concatenate([f[f"{grp}/data/{d}"][()].real for d in f[f"{grp}/data"].keys()])
        if name not in f[f"{grp}/shape"].keys():
            raise RuntimeError(f"estimator file has no quantity {name!r}")
        shape = f[f"{grp}/shape/{name}"][()]
        offset = int(f[f"{grp}/offset/{name}"][()])
        size = int(f[f"{grp}/size/{name}"][()])
        names = f[f"{grp}/names/{name}"][()]
        nw = int(f[f"{grp}/num_walker_props"][()])
        header = list(f[f"{grp}/walker_prop_header"][()])
        max_block = sum(int(f[f"{grp}/max_block/{d}"][()]) for d in f[f"{grp}/max_block"].keys())
    data = data[: max_block + 1]
    obs = data[:, offset:offset + size].reshape((-1,) + tuple(int(x) for x in shape))
    out = pd.DataFrame(np.hstack([data[:, :nw], obs]))
    out.columns = [bytes(n).decode("utf-8") for n in header + bytes(names).split()]
    return out
