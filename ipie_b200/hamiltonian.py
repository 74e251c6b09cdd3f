"""Generic real-Cholesky Hamiltonian, device resident.

Mirror of ipie's ``Generic`` factory / ``GenericRealChol``
(``hamiltonians/generic.py:31-102,153-157``): same constructor arguments
(``h1e`` (2, M, M), ``chol`` (M*M, X), ``ecore``), same attribute names.
Set-up arithmetic (``h1e_mod``, packing) runs once on the host in numpy; the
arrays the walker step reads are uploaded once and stay in HBM.
"""
from __future__ import annotations

import numpy as np
import torch


def tiled_triu_indices(M, rows=32, cols=4):
    """Upper-triangle (i <= j) pairs ordered by tiles of ``rows`` x ``cols``: consecutive packed
    entries then cover a small block of the matrix, so the symmetric scatter of VHS writes runs
    of contiguous elements instead of single ones.  The full tiles strictly above the diagonal
    come first (``rows * cols`` = 128 pairs each, so every warp's 32 consecutive pairs form an
    8 x 4 block that the VHS epilogue writes as 8-byte runs in both orientations); the tiles
    that touch the diagonal or the matrix edge follow.  32 x 4 measured fastest of the tile
    shapes (VHS 2.03 ms with 8 x 16, 1.64 ms with 16 x 8, 1.60 ms with 32 x 4 at 2048 walkers,
    c2 shapes, before the full tiles were moved first)."""
    full, rest = ([], []), ([], [])
    for I in range(0, M, rows):
        for J in range((I // cols) * cols, M, cols):
            i = np.arange(I, min(I + rows, M))[:, None]
            j = np.arange(J, min(J + cols, M))[None, :]
            keep = j >= i
            dst = full if (I + rows <= M and J + cols <= M and J >= I + rows) else rest
            dst[0].append(np.broadcast_to(i, keep.shape)[keep])
            dst[1].append(np.broadcast_to(j, keep.shape)[keep])
    ii, jj = full[0] + rest[0], full[1] + rest[1]
    return np.concatenate(ii), np.concatenate(jj)


class GenericRealChol:
    complex_chol = False

    def __init__(self, h1e, chol, ecore=0.0, device="cuda", verbose=False):
        h1e = np.asarray(h1e)
        chol = np.asarray(chol)
        assert h1e.shape[0] == 2, "h1e must carry both spin components"
        assert chol.dtype == np.float64, "GenericRealChol needs a float64 Cholesky tensor"
        self.H1 = h1e
        self.ecore = float(ecore)
        self.nbasis = h1e.shape[-1]
        self.nchol = chol.shape[-1]
        self.nfields = self.nchol
        assert self.nbasis ** 2 == chol.shape[0]
        self.chunked = False
        M, X = self.nbasis, self.nchol
        self.chol = np.ascontiguousarray(chol)  # host copy (set-up only)
        iu, ju = np.triu_indices(M)
        self.sym_idx = (iu, ju)  # ipie's packing order (host attribute)
        # the device copy is packed in tiled order (same entries, see tiled_triu_indices)
        ti, tj = tiled_triu_indices(M)
        packed = np.ascontiguousarray(self.chol.reshape(M, M, X)[ti, tj, :])
        # h1e_mod = h1e - 1/2 sum_kn L_ik,n L_jk,n  (hamiltonians/generic.py:31-43)
        view = self.chol.reshape(M, M * X)
        v0 = 0.5 * view @ view.T
        self.h1e_mod = np.array([h1e[0] - v0, h1e[1] - v0])
        self.device = torch.device(device)
        self.chol_packed = torch.from_numpy(packed).to(self.device)
        self.sym_idx_i = torch.from_numpy(ti.astype(np.int32)).to(self.device)
        self.sym_idx_j = torch.from_numpy(tj.astype(np.int32)).to(self.device)
        if verbose:
            print(f"# nbasis {M}  nchol {X}  packed Cholesky {packed.nbytes / 1e9:.3f} GB on {self.device}")

    @property
    def npacked(self):
        return self.nbasis * (self.nbasis + 1) // 2


class GenericComplexChol:
    """ipie's ``GenericComplexChol`` (``hamiltonians/generic.py:100-150``): complex Cholesky
    vectors L (M*M, X) and their Hermitian parts ``A_x = (L_x + L_x^H)/2``,
    ``B_x = i (L_x - L_x^H)/2``; 2X auxiliary fields (A first, then B).  The device keeps
    ``C = [A | B]`` (M*M, 2X) as real and imaginary parts, the left operand of the VHS."""

    complex_chol = True

    def __init__(self, h1e, chol, ecore=0.0, device="cuda", verbose=False):
        h1e = np.asarray(h1e)
        chol = np.asarray(chol, dtype=np.complex128)
        assert h1e.shape[0] == 2, "h1e must carry both spin components"
        self.H1 = h1e
        self.ecore = float(ecore)
        self.nbasis = h1e.shape[-1]
        self.nchol = chol.shape[-1]
        self.nfields = 2 * self.nchol
        assert self.nbasis ** 2 == chol.shape[0]
        self.chunked = False
        M, X = self.nbasis, self.nchol
        self.chol = np.ascontiguousarray(chol)  # host copy (set-up only)
        # h1e_mod = h1e - 1/2 L L^H, allocated with H1's dtype as ipie does (generic.py:116-118):
        # for a real H1 the (antisymmetric) imaginary part is dropped
        view = self.chol.reshape(M, M * X)
        v0 = 0.5 * view @ view.T.conj()
        h1e_mod = np.array([h1e[0] - v0, h1e[1] - v0])
        self.h1e_mod = h1e_mod if np.iscomplexobj(h1e) else h1e_mod.real.copy()
        L = self.chol.reshape(M, M, X)
        LH = L.transpose(1, 0, 2).conj()
        self.A = np.ascontiguousarray((0.5 * (L + LH)).reshape(M * M, X))
        self.B = np.ascontiguousarray((0.5j * (L - LH)).reshape(M * M, X))
        self.device = torch.device(device)
        C = np.concatenate([self.A, self.B], axis=1)
        self.c_re = torch.from_numpy(np.ascontiguousarray(C.real)).to(self.device)
        self.c_im = torch.from_numpy(np.ascontiguousarray(C.imag)).to(self.device)
        if verbose:
            print(f"# nbasis {M}  nchol {X}  complex Cholesky, {2 * C.real.nbytes / 1e9:.3f} GB of [A | B] on {self.device}")


def Generic(h1e, chol, ecore=0.0, shmem=False, chol_packed=None, verbose=False):
    """Factory with ipie's signature (``hamiltonians/generic.py:153-157``): complex Cholesky
    vectors give :class:`GenericComplexChol`, real ones :class:`GenericRealChol`."""
    chol = np.asarray(chol)
    if chol.dtype == np.complex128:
        return GenericComplexChol(h1e, chol, ecore, verbose=verbose)
    return GenericRealChol(h1e, chol, ecore, verbose=verbose)
