"""UHF walker batch, device resident.

Mirror of ipie's ``UHFWalkers`` (``walkers/uhf_walkers.py:27-161``) and the
parts of ``BaseWalkers`` (``walkers/base_walkers.py:86-179``) the walker step
uses.  Every per-walker array is a torch CUDA tensor with ipie's name, shape
and dtype; ``reortho`` runs the modified Gram-Schmidt kernel.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, ptr, stream

C128 = torch.complex128
F64 = torch.float64


class UHFWalkers:
    # phia/phib are properties: replacing either drops the cached Green's function
    @property
    def phia(self):
        return self._phia

    @phia.setter
    def phia(self, value):
        self._phia = value
        self._gf_key = None

    @property
    def phib(self):
        return self._phib

    @phib.setter
    def phib(self, value):
        self._phib = value
        self._gf_key = None

    def __init__(self, initial_walker, nup, ndown, nbasis, nwalkers, mpi_handler=None, verbose=False, device="cuda"):
        init = np.asarray(initial_walker)
        assert init.ndim == 2
        self.nup, self.ndown, self.nbasis, self.nwalkers = nup, ndown, nbasis, nwalkers
        self.mpi_handler = mpi_handler
        self.device = dev = torch.device(device)
        W, M = nwalkers, nbasis
        # orbitals Ghalfa/b and ovlp were last computed from (see gf_current)
        self._gf_key = None
        ia = torch.from_numpy(np.ascontiguousarray(init[:, :nup].astype(np.complex128)))
        ib = torch.from_numpy(np.ascontiguousarray(init[:, nup:].astype(np.complex128)))
        self.phia = ia.to(dev).unsqueeze(0).repeat(W, 1, 1).contiguous()
        self.phib = ib.to(dev).unsqueeze(0).repeat(W, 1, 1).contiguous()
        self.weight = torch.ones(W, dtype=F64, device=dev)
        self.unscaled_weight = torch.ones(W, dtype=F64, device=dev)
        self.phase = torch.ones(W, dtype=C128, device=dev)
        self.ovlp = torch.ones(W, dtype=C128, device=dev)
        self.sgn_ovlp = torch.ones(W, dtype=F64, device=dev)
        self.log_ovlp = torch.zeros(W, dtype=F64, device=dev)
        self.hybrid_energy = torch.zeros(W, dtype=C128, device=dev)
        self.detR = torch.ones(W, dtype=F64, device=dev)
        self.detR_shift = torch.zeros(W, dtype=F64, device=dev)
        self.log_detR = torch.zeros(W, dtype=F64, device=dev)
        self.log_shift = torch.zeros(W, dtype=F64, device=dev)
        self.Ghalfa = torch.zeros(W, nup, M, dtype=C128, device=dev)
        self.Ghalfb = torch.zeros(W, ndown, M, dtype=C128, device=dev)
        # device status word: numerical trouble bits written by the kernels
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.rhf = False  # ipie propagates both spin blocks in production (uhf_walkers.py:99)
        # spin_alias: phib is phia (same tensor) -- both blocks identical, computed once
        self.spin_alias = False
        self.buff_names = ["weight", "unscaled_weight", "phase", "hybrid_energy", "ovlp", "sgn_ovlp", "log_ovlp",
                           "phia", "phib"]

    def enable_spin_alias(self):
        """Share one tensor for identical alpha and beta blocks (RHF trial, walkers started from it).

        Every kernel then computes the block once and counts it twice; results equal
        propagating both blocks (ipie's production mode), which stay identical because
        they see the same operators and fields.
        """
        if self.nup != self.ndown or not torch.equal(self.phia, self.phib):
            raise ValueError("spin aliasing needs identical alpha and beta blocks")
        self.phib = self.phia
        self.Ghalfb = self.Ghalfa
        self.spin_alias = True

    def sync_alias(self):
        """Re-point the beta views after the alpha tensors were replaced."""
        if self.spin_alias:
            self.phib = self.phia
            self.Ghalfb = self.Ghalfa

    def _orbital_key(self, trial):
        return (self._phia._version, self._phib._version, id(trial))

    def mark_gf_current(self, trial):
        """Ghalfa/b and ovlp now belong to the current orbitals."""
        self._gf_key = self._orbital_key(trial)

    def gf_current(self, trial):
        """True while Ghalfa/b and ovlp are those of the current orbitals.

        Kept valid by the library's own updates (a propagation step ends with the
        Green's function of its new orbitals; reorthogonalisation leaves Ghalf
        unchanged and rescales ovlp; population control copies Ghalf with the
        orbitals).  Assigning ``phia``/``phib`` or changing them with in-place torch
        operations invalidates it; after writing them through raw device pointers
        call :meth:`invalidate_gf`.
        """
        return self._gf_key is not None and self._gf_key == self._orbital_key(trial)

    def invalidate_gf(self):
        self._gf_key = None

    def resample(self, src):
        """Walker d becomes walker ``src[d]`` (int32 device tensor; sources may repeat).

        Orbitals, Green's functions, overlaps, hybrid energies, phases and unscaled
        weights move together (out of place); the Green's-function cache stays valid.
        """
        was_current = self._gf_key is not None and self._gf_key[:2] == (self._phia._version, self._phib._version)
        key_trial = self._gf_key[2] if was_current else None
        alias = self.spin_alias
        new = {n: torch.empty_like(getattr(self, n)) for n in ("phia", "Ghalfa", "hybrid_energy", "ovlp", "phase",
                                                                 "unscaled_weight")}
        if not alias:
            new["phib"] = torch.empty_like(self.phib)
            new["Ghalfb"] = torch.empty_like(self.Ghalfb)
        call("ipie_b200_walker_gather", ptr(src), self.nwalkers, self.nbasis, self.nup, self.ndown,
             ptr(self.phia), ptr(self.phib), ptr(self.Ghalfa), ptr(self.Ghalfb), ptr(self.hybrid_energy),
             ptr(self.ovlp), ptr(self.phase), ptr(self.unscaled_weight), ptr(new["phia"]),
             ptr(new.get("phib", new["phia"])), ptr(new["Ghalfa"]), ptr(new.get("Ghalfb", new["Ghalfa"])),
             ptr(new["hybrid_energy"]), ptr(new["ovlp"]), ptr(new["phase"]), ptr(new["unscaled_weight"]), stream())
        for n, t in new.items():
            setattr(self, n, t)
        if alias:
            self.phib = self.phia
            self.Ghalfb = self.Ghalfa
        if was_current:
            self._gf_key = (self._phia._version, self._phib._version, key_trial)

    def build(self, trial):
        """``walkers.build``: initial overlaps and Green's functions (``uhf_walkers.py:101-102``)."""
        self.ovlp = trial.calc_greens_function(self)
        self.mark_gf_current(trial)

    def reortho(self):
        """Thin QR per spin block with positive diag(R); returns detR (``uhf_walkers.py:108-161``)."""
        call(
            "ipie_b200_reortho",
            ptr(self.phia), ptr(self.phib), self.nwalkers, self.nbasis, self.nup, self.ndown,
            ptr(self.detR_shift), ptr(self.detR), ptr(self.log_detR), ptr(self.ovlp), ptr(self.status), stream(),
        )
        return self.detR

    def orthogonalise(self, free_projection=False):
        """``BaseWalkers.orthogonalise`` (``base_walkers.py:166-179``), phaseless branch."""
        if free_projection:
            raise NotImplementedError("free projection is not part of the B200 walker step")
        return self.reortho()

    def check_status(self):
        """Raise if a kernel flagged non-finite values or a singular overlap since the last check."""
        s = int(self.status.item())
        if s:
            self.status.zero_()
            if s & 16:
                # device population control met a vanishing total weight (ipie pop_controller.py:103-107)
                raise ValueError("total walker weight fell below 1e-8 in population control")
            names = []
            for bit, name in ((1, "non-finite weight/overlap/energy"), (2, "singular overlap matrix"),
                              (4, "unsupported shape"), (8, "zero column in Gram-Schmidt")):
                if s & bit:
                    names.append(name)
            raise FloatingPointError("walker step reported: " + ", ".join(names))
