"""Population control (pair branch) for a device-resident walker batch.

Mirror of ipie's ``PopController`` (``walkers/pop_controller.py:33-125``) and
``pair_branch`` (``:304-429``) on one process.  ipie runs the pairing on the
host with one ``numpy.random.rand()`` per pair; that is kept so a run fed the
same seed makes the same decisions.  The walker copies run on the device.

Single-process message semantics (``qmc/comm.py:61-71``): every send in
ipie's pair branch carries the same tag (it is built from a rank index), and
the single-process communicator keeps the last send per tag, so every killed
walker receives the buffer of the highest-index cloned walker -- orbitals,
overlap, hybrid energy and weight included.  That is reproduced here.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, ptr, stream


def pair_branch_table(absw, max_weight, min_weight, rand=np.random.rand):
    """ipie's pairing walk (``pop_controller.py:338-391``): returns (new |w|, status 0/1/2) in walker order."""
    n = absw.size
    w = absw.astype(np.float64).copy()
    st = np.ones(n, dtype=np.int64)
    order = np.argsort(w, kind="mergesort")
    ws = w[order]
    ss = st[order]
    s, e = 0, n - 1
    while s < e:
        if ws[s] < min_weight or ws[e] > max_weight:
            wab = ws[s] + ws[e]
            r = rand()
            if r < ws[e] / wab:
                ws[e] = 0.5 * wab
                ss[e] = 2
                ws[s] = 0.0
                ss[s] = 0
            else:
                ws[s] = 0.5 * wab
                ss[s] = 2
                ws[e] = 0.0
                ss[e] = 0
            s += 1
            e -= 1
        else:
            break
    out_w = np.empty(n)
    out_s = np.empty(n, dtype=np.int64)
    out_w[order] = ws
    out_s[order] = ss
    return out_w, out_s


class PopController:
    def __init__(self, num_walkers_local, num_steps, mpi_handler=None, pop_control_method="pair_branch",
                 min_weight=0.1, max_weight=4, reconfiguration_freq=50, verbose=False):
        if pop_control_method != "pair_branch":
            raise NotImplementedError(f"population control {pop_control_method!r}: only pair_branch is provided")
        self.method = pop_control_method
        self.num_walkers_local = num_walkers_local
        self.num_steps = num_steps
        self.min_weight = min_weight
        self.max_weight = max_weight
        self.size = 1
        self.ntot_walkers = num_walkers_local
        self.target_weight = self.ntot_walkers
        self.total_weight = self.ntot_walkers
        self._src = None

    def pop_control(self, walkers, comm=None, rand=np.random.rand):
        """Rescale by total |w| / target, then pair branch (``pop_controller.py:78-125``)."""
        if self.ntot_walkers == 1:
            return
        w = walkers.weight.cpu().numpy()
        total_weight = float(np.sum(np.abs(w)))
        scale = total_weight / self.target_weight
        if total_weight < 1e-8:
            raise ValueError(f"Total weight is {total_weight:13.8e}: something is seriously wrong")
        self.total_weight = total_weight
        unscaled = w.copy()
        w = w / scale
        neww, status = pair_branch_table(np.abs(w), self.max_weight, self.min_weight, rand)
        cloned = np.nonzero(status == 2)[0]
        killed = np.nonzero(status == 0)[0]
        w[cloned] = neww[cloned]
        src = np.full(walkers.nwalkers, -1, dtype=np.int32)
        if cloned.size:
            src[killed] = cloned.max()
        walkers.unscaled_weight.copy_(torch.from_numpy(unscaled))
        walkers.weight.copy_(torch.from_numpy(w))
        if killed.size:
            if self._src is None or self._src.numel() != walkers.nwalkers:
                self._src = torch.empty(walkers.nwalkers, dtype=torch.int32, device=walkers.device)
            self._src.copy_(torch.from_numpy(src))
            call("ipie_b200_walker_copy", ptr(self._src), walkers.nwalkers, walkers.nbasis, walkers.nup, walkers.ndown,
                 ptr(walkers.phia), ptr(walkers.phib), ptr(walkers.weight), ptr(walkers.unscaled_weight),
                 ptr(walkers.hybrid_energy), ptr(walkers.ovlp), ptr(walkers.phase), stream())
        return neww, status
