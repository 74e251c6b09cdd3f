"""Population control for a device-resident walker batch.

Mirror of ipie's ``PopController`` (``walkers/pop_controller.py:33-125``) with
its three methods on one process: ``pair_branch`` (``:304-429``), ``comb``
(``:199-301``) and ``stochastic_reconfiguration`` (``:432-475``).  ipie
decides on the host from the |w| vector with numpy's global generator (one
``rand()`` per pair, one ``random()`` per comb, one ``rand()`` per
reconfiguration); that is kept so a run fed the same seed makes the same
decisions.  The walker copies run on the device.

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


def pair_branch_table(absw, max_weight, min_weight, rand=np.random.rand, pairs=None):
    """ipie's pairing walk (``pop_controller.py:338-391``): returns (new |w|, status 0/1/2) in walker order.

    ``pairs`` (a list), when given, receives each pair's decision as (low walker, high walker,
    high walker kept) in walker indices, so that another walker set can be branched the same way
    (:meth:`PopController.follow`)."""
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
            if pairs is not None:
                pairs.append((int(order[s]), int(order[e]), bool(r < ws[e] / wab)))
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


def apply_pairs(absw, pairs):
    """(new |w|, status) of a pair branch whose pairs and survivors are given (the ``pairs`` list of
    :func:`pair_branch_table`), applied to the weights ``absw``: each pair's survivor carries half
    the pair's summed weight."""
    neww = absw.astype(np.float64).copy()
    status = np.ones(neww.size, dtype=np.int64)
    for i, j, keep_j in pairs:
        half = 0.5 * (neww[i] + neww[j])
        keep, drop = (j, i) if keep_j else (i, j)
        neww[keep], status[keep] = half, 2
        neww[drop], status[drop] = 0.0, 0
    return neww, status


def comb_parent_counts(weights, target_weight, r):
    """Copies of each walker under the comb (``pop_controller.py:215-229``).

    Teeth ``(i + r) * total / target`` for i < target; walker iw takes every tooth
    in [cprobs[iw-1], cprobs[iw]), i.e. a right-sided search in the cumulative weights.
    """
    cprobs = np.cumsum(weights)
    total = cprobs[-1]  # ipie's builtin sum: the same sequential sum
    teeth = (np.arange(target_weight) + r) * (total / target_weight)
    iw = np.minimum(np.searchsorted(cprobs, teeth, side="right"), len(weights) - 1)
    return np.bincount(iw, minlength=len(weights)).astype(np.int64)


def reconfiguration_sources(absw, zeta):
    """Source walker of every slot under stochastic reconfiguration (``pop_controller.py:455-465``)."""
    n = absw.size
    cumulative = np.cumsum(absw)
    total = cumulative[-1]
    z = (np.arange(n) + zeta) / n / 1
    return np.searchsorted(cumulative, z * total), total / n / 1


METHODS = ("pair_branch", "comb", "stochastic_reconfiguration")


class PopController:
    """``device=True`` (pair branch only) decides on the GPU (``ipie_b200_pair_branch``) with device
    uniforms (Philox keyed by ``seed``): no host round trip, so a step with population control can be
    replayed from a CUDA graph; the total weight and the clip bound then stay on the device
    (``total_weight_dev``, and ``wbound``, the weight-clip bound tensor the caller hands in).

    ``paired`` selects what a killed walker of the pair branch receives: False (default) the buffer
    of the highest-index survivor, as ipie does in one process (every send carries the same tag and
    its single-process communicator keeps the last); True its own pair's survivor, as ipie does
    when the pairs span ranks.  The first reproduces ipie's single-process runs; it also copies
    one walker into every killed slot, which thins the population's diversity over long runs."""

    def __init__(self, num_walkers_local, num_steps, mpi_handler=None, pop_control_method="pair_branch",
                 min_weight=0.1, max_weight=4, reconfiguration_freq=50, verbose=False, device=False, seed=7,
                 paired=False, wbound=None):
        if pop_control_method not in METHODS:
            raise NotImplementedError(f"population control {pop_control_method!r}: one of {METHODS}")
        if device and pop_control_method != "pair_branch":
            raise NotImplementedError("population control on the device is pair branch only")
        self.device = bool(device)
        self.seed = int(seed)
        self.paired = bool(paired)
        self.wbound = wbound
        self._dev = None
        self.method = pop_control_method
        self.reconfiguration_counter = 0
        self.reconfiguration_freq = reconfiguration_freq
        self.num_walkers_local = num_walkers_local
        self.num_steps = num_steps
        self.min_weight = min_weight
        self.max_weight = max_weight
        self.size = 1
        self.ntot_walkers = num_walkers_local
        self.target_weight = self.ntot_walkers
        self.total_weight = self.ntot_walkers
        self._src = None
        self.leader = None  # see follow()
        self.last_pairs = []

    def follow(self, leader):
        """Branch with ``leader``'s pairs instead of drawing: each pair (i, j) the leader formed at
        its last pair branch is formed here too, from this walker set's own weights, and the same
        walker of the pair survives.  Two runs of one system that differ only in arithmetic
        (precision forms) then keep the same population and stay comparable step by step; the
        leader must branch first at every step.  Pair branch only."""
        if self.method != "pair_branch":
            raise NotImplementedError("follow() couples pair-branch population control")
        self.leader = leader

    def pop_control(self, walkers, comm=None, rand=None):
        """Rescale by total |w| / target, then the configured method (``pop_controller.py:78-125``).

        ``rand`` replaces numpy's global ``rand``/``random`` (tests replay draws with it).
        """
        if self.ntot_walkers == 1:
            return
        if self.device:
            return self._pair_branch_device(walkers)
        w = walkers.weight.cpu().numpy()
        absw = np.abs(w)
        if self.method == "comb":
            total_weight = float(np.cumsum(absw)[-1])  # ipie: builtin sum of the gathered |w|
        else:
            total_weight = float(np.sum(absw))
        scale = total_weight / self.target_weight
        if total_weight < 1e-8:
            raise ValueError(f"Total weight is {total_weight:13.8e}: something is seriously wrong")
        self.total_weight = total_weight
        unscaled = w.copy()
        w = w / scale
        walkers.unscaled_weight.copy_(torch.from_numpy(unscaled))
        if self.method == "pair_branch":
            return self._pair_branch(walkers, w, rand or np.random.rand)
        if self.method == "comb":
            return self._comb(walkers, w, absw / scale, rand or np.random.random)
        walkers.weight.copy_(torch.from_numpy(w))
        self.reconfiguration_counter += 1
        if self.reconfiguration_counter % self.reconfiguration_freq == 0:
            self.reconfiguration_counter = 0
            return self._reconfigure(walkers, np.abs(w), rand or np.random.rand)

    def _device_state(self, walkers):
        if self._dev is None or self._dev["src"].numel() != walkers.nwalkers:
            dev = walkers.device
            self._dev = {
                "src": torch.empty(walkers.nwalkers, dtype=torch.int32, device=dev),
                "counter": torch.zeros(1, dtype=torch.int64, device=dev),
                "total": torch.full((1,), float(self.target_weight), dtype=torch.float64, device=dev),
                "uniforms": None,
            }
        return self._dev

    @property
    def total_weight_dev(self):
        return None if self._dev is None else self._dev["total"]

    def _pair_branch_device(self, walkers, uniforms=None):
        """Rescale and pair on the device, then the walker copies; nothing returns to the host."""
        d = self._device_state(walkers)
        call("ipie_b200_pair_branch", walkers.nwalkers, ptr(walkers.weight), ptr(walkers.unscaled_weight),
             float(self.target_weight), float(self.min_weight), float(self.max_weight), self.seed, ptr(d["counter"]),
             int(self.paired), ptr(d["src"]), ptr(d["total"]), ptr(self.wbound), ptr(uniforms), ptr(walkers.status),
             stream())
        call("ipie_b200_walker_copy", ptr(d["src"]), walkers.nwalkers, walkers.nbasis, walkers.nup, walkers.ndown,
             ptr(walkers.phia), ptr(walkers.phib), ptr(walkers.weight), ptr(walkers.unscaled_weight),
             ptr(walkers.hybrid_energy), ptr(walkers.ovlp), ptr(walkers.phase), ptr(walkers.Ghalfa),
             ptr(walkers.Ghalfb), stream())

    def _copy(self, walkers, src):
        if self._src is None or self._src.numel() != walkers.nwalkers:
            self._src = torch.empty(walkers.nwalkers, dtype=torch.int32, device=walkers.device)
        self._src.copy_(torch.from_numpy(src.astype(np.int32)))
        call("ipie_b200_walker_copy", ptr(self._src), walkers.nwalkers, walkers.nbasis, walkers.nup, walkers.ndown,
             ptr(walkers.phia), ptr(walkers.phib), ptr(walkers.weight), ptr(walkers.unscaled_weight),
             ptr(walkers.hybrid_energy), ptr(walkers.ovlp), ptr(walkers.phase), ptr(walkers.Ghalfa),
             ptr(walkers.Ghalfb), stream())

    def _pair_branch(self, walkers, w, rand):
        if self.leader is not None:
            pairs = self.leader.last_pairs
            neww, status = apply_pairs(np.abs(w), pairs)
        else:
            self.last_pairs = pairs = []
            neww, status = pair_branch_table(np.abs(w), self.max_weight, self.min_weight, rand, pairs=pairs)
        cloned = np.nonzero(status == 2)[0]
        killed = np.nonzero(status == 0)[0]
        w[cloned] = neww[cloned]
        walkers.weight.copy_(torch.from_numpy(w))
        if killed.size:
            src = np.full(walkers.nwalkers, -1, dtype=np.int32)
            if self.paired:
                for i, j, keep_j in pairs:
                    keep, drop = (j, i) if keep_j else (i, j)
                    src[drop] = keep
            elif cloned.size:
                src[killed] = cloned.max()
            self._copy(walkers, src)
        return neww, status

    def _comb(self, walkers, w, global_weights, rand):
        """Walker kill[i] <- clone[i] (pairs zipped in index order), then every weight is 1."""
        parent = comb_parent_counts(global_weights, self.target_weight, rand())
        kill = np.where(parent == 0)[0]
        clone = np.where(parent > 1)[0]
        walkers.weight.copy_(torch.from_numpy(w))
        src = np.full(walkers.nwalkers, -1, dtype=np.int32)
        for c, k in zip(clone, kill):
            src[k] = c
        if (src >= 0).any():
            self._copy(walkers, src)
        walkers.weight.fill_(1.0)
        return parent

    def _reconfigure(self, walkers, absw, rand):
        """Resample every slot from the cumulative |w|; all weights become the mean."""
        src, mean_weight = reconfiguration_sources(absw, rand())
        if self._src is None or self._src.numel() != walkers.nwalkers:
            self._src = torch.empty(walkers.nwalkers, dtype=torch.int32, device=walkers.device)
        self._src.copy_(torch.from_numpy(src.astype(np.int32)))
        walkers.resample(self._src)
        walkers.weight.fill_(mean_weight)
        return src
