"""One walker step captured as a CUDA graph.

The per-step device work of the driver loop -- reortho (on its steps), the
whole propagation (force bias, fields, VHS, orbital update, Green's function
of the new orbitals, weights), the weight clip, population control decided on
the device (on its steps) and the block accumulation -- is a fixed sequence of
kernel launches on fixed buffers, so it is captured once per variant and
replayed.  The energy shift (and, with population control on the host, the
clip bound) is written to its device scalar before each replay; population
control decided on the host and the energy estimator run as ordinary launches
on the same stream.

The step ping-pongs the orbitals between two buffers, so two graphs exist
(one per buffer parity); each remembers the Python-side buffer assignment it
was captured from and the one it leaves, and a replay restores the latter.
A buffer that was replaced (e.g. by stochastic reconfiguration) simply leads
to a new capture.  Auxiliary fields come from the device-side counter of
``rng="device"``, which the graph advances on every replay, so graph and
ordinary launches give the same draws.
"""
from __future__ import annotations

import torch

from .propagation import _NoTimer

# attributes that one step may re-point (buffer swaps in the orbital update, ovlp)
_STATE = (("walkers", "phia"), ("walkers", "phib"), ("walkers", "Ghalfa"), ("walkers", "Ghalfb"),
          ("walkers", "ovlp"), ("ws", "phia_tmp"), ("ws", "phib_tmp"))


class StepGraphs:
    def __init__(self, propagator, walkers, hamiltonian, trial):
        if propagator.rng != "device":
            raise ValueError("graph capture needs rng='device' (host draws cannot be replayed)")
        self.prop, self.walkers, self.ham, self.trial = propagator, walkers, hamiltonian, trial
        self.graphs = {}
        self.captures = 0
        self.replays = 0
        self.launches_per_step = 0  # kernel launches recorded in the last captured step
        self.replayed_launches = 0  # kernel launches replayed so far (all variants)

    def _owner(self, name):
        return self.walkers if name == "walkers" else self.prop.ws

    def _objs(self):
        return tuple(getattr(self._owner(o), n) for o, n in _STATE)

    def _set(self, objs):
        for (o, n), t in zip(_STATE, objs):
            setattr(self._owner(o), n, t)

    def _body(self, reortho, pcontrol, accumulators):
        prop = self.prop
        if reortho:
            self.walkers.orthogonalise()
        prop.propagate_walkers(self.walkers, self.ham, self.trial, prop.ws.eshift)
        prop.clip_weights(self.walkers)
        if pcontrol is not None:
            pcontrol.pop_control(self.walkers)
        if accumulators is not None:
            accumulators.update(self.walkers)

    def step(self, eshift, wbound, reortho=False, pcontrol=None, accumulators=None):
        """One step: reortho first when ``reortho``, propagation + weight clip, then ``pcontrol``'s
        device population control and ``accumulators``' update when given.  ``eshift`` is a host
        scalar; ``wbound`` a host scalar, or None to keep the device bound (kept by population
        control on the device)."""
        from .trial import greens_function_into

        prop, w, trial = self.prop, self.walkers, self.trial
        if pcontrol is not None and not pcontrol.device:
            raise ValueError("only population control decided on the device can be captured")
        prop._workspace(w, self.ham)
        ws = prop.ws
        ws.eshift.fill_(float(eshift))
        if wbound is not None:
            ws.wbound.fill_(float(wbound))
        if not w.gf_current(trial):
            # the captured step starts from the cached Green's function
            greens_function_into(w, trial, w.ovlp)
            w.mark_gf_current(trial)
        if prop.rng_counter_dev is None:
            prop.rng_counter_dev = torch.full((1,), prop.rng_counter, dtype=torch.int64, device=w.device)
        pre = self._objs()
        key = tuple(id(t) for t in pre) + (bool(reortho), id(pcontrol), id(accumulators))
        entry = self.graphs.get(key)
        if entry is None:
            # capture runs the Python side of one step without executing it on the GPU
            from ._lib import launch_count

            timer, prop.timer = prop.timer, _NoTimer()
            counter = prop.rng_counter
            n0 = launch_count()
            g = torch.cuda.CUDAGraph()
            try:
                with torch.cuda.graph(g, capture_error_mode="thread_local"):
                    self._body(reortho, pcontrol, accumulators)
            finally:
                prop.timer = timer
                prop.rng_counter = counter
            self.launches_per_step = launch_count() - n0
            post = self._objs()
            self._set(pre)
            entry = (g, pre, post, self.launches_per_step)
            self.graphs[key] = entry
            self.captures += 1
        g, _, post, nl = entry
        g.replay()
        self.replays += 1
        self.replayed_launches += nl
        prop.rng_counter += 1
        self._set(post)
        w.sync_alias()
        w.mark_gf_current(trial)
