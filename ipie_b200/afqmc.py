"""AFQMC driver: ``AFQMC.build(...)`` and ``AFQMC.run()`` on one B200.

Mirror of ipie's ``AFQMC`` (``qmc/afqmc.py:297-392`` build, ``:508-633`` run):
same arguments, same step order (reortho every ``stabilize_freq`` steps,
propagate, weight clip, pair branch every ``pop_control_freq`` steps,
accumulate, energy every block, eshift update).  The block estimates are
kept in ``self.block_data`` (and written to an estimator file in ipie's HDF5
layout when ``run`` is given ``estimator_filename``) as rows of
``[Weight, WeightFactor, HybridEnergy, ENumer, EDenom, ETotal, E1Body, E2Body]``.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import call, ptr, stream
from .estimators import EnergyEstimator
from .pop_control import PopController
from .propagation import PhaselessGeneric
from .walkers import UHFWalkers

C128 = torch.complex128


@dataclass
class QMCParams:
    num_walkers: int
    total_num_walkers: int
    num_blocks: int
    num_steps_per_block: int
    timestep: float
    num_stblz: int
    pop_control_freq: int
    rng_seed: int | None


class WalkerAccumulator:
    """Block sums of weight, unscaled weight and weighted hybrid energy (ipie ``base_walkers.py:32-83``)."""

    def __init__(self, nsteps, device):
        self.nsteps_per_block = nsteps
        self.buffer = torch.zeros(7, dtype=C128, device=device)
        self._eshift = 0.0

    def update(self, walkers):
        call("ipie_b200_walker_sums", walkers.nwalkers, ptr(walkers.weight), ptr(walkers.unscaled_weight),
             ptr(walkers.hybrid_energy), None, ptr(self.buffer), 1, stream())

    def block_end(self, block):
        """Post-reduce hook (``base_walkers.py:69-80``) and the eshift of ``handler.py:231-236``."""
        v = self.buffer.cpu().numpy()
        factor = 1 if block == 0 else self.nsteps_per_block
        vals = np.array([v[0] / factor, v[1] / factor, v[2] / v[0]])
        self._eshift = vals[2]
        self.buffer.zero_()
        return vals

    @property
    def eshift(self):
        return np.real(self._eshift)


class AFQMC:
    def __init__(self, system, hamiltonian, trial, walkers, propagator, params, verbose=False):
        self.system = system
        self.hamiltonian = hamiltonian
        self.trial = trial
        self.walkers = walkers
        self.propagator = propagator
        self.params = params
        self.verbose = verbose
        if params.rng_seed is not None:
            np.random.seed(params.rng_seed)  # ipie qmc/utils.py:24-40 (seed + rank, rank 0)
        self.block_data = []
        self.timers = {}
        self.use_graph = False
        self.graphs = None
        self.population = "host"
        self.paired_copies = False

    @staticmethod
    def build(num_elec, hamiltonian, trial_wavefunction, walkers=None, num_walkers=100, seed=None,
              num_steps_per_block=25, num_blocks=100, timestep=0.005, stabilize_freq=5, pop_control_freq=5,
              verbose=True, mpi_handler=None, rng="numpy", spin_alias="auto", precision="fp64", graph=False,
              population="host", paired_copies=False):
        """ipie's ``AFQMC.build`` (``qmc/afqmc.py:297-392``) plus the B200 options: ``rng`` ("numpy":
        ipie's draws; "device": on-GPU draws), ``precision`` ("fp64" | "mixed"), ``spin_alias``,
        ``graph`` (replay each step's device work from a captured CUDA graph; needs rng="device") and
        ``population`` ("host": ipie's pair branch decided on the host with numpy's draws; "device":
        decided on the GPU with device draws, no host round trip, captured in the step graph) and
        ``paired_copies`` (a killed walker receives its own pair's survivor, ipie's multi-rank
        semantics, instead of the highest-index survivor, its single-process semantics)."""
        params = QMCParams(num_walkers, num_walkers, num_blocks, num_steps_per_block, timestep, stabilize_freq,
                           pop_control_freq, seed)
        if not trial_wavefunction.half_rotated:
            trial_wavefunction.half_rotate(hamiltonian)
        if walkers is None and getattr(trial_wavefunction, "multidet", False):
            # ipie starts them at the reference determinant, whose overlap with every excited
            # determinant is zero: the determinant sums here need walkers that overlap all of them
            raise NotImplementedError("with a particle-hole trial pass walkers that overlap every determinant "
                                      "(e.g. the perturbed reference); walkers at the reference determinant "
                                      "itself need Wick's theorem relative to it, which is not built")
        if walkers is None:
            init = np.asarray(trial_wavefunction.psi).copy()  # walkers_dispatch.py:42-58
            if getattr(trial_wavefunction, "ghf", False):
                from .ghf import GHFWalkers  # walkers_dispatch.py:61-72

                walkers = GHFWalkers(init, num_elec[0], num_elec[1], hamiltonian.nbasis, num_walkers,
                                     device=trial_wavefunction.device)
            else:
                walkers = UHFWalkers(init, num_elec[0], num_elec[1], hamiltonian.nbasis, num_walkers,
                                     device=trial_wavefunction.device)
            walkers.build(trial_wavefunction)
        if graph and getattr(walkers, "ghf", False):
            raise NotImplementedError("graph capture covers UHF walkers; GHF walkers step kernel by kernel")
        if graph and getattr(trial_wavefunction, "multidet", False):
            raise NotImplementedError("graph capture covers single-determinant trials; a particle-hole trial "
                                      "steps kernel by kernel")
        prop = PhaselessGeneric(timestep, rng=rng, seed=seed if seed is not None else 7, precision=precision)
        prop.build(hamiltonian, trial_wavefunction, walkers)
        # identical spin blocks (RHF trial, walkers started from it, equal one-body operators):
        # compute each block once (results equal propagating both, ipie's production mode)
        if spin_alias and getattr(trial_wavefunction, "spin_symmetric", False) and prop.spin_symmetric:
            if walkers.nup == walkers.ndown and torch.equal(walkers.phia, walkers.phib):
                walkers.enable_spin_alias()
        af = AFQMC(num_elec, hamiltonian, trial_wavefunction, walkers, prop, params, verbose=verbose)
        af.use_graph = bool(graph)
        if af.use_graph and rng != "device":
            raise ValueError("graph=True needs rng='device'")
        if population not in ("host", "device"):
            raise ValueError(f"population must be 'host' or 'device', not {population!r}")
        af.population = population
        af.paired_copies = bool(paired_copies)
        return af

    def _block(self, block, est, acc_vals):
        d = est.data.copy()
        est.post_reduce_hook(d)
        row = [acc_vals[0].real, acc_vals[1].real, acc_vals[2].real, d[0].real, d[1].real, d[2].real, d[3].real,
               d[4].real]
        self.block_data.append(row)
        if getattr(self, "estimator_filename", None):
            from .io import write_estimates

            write_estimates(self.estimator_filename, self.block_data, metadata=self.metadata())
        if self.verbose:
            print(f"{block:>17d} " + " ".join(f"{v: .16e}" for v in row))

    def setup_run(self, walkers=None):
        """Everything ``run`` does before its step loop (``afqmc.py:526-559``)."""
        if walkers is not None:
            self.walkers = walkers
        w, ham, trial, p = self.walkers, self.hamiltonian, self.trial, self.params
        self.eshift = 0.0
        w.orthogonalise()
        if self.population == "device":
            # the clip bound lives on the device from here on: 0.1 x the target weight until the
            # first population control writes 0.1 x the total weight
            ws = self.propagator._workspace(w, ham)
            ws.wbound.fill_(0.10 * p.num_walkers)
            seed = p.rng_seed if p.rng_seed is not None else 7
            self.pcontrol = PopController(p.num_walkers, p.num_steps_per_block, device=True, seed=seed + 7919,
                                          wbound=ws.wbound, paired=self.paired_copies)
        else:
            self.pcontrol = PopController(p.num_walkers, p.num_steps_per_block, paired=self.paired_copies)
        self.accumulators = WalkerAccumulator(p.num_steps_per_block, w.device)
        self.estimator = EnergyEstimator(precision=self.propagator.precision)
        self.estimator.compute_estimator(self.system, w, ham, trial)
        self.accumulators.update(w)
        self._block(0, self.estimator, self.accumulators.block_end(0))
        self.num_eqlb_steps = 2.0 / p.timestep

    def step(self, step):
        """Body of ``run``'s loop for step number ``step`` (1-based; ``afqmc.py:561-633``)."""
        w, ham, trial, prop, p = self.walkers, self.hamiltonian, self.trial, self.propagator, self.params
        reortho = step % p.num_stblz == 0
        popc = step % p.pop_control_freq == 0
        dev_pop = self.pcontrol.device
        # the clip bound: host scalar, or kept on the device by device population control
        wbound = None if dev_pop else self.pcontrol.total_weight * 0.10
        if self.use_graph and step > 1:
            if self.graphs is None:
                from .graphs import StepGraphs

                self.graphs = StepGraphs(prop, w, ham, trial)
            # the accumulation follows population control, so it joins the graph unless a
            # host-decided population control comes between them
            acc_in_graph = dev_pop or not popc
            self.graphs.step(np.real(self.eshift), wbound, reortho=reortho,
                             pcontrol=self.pcontrol if (popc and dev_pop) else None,
                             accumulators=self.accumulators if acc_in_graph else None)
            if popc and not dev_pop:
                self.pcontrol.pop_control(w)
            if not acc_in_graph:
                self.accumulators.update(w)
        else:
            if reortho:
                w.orthogonalise()
            prop.propagate_walkers(w, ham, trial, self.eshift)
            if step > 1:
                prop.clip_weights(w, wbound)
            if popc:
                self.pcontrol.pop_control(w)
            self.accumulators.update(w)
        if step % p.num_steps_per_block == 0:
            block = step // p.num_steps_per_block
            self.estimator.compute_estimator(self.system, w, ham, trial)
            self._block(block, self.estimator, self.accumulators.block_end(block))
            w.check_status()
        if step < self.num_eqlb_steps:
            self.eshift = self.accumulators.eshift
        else:
            self.eshift += self.accumulators.eshift - self.eshift

    def run(self, walkers=None, estimator_filename=None, verbose=True, additional_estimators=None):
        """The step loop (``afqmc.py:508-633``); with ``estimator_filename`` the block estimates are
        also written there after every block in ipie's estimator-file layout
        (:func:`ipie_b200.io.write_estimates`; ipie writes ``estimates.0.h5`` when no name is given,
        this driver writes nothing then)."""
        self.estimator_filename = estimator_filename
        self.setup_run(walkers)
        total_steps = self.params.num_steps_per_block * self.params.num_blocks
        t0 = time.time()
        for step in range(1, total_steps + 1):
            self.step(step)
        torch.cuda.synchronize()
        self.timers["run"] = time.time() - t0
        return np.array(self.block_data)

    def metadata(self):
        """JSON of the run parameters (the ``metadata`` entry of the estimator file)."""
        import json

        p = self.params
        return json.dumps({
            "system": {"nup": int(self.walkers.nup), "ndown": int(self.walkers.ndown)},
            "hamiltonian": {"nbasis": int(self.hamiltonian.nbasis), "nchol": int(self.hamiltonian.nchol),
                            "complex_chol": bool(getattr(self.hamiltonian, "complex_chol", False))},
            "qmc": {"nwalkers": p.num_walkers, "num_blocks": p.num_blocks, "num_steps": p.num_steps_per_block,
                    "timestep": p.timestep, "num_stblz": p.num_stblz, "pop_control_freq": p.pop_control_freq,
                    "rng_seed": p.rng_seed},
            "propagator": {"precision": self.propagator.precision, "rng": self.propagator.rng},
        }, indent=4)

    @staticmethod
    def build_from_hdf5(num_elec, ham_file, wfn_file, num_walkers=100, seed=None, num_steps_per_block=25,
                        num_blocks=100, timestep=0.005, stabilize_freq=5, pop_control_freq=5, num_dets_chunk=1,
                        num_dets_for_trial_props=100, pack_cholesky=True, verbose=True, **kwargs):
        """ipie's ``AFQMC.build_from_hdf5`` (``qmc/afqmc.py:394-475``): Hamiltonian and trial from
        files in ipie's or QMCPACK's HDF5 layouts (:mod:`ipie_b200.io`), then :meth:`build` with the
        electron counts read from the wavefunction file; ``kwargs`` go to :meth:`build`."""
        from .io import get_hamiltonian, get_trial_wavefunction

        ham = get_hamiltonian(ham_file, verbose=verbose, pack_chol=pack_cholesky)
        trial = get_trial_wavefunction(num_elec, ham.nbasis, wfn_file, ndet_chunks=num_dets_chunk,
                                       ndets_props=num_dets_for_trial_props, verbose=verbose)
        trial.half_rotate(ham)
        return AFQMC.build(trial.nelec, ham, trial, num_walkers=num_walkers, seed=seed,
                           num_steps_per_block=num_steps_per_block, num_blocks=num_blocks, timestep=timestep,
                           stabilize_freq=stabilize_freq, pop_control_freq=pop_control_freq, verbose=verbose,
                           **kwargs)
