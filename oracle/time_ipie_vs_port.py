"""Time ipie's own numpy walker step against the oracle port on the same bounded sample.

Test and measurement infrastructure, not product code.  The oracle port (``afqmc_oracle``) is
what ``bench.py`` times as the CPU baseline on the GPU host, where ipie's source is absent.
This script calibrates it: it runs ipie itself (its ``PhaselessGeneric.propagate_walkers`` and
``local_energy_single_det_uhf_batch`` on the numpy path, with the stand-ins for ``plum`` and
``h5py`` from ``tests/golden/_ref_shims``) and the port on the same sample of a workload, with
the same BLAS threads, and prints both rates as JSON.

    python oracle/time_ipie_vs_port.py /path/to/ipie-checkout [workload] [walkers] [repeats]

A sample is ``walkers`` walkers propagated one step plus the local energy of one walker,
amortised at one evaluation per 25 steps (the rate unit is walker-steps/s).
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def main():
    ref = sys.argv[1]
    wl = sys.argv[2] if len(sys.argv) > 2 else "c2_rhf_m200"
    nw = int(sys.argv[3]) if len(sys.argv) > 3 else 32
    reps = int(sys.argv[4]) if len(sys.argv) > 4 else 3
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden", "_ref_shims"))
    sys.path.insert(0, ref)
    sys.path.insert(0, ROOT)

    from ipie.estimators.greens_function_single_det import greens_function_single_det
    from ipie.estimators.local_energy_sd import local_energy_single_det_uhf_batch
    from ipie.hamiltonians.generic import Generic as HamGeneric
    from ipie.propagation.phaseless_generic import PhaselessGeneric
    from ipie.systems.generic import Generic
    from ipie.trial_wavefunction.single_det import SingleDet
    from ipie.utils.mpi import MPIHandler
    from ipie.walkers.walkers_dispatch import UHFWalkersTrial

    import bench
    from ipie_b200 import synthetic

    p = bench.WORKLOADS[wl]
    s = synthetic.generate(p["nbasis"], p["nocc"], p["nchol"], p["decay"], seed=7, uhf=p["uhf"], chol_scale="stable")
    ham = HamGeneric(h1e=s.h1e.copy(), chol=s.chol.copy(), ecore=s.ecore)
    trial = SingleDet(s.psi.copy(), (s.nup, s.ndown), s.nbasis)
    trial.half_rotate(ham)
    system = Generic((s.nup, s.ndown))

    def ipie_sample(walkers, prop, sub):
        t0 = time.perf_counter()
        prop.propagate_walkers(walkers, ham, trial, 0.0)
        t1 = time.perf_counter()
        greens_function_single_det(sub, trial)
        local_energy_single_det_uhf_batch(system, ham, sub, trial)
        t2 = time.perf_counter()
        return 1.0 / ((t1 - t0) / nw + (t2 - t1) / 25.0), t2 - t0

    np.random.seed(7)
    walkers = UHFWalkersTrial(trial, s.init.copy(), s.nup, s.ndown, s.nbasis, nw, MPIHandler())
    walkers.build(trial)
    sub = UHFWalkersTrial(trial, s.init.copy(), s.nup, s.ndown, s.nbasis, 1, MPIHandler())
    sub.build(trial)
    prop = PhaselessGeneric(0.005)
    prop.build(ham, trial, walkers, MPIHandler())
    ipie_sample(walkers, prop, sub)  # numba compilation and first-touch out of the timing
    ipie_runs = [ipie_sample(walkers, prop, sub) for _ in range(reps)]

    cpu = bench.CpuSample(wl, walkers=nw, energy_walkers=1)
    cpu.step()
    port_runs = [cpu.step() for _ in range(reps)]

    ipie_rate = float(np.median([r for r, _ in ipie_runs]))
    port_rate = float(np.median([r for r, _ in port_runs]))
    print(json.dumps({
        "workload": wl, "sample": cpu.sample, "repeats": reps,
        "ipie_walker_steps_per_s": ipie_rate, "port_walker_steps_per_s": port_rate,
        "port_over_ipie": port_rate / ipie_rate,
        "ipie_sample_s": [round(t, 3) for _, t in ipie_runs], "port_sample_s": [round(t, 3) for _, t in port_runs],
        "cores": os.cpu_count(), "blas_threads": bench.blas_threads(),
    }))


if __name__ == "__main__":
    main()
