"""Walker-step throughput of the B200 phaseless-AFQMC drop-in.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A "step" is one AFQMC step of ipie's driver loop over the whole walker batch:
reortho every 5 steps, propagation (Green's function, one-body, force bias,
field shift, VHS, exp(VHS), one-body, overlap, weights), weight clip, pair
branch every 5 steps, accumulation, and the local energy every 25 steps.
Default workload: nbasis 200, 32+32 electrons, 1600 Cholesky vectors,
2048 walkers, dt 0.005 (synthetic Hamiltonian, seeded).

``value`` is walker-steps/s over the timed steps with all state resident in
HBM (auxiliary fields drawn on the device); each step's propagation and weight
clip replay from a captured CUDA graph (the phase breakdown comes from a few
steps launched kernel by kernel).  ``e2e`` runs the same steps
through the public API with the auxiliary fields supplied from pinned host
memory each step and the weights read back each step.  ``--impl reference``
times the CPU oracle (numpy restatement of ipie's path) on the host cores.
With torchrun (N > 1) every rank runs an independent replica (weak scaling);
the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c2_rhf_m200": dict(nbasis=200, nocc=32, nchol=1600, decay=200.0, walkers=2048, uhf=False),
    "c1_uhf_m108": dict(nbasis=108, nocc=15, nchol=600, decay=100.0, walkers=640, uhf=True),
    "c4_rhf_m76": dict(nbasis=76, nocc=10, nchol=400, decay=30.0, walkers=512, uhf=False),
    "c0_rhf_m26": dict(nbasis=26, nocc=5, nchol=120, decay=30.0, walkers=64, uhf=False),
}


METRIC = "walker-steps/s at <=0.1 mEh energy shift (mixed vs plain FP64 phaseless AFQMC step)"


def line_config(wl, W, world, form="mixed"):
    """The bench line's ``config`` (shared by both arms so the driver compares like with like)."""
    p = WORKLOADS[wl]
    return {
        "workload": wl, "nbasis": p["nbasis"], "nalpha": p["nocc"], "nbeta": p["nocc"], "nchol": p["nchol"],
        "walkers_per_gpu": W, "dt": 0.005, "form": form, "parallelism": f"replicas{world}",
        "l2": "inputs larger than L2 (VHS 1.3 GB fp64 / 1.3 GB split fp32, walkers 0.2-0.4 GB)",
        "step": "reortho/5, propagate, clip, pair-branch/5, energy/25 (ipie driver order)",
    }


def flops_per_walker(M, na, nb, X, alias=False):
    """Algorithmic real FLOPs per walker (complex mult-add = 8, real x complex = 4).

    With ``alias`` (identical spin blocks computed once) the per-spin terms count
    one block: the work executed.  Without it: both blocks, ipie's work.
    """
    P = M * (M + 1) // 2
    spins = [n for n in (na, nb) if n > 0]
    if alias:
        spins = spins[:1]
    f = {
        "greens_function": sum(12 * M * n * n + 8 * n ** 3 for n in spins),
        "force_bias": sum(4 * X * n * M for n in spins),
        "one_body": sum(2 * 4 * M * M * n for n in spins),
        "taylor": sum(48 * M * M * n for n in spins),
        "vhs": 4 * P * X,
        "overlap": sum(4 * M * n * n + 8 * n ** 3 for n in spins),
    }
    f["orbitals"] = f["one_body"] + f["taylor"]  # fused launch: one-body + exp(VHS) + one-body
    energy = sum(4 * X * n * n * M + 8 * X * n * n + 4 * X * n * M for n in spins)
    return f, energy


def load_peaks():
    peaks = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        peaks.update({k: d[k] for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained") if k in d})
        peaks["source"] = "measured"
    # FP64 and TF32 peaks: measured in the run (gemm_peaks) before the forms are timed; these
    # are the values an earlier measurement on this pool's B200s gave, kept only as a fallback
    peaks["fp64_tflops"] = 35.47
    peaks["tf32_tflops"] = 755.8
    peaks["fp64_tf32_source"] = "earlier cuBLAS 8192^3 measurement on B200"
    return peaks


def _best_time(fn, iters=5):
    import torch

    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    out = 1e9
    for _ in range(iters):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out = min(out, a.elapsed_time(b) / 1e3)
    return out


def gemm_peaks(peaks):
    """cuBLAS FP64 and TF32 GEMM rates (8192^3, best of 5, CUDA events), measured in this run on
    this GPU: the denominators of the FP64 form's phases and of the TF32 products."""
    import torch

    n = 8192
    for key, dt, tf32 in (("fp64_tflops", torch.float64, False), ("tf32_tflops", torch.float32, True)):
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, device="cuda", dtype=dt)
        b = torch.randn(n, n, device="cuda", dtype=dt)
        peaks[key] = round(2 * n ** 3 / _best_time(lambda: a @ b) / 1e12, 2)
        torch.backends.cuda.matmul.allow_tf32 = prev
        del a, b
    torch.cuda.empty_cache()
    peaks["fp64_tf32_source"] = "measured in this run: cuBLAS 8192^3 GEMM, best of 5"
    return peaks


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(ngpus):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        # NCCL between GPUs; gloo when no GPU is visible (the CPU test of the multi-rank path)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            backend = "nccl"
        else:
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier_max(value, world):
    import torch

    if world == 1:
        return value
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# DRAM bytes (read + write) per launch of a phase's kernel from one ncu capture, scaled to the
# workload's walker count (the capture's traffic grows with the walkers it processes); the
# capture and its command are summarised under profiles/.
DRAM_TRAFFIC = {
    # FP16 orbital chain (transposed products) at 512 walkers: 220.1 MB read + 35.9 MB written per
    # launch (profiles/orbital_chain_t16_c2_w512.md), x4 for 2048 walkers (its traffic is per walker)
    ("c2_rhf_m200", "mixed", "orbitals"): 4 * (220.10e6 + 35.86e6),
    # block-tiled VHS product with TMA-store epilogue at 512 walkers: 244.9 MB read + 178.5 MB
    # written (profiles/vhs_blocks_tma_c2_w512.md); the Cholesky operand (~150 MB) is read once per
    # launch whatever the walker count, the fields and planes scale with it
    ("c2_rhf_m200", "mixed", "vhs"): 4 * (244.9e6 - 150.0e6 + 178.5e6) + 150.0e6,
}


def build_afqmc(wl, walkers, rng, seed, precision="fp64", pop_control_freq=5, graph=False, population="host",
                paired_copies=False):
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic

    p = WORKLOADS[wl]
    s = synthetic.generate(p["nbasis"], p["nocc"], p["nchol"], p["decay"], seed=7, uhf=p["uhf"], chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis)
    trial.half_rotate(ham)
    af = AFQMC.build((s.nup, s.ndown), ham, trial, num_walkers=walkers, seed=seed, num_steps_per_block=25,
                     num_blocks=10 ** 6, timestep=0.005, stabilize_freq=5, pop_control_freq=pop_control_freq,
                     verbose=False, rng=rng,
                     precision=precision, graph=graph, population=population, paired_copies=paired_copies)
    return af, s


class CpuSample:
    """ipie's numpy walker step restated (the oracle) on the host cores, on a bounded sample of a
    workload: ``walkers`` walkers propagated one step plus the local energy of ``energy_walkers``
    walkers, amortised at one evaluation per 25 steps as in the driver loop."""

    def __init__(self, wl, walkers=32, energy_walkers=1):
        from ipie_b200 import synthetic
        from oracle import afqmc_oracle as O

        p = WORKLOADS[wl]
        s = synthetic.generate(p["nbasis"], p["nocc"], p["nchol"], p["decay"], seed=7, uhf=p["uhf"],
                               chol_scale="stable")
        self.O = O
        self.S = O.System(s.nbasis, s.nup, s.ndown, s.h1e, s.chol, s.ecore, s.psi).build()
        self.w = O.Walkers.from_initial(s.init, s.nup, walkers)
        np.random.seed(7)
        O.greens_function(self.S, self.w)
        self.walkers, self.energy_walkers = walkers, energy_walkers
        self.sample = (f"{walkers} walkers x 1 propagation step + local energy of {energy_walkers} walker(s) "
                       f"(amortised 1 per 25 steps), same system")

    def step(self):
        """One sample: returns (walker-steps/s, seconds the sample took)."""
        O, S, w = self.O, self.S, self.w
        t0 = time.perf_counter()
        O.propagate_walkers(S, w, 0.0)
        t1 = time.perf_counter()
        sub = w.copy()
        n = self.energy_walkers
        sub.phia, sub.phib = w.phia[:n].copy(), w.phib[:n].copy()
        sub.log_shift = w.log_shift[:n]
        O.greens_function(S, sub)
        O.local_energy_single_det_uhf_batch(S, sub)
        t2 = time.perf_counter()
        t_prop = (t1 - t0) / self.walkers
        t_en = (t2 - t1) / n
        return 1.0 / (t_prop + t_en / 25.0), t2 - t0


def blas_threads():
    try:
        from threadpoolctl import threadpool_info

        info = threadpool_info()
        return max((i.get("num_threads", 1) for i in info), default=os.cpu_count())
    except Exception:
        return os.cpu_count()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = args.workload
    p = WORKLOADS[wl]
    cpu = CpuSample(wl, walkers=args.ref_walkers, energy_walkers=1)
    for _ in range(max(args.warmup, 0)):
        cpu.step()
    rates, secs = [], []
    for _ in range(max(args.steps, 1)):
        r, dt = cpu.step()
        rates.append(r)
        secs.append(dt)
    value = float(np.median(rates))
    cores = blas_threads()
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "walker-steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        # a step of this arm is one bounded sample (below), timed by the wall clock
        "ms_per_step": float(np.median(secs)) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": line_config(wl, args.walkers or p["walkers"], int(os.environ.get("WORLD_SIZE", "1"))),
        "reference_path": ("ipie's numpy walker step (the oracle: numpy restatement pinned to ipie's outputs) on "
                           "the host cores; ipie's own run of the same sample is timed against it on the build "
                           "host (the ipie source does not travel to the GPU host)"),
        "cpu_baseline": {"value": value, "unit": "walker-steps/s", "cores": cores, "kind": "port",
                         "sample": cpu.sample},
        "e2e": {"value": value, "unit": "walker-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def train_control_variate(wl, W, rank, steps=100, epochs=60):
    """Exchange control variate trained on (features, exchange) pairs of `steps` plain FP64 steps."""
    import time as _t

    from ipie_b200.control_variate import ExchangeControlVariate, generate_training_data

    t0 = _t.perf_counter()
    af, _ = build_afqmc(wl, W, "device", 1000 + rank, precision="fp64")
    af.setup_run()
    feats, ys, bases = generate_training_data(af, steps=steps)
    del af
    cv = ExchangeControlVariate(hidden=256, seed=rank)
    hist = cv.fit(feats, ys, bases, epochs=epochs, batch=4096, lr=2e-3)
    resid = (ys - bases)
    info = {"pairs": int(feats.shape[0]), "epochs": epochs,
            "var_y": float(ys.var().item()), "var_y_minus_linear": float(resid.var().item()),
            "holdout_mse_first": hist[0][1], "holdout_mse_last": hist[-1][1],
            "mse_units": "var(y - linear term)", "seconds": _t.perf_counter() - t0}
    return cv, info


def statistics_runs(wl, W, rank, steps, cv=None, dt=0.005):
    """Block energies of the FP64 and mixed forms over ``steps`` driver steps, run in lockstep with
    identical draws and the same population control: the FP64 run draws its pair branch, the mixed
    run forms the same pairs from its own weights (``PopController.follow``), so the two stay the
    same walk and differ only by precision.  The mixed + control-variate estimator is evaluated on
    the mixed run's walkers at the same block ends (the control variate changes the estimator, not
    the walk).

    Returns {form: block ETotal series (blocks 1..n)} and, per form, ipie's reblocking analysis
    (:func:`ipie_b200.analysis.reblock_mixed`) of the blocks after ipie's equilibration time 2/dt
    and of the paired differences to FP64 over the same blocks."""
    from ipie_b200.analysis import reblock_mixed

    runs = {}
    for form in ("fp64", "mixed"):
        af, _ = build_afqmc(wl, W, "device", 4242 + rank, precision=form, graph=True, paired_copies=True)
        af.setup_run()
        runs[form] = af
    runs["mixed"].pcontrol.follow(runs["fp64"].pcontrol)
    cv_est, e_cv = None, []
    if cv is not None:
        from ipie_b200.control_variate import ControlVariateEnergyEstimator

        cv_est = ControlVariateEnergyEstimator(cv.clone(), fraction=8, seed=99 + rank, precision="mixed")
    nblk = runs["fp64"].params.num_steps_per_block
    t0 = time.perf_counter()
    for step in range(1, steps + 1):
        for form in ("fp64", "mixed"):  # the leader branches first
            runs[form].step(step)
        if cv_est is not None and step % nblk == 0:
            af = runs["mixed"]
            d = cv_est.compute_estimator(af.system, af.walkers, af.hamiltonian, af.trial)
            e_cv.append(float((d[0] / d[1]).real))
    seconds = time.perf_counter() - t0
    series = {form: np.array(af.block_data)[1:, 5].real for form, af in runs.items()}
    if cv_est is not None:
        series["mixed_cv"] = np.array(e_cv)
    del runs
    n = min(len(v) for v in series.values())
    series = {k: v[:n] for k, v in series.items()}
    eq = min(int(round(2.0 / dt / nblk)), max(n - 8, 0))  # ipie's equilibration time, in blocks
    out = {"blocks": n, "equilibration_blocks": eq, "steps": steps, "seconds": seconds,
           "coupling": ("identical device draws; the mixed run takes the FP64 run's pair-branch pairs; killed "
                        "walkers receive their own pair's survivor (ipie's multi-rank copy semantics)"), "forms": {}}
    for form, v in series.items():
        rb = reblock_mixed(v[eq:])
        entry = {"energy_Eh": rb["mean"], "error_mEh": max(rb["error"], rb["error_ac"]) * 1e3,
                 "error_fp_mEh": rb["error"] * 1e3, "error_ac_mEh": rb["error_ac"] * 1e3,
                 "reblock_converged": rb["converged"], "block": rb["block"]}
        if form != "fp64":
            d = reblock_mixed(v[eq:] - series["fp64"][eq:])
            entry["vs_fp64_mEh"] = d["mean"] * 1e3
            entry["vs_fp64_err_mEh"] = max(d["error"], d["error_ac"]) * 1e3
            entry["vs_fp64_max_block_mEh"] = float(np.max(np.abs(v - series["fp64"]))) * 1e3
        out["forms"][form] = entry
    return series, out


def timed_run(wl, W, precision, args, rank, world, local, rng="device", with_clock=False, cv=None):
    """Build, warm up and time ``args.steps`` driver steps of one form; returns a result dict."""
    import torch

    from ipie_b200 import _lib
    from ipie_b200.propagation import PhaseTimer, _NoTimer

    # each step's propagation and weight clip replay from a captured CUDA graph (device draws)
    graph = rng == "device"
    # throughput mode: population control decided on the device (no host round trip, inside the
    # step graph), killed walkers copying their own pair's survivor
    af, _ = build_afqmc(wl, W, rng, 7 + rank, precision=precision, graph=graph, population="device",
                        paired_copies=True)
    af.setup_run()
    if cv is not None:
        from ipie_b200.control_variate import ControlVariateEnergyEstimator

        af.estimator = ControlVariateEnergyEstimator(cv.clone(), fraction=8, seed=7 + rank, precision="mixed")
    step = 0
    for _ in range(args.warmup):
        step += 1
        af.step(step)
    # one untimed energy evaluation so the estimator's one-time set-up (work buffers, trial
    # reference, control-variate parts) happens before the timed region
    af.estimator.compute_estimator(af.system, af.walkers, af.hamiltonian, af.trial)
    # phase breakdown: a few steps launched one kernel at a time with CUDA events between phases
    torch.cuda.synchronize()
    timer = PhaseTimer()
    af.propagator.timer = timer
    af.use_graph = False
    phase_steps = min(10, args.steps)
    l0 = _lib.launch_count()
    for _ in range(phase_steps):
        step += 1
        af.step(step)
    torch.cuda.synchronize()
    launches_per_step_eager = (_lib.launch_count() - l0) / phase_steps
    af.propagator.timer = _NoTimer()
    af.use_graph = graph
    nblocks0 = len(af.block_data)
    launches0 = _lib.launch_count()
    replayed0 = af.graphs.replayed_launches if af.graphs is not None else 0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local) if with_clock else None
    if clk:
        clk.__enter__()
    ev0.record()
    for _ in range(args.steps):
        step += 1
        af.step(step)
    ev1.record()
    torch.cuda.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    if world > 1:
        torch.distributed.barrier()
    # kernels launched in the timed region: ordinary launches plus the captured ones replayed
    launches = _lib.launch_count() - launches0
    if af.graphs is not None:
        launches += af.graphs.replayed_launches - replayed0
    res = {
        "t": barrier_max(ev0.elapsed_time(ev1) / 1e3, world),
        "phases": timer.summary(),
        "phase_steps": phase_steps,
        "launches": launches,
        "launches_per_step_eager": launches_per_step_eager,
        "graph": bool(graph),
        "blocks": np.array(af.block_data),
        "timed_blocks": np.array(af.block_data[nblocks0:]),
        "alias": bool(af.walkers.spin_alias),
        "clocks": clk.summary() if clk else None,
    }
    af.propagator.timer = _NoTimer()
    # untimed checks on the final walkers
    w, ham, trial = af.walkers, af.hamiltonian, af.trial
    if precision == "mixed" and cv is None:
        from ipie_b200.estimators import EnergyEstimator

        d64 = EnergyEstimator(precision="fp64").compute_estimator(None, w, ham, trial)
        dmx = EnergyEstimator(precision="mixed").compute_estimator(None, w, ham, trial)
        res["estimator_shift_mEh"] = abs(float((dmx[0] / dmx[1]).real - (d64[0] / d64[1]).real)) * 1e3
    if cv is not None:
        from ipie_b200.control_variate import EnergyParts, cv_estimator_error

        res["cv_error"] = cv_estimator_error(cv, EnergyParts(ham, trial, w), w, fraction=8, trials=64)
    del af
    torch.cuda.empty_cache()
    return res


# tensor pipe of each mixed-form phase: every product is a 3-pass head/remainder product on FP16
# operands (kind::f16, the bf16 tensor rate) -- force bias, VHS and the orbital chain
MIXED_PIPE = {"force_bias": "f16", "vhs": "f16", "orbitals": "f16"}


def phase_roofline(r, form, fl, fl_ipie, W, peaks, wl):
    """Roofline of the phase with the largest CUDA-event time in ``r`` (one timed form), and every
    tensor-core phase's fraction of its pipe's peak.

    ``achieved`` counts ALGORITHMIC FLOPs: the per-walker figure of ``flops_per_walker`` (identical
    RHF spin blocks counted once when they are computed once) x walkers x launches / event time.
    The mixed form executes each product as 3 passes (head x head, head x remainder, remainder x
    head): ``achieved_executed`` counts those; ``achieved_ipie_work`` counts both spin blocks."""
    phases = r["phases"]
    dom = max((k for k in phases if k in fl), key=lambda k: phases[k][1])
    n_launch, tot_ms = phases[dom]
    passes = 3 if form == "mixed" else 1

    def pipe_of(k):
        if form != "mixed":
            return "fp64", peaks["fp64_tflops"], f"cuBLAS DGEMM 8192^3 ({peaks['fp64_tf32_source']})"
        if MIXED_PIPE.get(k, "tf32") == "f16":
            return ("f16", peaks["bf16_tflops"],
                    f"{peaks['source']} cuBLAS bf16 8192^3 burst (MEASURED_PEAKS.json; fp16 runs at the bf16 rate)")
        return "tf32", peaks["tf32_tflops"], f"cuBLAS TF32 8192^3 ({peaks['fp64_tf32_source']})"

    def rate(k, per_walker):
        n, ms = phases[k]
        return per_walker * W * n / (ms / 1e3) / 1e12 if ms > 0 else 0.0

    pipe, peak, src = pipe_of(dom)
    achieved = rate(dom, fl[dom])
    tensor_phases = [k for k in sorted(phases) if k in fl and k != "greens_function" and phases[k][1] > 0]
    return {
        "kernel": dom, "bound": "tensor", "pipe": pipe + (" (3 passes)" if passes == 3 else " (DMMA)"),
        "achieved": round(achieved, 3), "peak": peak, "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
        "frac_of": "measured" if "measured" in src else "fallback",
        "achieved_executed": round(passes * achieved, 3),
        "achieved_ipie_work": round(rate(dom, fl_ipie[dom]), 3),
        "algorithmic_gflop_per_launch": round(fl[dom] * W * n_launch / max(n_launch, 1) / 1e9, 3),
        "launch_ms": round(tot_ms / max(n_launch, 1), 4),
        "traffic": DRAM_TRAFFIC.get((wl, form, dom)),
        "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum, scaled by walkers)",
        "peak_source": src,
        "phase_ms_per_step": {k: round(v[1] / r["phase_steps"], 4) for k, v in sorted(phases.items())},
        "phase_frac_of_peak": {k: round(rate(k, fl[k]) / pipe_of(k)[1], 4) for k in tensor_phases},
        "phase_frac_executed": {k: round(passes * rate(k, fl[k]) / pipe_of(k)[1], 4) for k in tensor_phases},
        "phase_pipe": {k: pipe_of(k)[0] for k in tensor_phases},
        "phase_timing": f"{r['phase_steps']} steps launched kernel by kernel with CUDA events between phases",
    }


def run_ours(args):
    import torch

    rank, world, local = dist_setup(args.gpus)
    wl = args.workload
    p = WORKLOADS[wl]
    W = args.walkers or p["walkers"]
    M, na, nb, X = p["nbasis"], p["nocc"], p["nocc"], p["nchol"]
    peaks = load_peaks()
    if torch.cuda.is_available():
        gemm_peaks(peaks)
    forms = ["fp64", "mixed"] if args.form == "both" else [args.form]

    runs = {}
    for form in forms:
        runs[form] = timed_run(wl, W, form, args, rank, world, local, with_clock=(form == forms[-1]))
    cv_info = None
    if args.form == "both" and not args.no_cv:
        cv, cv_info = train_control_variate(wl, W, rank, steps=args.cv_steps)
        runs["mixed_cv"] = timed_run(wl, W, "mixed", args, rank, world, local, cv=cv)
        cv_info["estimator_error"] = runs["mixed_cv"].pop("cv_error", None)
    else:
        cv = None
    head = "mixed" if "mixed" in runs else "fp64"
    r = runs[head]
    t = r["t"]
    value = W * args.steps * world / t

    alias = r["alias"]
    fl, fl_energy = flops_per_walker(M, na, nb, X, alias=alias)
    fl_ipie, fl_energy_ipie = flops_per_walker(M, na, nb, X, alias=False)
    roofline = phase_roofline(r, head, fl, fl_ipie, W, peaks, wl)
    step_flops = (sum(v for k, v in fl.items() if k != "orbitals") * W + fl_energy * W / 25.0)
    step_flops_ipie = (sum(v for k, v in fl_ipie.items() if k != "orbitals") * W + fl_energy_ipie * W / 25.0)

    forms_out = {}
    for form, rr in runs.items():
        forms_out[form] = {"walker_steps_per_s": W * args.steps * world / rr["t"], "ms_per_step": rr["t"] / args.steps * 1e3,
                           "gpu_launches": int(rr["launches"]), "cuda_graph_steps": rr["graph"],
                           "block_etotal": [round(float(x), 9) for x in rr["blocks"][:, 5]]}
    if "fp64" in runs and head != "fp64":
        forms_out["fp64"]["roofline"] = phase_roofline(runs["fp64"], "fp64", fl, fl_ipie, W, peaks, wl)
    shift = shift_err = None
    stats = None
    if "mixed" in runs and "fp64" in runs:
        a, b = runs["mixed"]["blocks"][:, 5], runs["fp64"]["blocks"][:, 5]
        n = min(len(a), len(b))
        # with population control a single flipped branching decision moves whole walkers
        forms_out["trajectory_shift_with_branching_mEh"] = float(np.max(np.abs(a[:n] - b[:n]))) * 1e3
        forms_out["mixed_over_fp64"] = forms_out["mixed"]["walker_steps_per_s"] / forms_out["fp64"]["walker_steps_per_s"]
        forms_out["mixed"]["estimator_shift_mEh"] = runs["mixed"].get("estimator_shift_mEh")
        if args.stat_steps > 0:
            series, stats = statistics_runs(wl, W, rank, args.stat_steps, cv=cv)
            stats["block_etotal"] = {k: [round(float(x), 9) for x in v] for k, v in series.items()}
            e0 = stats["forms"]["fp64"]["error_mEh"]
            for form, st in stats["forms"].items():
                if form not in forms_out:
                    continue
                # statistical efficiency 1/(sigma^2 t) against the FP64 form: >1 means the form reaches
                # a given error bar in less time; sigma from the reblocked block energies, t = ms/step
                t_ratio = forms_out["fp64"]["ms_per_step"] / forms_out[form]["ms_per_step"]
                st["efficiency_vs_fp64"] = (e0 / st["error_mEh"]) ** 2 * t_ratio if st["error_mEh"] > 0 else None
                forms_out[form]["statistics"] = st
                if form != "fp64":
                    st["within_0p1_mEh"] = bool(abs(st["vs_fp64_mEh"]) - 2 * st["vs_fp64_err_mEh"] <= 0.1)
            shift = abs(stats["forms"]["mixed"]["vs_fp64_mEh"])
            shift_err = stats["forms"]["mixed"]["vs_fp64_err_mEh"]
            if "mixed_cv" in stats["forms"] and "mixed_cv" in forms_out:
                st = stats["forms"]["mixed_cv"]
                gain = st["efficiency_vs_fp64"] / stats["forms"]["mixed"]["efficiency_vs_fp64"]
                st["cv_gain_over_mixed"] = gain
                st["note"] = ("the control variate's cheaper energy evaluations outweigh its added noise" if gain > 1
                              else "the control variate's added noise cancels its cheaper energy evaluations")
    if "mixed_cv" in runs and "fp64" in runs:
        forms_out["mixed_cv_over_fp64"] = (forms_out["mixed_cv"]["walker_steps_per_s"]
                                          / forms_out["fp64"]["walker_steps_per_s"])
        forms_out["mixed_cv"]["training"] = cv_info
    del cv

    # ---------------- end to end through the public API (headline form) ----------------
    e2e_steps = min(args.steps, args.e2e_steps)
    af2, _ = build_afqmc(wl, W, "host", 7 + rank, precision=head, population="device", paired_copies=True)
    rng = np.random.default_rng(1234 + rank)
    fields = [torch.from_numpy(rng.standard_normal((W, X))).pin_memory() for _ in range(args.warmup + e2e_steps)]
    af2.propagator.host_fields = iter(fields)
    wback = torch.empty(W, dtype=torch.float64).pin_memory()
    af2.setup_run()
    step = 0
    for _ in range(args.warmup):
        step += 1
        af2.step(step)
        wback.copy_(af2.walkers.weight)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        step += 1
        af2.step(step)
        wback.copy_(af2.walkers.weight, non_blocking=True)  # the step's result back to (pinned) host memory
    e1.record()
    torch.cuda.synchronize()
    t2 = barrier_max(e0.elapsed_time(e1) / 1e3, world)
    e2e_value = W * e2e_steps * world / t2
    del af2, fields
    torch.cuda.empty_cache()

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            sampler = CpuSample(wl, walkers=args.ref_walkers, energy_walkers=1)
            sampler.step()  # warm-up
            rcpu = float(np.median([sampler.step()[0] for _ in range(2)]))
            cpu = {"value": rcpu, "unit": "walker-steps/s", "cores": blas_threads(), "kind": "port",
                   "sample": sampler.sample + ", median of 2 after 1 warm-up"}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "walker-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f16+f64" if head == "mixed" else "f64",
            "data": "synthetic",
            "config": line_config(wl, W, world, head),
            "forms": forms_out,
            "energy_shift_mEh": shift,
            "energy_shift_err_mEh": shift_err,
            "energy_shift_method": (f"|mean of block E(mixed) - block E(fp64)| over the blocks after ipie's "
                                    f"equilibration time (2/dt) of two {args.stat_steps}-step runs with identical "
                                    "draws and no population control, reblocked error (ipie's reblock_mixed: "
                                    "Flyvbjerg-Petersen and autocorrelation, the larger); per form in "
                                    "forms.*.statistics; estimator-only shift on identical walkers in "
                                    "forms.mixed.estimator_shift_mEh"),
            "statistics": ({k: v for k, v in stats.items() if k != "forms"} if stats else None),
            "e2e": {"value": e2e_value, "unit": "walker-steps/s", "h2d_bytes_per_step": W * X * 8,
                    "d2h_bytes_per_step": W * 8, "steps": e2e_steps,
                    "fields": "host-supplied N(0,1) draws in pinned memory, one (W, X) array per step"},
            "roofline": roofline,
            "step_tflops": round(step_flops / (t / args.steps) / 1e12, 3),
            "work": {"spin_alias": alias, "executed_gflop_per_step": round(step_flops / 1e9, 1),
                     "ipie_equivalent_gflop_per_step": round(step_flops_ipie / 1e9, 1)},
            "cpu_baseline": cpu,
            "clocks": r["clocks"],
            "gpu_launches": int(r["launches"]),
            "finite_energies": bool(all(np.all(np.isfinite(rr["blocks"])) for rr in runs.values())),
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def measure_peaks():
    """torch/cuBLAS GEMM and copy peaks (the FP64/TF32 roofline denominators); prints JSON."""
    import torch

    def best(fn, iters=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        out = 1e9
        for _ in range(iters):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            out = min(out, a.elapsed_time(b) / 1e3)
        return out

    res = {}
    n = 8192
    for name, dt, tf32 in (("f64", torch.float64, False), ("f32", torch.float32, False), ("tf32", torch.float32, True),
                           ("bf16", torch.bfloat16, False)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, device="cuda").to(dt)
        b = torch.randn(n, n, device="cuda").to(dt)
        res[f"{name}_tflops_8192"] = 2 * n ** 3 / best(lambda: a @ b) / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    x = torch.empty(2 ** 28, device="cuda", dtype=torch.float64)
    y = torch.empty_like(x)
    res["copy_gbs"] = 2 * x.numel() * 8 / best(lambda: y.copy_(x)) / 1e9
    print(json.dumps(res))
    return 0


def profile_round(args):
    """A few driver steps of one form launched kernel by kernel (no CUDA graph, device draws): the
    target of the ncu captures summarised under profiles/, e.g.
    ncu --set full --clock-control none -k regex:orbital_chain16 -s 1 -c 1 python bench.py
    --profile-round --walkers 512"""
    import torch

    torch.cuda.set_device(0)
    wl = args.workload
    W = args.walkers or WORKLOADS[wl]["walkers"]
    af, _ = build_afqmc(wl, W, "device", 7, precision=args.form if args.form != "both" else "mixed",
                        population="device", paired_copies=True)
    af.setup_run()
    for step in range(1, 4):
        af.step(step)
    af.estimator.compute_estimator(af.system, af.walkers, af.hamiltonian, af.trial)
    torch.cuda.synchronize()
    af.walkers.check_status()
    print(json.dumps({"profile_round": wl, "walkers": W, "steps": 3, "energy_evaluations": 2}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100, help="timed steps; multiples of 25 include whole energy blocks")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2_rhf_m200", choices=sorted(WORKLOADS))
    ap.add_argument("--walkers", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=25)
    ap.add_argument("--ref-walkers", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cv", action="store_true", help="skip the learned control-variate form")
    ap.add_argument("--cv-steps", type=int, default=100, help="plain-method steps generating control-variate training data")
    ap.add_argument("--stat-steps", type=int, default=1000,
                    help="steps of the FP64/mixed/control-variate statistics runs (0: skip); 25 steps per block")
    ap.add_argument("--form", choices=["fp64", "mixed", "both"], default="both",
                    help="which forms to time; with both, the mixed form is the headline and the FP64 form its reference")
    ap.add_argument("--measure-peaks", action="store_true", help="print measured GEMM/copy peaks and exit")
    ap.add_argument("--profile-round", action="store_true",
                    help="run 3 steps + 2 energy evaluations of one form kernel by kernel (an ncu target) and exit")
    args = ap.parse_args()
    if args.measure_peaks:
        return measure_peaks()
    if args.profile_round:
        return profile_round(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
