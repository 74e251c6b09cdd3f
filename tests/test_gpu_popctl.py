"""Pair-branch population control decided on the device (``ipie_b200_pair_branch``).

The device pairing is held to ipie's pairing walk restated on the host (``pair_branch_table``,
``walkers/pop_controller.py:338-391``) fed the uniforms the kernel drew, with both copy
semantics; a run with it replays bitwise from CUDA graphs; a vanishing total weight raises
ipie's ``ValueError``.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from ipie_b200._lib import call, ptr, stream  # noqa: E402
from ipie_b200.pop_control import pair_branch_table  # noqa: E402

pytestmark = pytest.mark.gpu


def _device_branch(w0, paired, counter=0, seed=5):
    W = w0.size
    dev = "cuda"
    w = torch.from_numpy(w0.copy()).to(dev)
    unscaled = torch.zeros(W, dtype=torch.float64, device=dev)
    src = torch.full((W,), -7, dtype=torch.int32, device=dev)
    ctr = torch.full((1,), counter, dtype=torch.int64, device=dev)
    total = torch.zeros(1, dtype=torch.float64, device=dev)
    wb = torch.zeros(1, dtype=torch.float64, device=dev)
    u = torch.full((W // 2,), -1.0, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    call("ipie_b200_pair_branch", W, ptr(w), ptr(unscaled), float(W), 0.1, 4.0, seed, ptr(ctr), int(paired),
         ptr(src), ptr(total), ptr(wb), ptr(u), ptr(status), stream())
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in dict(w=w, unscaled=unscaled, src=src, ctr=ctr, total=total, wb=wb, u=u,
                                                  status=status).items()}


def _weights(W, seed):
    rng = np.random.default_rng(seed)
    w = np.exp(rng.normal(0.0, 1.3, size=W))
    w[rng.integers(0, W, size=W // 8)] = w[0]  # exact ties, as copies of one walker leave them
    return w * 1.7


@pytest.mark.parametrize("W", [2048, 37, 2])
@pytest.mark.parametrize("paired", [0, 1])
def test_device_pair_branch_matches_pairing_walk(W, paired):
    w0 = _weights(W, seed=W + paired)
    d = _device_branch(w0, paired)
    total = np.sum(np.abs(w0))
    assert d["status"][0] == 0
    assert abs(d["total"][0] - total) <= 1e-14 * total
    assert abs(d["wb"][0] - 0.1 * total) <= 1e-14 * total
    assert d["ctr"][0] == 1
    np.testing.assert_array_equal(d["unscaled"], w0)
    ws = w0 / (d["total"][0] / W)
    it = iter(d["u"])
    pairs = []
    neww, status = pair_branch_table(np.abs(ws), 4.0, 0.1, lambda: next(it), pairs=pairs)
    assert len(pairs) > 0 or W == 2
    assert np.all(d["u"][len(pairs):] == -1.0)  # one uniform per pair formed, nothing beyond
    killed = status == 0
    np.testing.assert_array_equal(d["src"] >= 0, killed)
    cloned = np.nonzero(status == 2)[0]
    if killed.any():
        if paired:
            # killed walker -> its pair's survivor
            want = {(i if keep_j else j): (j if keep_j else i) for i, j, keep_j in pairs}
            for k in np.nonzero(killed)[0]:
                assert d["src"][k] == want[k]
        else:
            assert np.all(d["src"][killed] == cloned.max())
    keep = ~killed
    ref = ws.copy()
    ref[cloned] = neww[cloned]
    np.testing.assert_allclose(d["w"][keep], ref[keep], rtol=1e-14, atol=0)


def test_device_pair_branch_draws_advance():
    w0 = _weights(512, seed=3)
    a = _device_branch(w0, 1, counter=0)
    b = _device_branch(w0, 1, counter=1)
    c = _device_branch(w0, 1, counter=0)
    n = int(np.sum(a["u"] >= 0))
    assert n > 0
    assert not np.array_equal(a["u"][:n], b["u"][:n])
    np.testing.assert_array_equal(a["u"], c["u"])
    np.testing.assert_array_equal(a["src"], c["src"])


def _afqmc(population, graph, paired=True):
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic

    s = synthetic.generate(30, (6, 4), 90, decay=30.0, seed=12, uhf=True, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (6, 4), 30)
    trial.half_rotate(ham)
    return AFQMC.build((6, 4), ham, trial, num_walkers=40, seed=4, num_steps_per_block=10, num_blocks=3,
                       verbose=False, rng="device", graph=graph, population=population, paired_copies=paired)


def test_device_population_control_replays_from_graphs():
    """Steps with reortho, device pair branch and accumulation captured in graphs give the same
    walk, bit for bit, as the same steps launched one by one."""
    runs = {}
    for graph in (False, True):
        af = _afqmc("device", graph)
        runs[graph] = (af.run(), af)
    (b0, a0), (b1, a1) = runs[False], runs[True]
    np.testing.assert_array_equal(b0, b1)
    assert torch.equal(a0.walkers.weight, a1.walkers.weight)
    assert torch.equal(a0.walkers.phia, a1.walkers.phia)
    assert a1.graphs.replays == 29
    # the variants: plain steps, reortho + pair branch steps (every 5th)
    assert a1.graphs.captures >= 2
    assert np.all(np.isfinite(b1))
    # population control happened: some walker was copied over another at least once
    assert float(a1.pcontrol.total_weight_dev.item()) > 0


def test_device_population_control_walk_close_to_host_walk():
    """The device pairing with device uniforms makes other decisions than numpy's draws, but both
    walks stay populated and give block energies of the same system within a few Eh."""
    af_d = _afqmc("device", False)
    af_h = _afqmc("host", False)
    bd, bh = af_d.run(), af_h.run()
    assert np.all(np.isfinite(bd)) and np.all(np.isfinite(bh))
    assert abs(bd[-1, 5] - bh[-1, 5]) < 5.0


def test_device_population_control_zero_weight_raises():
    af = _afqmc("device", False)
    af.setup_run()
    af.walkers.weight.zero_()
    af.pcontrol.pop_control(af.walkers)
    with pytest.raises(ValueError):
        af.walkers.check_status()
