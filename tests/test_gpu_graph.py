"""A walker step replayed from a captured CUDA graph equals the same step launched normally."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _run(precision, graph, steps=12):
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic

    s = synthetic.generate(64, (8, 8), 128, decay=30.0, seed=3, uhf=False, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (8, 8), 64)
    trial.half_rotate(ham)
    af = AFQMC.build((8, 8), ham, trial, num_walkers=48, seed=5, num_steps_per_block=6, num_blocks=2,
                     verbose=False, rng="device", precision=precision, graph=graph)
    af.setup_run()
    for step in range(1, steps + 1):  # reortho and pair branch at steps 5 and 10, energies at 6 and 12
        af.step(step)
    torch.cuda.synchronize()
    w = af.walkers
    return af, (np.array(af.block_data), w.weight.cpu().numpy(), w.phia.cpu().numpy(), w.ovlp.cpu().numpy(),
                w.Ghalfa.cpu().numpy())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_matches_launches(precision):
    af_g, got = _run(precision, True)
    _, ref = _run(precision, False)
    # one graph per orbital-buffer parity and step variant: plain steps (with the accumulation),
    # and the reortho steps 5 and 10 (pair branch decided on the host after the replay)
    assert af_g.graphs.captures == 4
    assert af_g.graphs.replays == 11
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    af_g.walkers.check_status()
