"""The learned exchange control variate: GPU MLP kernels vs the CPU oracle, and what training gains."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def test_mlp_forward_and_gradients_match_oracle():
    from ipie_b200.control_variate import ExchangeControlVariate
    from ipie_b200._lib import call, ptr, stream

    cv = ExchangeControlVariate(hidden=64, seed=4)
    B, F, H = 96, 16, 64
    rng = np.random.default_rng(0)
    x = rng.normal(size=(B, F)).astype(np.float32)
    y = rng.normal(size=B).astype(np.float32)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    acts = torch.empty(4 * B * H, dtype=torch.float32, device="cuda")
    out = torch.empty(B, dtype=torch.float32, device="cuda")
    work = torch.empty(B + 2 * B * H, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    call("ipie_b200_mlp_forward", ptr(xd), B, F, H, ptr(cv.wbf), ptr(cv.master), ptr(acts), ptr(out), stream())
    call("ipie_b200_mlp_backward", ptr(xd), ptr(yd), B, F, H, ptr(cv.wbf), ptr(acts), ptr(out), ptr(cv.grad),
         ptr(work), ptr(loss), stream())
    theta = cv.master.cpu().numpy().astype(np.float64)
    ref_out, _ = mlp_oracle.forward(x.astype(np.float64), theta, F, H)
    ref_loss, ref_g = mlp_oracle.mse_grad(x.astype(np.float64), y.astype(np.float64), theta, F, H)
    got_g = cv.grad.cpu().numpy()
    assert np.max(np.abs(out.cpu().numpy() - ref_out)) < 1e-4 * max(1.0, np.max(np.abs(ref_out)))
    assert abs(loss.item() - ref_loss) < 1e-4 * ref_loss
    assert np.max(np.abs(got_g - ref_g)) < 2e-4 * np.max(np.abs(ref_g))


def test_trained_control_variate_reduces_subsample_variance():
    """Train on walker data of the plain method; the subsampled exchange estimate's spread shrinks."""
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic
    from ipie_b200.control_variate import (EnergyParts, ExchangeControlVariate, generate_training_data,
                                           subsample_variances)

    s = synthetic.generate(40, (8, 8), 160, decay=30.0, seed=5, uhf=False, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (8, 8), 40)
    trial.half_rotate(ham)
    af = AFQMC.build((8, 8), ham, trial, num_walkers=256, seed=5, num_blocks=100, verbose=False, rng="device")
    af.setup_run()
    feats, ys, bases = generate_training_data(af, steps=40)
    # the exchange over the leading eighth of the Cholesky vectors already carries most of the spread
    assert (ys - bases).var().item() < 0.5 * ys.var().item()
    cv = ExchangeControlVariate(hidden=128, seed=1)
    hist = cv.fit(feats, ys, bases, epochs=40, batch=1024, lr=2e-3)
    # holdout MSE (units of var(y - base)) fell during training and beats the leading-vector term alone
    assert hist[-1][1] < hist[0][1]
    assert hist[-1][1] < 0.8
    for step in range(41, 51):
        af.step(step)
    parts = EnergyParts(ham, trial, af.walkers)
    sd_plain, sd_cv, exact, sd_lin = subsample_variances(cv, parts, af.walkers, fraction=8, trials=48)
    assert sd_cv < 0.3 * sd_plain, (sd_plain, sd_cv)
    # what the network gains over the method without it (the leading-vector term alone)
    assert sd_cv < 0.9 * sd_lin, (sd_lin, sd_cv)


def test_online_refit_follows_new_walkers():
    """The estimator's refit on exact subsamples lowers the network's error on walkers it was not
    trained on (training on early walkers, evaluating 60 steps later)."""
    from ipie_b200 import AFQMC, Generic, SingleDet, synthetic
    from ipie_b200.control_variate import (ControlVariateEnergyEstimator, EnergyParts, ExchangeControlVariate,
                                           generate_training_data)

    s = synthetic.generate(40, (8, 8), 160, decay=30.0, seed=6, uhf=False, chol_scale="stable")
    ham = Generic(s.h1e, s.chol, s.ecore)
    trial = SingleDet(s.psi, (8, 8), 40)
    trial.half_rotate(ham)
    af = AFQMC.build((8, 8), ham, trial, num_walkers=256, seed=6, num_blocks=100, verbose=False, rng="device")
    af.setup_run()
    feats, ys, bases = generate_training_data(af, steps=20)
    cv = ExchangeControlVariate(hidden=64, seed=2)
    cv.fit(feats, ys, bases, epochs=20, batch=1024, lr=2e-3)
    frozen = cv.clone()
    est = ControlVariateEnergyEstimator(cv, fraction=4, seed=3, refit=True, buffer_blocks=8, refit_steps=20,
                                        refit_lr=1e-3)
    step = 21
    for _ in range(6):
        for _ in range(10):
            af.step(step)
            step += 1
        est.compute_estimator(None, af.walkers, ham, trial)
    parts = EnergyParts(ham, trial, af.walkers)
    parts.compute(af.walkers)
    y = parts.exchange_term(af.walkers)
    err_frozen = float(((frozen.predict(parts.feat, parts.base).double() - y) ** 2).mean())
    err_refit = float(((cv.predict(parts.feat, parts.base).double() - y) ** 2).mean())
    assert np.isfinite(err_refit) and err_refit < err_frozen, (err_frozen, err_refit)
