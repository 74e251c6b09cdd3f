"""The mixed-precision form (FP16 and TF32 tensor cores) against the FP64 form.

Tolerances follow the arithmetic: the force bias, VHS, orbital and exchange
products are 3-pass FP16 or TF32 (~2^-22 relative per product); walker weights and
overlaps after a few steps stay within 1e-5 of the FP64 path; the local energy,
expanded around the trial, within 1e-6 (exact at the trial itself).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import afqmc_oracle as O  # noqa: E402
from tests.test_gpu_parity import _walker_pert, dev, gpu_objects, rel  # noqa: E402

pytestmark = pytest.mark.gpu


def _system(M=64, N=8, X=128, uhf=True):
    from ipie_b200 import synthetic

    return synthetic.generate(M, (N, N), X, decay=30.0, seed=21, uhf=uhf, chol_scale="stable")


def _mixed_objects(s, W):
    from ipie_b200.propagation import PhaselessGeneric

    ham, trial, walkers, prop = gpu_objects(s, W)
    pm = PhaselessGeneric(0.005, precision="mixed")
    pm.build(ham, trial, walkers)
    return ham, trial, walkers, prop, pm


def test_mixed_force_bias_3pass():
    s = _system()
    ham, trial, walkers, prop, pm = _mixed_objects(s, 40)
    pa, pb = _walker_pert(s, 40, 3)
    walkers.phia, walkers.phib = dev(pa), dev(pb)
    trial.calc_greens_function(walkers)
    ref = trial.calc_force_bias(ham, walkers)
    from ipie_b200._lib import call, ptr, stream

    ws = pm._workspace(walkers, ham)
    out = torch.empty_like(ref)
    (ra_hi, ra_lo, ra_s), (rb_hi, rb_lo, rb_s) = pm.rpad
    call("ipie_b200_construct_force_bias_mixed", ptr(ra_hi), ptr(ra_lo), ra_s, ptr(rb_hi), ptr(rb_lo), rb_s,
         ptr(walkers.Ghalfa), ptr(walkers.Ghalfb), ptr(ws.gwork), 40, s.nchol, s.nbasis, s.nup, s.ndown, ptr(out),
         ptr(walkers.status), stream())
    assert rel(out, ref) < 1e-5
    walkers.check_status()


def test_mixed_vhs_3pass():
    s = _system()
    W = 24
    ham, trial, walkers, prop, pm = _mixed_objects(s, W)
    ws = pm._workspace(walkers, ham)
    rng = np.random.default_rng(5)
    vb = dev(0.3 * (rng.normal(size=(W, s.nchol)) + 1j * rng.normal(size=(W, s.nchol))))
    xi = dev(rng.normal(size=(W, s.nchol)))
    from ipie_b200._lib import call, ptr, stream

    xs = torch.empty(s.nchol, W, dtype=torch.complex128, device="cuda")
    call("ipie_b200_field_shift_mixed", ptr(vb), ptr(xi), ptr(pm.mf_shift_dev), W, s.nchol, pm.sqrt_dt, 1.0, ptr(xs),
         ptr(ws.xs_hi), ptr(ws.xs_lo), ptr(ws.cmf), ptr(ws.cfb), stream())
    ref = prop.construct_VHS(ham, xs)
    M = s.nbasis
    # binary16 planes x v_scale (the FP16 orbital chain's operands), then fp32 TF32 planes
    assert pm.chain16
    v = ws.v_planar
    call("ipie_b200_construct_vhs_mixed", ptr(pm.cp_hi), ptr(pm.cp_lo), ptr(ham.sym_idx_i), ptr(ham.sym_idx_j),
         M, s.nchol, ptr(ws.xs_hi), ptr(ws.xs_lo), W, pm.sqrt_dt, pm.cp_scale, 1, pm.v_scale, ptr(v[0]), ptr(v[1]),
         ptr(v[2]), ptr(v[3]), ptr(walkers.status), stream())
    got = ((v[0].double() + v[1].double()) + 1j * (v[2].double() + v[3].double()))[:, :, :M] / pm.v_scale
    assert rel(got, ref) < 1e-5
    v32 = [torch.empty(W, M, M, dtype=torch.float32, device="cuda") for _ in range(4)]
    call("ipie_b200_construct_vhs_mixed", ptr(pm.cp_hi), ptr(pm.cp_lo), ptr(ham.sym_idx_i), ptr(ham.sym_idx_j),
         M, s.nchol, ptr(ws.xs_hi), ptr(ws.xs_lo), W, pm.sqrt_dt, pm.cp_scale, 0, 0.0, ptr(v32[0]), ptr(v32[1]),
         ptr(v32[2]), ptr(v32[3]), ptr(walkers.status), stream())
    got = (v32[0].double() + v32[1].double()) + 1j * (v32[2].double() + v32[3].double())
    assert rel(got, ref) < 1e-5
    walkers.check_status()


@pytest.mark.parametrize("M,X,W,persistent", [(64, 128, 24, 0), (108, 216, 70, 1), (76, 152, 130, 0),
                                              (200, 400, 9, 1), (200, 400, 200, 0)])
def test_mixed_vhs_blocks(M, X, W, persistent):
    """The block-tiled VHS (16 x 16 pair blocks, fields as the left operand) writes the same
    binary16 planes as the packed-pair product, with the pad columns zero; M = 108 and 76 end on
    partial blocks, W = 70 and 130 on partial walker tiles."""
    from ipie_b200 import synthetic
    from ipie_b200._lib import call, ptr, stream

    s = synthetic.generate(M, (8, 8), X, decay=30.0, seed=23, uhf=True, chol_scale="stable")
    ham, trial, walkers, prop, pm = _mixed_objects(s, W)
    assert pm.chain16
    ws = pm._workspace(walkers, ham)
    rng = np.random.default_rng(7)
    vb = dev(0.3 * (rng.normal(size=(W, X)) + 1j * rng.normal(size=(W, X))))
    xi = dev(rng.normal(size=(W, X)))
    xs = torch.empty(X, W, dtype=torch.complex128, device="cuda")
    call("ipie_b200_field_shift_mixed", ptr(vb), ptr(xi), ptr(pm.mf_shift_dev), W, X, pm.sqrt_dt, 1.0, ptr(xs),
         ptr(ws.xs_hi), ptr(ws.xs_lo), ptr(ws.cmf), ptr(ws.cfb), stream())
    ref = prop.construct_VHS(ham, xs)
    Mp = (M + 7) // 8 * 8
    planes = [torch.full((W, M, Mp), float("nan"), dtype=torch.float16, device="cuda") for _ in range(4)]
    call("ipie_b200_construct_vhs_blocks", ptr(pm.cb_hi), ptr(pm.cb_lo), M, X, ptr(ws.xs_hi), ptr(ws.xs_lo), W,
         pm.sqrt_dt, pm.cp_scale, pm.v_scale, *(ptr(v) for v in planes), persistent, ptr(walkers.status), stream())
    old = [torch.zeros(W, M, Mp, dtype=torch.float16, device="cuda") for _ in range(4)]
    call("ipie_b200_construct_vhs_mixed", ptr(pm.cp_hi), ptr(pm.cp_lo), ptr(ham.sym_idx_i), ptr(ham.sym_idx_j), M, X,
         ptr(ws.xs_hi), ptr(ws.xs_lo), W, pm.sqrt_dt, pm.cp_scale, 1, pm.v_scale, *(ptr(v) for v in old),
         ptr(walkers.status), stream())
    for k in range(4):
        assert not torch.isnan(planes[k]).any(), k  # every element written, pad columns included
        assert torch.count_nonzero(planes[k][:, :, M:]) == 0
    got = ((planes[0].double() + planes[1].double()) + 1j * (planes[2].double() + planes[3].double()))[:, :, :M]
    assert rel(got / pm.v_scale, ref) < 1e-5
    prev = ((old[0].double() + old[1].double()) + 1j * (old[2].double() + old[3].double()))[:, :, :M]
    # the same FP32 sums up to the order of the tensor cores' additions
    assert rel(got, prev) < 1e-6
    walkers.check_status()


@pytest.mark.parametrize("M,N,W", [(64, 8, 6), (200, 32, 6), (108, 15, 6), (128, 16, 5), (64, 4, 300),
                                   (200, 13, 5), (256, 24, 4), (260, 4, 3)])
def test_mixed_orbital_update_3pass(M, N, W):
    """One-launch chain (M <= 256: one or two 128-row tiles, orbital groups partly or wholly past N;
    W = 300 > SM count exercises the persistent walker loop) and the per-term launches (M = 260)
    against the oracle's one-body, Taylor-6, one-body."""
    from ipie_b200 import synthetic
    from ipie_b200._lib import call, ptr, stream

    s = synthetic.generate(M, (N, N), 2 * M, decay=30.0, seed=9, uhf=True, chol_scale="stable")
    ham, trial, walkers, prop, pm = _mixed_objects(s, W)
    pa, _ = _walker_pert(s, W, 4)
    rng = np.random.default_rng(2)
    xs = dev(rng.normal(size=(s.nchol, W)) + 0.2j * rng.normal(size=(s.nchol, W)))
    vhs = prop.construct_VHS(ham, xs)
    pa_d = dev(pa)  # keep the input alive until the kernels have run
    E = prop.expH1[0].real
    ref = np.einsum("pq,wqn->wpn", E, O.apply_exponential(np.einsum("pq,wqn->wpn", E, pa), vhs.cpu().numpy(), 6))
    planes = []
    for part in (vhs.real.contiguous(), vhs.imag.contiguous()):
        hi = torch.empty(part.shape, dtype=torch.float32, device="cuda")
        lo = torch.empty_like(hi)
        call("ipie_b200_split_tf32", ptr(part), ptr(hi), ptr(lo), part.numel(), stream())
        planes += [hi, lo]
    out = torch.empty_like(pa_d)
    work = torch.empty(4 * W * 2 * N * M, dtype=torch.float32, device="cuda")
    call("ipie_b200_propagate_orbitals_mixed", ptr(pm.e_hi[0]), ptr(pm.e_lo[0]), pm.lde, ptr(planes[0]), ptr(planes[1]),
         ptr(planes[2]), ptr(planes[3]), ptr(pa_d), ptr(out), ptr(work), W, M, N, 6, ptr(walkers.status), stream())
    assert rel(out, ref) < 1e-5
    walkers.check_status()


def _split16_padded(x, scale):
    """(W, M, M) real -> binary16 head/remainder (W, M, Mp) of x * scale, Mp = M rounded up to 8."""
    from ipie_b200._lib import call, ptr, stream

    W, M, _ = x.shape
    Mp = (M + 7) // 8 * 8
    xp = torch.zeros(W, M, Mp, dtype=torch.float64, device="cuda")
    xp[:, :, :M] = x
    hi = torch.empty(W, M, Mp, dtype=torch.float16, device="cuda")
    lo = torch.empty_like(hi)
    call("ipie_b200_split_f16", ptr(xp), ptr(hi), ptr(lo), xp.numel(), scale, stream())
    return hi, lo


@pytest.mark.parametrize("M,N,W,vmag", [(64, 8, 6, 1.0), (200, 32, 6, 1.0), (108, 15, 6, 1.0), (128, 16, 5, 1.0),
                                        (64, 4, 300, 1.0), (200, 13, 5, 1.0), (256, 24, 4, 1.0), (76, 10, 4, 1.0),
                                        (200, 32, 4, 1e-3), (200, 32, 4, 30.0)])
def test_mixed_orbital_chain16(M, N, W, vmag):
    """The FP16 orbital chain (one or two 128-row tiles, orbital groups partly or wholly past N,
    M not a multiple of 8, W = 300 > SM count for the persistent walker loop) against the oracle's
    one-body, Taylor-6, one-body; vmag scales the VHS by 1e-3 and 30 so that the Taylor terms
    span many binades (each term's B carries its own scale)."""
    import math

    from ipie_b200 import synthetic
    from ipie_b200._lib import call, ptr, stream

    s = synthetic.generate(M, (N, N), 2 * M, decay=30.0, seed=9, uhf=True, chol_scale="stable")
    ham, trial, walkers, prop, pm = _mixed_objects(s, W)
    assert pm.chain16
    pa, _ = _walker_pert(s, W, 4)
    rng = np.random.default_rng(2)
    xs = dev(rng.normal(size=(s.nchol, W)) + 0.2j * rng.normal(size=(s.nchol, W)))
    vhs = prop.construct_VHS(ham, xs) * vmag
    pa_d = dev(pa)
    E = prop.expH1[0].real
    ref = np.einsum("pq,wqn->wpn", E, O.apply_exponential(np.einsum("pq,wqn->wpn", E, pa), vhs.cpu().numpy(), 6))
    vmax = max(vhs.real.abs().max().item(), vhs.imag.abs().max().item())
    vs = 2.0 ** (14 - math.frexp(vmax)[1])
    vr = _split16_padded(vhs.real.contiguous(), vs)
    vi = _split16_padded(vhs.imag.contiguous(), vs)
    out = torch.empty_like(pa_d)
    call("ipie_b200_propagate_orbitals_mixed16", ptr(pm.e16_hi[0]), ptr(pm.e16_lo[0]), pm.e_scale, ptr(vr[0]),
         ptr(vr[1]), ptr(vi[0]), ptr(vi[1]), vs, ptr(pa_d), ptr(out), W, M, N, 6, ptr(walkers.status), stream())
    assert rel(out, ref) < 1e-5
    walkers.check_status()


def test_mixed_steps_track_fp64():
    """Three steps with identical draws: the mixed form stays within 1e-5 of the FP64 form."""
    s = _system(M=76, N=10, X=200, uhf=False)
    W = 32
    runs = {}
    for precision in ("fp64", "mixed"):
        from ipie_b200 import Generic, SingleDet, UHFWalkers
        from ipie_b200.propagation import PhaselessGeneric

        ham = Generic(s.h1e, s.chol, s.ecore)
        trial = SingleDet(s.psi, (s.nup, s.ndown), s.nbasis)
        trial.half_rotate(ham)
        walkers = UHFWalkers(s.init, s.nup, s.ndown, s.nbasis, W)
        walkers.build(trial)
        walkers.enable_spin_alias()
        prop = PhaselessGeneric(0.005, precision=precision)
        prop.build(ham, trial, walkers)
        for step in range(3):
            np.random.seed(70 + step)
            prop.propagate_walkers(walkers, ham, trial, -1.0 if step else 0.0)
        walkers.check_status()
        runs[precision] = (walkers.weight.cpu().numpy(), walkers.ovlp.cpu().numpy(), walkers.phia.cpu().numpy())
    a, b = runs["mixed"], runs["fp64"]
    assert rel(a[0], b[0]) < 1e-5
    assert rel(a[1], b[1]) < 1e-5
    assert rel(a[2], b[2]) < 1e-5


@pytest.mark.parametrize("uhf,N", [(False, 10), (True, 15), (False, 32)])
def test_mixed_local_energy(uhf, N):
    """Exchange in 3-pass TF32 (Coulomb in FP64) against the FP64 local energy."""
    from ipie_b200 import synthetic
    from ipie_b200.estimators import local_energy_mixed, local_energy_single_det_uhf_batch

    s = synthetic.generate(76, (N, N), 200, decay=30.0, seed=17, uhf=uhf, chol_scale="stable")
    W = 40
    ham, trial, walkers, prop = gpu_objects(s, W)
    pa, pb = _walker_pert(s, W, 6)
    walkers.phia, walkers.phib = dev(pa), dev(pb)
    trial.calc_greens_function(walkers)
    ref = local_energy_single_det_uhf_batch(None, ham, walkers, trial)
    # these walkers are random perturbations far from the trial: the expansion gains little here
    got = local_energy_mixed(None, ham, walkers, trial)
    assert rel(got, ref) < 1e-6
    plain = local_energy_mixed(None, ham, walkers, trial, reference=False)
    assert rel(plain, ref) < 2e-6
    walkers.check_status()


def test_mixed_local_energy_is_exact_at_the_trial():
    """Expanded around the trial, the tensor cores see G - G_T = 0 there: FP64 energies result."""
    from ipie_b200 import synthetic
    from ipie_b200.estimators import local_energy_mixed, local_energy_single_det_uhf_batch

    s = synthetic.generate(76, (10, 10), 200, decay=30.0, seed=17, uhf=False, chol_scale="stable")
    ham, trial, walkers, prop = gpu_objects(s, 8)
    trial.calc_greens_function(walkers)
    ref = local_energy_single_det_uhf_batch(None, ham, walkers, trial)
    got = local_energy_mixed(None, ham, walkers, trial)
    assert rel(got, ref) < 1e-12


@pytest.mark.parametrize("uhf,N", [(False, 10), (True, 15)])
def test_mixed_exchange_terms_match_fp64(uhf, N):
    """ipie_b200_exchange_mixed (with and without the trial expansion, full and leading-vector
    sums, on a walker subsample) against the FP64 exchange kernel."""
    from ipie_b200 import synthetic
    from ipie_b200.control_variate import EnergyParts

    s = synthetic.generate(76, (N, N), 200, decay=30.0, seed=21, uhf=uhf, chol_scale="stable")
    W = 24
    ham, trial, walkers, prop = gpu_objects(s, W)
    pa, pb = _walker_pert(s, W, 8)
    walkers.phia, walkers.phib = dev(0.3 * pa + 0.7 * s.init[:, :N][None]), dev(0.3 * pb + 0.7 * s.init[:, N:][None])
    trial.calc_greens_function(walkers)
    p64 = EnergyParts(ham, trial, walkers)
    pmx = EnergyParts(ham, trial, walkers, precision="mixed")
    idx = torch.tensor([1, 4, 5, 17, 23], dtype=torch.int32, device="cuda")
    # the leading-vector sum (a control-variate input) runs without the trial expansion: plain
    # 3-pass accuracy; the full sums are expanded around the trial
    for kw, tol in (({}, 1e-6), ({"nchol": 25}, 5e-6), ({"idx": idx}, 1e-6)):
        ref = p64.exchange_term(walkers, **kw)
        got = pmx.exchange_term(walkers, **kw)
        assert rel(got, ref) < tol, kw
    walkers.check_status()
