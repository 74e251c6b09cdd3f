"""Phaseless propagator for generic real-Cholesky Hamiltonians on B200.

Mirror of ipie's ``PhaselessGeneric`` / ``PhaselessBase``
(``propagation/phaseless_generic.py:28-97``, ``propagation/phaseless_base.py:242-385``):
``build``, ``propagate_walkers``, ``propagate_walkers_one_body``,
``propagate_walkers_two_body``, ``construct_VHS``, ``apply_VHS`` and
``update_weight`` keep ipie's names, arguments and order of operations.

Auxiliary fields: ``rng="numpy"`` (default) draws them exactly as ipie does,
``numpy.random.normal(0, 1, X*W).reshape(W, X)`` from numpy's global stream,
so a run fed the same seed consumes the same draws; ``rng="device"`` draws
them on the GPU (Philox4x32-10), which keeps a step free of host work;
``rng="host"`` takes caller-supplied (W, X) host arrays from the iterator
``propagator.host_fields`` and uploads one per step (the next step's array on a copy stream
while the current step computes).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg
import torch

from ._lib import call, lib, ptr, stream
from .trial import force_bias_into, greens_function_into, overlap_into

C128 = torch.complex128
F64 = torch.float64


def construct_mean_field_shift(hamiltonian, trial):
    """``mf = 1j L^T Re(G_a+G_b) - L^T Im(G_a+G_b)`` (ipie ``phaseless_base.py:153-172``); for a
    complex Cholesky ``mf = [1j A^T g ; 1j B^T g]`` (``:199-218``)."""
    if getattr(trial, "ghf", False):
        # Gaa + Gbb of the GHF trial's (2M, 2M) density (ipie phaseless_base.py:175-196)
        M = hamiltonian.nbasis
        g = (trial.Gfull[:M, :M] + trial.Gfull[M:, M:]).ravel()
    else:
        g = (trial.G[0] + trial.G[1]).ravel()
    if getattr(hamiltonian, "complex_chol", False):
        return np.concatenate([1.0j * (hamiltonian.A.T @ g), 1.0j * (hamiltonian.B.T @ g)])
    return 1.0j * (hamiltonian.chol.T @ g.real) - hamiltonian.chol.T @ g.imag


def construct_one_body_propagator(hamiltonian, mf_shift, dt):
    """``expH1_s = expm(-dt/2 (h1e_mod_s - 1j L.mf))`` (ipie ``phaseless_base.py:27-74``); for a
    complex Cholesky the shift is ``1j (A mf[:X] + B mf[X:])`` (``:78-106``)."""
    M = hamiltonian.nbasis
    if getattr(hamiltonian, "complex_chol", False):
        X = hamiltonian.nchol
        shift = 1.0j * np.einsum("mx,x->m", hamiltonian.A, mf_shift[:X]).reshape(M, M)
        shift = shift + 1.0j * np.einsum("mx,x->m", hamiltonian.B, mf_shift[X:]).reshape(M, M)
    else:
        shift = 1.0j * np.einsum("mx,x->m", hamiltonian.chol, mf_shift).reshape(M, M)
    H1 = hamiltonian.h1e_mod - np.array([shift, shift])
    return np.array([scipy.linalg.expm(-0.5 * dt * H1[0]), scipy.linalg.expm(-0.5 * dt * H1[1])])


class PhaseTimer:
    """CUDA-event timing of named step phases on the launching (current) stream."""

    def __init__(self):
        self.events = {}

    def start(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.events.setdefault(name, []).append([e, None])

    def stop(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.events[name][-1][1] = e

    def summary(self):
        """{phase: (launch groups, total ms)} after a device synchronize."""
        out = {}
        for k, v in self.events.items():
            out[k] = (len(v), sum(a.elapsed_time(b) for a, b in v))
        return out


class _NoTimer:
    def start(self, name):
        pass

    def stop(self, name):
        pass


class Workspace:
    """Scratch buffers of one walker batch, allocated once."""

    def __init__(self, W, M, na, nb, X, device):
        self.W, self.M, self.na, self.nb, self.X = W, M, na, nb, X
        dev = device
        self.phia_tmp = torch.empty(W, M, na, dtype=C128, device=dev)
        self.phib_tmp = torch.empty(W, M, nb, dtype=C128, device=dev)
        nmax = max(na, nb)
        self.taylor = torch.empty(2 * W * M * nmax, dtype=C128, device=dev)
        self.vbias = torch.empty(W, X, dtype=C128, device=dev)
        self.xi = torch.empty(W, X, dtype=F64, device=dev)
        self.xshifted = torch.empty(X, W, dtype=C128, device=dev)
        self.cmf = torch.empty(W, dtype=C128, device=dev)
        self.cfb = torch.empty(W, dtype=C128, device=dev)
        self.vhs = torch.empty(W, M, M, dtype=C128, device=dev)
        self.ovlp_new = torch.empty(W, dtype=C128, device=dev)
        self.eshift = torch.zeros(1, dtype=F64, device=dev)
        self.wbound = torch.full((1,), -1.0, dtype=F64, device=dev)
        self.xi_host = torch.empty(W, X, dtype=F64).pin_memory() if torch.cuda.is_available() else None
        self.xi_copied = torch.cuda.Event() if torch.cuda.is_available() else None
        self.dev = dev

    def add_mixed(self, chain16):
        """Buffers of the mixed form; ``chain16``: the orbital update runs as the FP16 chain
        (binary16 VHS planes), otherwise as TF32 products (fp32 planes and work)."""
        W, M, X, N = self.W, self.M, self.X, max(self.na, self.nb)
        f32, f16, dev = torch.float32, torch.float16, self.dev
        self.gwork = torch.empty(2 * W * 2 * 32 * M, dtype=f32, device=dev)
        Xp = (X + 7) // 8 * 8  # binary16 rows padded to 16 bytes
        # head and remainder in one allocation: the VHS product loads both tiles with one copy
        self.xs_hilo = torch.empty(2, W, 2, Xp, dtype=f16, device=dev)
        self.xs_hi, self.xs_lo = self.xs_hilo[0], self.xs_hilo[1]
        if chain16:
            Mp = (M + 7) // 8 * 8
            # re_hi, re_lo, im_hi, im_lo in one allocation: the chain loads the last columns of all
            # four planes of a walker with one copy
            self.v_planar = list(torch.empty(4, W, M, Mp, dtype=f16, device=dev).unbind(0))
            self.orb_work = torch.empty(0, dtype=f32, device=dev)
        else:
            self.v_planar = [torch.empty(W, M, M, dtype=f32, device=dev) for _ in range(4)]
            self.orb_work = torch.empty(4 * W * 2 * N * M, dtype=f32, device=dev)


class PhaselessGeneric:
    def __init__(self, time_step, exp_nmax=6, verbose=False, rng="numpy", seed=7, precision="fp64"):
        self.dt = time_step
        self.sqrt_dt = self.dt ** 0.5
        self.isqrt_dt = 1j * self.sqrt_dt
        self.exp_nmax = exp_nmax
        self.ebound = (2.0 / self.dt) ** 0.5
        self.fbbound = 1.0
        self.verbose = verbose
        self.rng = rng
        self.rng_seed = seed
        self.rng_counter = 0
        self.rng_counter_dev = None  # device copy of the counter block of rng="device"
        self.vbias = None
        self.ws = None
        self.timer = _NoTimer()
        self.fused = True  # one launch per spin for one-body + exp(VHS) + one-body
        self.vhs_flags = 1  # block-tiled mixed VHS: bit 0 = persistent CTAs (1.41 vs 1.50 ms at c2)
        # "fp64": the plain form (ipie's arithmetic); "mixed": force bias, VHS and the orbital
        # update as 3-pass TF32 tensor-core products, FP64 everywhere else
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
        self.precision = precision

    # ------------------------------------------------------------------ set-up
    def build(self, hamiltonian, trial=None, walkers=None, mpi_handler=None, verbose=False):
        """Mean-field shift and one-body propagator (ipie ``phaseless_base.py:256-272``)."""
        self.mf_shift = construct_mean_field_shift(hamiltonian, trial)
        self.expH1 = construct_one_body_propagator(hamiltonian, self.mf_shift, self.dt)
        dev = trial.device
        self.device = dev
        self.mf_shift_dev = torch.from_numpy(np.ascontiguousarray(self.mf_shift.astype(np.complex128))).to(dev)
        self.expH1_complex = bool(np.iscomplexobj(self.expH1) and np.abs(self.expH1.imag).max() > 0)
        e = self.expH1.astype(np.complex128) if self.expH1_complex else self.expH1.real.astype(np.float64)
        self.expH1_dev = torch.from_numpy(np.ascontiguousarray(e)).to(dev)
        # rows padded to an even length (16-byte aligned) for the fused orbital kernel
        M = hamiltonian.nbasis
        self.lda_e = M + (M & 1)
        if not self.expH1_complex:
            ep = np.zeros((2, M, self.lda_e))
            ep[:, :, :M] = self.expH1.real
            self.expH1_pad = torch.from_numpy(ep).to(dev)
        self.spin_symmetric = bool(np.array_equal(self.expH1[0], self.expH1[1]))
        if self.precision == "mixed":
            if getattr(trial, "multidet", False):
                raise NotImplementedError("the particle-hole trial propagates in FP64 (precision='fp64')")
            self._mixed_setup(hamiltonian, trial)
        if walkers is not None:
            self._workspace(walkers, hamiltonian)

    def _workspace(self, walkers, hamiltonian):
        W, M, X = walkers.nwalkers, walkers.nbasis, hamiltonian.nfields
        na, nb = walkers.nup, walkers.ndown
        ghf = getattr(walkers, "ghf", False)
        if ghf:
            # the propagated spin-diagonal blocks of the (2M, N) determinants
            M, na, nb = walkers.nbasis_spatial, walkers.nalpha, walkers.nbeta
        ws = self.ws
        if ws is None or (ws.W, ws.M, ws.na, ws.nb, ws.X) != (W, M, na, nb, X):
            self.ws = Workspace(W, M, na, nb, X, walkers.device)
            if ghf:
                self.ws.ghf_pa = torch.empty(W, M, na, dtype=C128, device=walkers.device)
                self.ws.ghf_pb = torch.empty(W, M, nb, dtype=C128, device=walkers.device)
            if self.precision == "mixed":
                self.ws.add_mixed(self.chain16)
        return self.ws

    def _mixed_setup(self, hamiltonian, trial):
        """Operands of the mixed form, prepared once: packed Cholesky FP16 hi/lo, half-rotated
        Cholesky FP16 hi/lo (padded), expH1 - I as FP16 hi/lo (the FP16 orbital chain, which
        takes blocks of M <= 256 and N <= 32) and as TF32 hi/lo (the per-term products)."""
        M, X = hamiltonian.nbasis, hamiltonian.nchol
        if getattr(hamiltonian, "complex_chol", False):
            raise NotImplementedError("the mixed form takes real Cholesky Hamiltonians (precision='fp64' for complex ones)")
        if M % 4 or X % 4 or self.expH1_complex:
            raise NotImplementedError("the mixed form needs nbasis and nchol multiples of 4 and a real expH1")
        dev = self.device
        P = hamiltonian.npacked
        f32 = torch.float32
        # packed Cholesky as the FP16 operand of the VHS product, scaled by a power of two that
        # puts its largest entry near 2^14; rows padded to a multiple of 8 halves
        Xp = (X + 7) // 8 * 8
        cmax = float(hamiltonian.chol_packed.abs().max().item()) or 1.0
        self.cp_scale = 2.0 ** (14 - int(np.ceil(np.log2(cmax))))
        cp = hamiltonian.chol_packed
        if Xp != X:
            cp = torch.zeros(P, Xp, dtype=cp.dtype, device=dev)
            cp[:, :X] = hamiltonian.chol_packed
        self.cp_hi = torch.empty(P, Xp, dtype=torch.float16, device=dev)
        self.cp_lo = torch.empty(P, Xp, dtype=torch.float16, device=dev)
        call("ipie_b200_split_f16", ptr(cp), ptr(self.cp_hi), ptr(self.cp_lo), P * Xp, self.cp_scale, stream())
        del cp
        from .estimators import _mixed_energy_operands

        # padded half-rotated Cholesky FP16 head/remainder: force bias and energy share it
        self.rpad = _mixed_energy_operands(trial, hamiltonian)
        self.lde = M
        # the one-body factor enters the mixed orbital update as E - I (the identity is added in FP64)
        e = torch.from_numpy(np.ascontiguousarray(self.expH1.real - np.eye(M)[None])).to(dev)
        self.chain16 = all(lib().ipie_b200_orbital_chain16_fits(M, n) == 1
                           for n in (trial.nalpha, trial.nbeta) if n > 0)
        if self.chain16:
            # binary16 operands of the orbital chain, rows padded to 8 halves: E - I with one
            # power-of-two scale, and the scale of the VHS planes from a bound on their entries,
            # |V| <= sqrt(dt) max_p sum_x |L_px| max|x_shifted| with |x_shifted| < 9 + the force-
            # bias cap (the normal draws stay below 9), so the planes never reach 2^15
            Mp = (M + 7) // 8 * 8
            ep = torch.zeros(2, M, Mp, dtype=torch.float64, device=dev)
            ep[:, :, :M] = e
            emax = float(e.abs().max().item())
            self.e_scale = 2.0 ** (14 - math.frexp(emax)[1]) if emax > 0 else 1.0
            self.e16_hi = torch.empty(2, M, Mp, dtype=torch.float16, device=dev)
            self.e16_lo = torch.empty(2, M, Mp, dtype=torch.float16, device=dev)
            call("ipie_b200_split_f16", ptr(ep), ptr(self.e16_hi), ptr(self.e16_lo), ep.numel(), self.e_scale, stream())
            l1 = float(hamiltonian.chol_packed.abs().sum(1).max().item())
            vbound = self.sqrt_dt * l1 * (9.0 + float(self.fbbound))
            self.v_scale = 2.0 ** (14 - math.frexp(vbound)[1]) if vbound > 0 else 1.0
            # the chain's VHS planes come from the block-tiled product (16 x 16 pair blocks)
            self.cb_hi, self.cb_lo = self._vhs_block_operand(hamiltonian, Xp)
        self.e_hi = torch.empty(2, M, M, dtype=f32, device=dev)
        self.e_lo = torch.empty(2, M, M, dtype=f32, device=dev)
        call("ipie_b200_split_tf32", ptr(e), ptr(self.e_hi), ptr(self.e_lo), e.numel(), stream())

    def _vhs_block_operand(self, hamiltonian, Xp):
        """Cholesky rows of the block-tiled VHS product: for every 16 x 16 block (I <= J) of
        orbital pairs, row-major, the packed row of (16 I + a, 16 J + b) (zeros past M), x cp_scale
        in binary16 head/remainder (``ipie_b200_vhs_block_pack``)."""
        from .hamiltonian import tiled_triu_indices

        M = hamiltonian.nbasis
        ti, tj = tiled_triu_indices(M)
        pidx = np.full((M + 16, M + 16), -1, dtype=np.int32)
        pidx[ti, tj] = np.arange(len(ti), dtype=np.int32)
        pidx[tj, ti] = np.arange(len(ti), dtype=np.int32)
        nb = (M + 15) // 16
        assert lib().ipie_b200_vhs_blocks(M) == nb * (nb + 1) // 2
        a = np.arange(16)
        rows = [pidx[16 * I + a[:, None], 16 * J + a[None, :]].ravel() for I in range(nb) for J in range(I, nb)]
        rowmap = torch.from_numpy(np.ascontiguousarray(np.concatenate(rows))).to(self.device)
        R = rowmap.numel()
        hilo = torch.empty(2, R, Xp, dtype=torch.float16, device=self.device)  # one allocation (see add_mixed)
        hi, lo = hilo[0], hilo[1]
        call("ipie_b200_vhs_block_pack", ptr(hamiltonian.chol_packed), ptr(rowmap), M, hamiltonian.nchol,
             self.cp_scale, ptr(hi), ptr(lo), stream())
        torch.cuda.current_stream().synchronize()
        return hi, lo

    # ------------------------------------------------------------- the step
    def propagate_walkers_one_body(self, walkers):
        """``phi_s <- expH1_s phi_s`` (ipie ``phaseless_base.py:274-280``)."""
        ws = self.ws
        self.timer.start("one_body")
        for s, (phi, tmp, n) in enumerate(((walkers.phia, ws.phia_tmp, walkers.nup), (walkers.phib, ws.phib_tmp, walkers.ndown))):
            if n == 0 or (s == 1 and walkers.spin_alias):
                continue
            call("ipie_b200_propagate_one_body", ptr(self.expH1_dev[s]), int(self.expH1_complex), ptr(phi), ptr(tmp),
                 walkers.nwalkers, walkers.nbasis, n, stream())
        self.timer.stop("one_body")
        walkers.phia, ws.phia_tmp = ws.phia_tmp, walkers.phia
        if walkers.ndown > 0 and not walkers.spin_alias:
            walkers.phib, ws.phib_tmp = ws.phib_tmp, walkers.phib
        walkers.sync_alias()

    def draw_fields(self, walkers, hamiltonian):
        """N(0,1) auxiliary fields (W, nfields) into the workspace (ipie ``phaseless_base.py:296-298``)."""
        ws = self.ws
        W, X = walkers.nwalkers, hamiltonian.nfields
        if self.rng == "numpy":
            xi = np.random.normal(0.0, 1.0, X * W).reshape(W, X)
            ws.xi_copied.synchronize()  # the previous step's upload has left the pinned buffer
            ws.xi_host.numpy()[...] = xi
            ws.xi.copy_(ws.xi_host, non_blocking=True)
            ws.xi_copied.record()
        elif self.rng == "host":
            return self._host_fields(ws)
        else:
            # the counter lives on the device so that a step captured in a CUDA graph draws a
            # new block on every replay (same sequence as counting on the host)
            if self.rng_counter_dev is None:
                self.rng_counter_dev = torch.full((1,), self.rng_counter, dtype=torch.int64, device=ws.xi.device)
            call("ipie_b200_normal_fill_dev", ptr(ws.xi), W * X, self.rng_seed, ptr(self.rng_counter_dev), stream())
            self.rng_counter += 1
        return ws.xi

    def _host_fields(self, ws):
        """This step's caller-supplied fields, uploaded while the previous step computed: each call
        returns the buffer filled for it and starts the next array's copy into the other buffer on
        a copy stream (after the compute stream has consumed that buffer), so the host-to-device
        transfer overlaps the step instead of preceding it."""
        cur = torch.cuda.current_stream()
        src = self.host_fields
        pending = getattr(ws, "xi_pending", None)
        if pending is not None and pending[0] is not src:
            # the caller replaced the iterator: the array prefetched from the old one is not this
            # step's (the copy still lands in a buffer that nothing reads before it is rewritten)
            cur.wait_event(pending[2])
            pending = None
        if pending is None:
            ws.xi.copy_(next(src), non_blocking=True)  # (W, X) float64, pinned host memory
            buf = ws.xi
        else:
            _, buf, ready = pending
            cur.wait_event(ready)
        nxt = next(src, None)
        if nxt is None:
            ws.xi_pending = None
            return buf
        if getattr(ws, "xi_alt", None) is None:
            ws.xi_alt = torch.empty_like(ws.xi)
            ws.copy_stream = torch.cuda.Stream(device=ws.xi.device)
        other = ws.xi_alt if buf is ws.xi else ws.xi
        free = torch.cuda.Event()
        free.record(cur)  # the previous step's field shift, which read `other`, is behind this point
        ws.copy_stream.wait_event(free)
        with torch.cuda.stream(ws.copy_stream):
            other.copy_(nxt, non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(ws.copy_stream)
        ws.xi_pending = (src, other, ready)
        return buf

    def propagate_walkers_two_body(self, walkers, hamiltonian, trial):
        """Force bias, shifted fields, VHS and exp(VHS) (ipie ``phaseless_base.py:282-310``)."""
        ws = self.ws
        W, X = walkers.nwalkers, hamiltonian.nfields
        self.timer.start("force_bias")
        force_bias_into(hamiltonian, walkers, trial, ws.vbias)
        self.timer.stop("force_bias")
        self.vbias = ws.vbias
        self.timer.start("rng")
        xi = self.draw_fields(walkers, hamiltonian)
        self.timer.stop("rng")
        self.timer.start("field_shift")
        call("ipie_b200_field_shift", ptr(ws.vbias), ptr(xi), ptr(self.mf_shift_dev), W, X, self.sqrt_dt, self.fbbound,
             ptr(ws.xshifted), ptr(ws.cmf), ptr(ws.cfb), stream())
        self.timer.stop("field_shift")
        self.apply_VHS(walkers, hamiltonian, ws.xshifted)
        return ws.cmf, ws.cfb

    def construct_VHS(self, hamiltonian, xshifted, out=None):
        """``VHS = i sqrt(dt) L . xshifted`` unpacked to (W, M, M) (ipie ``phaseless_generic.py:66-97``)."""
        W = xshifted.shape[-1]
        M = hamiltonian.nbasis
        if out is None:
            out = torch.empty(W, M, M, dtype=C128, device=xshifted.device)
        if getattr(hamiltonian, "complex_chol", False):
            # V = i sqrt(dt) (A xs[:X] + B xs[X:]) (ipie phaseless_generic.py:99-111)
            call("ipie_b200_construct_vhs_complex", ptr(hamiltonian.c_re), ptr(hamiltonian.c_im), M,
                 hamiltonian.nfields, ptr(xshifted.contiguous()), W, self.sqrt_dt, ptr(out), stream())
            return out
        call("ipie_b200_construct_vhs", ptr(hamiltonian.chol_packed), ptr(hamiltonian.sym_idx_i),
             ptr(hamiltonian.sym_idx_j), M, hamiltonian.nchol, ptr(xshifted.contiguous()), W, self.sqrt_dt, ptr(out),
             stream())
        return out

    def apply_VHS(self, walkers, hamiltonian, xshifted):
        """Build VHS and apply exp(VHS) to both spin blocks (ipie ``phaseless_generic.py:35-58``)."""
        assert walkers.nwalkers == xshifted.shape[-1]
        ws = self.ws
        self.timer.start("vhs")
        vhs = self.construct_VHS(hamiltonian, xshifted, out=ws.vhs)
        self.timer.stop("vhs")
        self.timer.start("taylor")
        for phi_name, tmp_name, n in (("phia", "phia_tmp", walkers.nup), ("phib", "phib_tmp", walkers.ndown)):
            if n == 0 or (phi_name == "phib" and walkers.spin_alias):
                continue
            phi, tmp = getattr(walkers, phi_name), getattr(ws, tmp_name)
            call("ipie_b200_apply_exponential_batch", ptr(vhs), ptr(phi), ptr(tmp), ptr(ws.taylor), walkers.nwalkers,
                 walkers.nbasis, n, self.exp_nmax, stream())
            setattr(walkers, phi_name, tmp)
            setattr(ws, tmp_name, phi)
        walkers.sync_alias()
        self.timer.stop("taylor")

    def propagate_walkers(self, walkers, hamiltonian, trial, eshift):
        """One phaseless step (ipie ``phaseless_base.py:312-338``).

        The two one-body half steps and exp(VHS) run as one fused launch per spin
        block (``ipie_b200_propagate_orbitals``); the force bias reads the Green's
        function of the step's starting orbitals, as in ipie, so moving the first
        one-body factor after it changes nothing.
        """
        if getattr(walkers, "ghf", False):
            return self._propagate_ghf(walkers, hamiltonian, trial, eshift)
        ws = self._workspace(walkers, hamiltonian)
        # The step's starting Green's function and overlap: the previous step ended with those of
        # the current orbitals (reortho and pair branch keep them consistent), so they are only
        # recomputed when the orbitals were replaced.  walkers.ovlp is overwritten by update_weight.
        # (a particle-hole trial's full Green's functions do not travel with population control's
        # copies, so they are recomputed every step)
        if not walkers.gf_current(trial) or getattr(trial, "multidet", False):
            self.timer.start("greens_function")
            greens_function_into(walkers, trial, walkers.ovlp)
            self.timer.stop("greens_function")
        walkers.invalidate_gf()  # the orbitals change below
        if self.precision == "mixed":
            cmf, cfb = self._mixed_two_body(walkers, hamiltonian, trial)
        elif not self.fused_ok(walkers):
            self.propagate_walkers_one_body(walkers)
            cmf, cfb = self.propagate_walkers_two_body(walkers, hamiltonian, trial)
            self.propagate_walkers_one_body(walkers)
        else:
            W, X = walkers.nwalkers, hamiltonian.nfields
            self.timer.start("force_bias")
            force_bias_into(hamiltonian, walkers, trial, ws.vbias)
            self.timer.stop("force_bias")
            self.vbias = ws.vbias
            self.timer.start("rng")
            xi = self.draw_fields(walkers, hamiltonian)
            self.timer.stop("rng")
            self.timer.start("field_shift")
            call("ipie_b200_field_shift", ptr(ws.vbias), ptr(xi), ptr(self.mf_shift_dev), W, X, self.sqrt_dt,
                 self.fbbound, ptr(ws.xshifted), ptr(ws.cmf), ptr(ws.cfb), stream())
            self.timer.stop("field_shift")
            self.timer.start("vhs")
            self.construct_VHS(hamiltonian, ws.xshifted, out=ws.vhs)
            self.timer.stop("vhs")
            self.timer.start("orbitals")
            for s_, (phi_name, tmp_name, n) in enumerate((("phia", "phia_tmp", walkers.nup),
                                                           ("phib", "phib_tmp", walkers.ndown))):
                if n == 0 or (s_ == 1 and walkers.spin_alias):
                    continue
                phi, tmp = getattr(walkers, phi_name), getattr(ws, tmp_name)
                call("ipie_b200_propagate_orbitals", ptr(ws.vhs), ptr(self.expH1_pad[s_]), self.lda_e, ptr(phi),
                     ptr(tmp), W, walkers.nbasis, n, self.exp_nmax, 1, 1, stream())
                setattr(walkers, phi_name, tmp)
                setattr(ws, tmp_name, phi)
            walkers.sync_alias()
            self.timer.stop("orbitals")
            cmf, cfb = ws.cmf, ws.cfb
        # Green's function of the new orbitals: its overlap is ovlp_new (ipie's calc_overlap) and its
        # Ghalf is the next step's (ipie recomputes it at the next step's start)
        self.timer.start("greens_function")
        greens_function_into(walkers, trial, ws.ovlp_new)
        self.timer.stop("greens_function")
        walkers.mark_gf_current(trial)
        self.update_weight(walkers, walkers.ovlp, ws.ovlp_new, cfb, cmf, eshift)

    def _propagate_ghf(self, walkers, hamiltonian, trial, eshift):
        """One step of GHF walkers (ipie ``phaseless_base.py:312-338`` with its GHF dispatches):
        Green's function and force bias of the whole (2M, N) determinants, one-body factors and
        exp(VHS) on their spin-diagonal blocks only (ipie's ``phia``/``phib`` views), copied out
        and back by ``ipie_b200_ghf_blocks``."""
        if self.precision == "mixed":
            raise NotImplementedError("GHF walkers run in the FP64 form")
        ws = self._workspace(walkers, hamiltonian)
        if not walkers.gf_current(trial):
            greens_function_into(walkers, trial, walkers.ovlp)
        walkers.invalidate_gf()
        W, X, M = walkers.nwalkers, hamiltonian.nfields, hamiltonian.nbasis
        na, nb = walkers.nalpha, walkers.nbeta
        self.timer.start("force_bias")
        force_bias_into(hamiltonian, walkers, trial, ws.vbias)
        self.timer.stop("force_bias")
        self.vbias = ws.vbias
        xi = self.draw_fields(walkers, hamiltonian)
        call("ipie_b200_field_shift", ptr(ws.vbias), ptr(xi), ptr(self.mf_shift_dev), W, X, self.sqrt_dt, self.fbbound,
             ptr(ws.xshifted), ptr(ws.cmf), ptr(ws.cfb), stream())
        self.timer.start("vhs")
        self.construct_VHS(hamiltonian, ws.xshifted, out=ws.vhs)
        self.timer.stop("vhs")
        self.timer.start("orbitals")
        call("ipie_b200_ghf_blocks", ptr(walkers.phia), W, M, na, nb, ptr(ws.ghf_pa), ptr(ws.ghf_pb), 0, stream())
        for s_, (src, dst, n) in enumerate(((ws.ghf_pa, ws.phia_tmp, na), (ws.ghf_pb, ws.phib_tmp, nb))):
            if n == 0:
                continue
            if self.fused and not self.expH1_complex and M <= 256 and n <= 32:
                call("ipie_b200_propagate_orbitals", ptr(ws.vhs), ptr(self.expH1_pad[s_]), self.lda_e, ptr(src),
                     ptr(dst), W, M, n, self.exp_nmax, 1, 1, stream())
            else:
                cplx = int(self.expH1_complex)
                call("ipie_b200_propagate_one_body", ptr(self.expH1_dev[s_]), cplx, ptr(src), ptr(dst), W, M, n,
                     stream())
                call("ipie_b200_apply_exponential_batch", ptr(ws.vhs), ptr(dst), ptr(src), ptr(ws.taylor), W, M, n,
                     self.exp_nmax, stream())
                call("ipie_b200_propagate_one_body", ptr(self.expH1_dev[s_]), cplx, ptr(src), ptr(dst), W, M, n,
                     stream())
        call("ipie_b200_ghf_blocks", ptr(walkers.phia), W, M, na, nb, ptr(ws.phia_tmp), ptr(ws.phib_tmp), 1, stream())
        self.timer.stop("orbitals")
        greens_function_into(walkers, trial, ws.ovlp_new)
        walkers.mark_gf_current(trial)
        self.update_weight(walkers, walkers.ovlp, ws.ovlp_new, ws.cfb, ws.cmf, eshift)

    def _mixed_two_body(self, walkers, hamiltonian, trial):
        """Force bias (TF32), shifted fields, VHS and the orbital update (3-pass TF32) of the mixed form."""
        ws = self.ws
        W, X, M = walkers.nwalkers, hamiltonian.nchol, walkers.nbasis
        self.timer.start("force_bias")
        (ra_hi, ra_lo, ra_s), (rb_hi, rb_lo, rb_s) = self.rpad
        call("ipie_b200_construct_force_bias_mixed", ptr(ra_hi), ptr(ra_lo), ra_s, ptr(rb_hi), ptr(rb_lo), rb_s,
             ptr(walkers.Ghalfa), ptr(walkers.Ghalfb), ptr(ws.gwork), W, X, M, walkers.nup, walkers.ndown,
             ptr(ws.vbias), ptr(walkers.status), stream())
        self.timer.stop("force_bias")
        self.vbias = ws.vbias
        self.timer.start("rng")
        xi = self.draw_fields(walkers, hamiltonian)
        self.timer.stop("rng")
        self.timer.start("field_shift")
        call("ipie_b200_field_shift_mixed", ptr(ws.vbias), ptr(xi), ptr(self.mf_shift_dev), W, X, self.sqrt_dt,
             self.fbbound, None, ptr(ws.xs_hi), ptr(ws.xs_lo), ptr(ws.cmf), ptr(ws.cfb), stream())
        self.timer.stop("field_shift")
        self.timer.start("vhs")
        v = ws.v_planar
        if self.chain16:
            call("ipie_b200_construct_vhs_blocks", ptr(self.cb_hi), ptr(self.cb_lo), M, X, ptr(ws.xs_hi),
                 ptr(ws.xs_lo), W, self.sqrt_dt, self.cp_scale, self.v_scale, ptr(v[0]), ptr(v[1]), ptr(v[2]),
                 ptr(v[3]), self.vhs_flags, ptr(walkers.status), stream())
        else:
            call("ipie_b200_construct_vhs_mixed", ptr(self.cp_hi), ptr(self.cp_lo), ptr(hamiltonian.sym_idx_i),
                 ptr(hamiltonian.sym_idx_j), M, X, ptr(ws.xs_hi), ptr(ws.xs_lo), W, self.sqrt_dt, self.cp_scale, 0,
                 0.0, ptr(v[0]), ptr(v[1]), ptr(v[2]), ptr(v[3]), ptr(walkers.status), stream())
        self.timer.stop("vhs")
        self.timer.start("orbitals")
        for s_, (phi_name, tmp_name, n) in enumerate((("phia", "phia_tmp", walkers.nup),
                                                       ("phib", "phib_tmp", walkers.ndown))):
            if n == 0 or (s_ == 1 and walkers.spin_alias):
                continue
            phi, tmp = getattr(walkers, phi_name), getattr(ws, tmp_name)
            if self.chain16:
                call("ipie_b200_propagate_orbitals_mixed16", ptr(self.e16_hi[s_]), ptr(self.e16_lo[s_]), self.e_scale,
                     ptr(v[0]), ptr(v[1]), ptr(v[2]), ptr(v[3]), self.v_scale, ptr(phi), ptr(tmp), W, M, n,
                     self.exp_nmax, ptr(walkers.status), stream())
            else:
                call("ipie_b200_propagate_orbitals_mixed", ptr(self.e_hi[s_]), ptr(self.e_lo[s_]), self.lde,
                     ptr(v[0]), ptr(v[1]), ptr(v[2]), ptr(v[3]), ptr(phi), ptr(tmp), ptr(ws.orb_work), W, M, n,
                     self.exp_nmax, ptr(walkers.status), stream())
            setattr(walkers, phi_name, tmp)
            setattr(ws, tmp_name, phi)
        walkers.sync_alias()
        self.timer.stop("orbitals")
        return ws.cmf, ws.cfb

    def fused_ok(self, walkers):
        """The fused orbital kernel covers real expH1, M <= 256 and N <= 32."""
        return (self.fused and not self.expH1_complex and walkers.nbasis <= 256
                and max(walkers.nup, walkers.ndown) <= 32)

    def update_weight(self, walkers, ovlp, ovlp_new, cfb, cmf, eshift):
        """Hybrid energy, bound, importance function and cosine projection (ipie ``phaseless_base.py:340-358``).

        ``ovlp`` is overwritten with ``ovlp_new`` and becomes ``walkers.ovlp``.
        """
        ws = self.ws
        if eshift is ws.eshift:
            pass  # already on the device (set before a captured step is replayed)
        elif isinstance(eshift, torch.Tensor):
            ws.eshift.copy_(eshift.reshape(1).to(F64))
        else:
            ws.eshift.fill_(float(np.real(eshift)))
        call("ipie_b200_update_weight", walkers.nwalkers, ptr(ovlp_new), ptr(cfb), ptr(cmf), ptr(ws.eshift), self.dt,
             self.ebound, None, ptr(ovlp), ptr(walkers.hybrid_energy), ptr(walkers.weight), ptr(walkers.status),
             stream())
        walkers.ovlp = ovlp

    def clip_weights(self, walkers, wbound=None):
        """Driver weight clip to ``+-wbound`` (ipie ``qmc/afqmc.py:581-585``); ``None`` keeps the bound
        already in the workspace (set before a captured step is replayed)."""
        if wbound is not None:
            self.ws.wbound.fill_(float(wbound))
        call("ipie_b200_clip_weight", walkers.nwalkers, ptr(self.ws.wbound), ptr(walkers.weight), stream())
