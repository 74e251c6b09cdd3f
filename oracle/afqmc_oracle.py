"""numpy restatement of ipie's phaseless-AFQMC walker step (CPU oracle).

TEST INFRASTRUCTURE ONLY.  This module is the checker the CUDA path is compared
against; it is imported by ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` and by nothing in ``ipie_b200``.

Every function restates one piece of ipie's CPU code path for a generic real
Cholesky Hamiltonian (``GenericRealChol``) with a single-determinant trial
(``SingleDet``) and UHF-style walkers (``UHFWalkers`` with ``rhf = False``, the
production setting).  Citations are ``file:line`` inside the ipie project.
Loops that ipie runs per walker are batched here with numpy stacks; the
arithmetic is the same.

Random numbers: the auxiliary fields are drawn exactly as ipie draws them,
``numpy.random.normal(0, 1, X*W).reshape(W, X)`` per step from the global
MT19937 stream, and pair branching consumes one ``numpy.random.rand()`` per
pair (``propagation/phaseless_base.py:296-298``,
``walkers/pop_controller.py:362``).  Seeding ``numpy.random.seed(s)`` before
a run therefore reproduces ipie's draw sequence.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg


# --------------------------------------------------------------------------
# Hamiltonian and trial set-up
# --------------------------------------------------------------------------
def construct_h1e_mod(chol: np.ndarray, h1e: np.ndarray) -> np.ndarray:
    """``h1e_mod = h1e - 1/2 sum_kn L_ik,n L_jk,n``.

    ipie: ``hamiltonians/generic.py:31-43``.  ``chol`` is (M*M, X).
    """
    M = h1e.shape[-1]
    X = chol.shape[-1]
    view = chol.reshape(M, M * X)
    v0 = 0.5 * view @ view.T.conj()
    return np.array([h1e[0] - v0, h1e[1] - v0])


def pack_cholesky(chol: np.ndarray, M: int) -> np.ndarray:
    """Upper-triangle packing ``chol_packed[t] = L[i_t, j_t]`` with numpy triu order.

    ipie: ``hamiltonians/generic.py:64-72`` and ``utils/pack_numba.py:36-45``.
    """
    X = chol.shape[-1]
    iu, ju = np.triu_indices(M)
    return chol.reshape(M, M, X)[iu, ju, :].copy()


def gab_mod(A: np.ndarray, B: np.ndarray):
    """Trial density ``G = A* (B^T A*)^-1 B^T``; ipie ``estimators/utils.py:99-132``."""
    O = B.T @ A.conj()
    ghalf = scipy.linalg.inv(O) @ B.T
    return A.conj() @ ghalf, ghalf


def trial_density(psi: np.ndarray, na: int, nb: int):
    """``gab_spin(psi, psi, na, nb)``; ipie ``estimators/utils.py:135-142``."""
    Ga, Gha = gab_mod(psi[:, :na], psi[:, :na])
    if nb > 0:
        Gb, Ghb = gab_mod(psi[:, na:], psi[:, na:])
    else:
        Gb = np.zeros_like(Ga)
        Ghb = np.zeros((0, Gha.shape[1]), dtype=Gha.dtype)
    return np.array([Ga, Gb]), [Gha, Ghb]


def half_rotate(psia: np.ndarray, psib: np.ndarray, chol: np.ndarray, h1e: np.ndarray):
    """Half-rotated one-body and Cholesky integrals.

    ``rH1_s[i, q] = sum_p psi*_pi h1_pq``; ``rchol_s[x, i*M + n] = sum_m psi*_mi L[m, n, x]``.
    ipie: ``trial_wavefunction/half_rotate.py:11-116`` (via ``single_det.py:88-112``).
    The dtype follows ipie's ``integral_type`` rule (``half_rotate.py:39-41``).
    """
    M = psia.shape[0]
    X = chol.shape[-1]
    L = chol.reshape(M, M, X)
    rH1a = np.einsum("pi,pq->iq", psia.conj(), h1e[0], optimize=True)
    rH1b = np.einsum("pi,pq->iq", psib.conj(), h1e[1], optimize=True)
    rchola = np.einsum("mi,mnx->xin", psia.conj(), L, optimize=True).reshape(X, -1)
    rcholb = np.einsum("mi,mnx->xin", psib.conj(), L, optimize=True).reshape(X, -1)
    if not np.iscomplexobj(psia) and not np.iscomplexobj(psib):
        rchola = rchola.real.copy()
        rcholb = rcholb.real.copy()
    return rH1a, rH1b, rchola, rcholb


def mean_field_shift(chol: np.ndarray, G: np.ndarray) -> np.ndarray:
    """``mf = 1j * L^T Re(G_a+G_b) - L^T Im(G_a+G_b)``; ipie ``propagation/phaseless_base.py:153-172``."""
    g = (G[0] + G[1]).ravel()
    return 1.0j * (chol.T @ g.real) - chol.T @ g.imag


def one_body_propagator(h1e_mod: np.ndarray, chol: np.ndarray, mf: np.ndarray, dt: float, M: int):
    """``expH1_s = expm(-dt/2 (h1e_mod_s - 1j L.mf))``; ipie ``phaseless_base.py:27-74``."""
    shift = 1.0j * np.einsum("mx,x->m", chol, mf).reshape(M, M)
    H1 = h1e_mod - np.array([shift, shift])
    return np.array([scipy.linalg.expm(-0.5 * dt * H1[0]), scipy.linalg.expm(-0.5 * dt * H1[1])])


@dataclass
class System:
    """Everything the walker step reads besides walker state (host arrays)."""

    nbasis: int
    nup: int
    ndown: int
    h1e: np.ndarray
    chol: np.ndarray  # (M*M, X) float64
    ecore: float
    psi: np.ndarray  # (M, nup+ndown) trial orbitals
    dt: float = 0.005
    exp_nmax: int = 6
    # derived
    chol_packed: np.ndarray = field(default=None)
    h1e_mod: np.ndarray = field(default=None)
    psi0a: np.ndarray = field(default=None)
    psi0b: np.ndarray = field(default=None)
    rH1a: np.ndarray = field(default=None)
    rH1b: np.ndarray = field(default=None)
    rchola: np.ndarray = field(default=None)
    rcholb: np.ndarray = field(default=None)
    G: np.ndarray = field(default=None)
    mf_shift: np.ndarray = field(default=None)
    expH1: np.ndarray = field(default=None)

    def build(self):
        """Mirror of ``Generic(...)``, ``SingleDet(...)``, ``half_rotate`` and ``PhaselessBase.build``."""
        M = self.nbasis
        psi = self.psi
        # ipie drops a negligible imaginary part of the trial (trial_wavefunction/single_det.py:41-44).
        if np.iscomplexobj(psi) and np.sum(psi.imag.ravel() ** 2) <= 1e-8:
            psi = np.array(psi.real, dtype=np.float64)
        self.psi = psi
        self.psi0a = np.ascontiguousarray(psi[:, : self.nup])
        self.psi0b = np.ascontiguousarray(psi[:, self.nup:])
        self.chol_packed = pack_cholesky(self.chol, M)
        self.h1e_mod = construct_h1e_mod(self.chol, self.h1e)
        self.G, _ = trial_density(psi, self.nup, self.ndown)
        self.rH1a, self.rH1b, self.rchola, self.rcholb = half_rotate(self.psi0a, self.psi0b, self.chol, self.h1e)
        self.mf_shift = mean_field_shift(self.chol, self.G)
        self.expH1 = one_body_propagator(self.h1e_mod, self.chol, self.mf_shift, self.dt, M)
        return self

    @property
    def nchol(self):
        return self.chol.shape[-1]

    # the pieces that differ for a complex Cholesky Hamiltonian (oracle/complex_chol_oracle.py)
    @property
    def nfields(self):
        return self.nchol

    def vbias(self, w):
        return force_bias(self, w)

    def vhs(self, xshifted):
        return construct_vhs(self, xshifted)

    def local_energy(self, w):
        return local_energy_single_det_uhf_batch(self, w)


@dataclass
class Walkers:
    """Walker-batch state; the arrays ipie's ``UHFWalkers`` carries (``walkers/uhf_walkers.py:46-99``)."""

    phia: np.ndarray
    phib: np.ndarray
    weight: np.ndarray
    unscaled_weight: np.ndarray
    phase: np.ndarray
    hybrid_energy: np.ndarray
    ovlp: np.ndarray
    sgn_ovlp: np.ndarray
    log_ovlp: np.ndarray
    log_shift: np.ndarray
    detR_shift: np.ndarray
    detR: np.ndarray
    log_detR: np.ndarray
    Ghalfa: np.ndarray = None
    Ghalfb: np.ndarray = None

    @property
    def nwalkers(self):
        return self.phia.shape[0]

    @staticmethod
    def from_initial(init: np.ndarray, nup: int, nwalkers: int) -> "Walkers":
        """``UHFWalkers.__init__`` + ``BaseWalkers.__init__`` (``uhf_walkers.py:67-74``, ``base_walkers.py:108-126``)."""
        W = nwalkers
        phia = np.array([init[:, :nup].copy() for _ in range(W)], dtype=np.complex128)
        phib = np.array([init[:, nup:].copy() for _ in range(W)], dtype=np.complex128)
        return Walkers(
            phia=phia,
            phib=phib,
            weight=np.ones(W),
            unscaled_weight=np.ones(W),
            phase=np.ones(W, dtype=np.complex128),
            hybrid_energy=np.zeros(W),
            ovlp=np.ones(W),
            sgn_ovlp=np.ones(W),
            log_ovlp=np.zeros(W),
            log_shift=np.zeros(W),
            detR_shift=np.zeros(W),
            detR=np.ones(W),
            log_detR=np.zeros(W),
        )

    def copy(self) -> "Walkers":
        kw = {}
        for k in self.__dataclass_fields__:
            v = getattr(self, k)
            kw[k] = None if v is None else np.array(v, copy=True)
        return Walkers(**kw)


# --------------------------------------------------------------------------
# Green's function, overlap
# --------------------------------------------------------------------------
def greens_function(sys_: System, w: Walkers) -> np.ndarray:
    """Half-rotated Green's function and overlap.

    ``O_s = phi_s^T psi_s*``; ``Ghalf_s = O_s^-1 phi_s^T``;
    ``ovlp = sign_a sign_b exp(logdet_a + logdet_b - log_shift)``.
    ipie: ``estimators/greens_function_single_det.py:62-103`` (per-walker loop
    batched here) and ``:106-154`` (its batched twin).  Sets ``w.Ghalfa/b``.
    """
    Oa = np.einsum("wmi,mj->wij", w.phia, sys_.psi0a.conj(), optimize=True)
    w.Ghalfa = np.linalg.inv(Oa) @ np.transpose(w.phia, (0, 2, 1))
    sa, la = np.linalg.slogdet(Oa)
    if sys_.ndown > 0:
        Ob = np.einsum("wmi,mj->wij", w.phib, sys_.psi0b.conj(), optimize=True)
        w.Ghalfb = np.linalg.inv(Ob) @ np.transpose(w.phib, (0, 2, 1))
        sb, lb = np.linalg.slogdet(Ob)
        return sa * sb * np.exp(la + lb - w.log_shift)
    w.Ghalfb = np.zeros((w.nwalkers, 0, sys_.nbasis), dtype=np.complex128)
    return sa * np.exp(la - w.log_shift)


def overlap(sys_: System, w: Walkers) -> np.ndarray:
    """Walker-trial overlap without the Green's function; ipie ``propagation/overlap.py:29-59``."""
    Oa = np.einsum("wmi,mj->wij", w.phia, sys_.psi0a.conj(), optimize=True)
    sa, la = np.linalg.slogdet(Oa)
    if sys_.ndown > 0:
        Ob = np.einsum("wmi,mj->wij", w.phib, sys_.psi0b.conj(), optimize=True)
        sb, lb = np.linalg.slogdet(Ob)
        return sa * sb * np.exp(la + lb - w.log_shift)
    return sa * np.exp(la - w.log_shift)


# --------------------------------------------------------------------------
# Force bias, VHS, exponential, one-body
# --------------------------------------------------------------------------
def force_bias(sys_: System, w: Walkers) -> np.ndarray:
    """``vbias[w, x] = sum_s rchol_s[x, :] . Ghalf_s[w, :]`` as separate real/imag GEMMs.

    ipie: ``propagation/force_bias.py:79-121`` (the ``rhf = False`` branch).
    ipie assigns the two products to ``.real`` and ``.imag`` of a complex
    array, so for a complex (complex-trial) ``rchol`` only the real part of
    each product survives; ``rchol.real`` reproduces that exactly.
    """
    W = w.nwalkers
    ra = sys_.rchola.real
    rb = sys_.rcholb.real
    Ga = w.Ghalfa.reshape(W, -1)
    Gb = w.Ghalfb.reshape(W, -1)
    vre = ra @ Ga.real.T + rb @ Gb.real.T
    vim = ra @ Ga.imag.T + rb @ Gb.imag.T
    v = np.empty((W, sys_.nchol), dtype=np.complex128)
    v.real = vre.T
    v.imag = vim.T
    return v


def apply_bound_force_bias(xbar: np.ndarray, max_bound: float = 1.0) -> np.ndarray:
    """Rescale ``|xbar| > max_bound`` entries to unit modulus; ipie ``phaseless_base.py:360-368``."""
    absxbar = np.abs(xbar)
    idx = absxbar > max_bound
    nonzeros = absxbar > 1e-13
    resc = xbar.copy()
    resc[nonzeros] = resc[nonzeros] / absxbar[nonzeros]
    return np.where(idx, resc, xbar)


def construct_vhs(sys_: System, xshifted: np.ndarray) -> np.ndarray:
    """``VHS[w] = 1j sqrt(dt) sum_x L_x xshifted[x, w]`` from the packed Cholesky, unpacked symmetric.

    ipie: ``propagation/phaseless_generic.py:66-97`` and ``utils/pack_numba.py:22-33``.
    ``xshifted`` is (X, W).
    """
    M = sys_.nbasis
    W = xshifted.shape[-1]
    vp = (sys_.chol_packed @ xshifted.real).astype(np.complex128)
    vp += 1.0j * (sys_.chol_packed @ xshifted.imag)
    vp = (1.0j * math.sqrt(sys_.dt)) * vp.T.reshape(W, -1)
    iu, ju = np.triu_indices(M)
    vhs = np.zeros((W, M, M), dtype=np.complex128)
    vhs[:, iu, ju] = vp
    vhs[:, ju, iu] = vp
    return vhs


def apply_exponential(phi: np.ndarray, vhs: np.ndarray, exp_nmax: int) -> np.ndarray:
    """Order-``exp_nmax`` Taylor series ``phi <- sum_n VHS^n phi / n!`` (recurrence form).

    ipie: ``propagation/operations.py:58-82`` (per walker) / ``:85-117`` (batched).
    """
    temp = phi.copy()
    for n in range(1, exp_nmax + 1):
        temp = (vhs @ temp) / n
        phi = phi + temp
    return phi


def propagate_one_body(phi: np.ndarray, expH1_s: np.ndarray) -> np.ndarray:
    """``phi_w <- expH1 . phi_w``; ipie ``propagation/operations.py:26-55``."""
    return np.einsum("ik,wkj->wij", expH1_s, phi, optimize=True)


def propagate_walkers_two_body(sys_: System, w: Walkers, xi: np.ndarray | None = None):
    """Force bias, field draw, VHS, exponential; returns ``(cmf, cfb)``.

    ipie: ``propagation/phaseless_base.py:282-310`` and ``phaseless_generic.py:35-58``.
    If ``xi`` (W, nfields) is not given it is drawn from numpy's global stream as ipie does.
    """
    W, X = w.nwalkers, sys_.nfields
    sqrt_dt = math.sqrt(sys_.dt)
    vbias = sys_.vbias(w)
    xbar = -sqrt_dt * (1.0j * vbias - sys_.mf_shift)
    xbar = apply_bound_force_bias(xbar, 1.0)
    if xi is None:
        xi = np.random.normal(0.0, 1.0, X * W).reshape(W, X)
    xshifted = xi - xbar
    cmf = -sqrt_dt * np.einsum("wx,x->w", xshifted, sys_.mf_shift)
    cfb = np.einsum("wx,wx->w", xi, xbar) - 0.5 * np.einsum("wx,wx->w", xbar, xbar)
    xshifted = xshifted.T.copy()
    vhs = sys_.vhs(xshifted)
    w.phia = apply_exponential(w.phia, vhs, sys_.exp_nmax)
    if sys_.ndown > 0:
        w.phib = apply_exponential(w.phib, vhs, sys_.exp_nmax)
    return cmf, cfb


def apply_bound_hybrid(ehyb: np.ndarray, eshift: float, ebound: float) -> np.ndarray:
    """Clip ``Re(E_hyb)`` to ``eshift +- sqrt(2/dt)`` unless ``|eshift| < 1e-10``; ipie ``phaseless_base.py:370-380``."""
    if abs(eshift) < 1e-10:
        return ehyb
    emax = eshift.real + ebound
    emin = eshift.real - ebound
    return np.clip(ehyb.real, emin, emax) + 1.0j * ehyb.imag


def update_weight(sys_: System, w: Walkers, ovlp, ovlp_new, cfb, cmf, eshift):
    """Hybrid energy, importance function, cosine projection; ipie ``phaseless_base.py:340-358``."""
    dt = sys_.dt
    ratio = ovlp_new / ovlp
    ehyb = -(np.log(ratio) + cfb + cmf) / dt
    ehyb = apply_bound_hybrid(ehyb, eshift, (2.0 / dt) ** 0.5)
    imp = np.exp(-dt * (0.5 * (ehyb + w.hybrid_energy) - eshift))
    magn = np.abs(imp)
    w.hybrid_energy = ehyb
    dtheta = (-dt * ehyb - cfb).imag
    cosine_fac = np.clip(np.cos(dtheta), 0.0, None)
    w.weight = w.weight * magn * cosine_fac
    w.ovlp = ovlp_new


def propagate_walkers(sys_: System, w: Walkers, eshift: float, xi: np.ndarray | None = None):
    """One phaseless step; ipie ``propagation/phaseless_base.py:312-338``."""
    ovlp = greens_function(sys_, w)
    w.phia = propagate_one_body(w.phia, sys_.expH1[0])
    if sys_.ndown > 0:
        w.phib = propagate_one_body(w.phib, sys_.expH1[1])
    cmf, cfb = propagate_walkers_two_body(sys_, w, xi)
    w.phia = propagate_one_body(w.phia, sys_.expH1[0])
    if sys_.ndown > 0:
        w.phib = propagate_one_body(w.phib, sys_.expH1[1])
    ovlp_new = overlap(sys_, w)
    update_weight(sys_, w, ovlp, ovlp_new, cfb, cmf, eshift)


# --------------------------------------------------------------------------
# Reorthogonalisation
# --------------------------------------------------------------------------
def reortho(sys_: System, w: Walkers) -> np.ndarray:
    """Thin QR with ``diag(R) > 0`` and overlap rescaling by ``det R``.

    ipie: ``walkers/uhf_walkers.py:108-143`` (CPU branch; scipy ``qr`` economic,
    ``utils/backend.py:75-78``).
    """
    W = w.nwalkers
    detR = np.empty(W)
    for iw in range(W):
        q, r = scipy.linalg.qr(w.phia[iw], mode="economic")
        d = np.diag(r)
        w.phia[iw] = q @ np.diag(np.sign(d))
        log_det = np.sum(np.log(np.abs(d)))
        if sys_.ndown > 0:
            q, r = scipy.linalg.qr(w.phib[iw], mode="economic")
            d = np.diag(r)
            w.phib[iw] = q @ np.diag(np.sign(d))
            log_det += np.sum(np.log(np.abs(d)))
        detR[iw] = np.exp(log_det - w.detR_shift[iw])
        w.log_detR[iw] += np.log(detR[iw])
        w.detR[iw] = detR[iw]
        w.ovlp[iw] = w.ovlp[iw] / detR[iw]
    return detR


# --------------------------------------------------------------------------
# Population control (pair branch), single-process semantics
# --------------------------------------------------------------------------
_BUFF_NAMES = ["weight", "unscaled_weight", "phase", "hybrid_energy", "ovlp", "sgn_ovlp", "log_ovlp", "phia", "phib"]


def get_buffer(w: Walkers, iw: int) -> np.ndarray:
    """Pack one walker; ipie ``walkers/pop_controller.py:128-158`` with ``buff_names`` from
    ``base_walkers.py:128-136`` + ``uhf_walkers.py:94``."""
    parts = []
    for name in _BUFF_NAMES:
        v = getattr(w, name)[iw]
        parts.append(np.asarray(v, dtype=np.complex128).ravel())
    return np.concatenate(parts)


def set_buffer(w: Walkers, iw: int, buff: np.ndarray):
    """Unpack one walker; ipie ``walkers/pop_controller.py:161-196``."""
    s = 0
    for name in _BUFF_NAMES:
        arr = getattr(w, name)
        if arr.ndim > 1:
            n = arr[iw].size
            arr[iw] = buff[s: s + n].reshape(arr[iw].shape)
            s += n
        else:
            if np.iscomplexobj(arr):
                arr[iw] = buff[s]
            else:
                arr[iw] = buff[s].real
            s += 1


def pair_branch_table(absw: np.ndarray, max_weight: float, min_weight: float, rand=np.random.rand):
    """Pairing table of ipie's pair branch on one process.

    Returns ``(new_abs_weight, status)`` in walker order: status 2 = cloned,
    0 = killed, 1 = untouched.  ipie: ``walkers/pop_controller.py:338-391``.
    """
    n = absw.size
    g = np.zeros((n, 2))
    g[:, 0] = absw
    g[:, 1] = 1
    sort = np.argsort(g[:, 0], kind="mergesort")
    isort = np.argsort(sort, kind="mergesort")
    g = g[sort]
    s, e = 0, n - 1
    while s < e:
        if g[s][0] < min_weight or g[e][0] > max_weight:
            wab = g[s][0] + g[e][0]
            r = rand()
            if r < g[e][0] / wab:
                g[e][0] = 0.5 * wab
                g[e][1] = 2
                g[s][0] = 0.0
                g[s][1] = 0
            else:
                g[s][0] = 0.5 * wab
                g[s][1] = 2
                g[e][0] = 0.0
                g[e][1] = 0
            s += 1
            e -= 1
        else:
            break
    g = g[isort]
    return g[:, 0].copy(), g[:, 1].astype(np.int64)


def pair_branch(w: Walkers, max_weight: float = 4.0, min_weight: float = 0.1, rand=np.random.rand):
    """Clone/kill walkers with ipie's single-process message semantics.

    ipie: ``walkers/pop_controller.py:304-429`` with ``FakeComm``
    (``qmc/comm.py:61-71``).  On one process every send and receive carries
    the same tag (the tag is built from a *rank* index), and ``FakeComm``
    keeps only the last send per tag, so every killed walker receives the
    buffer of the highest-index cloned walker, weight included.
    """
    neww, status = pair_branch_table(np.abs(w.weight), max_weight, min_weight, rand)
    last = None
    for iw in range(w.nwalkers):
        if status[iw] > 1:
            w.weight[iw] = neww[iw]
            last = get_buffer(w, iw)
    for iw in range(w.nwalkers):
        if status[iw] == 0 and last is not None:
            set_buffer(w, iw, last.copy())
    return neww, status


def comb_parent_counts(weights: np.ndarray, target_weight: int, r: float) -> np.ndarray:
    """Copies of each walker under the comb (Booth & Gubernatis, PRE 80, 046704 (2009)).

    ipie: ``walkers/pop_controller.py:199-243``.  The comb teeth are
    ``(i + r) * total / target`` for i < target; walker iw receives every tooth in
    [cprobs[iw-1], cprobs[iw]).  ipie walks the teeth with a while loop; the
    same assignment is a right-sided search in the cumulative weights.
    """
    cprobs = np.cumsum(weights)
    total_weight = cprobs[-1]  # ipie's builtin sum(weights): the same sequential sum
    teeth = (np.arange(target_weight) + r) * (total_weight / target_weight)
    iw = np.searchsorted(cprobs, teeth, side="right")
    return np.bincount(iw, minlength=len(weights))[: len(weights)].astype(np.int64)


def comb(w: Walkers, weights: np.ndarray, target_weight: int, rand=np.random.random):
    """Comb pop control on one process: walker ``kill[i]`` becomes a copy of ``clone[i]``
    (pairs in index order, as ipie zips them), then every weight is reset to 1.

    ipie: ``walkers/pop_controller.py:199-301``; each send carries its own tag
    ``i`` there, so single-process copies are exact.
    """
    parent_ix = comb_parent_counts(weights, target_weight, rand())
    kill = np.where(parent_ix == 0)[0]
    clone = np.where(parent_ix > 1)[0]
    buffers = [get_buffer(w, c) for c, _ in zip(clone, kill)]
    for (c, k), buff in zip(zip(clone, kill), buffers):
        set_buffer(w, k, buff)
    w.weight.fill(1.0)
    return parent_ix


def stochastic_reconfiguration(w: Walkers, rand=np.random.rand):
    """Resample W walkers with a uniform comb on the cumulative |w|; all get the mean weight.

    ipie: ``walkers/pop_controller.py:432-475`` on one process.
    """
    nwalkers = w.nwalkers
    buffers = np.array([get_buffer(w, i) for i in range(nwalkers)])
    cumulative_weights = np.cumsum(np.abs(buffers[:, 0]))
    total_weight = cumulative_weights[-1]
    new_average_weight = total_weight / nwalkers / 1
    zeta = rand()
    new_ix = np.empty(nwalkers, dtype=np.int64)
    for i in range(nwalkers):
        z = (i + zeta) / nwalkers / 1
        new_ix[i] = np.searchsorted(cumulative_weights, z * total_weight)
    for i in range(nwalkers):
        b = buffers[new_ix[i]].copy()
        b[0] = new_average_weight
        set_buffer(w, i, b)
    return new_ix


class PopController:
    """Weight rescaling + pair branch / comb / stochastic reconfiguration;
    ipie ``walkers/pop_controller.py:33-125``."""

    def __init__(self, num_walkers: int, min_weight: float = 0.1, max_weight: float = 4.0,
                 method: str = "pair_branch", reconfiguration_freq: int = 50):
        self.ntot_walkers = num_walkers
        self.target_weight = num_walkers
        self.total_weight = num_walkers
        self.min_weight = min_weight
        self.max_weight = max_weight
        self.method = method
        self.reconfiguration_counter = 0
        self.reconfiguration_freq = reconfiguration_freq

    def pop_control(self, w: Walkers, rand=np.random.rand):
        if self.ntot_walkers == 1:
            return
        absw = np.abs(w.weight)
        if self.method == "comb":
            total_weight = float(np.cumsum(absw)[-1])  # builtin sum over the gathered weights
        else:
            total_weight = float(np.sum(absw))
        scale = total_weight / self.target_weight
        if total_weight < 1e-8:
            raise ValueError(f"Total weight is {total_weight:13.8e}")
        self.total_weight = total_weight
        w.unscaled_weight = w.weight
        w.weight = w.weight / scale
        if self.method == "comb":
            comb(w, absw / scale, self.target_weight, rand)
        elif self.method == "pair_branch":
            pair_branch(w, self.max_weight, self.min_weight, rand)
        elif self.method == "stochastic_reconfiguration":
            self.reconfiguration_counter += 1
            if self.reconfiguration_counter % self.reconfiguration_freq == 0:
                stochastic_reconfiguration(w, rand)
                self.reconfiguration_counter = 0


# --------------------------------------------------------------------------
# Local energy
# --------------------------------------------------------------------------
def exx_kernel(rchol: np.ndarray, Ghalf: np.ndarray) -> np.ndarray:
    """``exx_w = 1/2 sum_x sum_ij T_ij T_ji`` with ``T = rchol_x (N x M) . Ghalf_w^T``.

    ipie: ``estimators/local_energy_sd.py:263-303``.
    """
    W, N, M = Ghalf.shape
    X = rchol.shape[0]
    r = rchol.reshape(X * N, M)
    exx = np.zeros(W, dtype=np.complex128)
    for iw in range(W):
        if np.iscomplexobj(r):
            T = (r @ Ghalf[iw].T).reshape(X, N, N)
        else:  # real rchol: two real GEMMs, as ipie's numba kernel splits them
            T = (r @ Ghalf[iw].real.T + 1.0j * (r @ Ghalf[iw].imag.T)).reshape(X, N, N)
        exx[iw] = np.sum(T * np.transpose(T, (0, 2, 1)))
    return 0.5 * exx


def ecoul_kernel_uhf(rchola, rcholb, Ghalfa, Ghalfb) -> np.ndarray:
    """``ecoul_w = 1/2 (X_a + X_b).(X_a + X_b)`` (no conjugation); ipie ``local_energy_sd.py:158-201``."""
    W = Ghalfa.shape[0]
    Xv = Ghalfa.reshape(W, -1) @ rchola.T + Ghalfb.reshape(W, -1) @ rcholb.T
    return 0.5 * np.einsum("wx,wx->w", Xv, Xv)


def local_energy_single_det_uhf_batch(sys_: System, w: Walkers) -> np.ndarray:
    """(W, 3) complex ``[e1b + e2b, e1b, e2b]``; ipie ``estimators/local_energy_sd.py:358-403``."""
    W = w.nwalkers
    e1b = w.Ghalfa.reshape(W, -1) @ sys_.rH1a.ravel()
    e1b = e1b + w.Ghalfb.reshape(W, -1) @ sys_.rH1b.ravel()
    e1b = e1b + sys_.ecore
    ecoul = ecoul_kernel_uhf(sys_.rchola, sys_.rcholb, w.Ghalfa, w.Ghalfb)
    exx = exx_kernel(sys_.rchola, w.Ghalfa) + exx_kernel(sys_.rcholb, w.Ghalfb)
    e2b = ecoul - exx
    out = np.zeros((W, 3), dtype=np.complex128)
    out[:, 0] = e1b + e2b
    out[:, 1] = e1b
    out[:, 2] = e2b
    return out


def local_energy_single_det_rhf_batch(sys_: System, w: Walkers) -> np.ndarray:
    """RHF variant (spin-alpha only, doubled); ipie ``estimators/local_energy_sd.py:44-73,106-155``."""
    W = w.nwalkers
    Ga = w.Ghalfa.reshape(W, -1)
    e1b = 2.0 * Ga @ sys_.rH1a.ravel() + sys_.ecore
    Xv = sys_.rchola @ Ga.real.T + 1.0j * (sys_.rchola @ Ga.imag.T)
    ecoul = 2.0 * np.einsum("xw,xw->w", Xv, Xv)
    exx = 2.0 * exx_kernel(sys_.rchola, w.Ghalfa)
    e2b = ecoul - exx
    out = np.zeros((W, 3), dtype=np.complex128)
    out[:, 0] = e1b + e2b
    out[:, 1] = e1b
    out[:, 2] = e2b
    return out


def local_energy_of_density(sys_: System, Ghalfa: np.ndarray, Ghalfb: np.ndarray):
    """Local energy of one pair of half-rotated densities, e.g. the trial's own ``Ghalf``.

    Same arithmetic as :func:`local_energy_single_det_uhf_batch` for one walker;
    ipie's equivalent single-density entry point is
    ``estimators/generic.py`` ``local_energy_cholesky_opt``.
    """
    w = Walkers.from_initial(np.zeros((sys_.nbasis, sys_.nup + sys_.ndown)), sys_.nup, 1)
    w.Ghalfa = Ghalfa[None].astype(np.complex128)
    w.Ghalfb = Ghalfb[None].astype(np.complex128)
    return local_energy_single_det_uhf_batch(sys_, w)[0]


# --------------------------------------------------------------------------
# Driver
# --------------------------------------------------------------------------
class Accumulator:
    """Per-block sums of weight, unscaled weight and weighted hybrid energy.

    ipie: ``walkers/base_walkers.py:32-83`` and the block reduction in
    ``estimators/handler.py:211-242``.
    """

    def __init__(self, nsteps_per_block: int):
        self.buffer = np.zeros(3, dtype=np.complex128)
        self.nsteps = nsteps_per_block
        self._eshift = 0.0

    def update(self, w: Walkers):
        self.buffer += np.array([np.sum(w.weight), np.sum(w.unscaled_weight), np.sum(w.weight * w.hybrid_energy)])

    def block_end(self, block: int):
        factor = 1 if block == 0 else self.nsteps
        vals = self.buffer.copy()
        vals[2] = vals[2] / vals[0]
        vals[0] = vals[0] / factor
        vals[1] = vals[1] / factor
        self._eshift = vals[2]
        self.buffer[:] = 0.0
        return vals

    @property
    def eshift(self):
        return np.real(self._eshift)


def energy_estimate(sys_: System, w: Walkers):
    """``EnergyEstimator.compute_estimator``: GF recomputed, weighted sums; ipie ``estimators/energy.py:156-165``."""
    greens_function(sys_, w)
    e = sys_.local_energy(w)
    return {
        "ENumer": np.sum(w.weight * e[:, 0].real),
        "EDenom": np.sum(w.weight),
        "E1Body": np.sum(w.weight * e[:, 1].real),
        "E2Body": np.sum(w.weight * e[:, 2].real),
        "energies": e,
    }


def run_afqmc(
    sys_: System,
    w: Walkers,
    num_blocks: int,
    num_steps_per_block: int = 25,
    stabilize_freq: int = 5,
    pop_control_freq: int = 5,
    seed: int | None = None,
    xi_source=None,
    rand=None,
    on_step=None,
):
    """``AFQMC.run`` without the HDF5 estimator file; ipie ``qmc/afqmc.py:508-633``.

    Returns a list of per-block dicts with ``ETotal`` etc.  ``xi_source(step)``
    may supply the (W, X) field draws; by default they come from numpy's
    global stream after ``numpy.random.seed(seed)`` (ipie seeds it in
    ``AFQMCBase.__init__`` via ``qmc/utils.py:24-40``).
    """
    if seed is not None:
        np.random.seed(seed)
    rand = rand if rand is not None else np.random.rand
    eshift = 0.0
    reortho(sys_, w)
    pc = PopController(w.nwalkers)
    acc = Accumulator(num_steps_per_block)
    blocks = []
    est = energy_estimate(sys_, w)
    acc.update(w)
    vals = acc.block_end(0)
    blocks.append(_block_record(0, est, vals))
    num_eqlb_steps = 2.0 / sys_.dt
    total = num_steps_per_block * num_blocks
    for step in range(1, total + 1):
        if step % stabilize_freq == 0:
            reortho(sys_, w)
        xi = None if xi_source is None else xi_source(step)
        propagate_walkers(sys_, w, eshift, xi)
        if step > 1:
            wbound = pc.total_weight * 0.10
            w.weight = np.clip(w.weight, -wbound, wbound)
        if step % pop_control_freq == 0:
            pc.pop_control(w, rand)
        acc.update(w)
        if step % num_steps_per_block == 0:
            est = energy_estimate(sys_, w)
            vals = acc.block_end(step // num_steps_per_block)
            blocks.append(_block_record(step // num_steps_per_block, est, vals))
        if step < num_eqlb_steps:
            eshift = acc.eshift
        else:
            eshift += acc.eshift - eshift
        if on_step is not None:
            on_step(step, w)
    return blocks


def _block_record(block, est, vals):
    return {
        "block": block,
        "Weight": vals[0].real,
        "WeightFactor": vals[1].real,
        "HybridEnergy": vals[2].real,
        "ENumer": est["ENumer"],
        "EDenom": est["EDenom"],
        "ETotal": est["ENumer"] / est["EDenom"],
        "E1Body": est["E1Body"] / est["EDenom"],
        "E2Body": est["E2Body"] / est["EDenom"],
    }
