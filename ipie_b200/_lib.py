"""ctypes binding of the in-tree CUDA library ``libipie_b200.so``.

The library is the product's compute path; there is no fallback.  If the
shared object is missing or fails to load, importing the compute entry points
raises immediately.  Every call passes raw device pointers of contiguous
torch tensors and torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libipie_b200.so")

P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double

# name -> argtypes (restype int unless noted)
SIGNATURES = {
    "ipie_b200_greens_function_single_det_batch": [P, P, I, I, I, I, P, P, P, P, P, P, P, P, P],
    "ipie_b200_calc_overlap_single_det_uhf": [P, P, I, I, I, I, P, P, P, P, P, P],
    "ipie_b200_construct_force_bias_batch_single_det": [P, P, P, P, I, I, I, I, I, P, P],
    "ipie_b200_field_shift": [P, P, P, I, I, D, D, P, P, P, P],
    "ipie_b200_construct_vhs": [P, P, P, I, I, P, I, D, P, P],
    "ipie_b200_apply_exponential_batch": [P, P, P, P, I, I, I, I, P],
    "ipie_b200_propagate_one_body": [P, I, P, P, I, I, I, P],
    "ipie_b200_propagate_orbitals": [P, P, I, P, P, I, I, I, I, I, I, P],
    "ipie_b200_update_weight": [I, P, P, P, P, D, D, P, P, P, P, P, P],
    "ipie_b200_clip_weight": [I, P, P, P],
    "ipie_b200_reortho": [P, P, I, I, I, I, P, P, P, P, P, P],
    "ipie_b200_walker_copy": [P, I, I, I, I, P, P, P, P, P, P, P, P, P, P],
    "ipie_b200_walker_gather": [P, I, I, I, I] + [P] * 17,
    "ipie_b200_exchange_rows": [I, I, I, I],
    "ipie_b200_exchange": [P, P, I, I, I, I, P, P],
    "ipie_b200_exchange_noalloc": [P, P, I, I, I, I, P, P],
    "ipie_b200_local_energy_single_det_batch": [I, P, P, P, P, D, P, P, I, I, I, I, I, P, P, P, P],
    "ipie_b200_walker_sums": [I, P, P, P, P, P, I, P],
    "ipie_b200_construct_force_bias_mixed": [P, P, D, P, P, D, P, P, P, I, I, I, I, I, P, P, P],
    "ipie_b200_field_shift_mixed": [P, P, P, I, I, D, D, P, P, P, P, P, P],
    "ipie_b200_construct_vhs_mixed": [P, P, P, P, I, I, P, P, I, D, D, I, D, P, P, P, P, P, P],
    "ipie_b200_orbital_chain16_fits": [I, I],
    "ipie_b200_vhs_blocks": [I],
    "ipie_b200_ghf_blocks": [P, I, I, I, I, P, P, I, P],
    "ipie_b200_vhs_block_pack": [P, P, I, I, D, P, P, P],
    "ipie_b200_construct_vhs_blocks": [P, P, I, I, P, P, I, D, D, D, P, P, P, P, I, P, P],
    "ipie_b200_propagate_orbitals_mixed16": [P, P, D, P, P, P, P, D, P, P, I, I, I, I, P, P],
    "ipie_b200_propagate_orbitals_mixed": [P, P, I, P, P, P, P, P, P, P, I, I, I, I, P, P],
    "ipie_b200_rchol_pad_split": [P, I, I, I, D, P, P, P],
    "ipie_b200_exchange_mixed": [P, P, D, P, P, P, P, I, I, I, I, P, P, P, P, P],
    "ipie_b200_local_energy_mixed": [I, P, P, P, P, D, P, P, D, P, P, D, P, P, P, P, P, P, P, I, I, I, I, I, P, P, P,
                                     P, P],
    "ipie_b200_energy_combine": [I, I, I, I, I, P, P, P, P, D, P, P, I, D, D, D, P, P, P],
    "ipie_b200_mlp_forward": [P, I, I, I, P, P, P, P, P],
    "ipie_b200_mlp_backward": [P, P, I, I, I, P, P, P, P, P, P, P],
    "ipie_b200_mlp_adam": [P, P, P, P, P, ctypes.c_longlong, ctypes.c_float, I, P],
    "ipie_b200_normalize_features": [P, ctypes.c_longlong, I, P, P, P],
    "ipie_b200_cv_features": [I, I, I, I, I, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P],
    "ipie_b200_gather_walkers": [P, P, I, ctypes.c_longlong, P, P],
    "ipie_b200_cv_sums": [I, P, P, P, I, P, P, P, P],
    "ipie_b200_local_energy_vjp": [I, P, P, P, P, P, P, I, I, I, I, I, P, P, P, P, P],
    "ipie_b200_onebody_adjoint": [I, I, I, I, P, P, P, P, P, P, P, P],
    "ipie_b200_rotate_onebody": [P, P, I, I, P, P],
    "ipie_b200_split_tf32": [P, P, P, ctypes.c_longlong, P],
    "ipie_b200_umma_gemm_test": [P, P, P, P, P, P, P, I, I, I, I, I, P, P],
    "ipie_b200_split_f16": [P, P, P, ctypes.c_longlong, D, P],
    "ipie_b200_force_bias_complex": [P, P, P, I, I, I, P, I, I, I, P],
    "ipie_b200_construct_vhs_complex": [P, P, I, I, P, I, D, P, P],
    "ipie_b200_energy_complex": [P, P, I, I, I, P, P, D, P, P, I, P, P, P],
    "ipie_b200_exchange_complex": [P, P, I, I, I, I, P, P, I, P],
    "ipie_b200_umma_gemm_f16_test": [P, P, P, P, P, I, I, I, I, P, P],
    "ipie_b200_normal_fill": [P, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.c_ulonglong, P],
    "ipie_b200_normal_fill_dev": [P, ctypes.c_longlong, ctypes.c_ulonglong, P, P],
    "ipie_b200_pair_branch": [I, P, P, D, D, D, ctypes.c_ulonglong, P, I, P, P, P, P, P, P],
    "ipie_b200_ad_greens_function": [P, P, ctypes.c_longlong, I, I, I, P, P, P, P, P, P, P],
    "ipie_b200_ad_field_shift": [P, P, P, P, I, I, D, D, P, P, P, P, P, P, P],
    "ipie_b200_ad_update_weight": [I, P, P, P, P, P, P, P, P, D, D, P, P, P, P],
    "ipie_b200_ad_reortho": [P, P, ctypes.c_longlong, I, I, I, P, P],
    "ipie_b200_ad_block_vhs": [P, P, I, I, P, P],
    "ipie_b200_ad_axpy": [P, P, D, ctypes.c_longlong, P, P],
    "ipie_b200_ad_gather": [P, I, ctypes.c_longlong, P, P, P],
    "ipie_b200_multidet_accumulate": [I, I, I, I, D, D, P, P, P, P, P, P, P, P, P, P, P],
    "ipie_b200_multidet_finalize": [I, I, P, P, P, P, P, P],
}

_lib = None


class CudaLibError(RuntimeError):
    pass


def lib():
    """The loaded library (loads it on first use; raises if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CudaLibError(
                f"{LIB_PATH} is missing: build it with `python -m ipie_b200.build` (needs nvcc); "
                "ipie_b200 has no CPU fallback"
            )
        lb = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lb, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        lb.ipie_b200_version.restype = ctypes.c_char_p
        lb.ipie_b200_version.argtypes = []
        lb.ipie_b200_launch_count.restype = ctypes.c_longlong
        lb.ipie_b200_launch_count.argtypes = []
        _lib = lb
    return _lib


def ptr(t):
    """Device pointer of a contiguous CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise CudaLibError("ipie_b200 kernels take CUDA tensors only")
    if not t.is_contiguous():
        raise CudaLibError("ipie_b200 kernels take contiguous tensors only")
    if t.is_conj() or t.is_neg():
        # a lazy view: its memory still holds the unconjugated (or unnegated) values
        raise CudaLibError("ipie_b200 kernels take materialised tensors (call resolve_conj() / resolve_neg())")
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def check(rc: int, what: str):
    if rc != 0:
        raise CudaLibError(f"{what} failed with CUDA error {rc} ({_err_name(rc)})")


def _err_name(rc):
    try:
        return torch.cuda.cudart().cudaGetErrorString(rc)
    except Exception:  # pragma: no cover - best effort
        return "?"


def call(name: str, *args):
    rc = getattr(lib(), name)(*args)
    check(rc, name)


def launch_count() -> int:
    """Kernels enqueued by the library so far (host-side counter)."""
    return int(lib().ipie_b200_launch_count())
