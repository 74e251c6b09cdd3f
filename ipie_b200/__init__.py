"""B200-native phaseless-AFQMC walker step behind ipie's surfaces.

The compute path is the in-tree CUDA library ``libipie_b200.so`` (sm_100a),
reached through a thin ctypes layer (``ipie_b200._lib``).  Host classes mirror
ipie's: ``Generic``/``GenericRealChol``/``GenericComplexChol``, ``SingleDet``/``SingleDetGHF``,
``UHFWalkers``/``GHFWalkers``,
``PhaselessGeneric``, ``PopController``, the single-determinant local energies,
``EnergyEstimator`` and ``AFQMC``.
"""
__version__ = "0.1.0"

_LAZY = {
    "Generic": "hamiltonian",
    "GenericRealChol": "hamiltonian",
    "GenericComplexChol": "hamiltonian",
    "SingleDet": "trial",
    "SingleDetGHF": "ghf",
    "UHFWalkers": "walkers",
    "GHFWalkers": "ghf",
    "PhaselessGeneric": "propagation",
    "PopController": "pop_control",
    "EnergyEstimator": "estimators",
    "local_energy_batch": "estimators",
    "local_energy_single_det_uhf_batch": "estimators",
    "local_energy_single_det_rhf_batch": "estimators",
    "local_energy_single_det_batch_gpu": "estimators",
    "AFQMC": "afqmc",
}


def __getattr__(name):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(name)
    import importlib

    return getattr(importlib.import_module(f"{__name__}.{mod}"), name)


def greens_function_single_det_batch(walker_batch, trial, build_full=False):
    """ipie ``estimators/greens_function_single_det.py:106-154``: sets ``Ghalfa/b``, returns overlaps."""
    return trial.calc_greens_function(walker_batch, build_full=build_full)
