"""culbm_b200 — D3Q27 lattice Boltzmann (BGK) solver for one NVIDIA B200.

A drop-in for the single-device hot path of cuLBM (single_dev_expt_main):
hand-written sm_100a CUDA kernels behind the C ABI of ``include/culbm.h``
(``libculbm.so``), a CLI driver with the reference's flags
(``culbm_b200/bin/single_dev_expt_main``) and this Python front end.
"""
from ._capi import CulbmError, STORAGE  # noqa: F401
from .simulation import Simulation  # noqa: F401

__all__ = ["Simulation", "CulbmError", "STORAGE"]
