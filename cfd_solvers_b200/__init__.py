"""B200-native in-place Esoteric-Pull lattice-Boltzmann engine.

The compute path is the sm_100a CUDA library ``libcfdx_lbm.so`` (C ABI in
``include/cfdx_lbm.h``); this package holds its ctypes binding and a Python
front end that mirrors the reference's ``cfd::lbm`` solver API.  There is no
CPU fallback: without the built library or a CUDA device every solver call
raises.
"""
from .bindings import CfdxError, CheckpointError, CudaError, NonFiniteError, SolverLibrary, load
from .lbm import (
    DeviceAccelerationView,
    DeviceMacroscopicView,
    DeviceTransferStats,
    EsotericPullCudaSolver,
    InPlaceLbmConfig,
    MacroscopicFields,
    cavity_flags,
    release_scratch,
    smagorinsky_k,
    trt_tau_minus,
)
from .slabs import DistributedEsotericPullSolver, SlabSolver

__all__ = [
    "CfdxError",
    "CheckpointError",
    "CudaError",
    "NonFiniteError",
    "SolverLibrary",
    "load",
    "DeviceAccelerationView",
    "DeviceMacroscopicView",
    "DeviceTransferStats",
    "EsotericPullCudaSolver",
    "InPlaceLbmConfig",
    "MacroscopicFields",
    "cavity_flags",
    "release_scratch",
    "smagorinsky_k",
    "trt_tau_minus",
    "DistributedEsotericPullSolver",
    "SlabSolver",
]
