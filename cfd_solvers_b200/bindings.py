"""ctypes bindings for the B200 engine's C ABI (include/cfdx_lbm.h).

Mirrors the reference's dependency-free ctypes binding
(python/cfd_solvers/bindings.py:1-33): a ``SolverLibrary`` wrapping the shared
library, a ``load(path=None)`` that honours ``CFD_SOLVERS_LIBRARY``, and
``RuntimeError``-style failures carrying the library's error text.  Error
statuses map onto the exception types the reference C++ solver throws
(``std::invalid_argument`` -> ValueError, ``std::out_of_range`` -> IndexError,
``std::bad_alloc`` -> MemoryError).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_LIBRARY = HERE / "libcfdx_lbm.so"

OK = 0
ERR_INVALID = 1
ERR_UNKNOWN = 2
ERR_CUDA = 3
ERR_OOM = 4
ERR_NONFINITE = 5
ERR_IO = 6
ERR_RANGE = 7

D3Q19 = 19
D3Q27 = 27
STORE_F32 = 0
STORE_F64 = 1
STORE_F16S = 2
BGK = 0
TRT = 1
HOST = 0
DEVICE = 1
ROUND_NEAREST = 0
ROUND_STOCHASTIC = 1
FLUID = 0
WALL = 1
MAX_WALL_IDS = 16
REDUCE_COUNT = 7
SIDE_LOWER = 0
STEP_EDGES = 1     # CFDX_STEP_EDGES: a slab's edge planes (the cells its halo messages carry)
STEP_INTERIOR = 2  # CFDX_STEP_INTERIOR: the remaining planes of that step
SIDE_UPPER = 1


class CfdxError(RuntimeError):
    """A failure reported by the C ABI (status code and message)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class NonFiniteError(CfdxError):
    """A reduction met NaN/Inf populations (CFDX_ERR_NONFINITE)."""


class CudaError(CfdxError):
    """A CUDA runtime failure, including "no CUDA device" (CFDX_ERR_CUDA)."""


class CheckpointError(CfdxError):
    """A checkpoint could not be written or read (CFDX_ERR_IO)."""


class cfdx_lbm_config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_size_t),
        ("ny", ctypes.c_size_t),
        ("nz", ctypes.c_size_t),
        ("tau", ctypes.c_float),
        ("acceleration_x", ctypes.c_float),
        ("acceleration_y", ctypes.c_float),
        ("acceleration_z", ctypes.c_float),
        ("smagorinsky_les", ctypes.c_int),
        ("lattice", ctypes.c_int),
        ("collision", ctypes.c_int),
        ("storage", ctypes.c_int),
        ("smagorinsky_cs", ctypes.c_float),
        ("trt_magic", ctypes.c_float),
        ("trt_tau_minus", ctypes.c_float),
        ("device", ctypes.c_int),
        ("fp16_rounding", ctypes.c_int),
        ("rounding_seed", ctypes.c_uint32),
    ]


class cfdx_lbm_info(ctypes.Structure):
    _fields_ = [
        ("cells", ctypes.c_size_t),
        ("q", ctypes.c_int),
        ("storage", ctypes.c_int),
        ("time_step", ctypes.c_uint64),
        ("population_bytes", ctypes.c_size_t),
        ("resident_bytes", ctypes.c_size_t),
        ("host_to_device_bytes", ctypes.c_uint64),
        ("device_to_host_bytes", ctypes.c_uint64),
        ("synchronizations", ctypes.c_uint64),
        ("fluid_flags", ctypes.c_int),
    ]


class cfdx_halo_entry(ctypes.Structure):
    _fields_ = [("plane", ctypes.c_uint32), ("direction", ctypes.c_uint32)]


class cfdx_slot_audit(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("slots", "touched", "read_twice", "written_twice", "read_only",
                                               "write_only", "foreign", "out_of_range")]


class cfdx_voxel_grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_size_t), ("ny", ctypes.c_size_t), ("nz", ctypes.c_size_t),
                ("minimum", ctypes.c_double * 3), ("maximum", ctypes.c_double * 3)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_sz = ctypes.c_size_t
_H = ctypes.c_void_p  # opaque handle

# name -> (restype, argtypes); the set of symbols include/cfdx_lbm.h declares.
SIGNATURES = {
    "cfdx_version": (ctypes.c_char_p, []),
    "cfdx_last_error": (_i, [ctypes.c_char_p, _sz]),
    "cfdx_lbm_config_default": (_i, [ctypes.POINTER(cfdx_lbm_config)]),
    "cfdx_lbm_create": (_i, [ctypes.POINTER(cfdx_lbm_config), ctypes.POINTER(_H), ctypes.c_char_p, _sz]),
    "cfdx_lbm_destroy": (_i, [_H]),
    "cfdx_lbm_init_uniform": (_i, [_H, _f, _f, _f, _f]),
    "cfdx_lbm_init_taylor_green": (_i, [_H, _f]),
    "cfdx_lbm_init_fields": (_i, [_H, _vp, _i]),
    "cfdx_lbm_set_flags": (_i, [_H, _vp, _i]),
    "cfdx_lbm_set_wall_velocity": (_i, [_H, _i, _f, _f, _f]),
    "cfdx_lbm_set_local_acceleration": (_i, [_H, _vp, _i]),
    "cfdx_lbm_device_local_acceleration": (_i, [_H, ctypes.POINTER(_vp)]),
    "cfdx_lbm_clear_device_acceleration": (_i, [_H]),
    "cfdx_lbm_set_solid_fraction": (_i, [_H, _vp, _i]),
    "cfdx_lbm_set_storage_scale": (_i, [_H, _vp]),
    "cfdx_lbm_step": (_i, [_H, ctypes.c_uint64]),
    "cfdx_lbm_synchronize": (_i, [_H]),
    "cfdx_lbm_macroscopic": (_i, [_H, _vp, _vp, _vp, _vp, _i]),
    "cfdx_lbm_macroscopic_f64": (_i, [_H, _vp, _vp, _vp, _vp, _i]),
    "cfdx_lbm_refresh_device_macroscopic": (_i, [_H] + [ctypes.POINTER(_vp)] * 4),
    "cfdx_lbm_reduce": (_i, [_H, ctypes.POINTER(ctypes.c_double)]),
    "cfdx_lbm_checksum": (_i, [_H, ctypes.POINTER(ctypes.c_double)]),
    "cfdx_lbm_logical_populations": (_i, [_H, _vp, _i]),
    "cfdx_lbm_get_info": (_i, [_H, ctypes.POINTER(cfdx_lbm_info)]),
    "cfdx_lbm_stream": (_i, [_H, ctypes.POINTER(_vp)]),
    "cfdx_lbm_raw_populations": (_i, [_H, ctypes.POINTER(_vp), ctypes.POINTER(_sz)]),
    "cfdx_lbm_set_launch_shape": (_i, [_H, _i, _i, _i]),
    "cfdx_lbm_set_step_planes": (_i, [_H, _i]),
    "cfdx_lbm_step_phase": (_i, [_H, _i]),
    "cfdx_lbm_reduce_noalloc": (_i, [_H, ctypes.POINTER(ctypes.c_double)]),
    "cfdx_lbm_set_tau": (_i, [_H, ctypes.c_float]),
    "cfdx_lbm_checkpoint_save": (_i, [_H, ctypes.c_char_p]),
    "cfdx_lbm_checkpoint_load": (_i, [_H, ctypes.c_char_p]),
    "cfdx_lbm_adjoint_forward": (_i, [_H, ctypes.c_uint64, ctypes.c_uint32]),
    "cfdx_lbm_adjoint_set_subinterval": (_i, [_H, ctypes.c_uint32]),
    "cfdx_lbm_adjoint_backward": (_i, [_H, _vp, _vp, _vp, _vp, _i, _vp, _i, ctypes.POINTER(ctypes.c_double)]),
    "cfdx_lbm_adjoint_memory": (_i, [_H, ctypes.POINTER(_sz)]),
    "cfdx_lbm_adjoint_release": (_i, [_H]),
    "cfdx_lbm_create_slab": (_i, [ctypes.POINTER(cfdx_lbm_config), ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_H),
                                  ctypes.c_char_p, _sz]),
    "cfdx_lbm_slab_info": (_i, [_H] + [ctypes.POINTER(ctypes.c_uint32)] * 3),
    "cfdx_halo_plan": (_i, [_i, _i, _i, ctypes.c_uint32, ctypes.POINTER(cfdx_halo_entry),
                            ctypes.POINTER(cfdx_halo_entry), _i, ctypes.POINTER(_i)]),
    "cfdx_lbm_halo_bytes": (_i, [_H, ctypes.POINTER(_sz)]),
    "cfdx_lbm_halo_pack": (_i, [_H, _i, _vp]),
    "cfdx_lbm_halo_unpack": (_i, [_H, _i, _vp]),
    "cfdx_lbm_halo_exchange": (_i, [_H, _H]),
    "cfdx_voxelize": (_i, [_vp, _sz, ctypes.POINTER(cfdx_voxel_grid), ctypes.c_uint32, ctypes.c_uint32,
                           ctypes.c_uint8, _vp, _i, _i]),
    "cfdx_lbm_set_flags_surface": (_i, [_H, _vp, _sz, _vp, _vp, ctypes.c_uint8, _vp, _i]),
    "cfdx_write_vtk_3d": (_i, [ctypes.c_char_p, _sz, _sz, _sz, _vp, _vp, _vp, ctypes.c_char_p, _i]),
    "cfdx_write_json_state_3d": (_i, [ctypes.c_char_p, _sz, _sz, _sz, ctypes.c_uint64, _vp, _vp, ctypes.c_char_p]),
    "cfdx_q_criterion": (_i, [_vp, _sz, _sz, _sz, ctypes.c_double, ctypes.c_double, ctypes.c_double, _vp, _i, _i]),
    "cfdx_lbm_q_criterion": (_i, [_H, ctypes.c_double, ctypes.c_double, ctypes.c_double, _vp, _i]),
    "cfdx_thermal_create": (_i, [_H, ctypes.c_float, ctypes.POINTER(_vp), ctypes.c_char_p, _sz]),
    "cfdx_thermal_destroy": (_i, [_vp]),
    "cfdx_thermal_init_uniform": (_i, [_vp, ctypes.c_float]),
    "cfdx_thermal_init_field": (_i, [_vp, _vp, _i]),
    "cfdx_thermal_step": (_i, [_vp, _vp, _vp, _vp, ctypes.c_uint64]),
    "cfdx_thermal_refresh_device_scalar": (_i, [_vp, ctypes.POINTER(_vp)]),
    "cfdx_thermal_temperature": (_i, [_vp, _vp, _i]),
    "cfdx_thermal_add_boussinesq": (_i, [_vp, _vp, _vp, _vp] + [ctypes.c_float] * 5),
    "cfdx_thermal_total": (_i, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "cfdx_thermal_info": (_i, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(ctypes.c_uint64),
                               ctypes.POINTER(ctypes.c_uint64)]),
    "cfdx_surface_create": (_i, [_H, ctypes.POINTER(_vp), ctypes.c_char_p, _sz]),
    "cfdx_surface_destroy": (_i, [_vp]),
    "cfdx_surface_init_uniform": (_i, [_vp, ctypes.c_float]),
    "cfdx_surface_init_half_space_x": (_i, [_vp, ctypes.c_float]),
    "cfdx_surface_init_field": (_i, [_vp, _vp, _i]),
    "cfdx_surface_advect": (_i, [_vp, _vp, _vp, _vp, ctypes.c_float]),
    "cfdx_surface_device_fill": (_i, [_vp, ctypes.POINTER(_vp)]),
    "cfdx_surface_refresh_geometry": (_i, [_vp, ctypes.POINTER(_vp)]),
    "cfdx_surface_add_tension": (_i, [_vp, _vp, _vp, _vp, ctypes.c_float, ctypes.c_float]),
    "cfdx_surface_volume": (_i, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "cfdx_surface_fill": (_i, [_vp, _vp, _i, _i]),
    "cfdx_surface_info": (_i, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(ctypes.c_uint64),
                               ctypes.POINTER(ctypes.c_uint64)]),
    "cfdx_particles_create": (_i, [_H, _sz, ctypes.POINTER(_vp), ctypes.c_char_p, _sz]),
    "cfdx_particles_destroy": (_i, [_vp]),
    "cfdx_particles_upload": (_i, [_vp, _vp, _sz]),
    "cfdx_particles_download": (_i, [_vp, _vp, _sz]),
    "cfdx_particles_device_state": (_i, [_vp, ctypes.POINTER(_vp)]),
    "cfdx_particles_advance": (_i, [_vp] + [_vp] * 6 + [ctypes.c_float, _i] + [ctypes.c_float] * 3),
    "cfdx_particles_info": (_i, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.POINTER(ctypes.c_uint64)]),
    "cfdx_diagnostics_create": (_i, [_H, ctypes.POINTER(_vp), ctypes.c_char_p, _sz]),
    "cfdx_diagnostics_destroy": (_i, [_vp]),
    "cfdx_diagnostics_q_criterion": (_i, [_vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "cfdx_diagnostics_info": (_i, [_vp, ctypes.POINTER(_sz)]),
    "cfdx_lbm_debug_slot_audit": (_i, [_H, _i, ctypes.POINTER(cfdx_slot_audit)]),
    "cfdx_debug_audit_classify": (_i, [ctypes.c_uint32] * 5 + [ctypes.POINTER(ctypes.c_uint)]),
    "cfdx_release_scratch": (_i, [_i]),
    "cfdx_debug_fail_allocations": (_i, [_i]),
    "cfdx_lbm_debug_force_wide_slots": (_i, [_H, _i]),
    "cfdx_debug_retry_allocations": (_i, [_i, ctypes.POINTER(ctypes.c_ulonglong)]),
}


class SolverLibrary:
    """The loaded C ABI.  Every wrapped call raises on a non-zero status."""

    def __init__(self, path):
        self.path = Path(path)
        self._lib = ctypes.CDLL(os.fspath(self.path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(self._lib, name)
            fn.restype = res
            fn.argtypes = args

    @property
    def version(self) -> str:
        return self._lib.cfdx_version().decode("utf-8")

    @property
    def raw(self):
        """The underlying ctypes.CDLL (every symbol of include/cfdx_lbm.h)."""
        return self._lib

    def last_error(self) -> tuple[int, str]:
        buf = ctypes.create_string_buffer(1024)
        status = self._lib.cfdx_last_error(buf, len(buf))
        return status, buf.value.decode("utf-8", errors="replace")

    def check(self, status: int, what: str = ""):
        if status == OK:
            return
        _, message = self.last_error()
        message = f"{what}: {message}" if what else message
        if status == ERR_INVALID:
            raise ValueError(message)
        if status == ERR_RANGE:
            raise IndexError(message)
        if status == ERR_OOM:
            raise MemoryError(message)
        if status == ERR_NONFINITE:
            raise NonFiniteError(status, message)
        if status == ERR_CUDA:
            raise CudaError(status, message)
        if status == ERR_IO:
            raise CheckpointError(status, message)
        raise CfdxError(status, message)

    def call(self, name: str, *args):
        self.check(getattr(self._lib, name)(*args), name)


_loaded: dict[str, SolverLibrary] = {}


def load(path=None) -> SolverLibrary:
    """Loads the engine library: ``path``, else ``$CFD_SOLVERS_LIBRARY``, else the in-tree build.

    Fails loudly when the library is missing; there is no CPU fallback.
    """
    path = Path(path or os.environ.get("CFD_SOLVERS_LIBRARY") or DEFAULT_LIBRARY)
    if not path.exists():
        raise RuntimeError(f"{path} is not built: run `python -m cfd_solvers_b200.build` (nvcc, sm_100a)")
    key = os.fspath(path.resolve())
    if key not in _loaded:
        _loaded[key] = SolverLibrary(path)
    return _loaded[key]
