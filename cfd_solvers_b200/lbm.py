"""Python front end of the B200 in-place Esoteric-Pull solver.

``EsotericPullCudaSolver`` keeps the method names, argument meaning and error
behaviour of the reference classes

* ``cfd::lbm::EsotericPullSolver<D>``     (include/cfd/solvers/lbm/esoteric_pull.hpp:104-515)
* ``cfd::lbm::EsotericPullSyclSolver<D>`` (include/cfd/solvers/lbm/esoteric_pull_sycl.hpp:18-475)

so reference-style driver code ports line for line.  All compute runs in the
sm_100a kernels of ``libcfdx_lbm.so`` behind the C ABI; this module only
marshals arguments.  Host arrays are numpy; device arrays may be passed as
torch CUDA tensors (anything with ``data_ptr()``) and are borrowed for the
duration of the call.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from dataclasses import dataclass
from typing import NamedTuple, Optional

import numpy as np

from . import bindings as B


@dataclass
class InPlaceLbmConfig:
    """The reference's InPlaceLbmConfig (esoteric_pull.hpp:20-29) plus the B200 extensions."""

    nx: int = 128
    ny: int = 128
    nz: int = 128
    tau: float = 0.6
    acceleration_x: float = 0.0
    acceleration_y: float = 0.0
    acceleration_z: float = 0.0
    smagorinsky_les: bool = False
    # extensions
    lattice: str = "d3q19"        # "d3q19" | "d3q27"
    collision: str = "bgk"        # "bgk" | "trt"
    storage: str = "fp32"         # "fp32" | "fp16s" | "fp64"
    smagorinsky_cs: float = 0.0   # <= 0: reference coefficient (Cs = sqrt(8/27)/pi)
    trt_magic: float = 3.0 / 16.0
    trt_tau_minus: float = 0.0    # > 0: fixed antisymmetric relaxation time
    device: int = 0
    fp16_rounding: str = "stochastic"  # FP16S stores: "stochastic" (unbiased) | "nearest"
    rounding_seed: int = 0

    @property
    def q(self) -> int:
        return _LATTICE[self.lattice]


class MacroscopicFields(NamedTuple):
    """rho, ux, uy, uz per cell (reference MacroscopicFields, esoteric_pull.hpp:31-36)."""

    rho: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    uz: np.ndarray


class DeviceMacroscopicView(NamedTuple):
    """Device pointers of rho|ux|uy|uz (reference esoteric_pull_sycl.hpp:218-224)."""

    rho: int
    ux: int
    uy: int
    uz: int
    cells: int


class DeviceAccelerationView(NamedTuple):
    """Device pointers of ax|ay|az (reference esoteric_pull_sycl.hpp:342-347)."""

    ax: int
    ay: int
    az: int
    cells: int


class DeviceTransferStats(NamedTuple):
    """Host<->device traffic of one solver (reference core/device_residency.hpp:11-42)."""

    host_to_device_bytes: int
    device_to_host_bytes: int
    synchronizations: int

    def host_transfer_bytes(self) -> int:
        return self.host_to_device_bytes + self.device_to_host_bytes


_LATTICE = {"d3q19": B.D3Q19, "d3q27": B.D3Q27}
_COLLISION = {"bgk": B.BGK, "trt": B.TRT}
_STORAGE = {"fp32": B.STORE_F32, "fp64": B.STORE_F64, "fp16s": B.STORE_F16S}


def _host(array, dtype, count, name):
    a = np.ascontiguousarray(array, dtype=dtype).reshape(-1)
    if a.size != count:
        raise ValueError(f"{name} size mismatch: expected {count}, got {a.size}")
    return a


def _is_device(array) -> bool:
    return hasattr(array, "data_ptr") and getattr(getattr(array, "device", None), "type", "cpu") == "cuda"


class EsotericPullCudaSolver:
    """Single-lattice in-place Esoteric-Pull solver on one B200 (sm_100a)."""

    def __init__(self, config: InPlaceLbmConfig | None = None, library=None, **kwargs):
        if config is None:
            config = InPlaceLbmConfig(**kwargs)
        elif kwargs:
            raise TypeError("pass either a config or keyword arguments")
        if config.lattice not in _LATTICE:
            raise ValueError("lattice must be d3q19 or d3q27")
        if config.collision not in _COLLISION:
            raise ValueError("collision must be bgk or trt")
        if config.storage not in _STORAGE:
            raise ValueError("storage must be fp32, fp16s or fp64")
        self._lib = library or B.load()
        self._config = config
        c = B.cfdx_lbm_config()
        self._lib.raw.cfdx_lbm_config_default(ctypes.byref(c))
        c.nx, c.ny, c.nz = int(config.nx), int(config.ny), int(config.nz)
        c.tau = config.tau
        c.acceleration_x = config.acceleration_x
        c.acceleration_y = config.acceleration_y
        c.acceleration_z = config.acceleration_z
        c.smagorinsky_les = int(bool(config.smagorinsky_les))
        c.lattice = _LATTICE[config.lattice]
        c.collision = _COLLISION[config.collision]
        c.storage = _STORAGE[config.storage]
        c.smagorinsky_cs = config.smagorinsky_cs
        c.trt_magic = config.trt_magic
        c.trt_tau_minus = config.trt_tau_minus
        c.device = config.device
        if config.fp16_rounding not in ("stochastic", "nearest"):
            raise ValueError("fp16_rounding must be stochastic or nearest")
        c.fp16_rounding = B.ROUND_STOCHASTIC if config.fp16_rounding == "stochastic" else B.ROUND_NEAREST
        c.rounding_seed = int(config.rounding_seed) & 0xFFFFFFFF
        self._h = None
        self._h = self._create(c)
        self._q = c.lattice
        self._cells = self._local_cells(c)
        self._has_mask = False
        self._has_local = False
        self._mask = None

    def _create(self, c: B.cfdx_lbm_config):
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        self._lib.check(self._lib.raw.cfdx_lbm_create(ctypes.byref(c), ctypes.byref(handle), err, len(err)),
                        "cfdx_lbm_create")
        return handle

    def _local_cells(self, c: B.cfdx_lbm_config) -> int:
        return c.nx * c.ny * c.nz

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.raw.cfdx_lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name, *args):
        if not self._h:
            raise RuntimeError("solver is closed")
        self._lib.call(name, self._h, *args)

    def _pointer(self, array, dtype, count, name):
        """(pointer, where, keepalive) for a host numpy or device torch array."""
        if _is_device(array):
            if array.numel() != count:
                raise ValueError(f"{name} size mismatch: expected {count}, got {array.numel()}")
            if not array.is_contiguous():
                raise ValueError(f"{name} must be contiguous")
            import torch

            # The library reads device buffers on its own stream: finish the
            # work that produced them on torch's stream first.
            torch.cuda.current_stream(array.device).synchronize()
            return ctypes.c_void_p(array.data_ptr()), B.DEVICE, array
        a = _host(array, dtype, count, name)
        return ctypes.c_void_p(a.ctypes.data), B.HOST, a

    # ------------------------------------------------- reference API (CPU class)
    def initialize_uniform(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        self._call("cfdx_lbm_init_uniform", rho, ux, uy, uz)

    def initialize_taylor_green(self, amplitude=0.03):
        self._call("cfdx_lbm_init_taylor_green", amplitude)

    def initialize_fields(self, rho, ux, uy, uz):
        fields = np.concatenate([_host(v, np.float32, self._cells, n) for v, n in
                                 ((rho, "rho"), (ux, "ux"), (uy, "uy"), (uz, "uz"))])
        self._call("cfdx_lbm_init_fields", ctypes.c_void_p(fields.ctypes.data), B.HOST)

    def step(self, count: int = 1):
        self._call("cfdx_lbm_step", int(count))

    def set_local_body_acceleration(self, ax, ay, az):
        if any(_is_device(v) for v in (ax, ay, az)):
            import torch

            a = torch.cat([ax.reshape(-1), ay.reshape(-1), az.reshape(-1)]).float().contiguous()
        else:
            a = np.concatenate([_host(v, np.float32, self._cells, "local LBM acceleration field")
                                for v in (ax, ay, az)])
        ptr, where, _keep = self._pointer(a, np.float32, 3 * self._cells, "local LBM acceleration field")
        self._call("cfdx_lbm_set_local_acceleration", ptr, where)
        self._has_local = True

    def clear_local_body_acceleration(self):
        self._call("cfdx_lbm_set_local_acceleration", None, B.HOST)
        self._has_local = False

    def has_local_body_acceleration(self) -> bool:
        return self._has_local

    def set_solid_mask(self, mask):
        """Stationary half-way bounce-back walls where mask != 0 (esoteric_pull.hpp:161-169)."""
        m = _host(mask, np.uint8, self._cells, "LBM solid mask")
        self.set_flags(np.where(m != 0, B.WALL, B.FLUID).astype(np.uint8))
        self._mask = m.copy()

    def clear_solid_mask(self):
        self._call("cfdx_lbm_set_flags", None, B.HOST)
        self._has_mask = False
        self._mask = None

    def has_solid_mask(self) -> bool:
        return self._has_mask

    def solid_mask(self):
        return self._mask

    def compute_macroscopic(self) -> MacroscopicFields:
        if self._config.storage == "fp64":
            out = [np.zeros(self._cells, np.float64) for _ in range(4)]
            self._call("cfdx_lbm_macroscopic_f64", *[ctypes.c_void_p(o.ctypes.data) for o in out], B.HOST)
        else:
            out = [np.zeros(self._cells, np.float32) for _ in range(4)]
            self._call("cfdx_lbm_macroscopic", *[ctypes.c_void_p(o.ctypes.data) for o in out], B.HOST)
        return MacroscopicFields(*out)

    def reduce(self) -> dict:
        """FP64 reductions over fluid cells (mass, momentum, KE, max speed, non-finite count)."""
        out = (ctypes.c_double * B.REDUCE_COUNT)()
        self._call("cfdx_lbm_reduce", out)
        return {"mass": out[0], "momentum": (out[1], out[2], out[3]), "kinetic_energy": out[4],
                "max_speed": out[5], "nonfinite": int(out[6])}

    def mass(self) -> float:
        return self.reduce()["mass"]

    def kinetic_energy(self) -> float:
        return self.reduce()["kinetic_energy"]

    def max_speed(self) -> float:
        return float(np.float32(self.reduce()["max_speed"]))

    def checksum(self) -> float:
        """mass + kinetic energy (examples/phase02_lbm_taylor_green.cpp:3)."""
        out = ctypes.c_double()
        self._call("cfdx_lbm_checksum", ctypes.byref(out))
        return out.value

    def logical_populations(self) -> np.ndarray:
        out = np.zeros(self._q * self._cells, np.float32)
        self._call("cfdx_lbm_logical_populations", ctypes.c_void_p(out.ctypes.data), B.HOST)
        return out

    @property
    def config(self) -> InPlaceLbmConfig:
        return self._config

    def cells(self) -> int:
        return self._cells

    def _info(self) -> B.cfdx_lbm_info:
        info = B.cfdx_lbm_info()
        self._call("cfdx_lbm_get_info", ctypes.byref(info))
        return info

    def time_step(self) -> int:
        return int(self._info().time_step)

    def population_bytes(self) -> int:
        return int(self._info().population_bytes)

    def two_lattice_population_bytes(self) -> int:
        return 2 * self.population_bytes()

    # ------------------------------------------------ reference API (SYCL class)
    def wait(self):
        self._call("cfdx_lbm_synchronize")

    def download_macroscopic(self) -> MacroscopicFields:
        return self.compute_macroscopic()

    def total_mass(self) -> float:
        return self.mass()

    def refresh_device_macroscopic(self) -> DeviceMacroscopicView:
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        self._call("cfdx_lbm_refresh_device_macroscopic", *[ctypes.byref(p) for p in ptrs])
        return DeviceMacroscopicView(*(p.value for p in ptrs), self._cells)

    def device_local_acceleration(self, clear: bool = False) -> DeviceAccelerationView:
        p = ctypes.c_void_p()
        self._call("cfdx_lbm_device_local_acceleration", ctypes.byref(p))
        if clear:
            self._call("cfdx_lbm_clear_device_acceleration")  # a device memset, no host transfer
        self._has_local = True
        base = p.value
        step = 4 * self._cells
        return DeviceAccelerationView(base, base + step, base + 2 * step, self._cells)

    def debug_slot_audit(self, parity: int) -> dict:
        """Slot-ownership audit of the step of `parity` (cfdx_lbm_debug_slot_audit): per-class slot
        counts.  A race-free step has written_twice == foreign == 0; read_only and write_only
        count the links into wall cells (one of each per link)."""
        out = B.cfdx_slot_audit()
        self._call("cfdx_lbm_debug_slot_audit", int(parity), ctypes.byref(out))
        return {k: int(getattr(out, k)) for k, _ in B.cfdx_slot_audit._fields_}

    def resident_bytes(self) -> int:
        return int(self._info().resident_bytes)

    def transfer_stats(self) -> DeviceTransferStats:
        i = self._info()
        return DeviceTransferStats(int(i.host_to_device_bytes), int(i.device_to_host_bytes), int(i.synchronizations))

    def device_name(self) -> str:
        try:
            import torch

            return torch.cuda.get_device_name(self._config.device)
        except Exception:  # pragma: no cover - informational only
            return "cuda"

    # ------------------------------------------------------------ extensions
    def set_flags(self, flags):
        """Cell flags: 0 fluid, 1 wall, 2..15 moving wall (velocity from set_wall_velocity)."""
        ptr, where, _keep = self._pointer(flags, np.uint8, self._cells, "LBM flag field")
        self._call("cfdx_lbm_set_flags", ptr, where)
        self._has_mask = True

    def set_solid_surface(self, triangles, minimum=(0.0, 0.0, 0.0), maximum=(1.0, 1.0, 1.0), solid_id: int = 1,
                          base_flags=None):
        """Flags from a closed triangle surface voxelized on the GPU over the box [minimum, maximum].

        Cells inside get `solid_id` (1 wall, 2..15 moving wall), the others
        `base_flags` (e.g. channel walls; host or device array of the handle's
        cells) or fluid.  Reference: voxelize_surface + set_solid_mask
        (examples/real_lbm3d_model.cpp:146-150).
        """
        from .geometry import as_surface

        t = as_surface(triangles)
        lo = np.ascontiguousarray(minimum, np.float64)
        hi = np.ascontiguousarray(maximum, np.float64)
        if base_flags is None:
            ptr, where, keep = None, B.HOST, None
        else:
            ptr, where, keep = self._pointer(base_flags, np.uint8, self._cells, "base flag field")
        self._call("cfdx_lbm_set_flags_surface", ctypes.c_void_p(t.ctypes.data), len(t),
                   ctypes.c_void_p(lo.ctypes.data), ctypes.c_void_p(hi.ctypes.data), int(solid_id), ptr, where)
        self._has_mask = True
        del keep

    # ------------------------------------------------------------ export
    def q_criterion(self, dx: float = 1.0, dy: float = 1.0, dz: float = 1.0, out=None):
        """Q-criterion of the current velocity, computed on the device (reference q_criterion_3d).

        Returns a float64 numpy array, or fills `out` (a float64 CUDA tensor of the cells).
        """
        if out is not None:
            if not _is_device(out) or out.numel() != self._cells:
                raise ValueError("out must be a CUDA tensor of one float64 per cell")
            self._call("cfdx_lbm_q_criterion", float(dx), float(dy), float(dz), ctypes.c_void_p(out.data_ptr()),
                       B.DEVICE)
            return out
        q = np.zeros(self._cells, np.float64)
        self._call("cfdx_lbm_q_criterion", float(dx), float(dy), float(dz), ctypes.c_void_p(q.ctypes.data), B.HOST)
        return q

    def _export_field(self, field: str):
        from .export import speed

        f = self.compute_macroscopic()
        if field == "speed":
            return speed(f), f
        if field == "rho":
            return np.asarray(f.rho, np.float64), f
        if field == "q_criterion":
            return self.q_criterion(), f
        raise ValueError("field must be speed, rho or q_criterion")

    def write_vtk(self, path, field: str = "speed", velocity: bool = True, solid: bool = True, binary: bool = False):
        """Legacy-VTK file of `field` (speed, rho or q_criterion), the velocity and the wall cells
        (rho = 0), as the reference's examples write frames (examples/real_lbm3d_model.cpp:120-125)."""
        from .export import write_vtk_structured_3d

        s, f = self._export_field(field)
        c = self._config
        write_vtk_structured_3d(path, c.nx, c.ny, self._cells // (c.nx * c.ny), s,
                                (f.ux, f.uy, f.uz) if velocity else None,
                                (np.asarray(f.rho) == 0).astype(np.uint8) if solid else None, field, binary,
                                library=self._lib)

    def write_json_state(self, path, field: str = "speed", solid: bool = True):
        """The JSON live state of `field` at the current time step (reference write_json_state_3d)."""
        from .export import write_json_state_3d

        s, f = self._export_field(field)
        c = self._config
        write_json_state_3d(path, c.nx, c.ny, self._cells // (c.nx * c.ny), self.time_step(), s,
                            (np.asarray(f.rho) == 0).astype(np.uint8) if solid else None, field, library=self._lib)

    def set_wall_velocity(self, wall_id: int, ux: float, uy: float, uz: float):
        self._call("cfdx_lbm_set_wall_velocity", int(wall_id), ux, uy, uz)

    def set_solid_fraction(self, ns):
        """Gray-LBM partial bounce-back fraction n_s per cell (None clears)."""
        if ns is None:
            self._call("cfdx_lbm_set_solid_fraction", None, B.HOST)
            return
        ptr, where, _keep = self._pointer(ns, np.float32, self._cells, "solid fraction field")
        self._call("cfdx_lbm_set_solid_fraction", ptr, where)

    def set_storage_scale(self, scale=None):
        if scale is None:
            self._call("cfdx_lbm_set_storage_scale", None)
            return
        s = _host(scale, np.float32, self._q, "storage scale")
        self._call("cfdx_lbm_set_storage_scale", ctypes.c_void_p(s.ctypes.data))

    def set_launch_shape(self, block_x: int = 0, block_y: int = 0, variant: int = 0):
        """Threads per block and step-kernel variant (0 auto, 1 one cell, 2 paired cells,
        3 / 4 the wall-aware FP16 pair kernel with / without its shared-memory prefetch)."""
        self._call("cfdx_lbm_set_launch_shape", int(block_x), int(block_y), int(variant))

    def set_step_planes(self, planes: int = 0):
        """z-planes per thread of the z-marching FP16 pair kernel (0: default)."""
        self._call("cfdx_lbm_set_step_planes", int(planes))

    def save_checkpoint(self, path):
        """CFDCHK3 checkpoint of the current state (reference DistributedPullSolver::save_checkpoint)."""
        self._call("cfdx_lbm_checkpoint_save", str(path).encode())

    def load_checkpoint(self, path):
        """Restores a CFDCHK3 checkpoint written for this configuration (time step and populations)."""
        self._call("cfdx_lbm_checkpoint_load", str(path).encode())

    def set_tau(self, tau: float):
        """Symmetric relaxation time of the following steps (the adjoint's dJ/dtau variable)."""
        self._call("cfdx_lbm_set_tau", float(tau))
        self._config = dataclasses.replace(self._config, tau=float(tau))

    # ------------------------------------------------------ discrete adjoint
    def adjoint_forward(self, steps: int, interval: int = 64, subinterval: int = 0):
        """Run `steps` steps keeping a checkpoint every `interval` steps for adjoint_backward.

        `subinterval` m (2 <= m < interval) makes the reverse sweep recompute
        each segment in two levels, holding about interval/m + m lattice
        frames instead of interval - 1, at about twice the recompute steps;
        0 keeps one level.  The gradients are the same bit for bit.
        """
        self._call("cfdx_lbm_adjoint_set_subinterval", int(subinterval))
        self._call("cfdx_lbm_adjoint_forward", int(steps), int(interval))

    def adjoint_backward(self, g_ux, g_uy, g_uz, g_rho=None, grad_ns_out=None):
        """dJ/dn_s (per cell, float64) and dJ/dtau for dJ/du and dJ/drho of the final state.

        Seeds are host numpy arrays or CUDA tensors (N float32 each).  The
        n_s gradient is returned as a numpy array, or written into
        `grad_ns_out` (a float64 CUDA tensor of N elements) when given.
        """
        n = self._cells
        keep = []
        ptrs = []
        where = None
        for name, g in (("g_rho", g_rho), ("g_ux", g_ux), ("g_uy", g_uy), ("g_uz", g_uz)):
            if g is None:
                ptrs.append(None)
                continue
            if _is_device(g):
                g = g.float().contiguous()
            ptr, w, k = self._pointer(g, np.float32, n, name)
            if where is not None and w != where:
                raise ValueError("adjoint seeds must all be host arrays or all device tensors")
            where = w
            keep.append(k)
            ptrs.append(ptr)
        tau = ctypes.c_double()
        if grad_ns_out is not None:
            if not _is_device(grad_ns_out) or grad_ns_out.numel() != n or not grad_ns_out.is_contiguous():
                raise ValueError("grad_ns_out must be a contiguous CUDA tensor of N float64 values")
            self._call("cfdx_lbm_adjoint_backward", *ptrs, where, ctypes.c_void_p(grad_ns_out.data_ptr()), B.DEVICE,
                       ctypes.byref(tau))
            return grad_ns_out, tau.value
        out = np.zeros(n, np.float64)
        self._call("cfdx_lbm_adjoint_backward", *ptrs, where, ctypes.c_void_p(out.ctypes.data), B.HOST,
                   ctypes.byref(tau))
        return out, tau.value

    def adjoint_memory(self) -> int:
        n = ctypes.c_size_t()
        self._call("cfdx_lbm_adjoint_memory", ctypes.byref(n))
        return n.value

    def adjoint_release(self):
        self._call("cfdx_lbm_adjoint_release")

    def stream(self) -> int:
        p = ctypes.c_void_p()
        self._call("cfdx_lbm_stream", ctypes.byref(p))
        return p.value or 0

    def raw_populations(self) -> tuple[int, int]:
        p = ctypes.c_void_p()
        n = ctypes.c_size_t()
        self._call("cfdx_lbm_raw_populations", ctypes.byref(p), ctypes.byref(n))
        return p.value, n.value

    @property
    def handle(self):
        return self._h

    @property
    def library(self) -> B.SolverLibrary:
        return self._lib


def release_scratch(device: int = 0, library=None):
    """Return the unused memory of the library's per-device scratch pool to the driver
    (cfdx_release_scratch).  The voxelizer and the Q-criterion take their temporary buffers from
    that pool, which keeps up to 8 GiB mapped between calls."""
    lib = library or B.load()
    lib.call("cfdx_release_scratch", int(device))


def smagorinsky_k(cs: float) -> float:
    """Smagorinsky coefficient K = 18 sqrt(2) Cs^2 of tau_eff = (tau + sqrt(tau^2 + K sqrt(Q)/rho)) / 2."""
    return 18.0 * math.sqrt(2.0) * cs * cs


def trt_tau_minus(tau: float, magic: float = 3.0 / 16.0) -> float:
    """Antisymmetric relaxation time from the TRT magic parameter Lambda = (tau+ - 1/2)(tau- - 1/2)."""
    return 0.5 + magic / (tau - 0.5)


def cavity_flags(nx: int, ny: int, nz: int, lid_id: int = 2) -> np.ndarray:
    """Lid-driven cavity: walls on x=0, x=nx-1, y=0, z=0, z=nz-1 and a moving lid (id) on y=ny-1."""
    fl = np.zeros((nz, ny, nx), np.uint8)
    fl[:, :, 0] = B.WALL
    fl[:, :, nx - 1] = B.WALL
    fl[:, 0, :] = B.WALL
    fl[0, :, :] = B.WALL
    fl[nz - 1, :, :] = B.WALL
    fl[:, ny - 1, :] = lid_id
    return fl.reshape(-1)
