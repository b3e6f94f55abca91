"""Device-resident coupling to the flow: temperature, free surface, particles, diagnostics.

The reference couples its SYCL flow solver to resident transport solvers through two device
views: the macroscopic velocity the step produced (``refresh_device_macroscopic``) and a per-cell
acceleration field the step consumes (``device_local_acceleration``), so no field crosses the
host (include/cfd/solvers/lbm/esoteric_pull_sycl.hpp:218-372,
include/cfd/solvers/lbm/resident_multiphysics_sycl.hpp:51-200).  The engine exposes the same two
views; :class:`ResidentThermalD3Q7` is the reference's ``ResidentThermalD3Q7Sycl`` on them: a
two-grid D3Q7 advection-diffusion lattice (c_s^2 = 1/4, tau = 1/2 + 4 D) stepped with the flow's
device velocity on the flow's CUDA stream, with Boussinesq buoyancy added into the flow's
acceleration field.  :class:`ResidentFreeSurface3D`, :class:`ResidentParticles3D` and
:class:`ResidentFlowDiagnostics3D` are the reference's ``ResidentFreeSurfaceSycl3D``,
``ResidentParticlesSycl3D`` and ``ResidentFlowDiagnosticsSycl3D``
(resident_multiphysics_sycl.hpp:202-405) on the same views.
"""
from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np

from . import bindings as B
from .lbm import DeviceAccelerationView, DeviceMacroscopicView, DeviceTransferStats, EsotericPullCudaSolver


class ParticleVector3(NamedTuple):
    """A 3-vector (the reference's ParticleVector3, used for gravity)."""

    x: float
    y: float
    z: float


class ImmersedBoundaryParticle(NamedTuple):
    """A point particle (the reference's ImmersedBoundaryParticle, particles.hpp:13-18)."""

    position: ParticleVector3 = ParticleVector3(0.0, 0.0, 0.0)
    velocity: ParticleVector3 = ParticleVector3(0.0, 0.0, 0.0)
    mass: float = 1.0
    response_time: float = 1.0


class _Resident:
    """A handle of the C ABI borrowing `flow`'s device and stream; close it before the flow."""

    _prefix = ""

    def _open(self, flow: EsotericPullCudaSolver, create: str, *args):
        self._flow = flow
        self._lib = flow.library
        self._cells = flow.cells()
        self._h = None
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        self._lib.check(getattr(self._lib.raw, create)(flow.handle, *args, ctypes.byref(handle), err, len(err)), create)
        self._h = handle

    def close(self):
        if getattr(self, "_h", None):
            getattr(self._lib.raw, self._prefix + "destroy")(self._h)
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
            raise RuntimeError(f"{type(self).__name__} is closed")
        self._lib.call(self._prefix + name, self._h, *args)

    def _check_cells(self, view, message):
        if view.cells != self._cells:
            raise ValueError(message)

    def _info3(self):
        r, h2d, d2h = ctypes.c_size_t(), ctypes.c_uint64(), ctypes.c_uint64()
        self._call("info", ctypes.byref(r), ctypes.byref(h2d), ctypes.byref(d2h))
        return r.value, h2d.value, d2h.value


class ResidentFreeSurface3D(_Resident):
    """Fill fraction in [0, 1] on `flow`'s grid (reference ResidentFreeSurfaceSycl3D,
    resident_multiphysics_sycl.hpp:202-330): upwind advection by the device velocity, normals and
    curvature, surface-tension acceleration into the device force field, FP64 volume."""

    _prefix = "cfdx_surface_"

    def __init__(self, flow: EsotericPullCudaSolver):
        self._open(flow, "cfdx_surface_create")

    def initialize_uniform(self, fill: float):
        self._call("init_uniform", float(fill))

    def initialize_half_space_x(self, interface_x: float):
        self._call("init_half_space_x", float(interface_x))

    def initialize_field(self, fill):
        f = np.ascontiguousarray(fill, np.float32).reshape(-1)
        if f.size != self._cells:
            raise ValueError("fill field size mismatch")
        self._call("init_field", ctypes.c_void_p(f.ctypes.data), B.HOST)

    def advect(self, flow: DeviceMacroscopicView, dt: float):
        self._check_cells(flow, "invalid resident free-surface advection")
        self._call("advect", ctypes.c_void_p(flow.ux), ctypes.c_void_p(flow.uy), ctypes.c_void_p(flow.uz), float(dt))

    def fill_device(self) -> int:
        p = ctypes.c_void_p()
        self._call("device_fill", ctypes.byref(p))
        return p.value

    def refresh_geometry(self) -> int:
        """Recompute normals and curvature; the device pointer to [nx | ny | nz | curvature]."""
        p = ctypes.c_void_p()
        self._call("refresh_geometry", ctypes.byref(p))
        return p.value

    def add_surface_tension_acceleration(self, force: DeviceAccelerationView, surface_tension: float,
                                         density: float = 1.0):
        self._check_cells(force, "invalid resident surface-tension coupling")
        self._call("add_tension", ctypes.c_void_p(force.ax), ctypes.c_void_p(force.ay), ctypes.c_void_p(force.az),
                   float(surface_tension), float(density))

    def volume(self) -> float:
        out = ctypes.c_double()
        self._call("volume", ctypes.byref(out))
        return out.value

    def _copy(self, which: int) -> np.ndarray:
        out = np.zeros(self._cells, np.float32)
        self._call("fill", ctypes.c_void_p(out.ctypes.data), int(which), B.HOST)
        return out

    def fill(self) -> np.ndarray:
        return self._copy(0)

    def geometry(self) -> dict:
        """Normals and curvature of the last refresh_geometry / add_surface_tension_acceleration."""
        return {k: self._copy(i + 1) for i, k in enumerate(("normal_x", "normal_y", "normal_z", "curvature"))}

    def resident_bytes(self) -> int:
        return self._info3()[0]

    def transfer_stats(self) -> DeviceTransferStats:
        _, h2d, d2h = self._info3()
        return DeviceTransferStats(h2d, d2h, 0)


class ResidentParticles3D(_Resident):
    """Point particles on `flow`'s grid (reference ResidentParticlesSycl3D,
    resident_multiphysics_sycl.hpp:333-382): trilinear interpolation of the device velocity, drag
    m (u - v) / tau_p plus gravity, periodic positions, two-way drag spreading with atomics."""

    _prefix = "cfdx_particles_"

    def __init__(self, flow: EsotericPullCudaSolver, count: int):
        self._open(flow, "cfdx_particles_create", int(count))
        self._count = int(count)
        self._transfers = [0, 0]

    def __len__(self):
        return self._count

    def size(self) -> int:
        return self._count

    @staticmethod
    def _records(particles) -> np.ndarray:
        rows = [(*p.position, *p.velocity, p.mass, p.response_time) for p in particles]
        return np.ascontiguousarray(np.asarray(rows, np.float64).reshape(-1, 8))

    def upload(self, particles):
        recs = particles if isinstance(particles, np.ndarray) else self._records(particles)
        recs = np.ascontiguousarray(recs, np.float64).reshape(-1, 8)
        self._call("upload", ctypes.c_void_p(recs.ctypes.data), recs.shape[0])

    def download_records(self) -> np.ndarray:
        out = np.zeros((self._count, 8), np.float64)
        self._call("download", ctypes.c_void_p(out.ctypes.data), self._count)
        return out

    def download(self) -> list:
        return [ImmersedBoundaryParticle(ParticleVector3(*r[0:3]), ParticleVector3(*r[3:6]), float(r[6]), float(r[7]))
                for r in self.download_records()]

    def device_state(self) -> int:
        p = ctypes.c_void_p()
        self._call("device_state", ctypes.byref(p))
        return p.value

    def advance(self, flow: DeviceMacroscopicView, force: DeviceAccelerationView, dt: float, two_way: bool,
                gravity=ParticleVector3(0.0, 0.0, 0.0)):
        if flow.cells != self._cells or force.cells != flow.cells:
            raise ValueError("invalid resident particle coupling")
        gx, gy, gz = (float(v) for v in gravity)
        self._call("advance", ctypes.c_void_p(flow.ux), ctypes.c_void_p(flow.uy), ctypes.c_void_p(flow.uz),
                   ctypes.c_void_p(force.ax), ctypes.c_void_p(force.ay), ctypes.c_void_p(force.az), float(dt),
                   1 if two_way else 0, gx, gy, gz)

    def resident_bytes(self) -> int:
        return self._info3()[0]

    def transfer_stats(self) -> DeviceTransferStats:
        _, h2d, d2h = self._info3()
        return DeviceTransferStats(h2d - self._transfers[0], d2h - self._transfers[1], 0)

    def reset_transfer_stats(self):
        _, h2d, d2h = self._info3()
        self._transfers = [h2d, d2h]


class ResidentFlowDiagnostics3D(_Resident):
    """FP32 Q-criterion of a device velocity (reference ResidentFlowDiagnosticsSycl3D,
    resident_multiphysics_sycl.hpp:384-405)."""

    _prefix = "cfdx_diagnostics_"

    def __init__(self, flow: EsotericPullCudaSolver):
        self._open(flow, "cfdx_diagnostics_create")

    def q_criterion(self, flow: DeviceMacroscopicView) -> int:
        """Device pointer to Q (owned by the handle, overwritten by the next call)."""
        self._check_cells(flow, "diagnostic/flow lattice size mismatch")
        p = ctypes.c_void_p()
        self._call("q_criterion", ctypes.c_void_p(flow.ux), ctypes.c_void_p(flow.uy), ctypes.c_void_p(flow.uz),
                   ctypes.byref(p))
        return p.value

    def resident_bytes(self) -> int:
        r = ctypes.c_size_t()
        self._call("info", ctypes.byref(r))
        return r.value


class ResidentThermalD3Q7:
    """Temperature lattice on `flow`'s grid, device and stream (reference ResidentThermalD3Q7Sycl).

    Destroy it (``close``) before its flow solver.
    """

    def __init__(self, flow: EsotericPullCudaSolver, diffusivity: float = 0.01):
        self._flow = flow
        self._lib = flow.library
        self._cells = flow.cells()
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        self._h = None
        self._lib.check(self._lib.raw.cfdx_thermal_create(flow.handle, float(diffusivity), ctypes.byref(handle), err,
                                                          len(err)), "cfdx_thermal_create")
        self._h = handle
        self.diffusivity = float(diffusivity)

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.raw.cfdx_thermal_destroy(self._h)
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
            raise RuntimeError("thermal lattice is closed")
        self._lib.call(name, self._h, *args)

    # ------------------------------------------------------------ reference API
    def initialize_uniform(self, temperature: float):
        self._call("cfdx_thermal_init_uniform", float(temperature))

    def initialize_field(self, temperature):
        t = np.ascontiguousarray(temperature, np.float32).reshape(-1)
        if t.size != self._cells:
            raise ValueError("temperature field size mismatch")
        self._call("cfdx_thermal_init_field", ctypes.c_void_p(t.ctypes.data), B.HOST)

    def step(self, flow: DeviceMacroscopicView, count: int = 1):
        """`count` steps advected by the device velocity of `flow` (refresh_device_macroscopic())."""
        if flow.cells != self._cells:
            raise ValueError("thermal/flow lattice size mismatch")
        self._call("cfdx_thermal_step", ctypes.c_void_p(flow.ux), ctypes.c_void_p(flow.uy), ctypes.c_void_p(flow.uz),
                   int(count))

    def refresh_device_scalar(self) -> int:
        """Device pointer to the temperature field (owned by the lattice)."""
        p = ctypes.c_void_p()
        self._call("cfdx_thermal_refresh_device_scalar", ctypes.byref(p))
        return p.value

    def temperature(self) -> np.ndarray:
        out = np.zeros(self._cells, np.float32)
        self._call("cfdx_thermal_temperature", ctypes.c_void_p(out.ctypes.data), B.HOST)
        return out

    def add_boussinesq_acceleration(self, force: DeviceAccelerationView, reference_temperature: float, beta: float,
                                    gravity):
        """force += -beta (T - T_ref) * gravity, per cell, on the device."""
        if force.cells != self._cells:
            raise ValueError("invalid resident Boussinesq coupling")
        gx, gy, gz = (float(v) for v in gravity)
        self._call("cfdx_thermal_add_boussinesq", ctypes.c_void_p(force.ax), ctypes.c_void_p(force.ay),
                   ctypes.c_void_p(force.az), float(reference_temperature), float(beta), gx, gy, gz)

    def total_scalar(self) -> float:
        out = ctypes.c_double()
        self._call("cfdx_thermal_total", ctypes.byref(out))
        return out.value

    def _info(self):
        r, h2d, d2h = ctypes.c_size_t(), ctypes.c_uint64(), ctypes.c_uint64()
        self._call("cfdx_thermal_info", ctypes.byref(r), ctypes.byref(h2d), ctypes.byref(d2h))
        return r.value, h2d.value, d2h.value

    def resident_bytes(self) -> int:
        return self._info()[0]

    def transfer_stats(self) -> DeviceTransferStats:
        _, h2d, d2h = self._info()
        return DeviceTransferStats(h2d, d2h, 0)


__all__ = ["ImmersedBoundaryParticle", "ParticleVector3", "ResidentFlowDiagnostics3D", "ResidentFreeSurface3D",
           "ResidentParticles3D", "ResidentThermalD3Q7"]
