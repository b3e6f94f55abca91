"""Device-resident coupling to the flow: the D3Q7 temperature lattice.

The reference couples its SYCL flow solver to resident transport solvers through two device
views: the macroscopic velocity the step produced (``refresh_device_macroscopic``) and a per-cell
acceleration field the step consumes (``device_local_acceleration``), so no field crosses the
host (include/cfd/solvers/lbm/esoteric_pull_sycl.hpp:218-372,
include/cfd/solvers/lbm/resident_multiphysics_sycl.hpp:51-200).  The engine exposes the same two
views; :class:`ResidentThermalD3Q7` is the reference's ``ResidentThermalD3Q7Sycl`` on them: a
two-grid D3Q7 advection-diffusion lattice (c_s^2 = 1/4, tau = 1/2 + 4 D) stepped with the flow's
device velocity on the flow's CUDA stream, with Boussinesq buoyancy added into the flow's
acceleration field.
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


__all__ = ["ParticleVector3", "ResidentThermalD3Q7"]
