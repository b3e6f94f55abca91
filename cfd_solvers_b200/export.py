"""Field export: legacy VTK, the JSON live state and the Q-criterion.

Mirrors the reference's LBM visualisation surface (include/cfd/solvers/lbm/visualization.hpp:14-22,
src/lbm/visualization.cpp:39-148) with the reference's function names.  The writers are
the native ones of libcfdx_lbm.so (``cfdx_write_vtk_3d`` / ``cfdx_write_json_state_3d``;
ASCII output equals the reference's byte for byte, ``binary=True`` writes the big-endian
binary legacy format for large lattices); the Q-criterion runs on the GPU
(``cfdx_q_criterion``; equal to the reference's bit for bit).
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Optional

import numpy as np

from . import bindings as B


def _velocity(velocity, cells: int) -> Optional[np.ndarray]:
    """(cells, 3) float64 C-contiguous, from (cells, 3) or a (ux, uy, uz) triple."""
    if velocity is None:
        return None
    if isinstance(velocity, (tuple, list)) and len(velocity) == 3:
        v = np.stack([np.asarray(c, np.float64).reshape(-1) for c in velocity], axis=1)
    else:
        v = np.asarray(velocity, np.float64).reshape(-1, 3)
    if v.shape[0] != cells:
        raise ValueError("LBM 3-D VTK field size mismatch")
    return np.ascontiguousarray(v)


def write_vtk_structured_3d(path, nx: int, ny: int, nz: int, scalar, velocity=None, solid=None,
                            scalar_name: str = "field", binary: bool = False, library=None):
    """Legacy-VTK structured points: one scalar, optional velocity and solid flags (reference :39-67)."""
    lib = library or B.load()
    cells = nx * ny * nz
    s = np.ascontiguousarray(scalar, np.float64).reshape(-1)
    if s.size != cells:
        raise ValueError("LBM 3-D VTK field size mismatch")
    v = _velocity(velocity, cells)
    m = None if solid is None else np.ascontiguousarray(solid, np.uint8).reshape(-1)
    if m is not None and m.size != cells:
        raise ValueError("LBM 3-D VTK field size mismatch")
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    lib.call("cfdx_write_vtk_3d", str(path).encode(), nx, ny, nz, ctypes.c_void_p(s.ctypes.data),
             None if v is None else ctypes.c_void_p(v.ctypes.data),
             None if m is None else ctypes.c_void_p(m.ctypes.data), scalar_name.encode(), int(bool(binary)))


def write_json_state_3d(path, nx: int, ny: int, nz: int, step: int, scalar, solid=None, scalar_name: str = "field",
                        library=None):
    """The JSON live state, published through a temporary file (reference :68-109)."""
    lib = library or B.load()
    cells = nx * ny * nz
    s = np.ascontiguousarray(scalar, np.float64).reshape(-1)
    m = None if solid is None else np.ascontiguousarray(solid, np.uint8).reshape(-1)
    if s.size != cells or (m is not None and m.size != cells):
        raise ValueError("LBM 3-D live state size mismatch")
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    lib.call("cfdx_write_json_state_3d", str(path).encode(), nx, ny, nz, int(step), ctypes.c_void_p(s.ctypes.data),
             None if m is None else ctypes.c_void_p(m.ctypes.data), scalar_name.encode())


def q_criterion_3d(nx: int, ny: int, nz: int, velocity, dx: float = 1.0, dy: float = 1.0, dz: float = 1.0,
                   device: int = 0, out=None, library=None):
    """Q = (|Omega|^2 - |S|^2) / 2 with central differences, 0 on the outer layer (reference :122-148).

    `velocity` is (cells, 3) / a (ux, uy, uz) triple on the host, or a (cells, 3) CUDA
    tensor; the result is a float64 numpy array, or `out` (a float64 CUDA tensor).
    """
    lib = library or B.load()
    cells = nx * ny * nz
    on_device = hasattr(velocity, "data_ptr") and velocity.device.type == "cuda"
    if on_device:
        import torch

        v = velocity.to(torch.float64).contiguous().reshape(-1, 3)
        if v.shape[0] != cells:
            raise ValueError("invalid LBM Q-criterion grid")
        q = out if out is not None else torch.empty(cells, dtype=torch.float64, device=v.device)
        torch.cuda.current_stream(v.device).synchronize()
        lib.call("cfdx_q_criterion", ctypes.c_void_p(v.data_ptr()), nx, ny, nz, dx, dy, dz,
                 ctypes.c_void_p(q.data_ptr()), B.DEVICE, v.device.index or 0)
        return q
    v = _velocity(velocity, cells)
    q = np.zeros(cells, np.float64)
    lib.call("cfdx_q_criterion", ctypes.c_void_p(v.ctypes.data), nx, ny, nz, dx, dy, dz, ctypes.c_void_p(q.ctypes.data),
             B.HOST, int(device))
    return q


def speed(fields) -> np.ndarray:
    """|u| per cell in FP64 from float fields, as the reference's examples compute it
    (tests/test_real_3d_model.cpp:49-51)."""
    ux, uy, uz = (np.asarray(c).astype(np.float64) for c in (fields.ux, fields.uy, fields.uz))
    return np.sqrt(ux * ux + uy * uy + uz * uz)


__all__ = ["q_criterion_3d", "speed", "write_json_state_3d", "write_vtk_structured_3d"]
