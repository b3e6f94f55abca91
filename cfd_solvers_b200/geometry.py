"""Triangle surfaces -> lattice flags: readers, transforms and the device voxelizer.

The reference feeds real geometries into its LBM solver through
``cfd::io::read_ascii_stl`` / ``read_obj_triangles`` (src/io/mesh_io.cpp:17-18),
``cfd::lbm::transform_surface`` and ``voxelize_surface`` (src/lbm/voxelize.cpp:4-6),
then ``set_solid_mask`` (examples/real_lbm3d_model.cpp:146-150).  Here a surface is
a float64 array of shape (triangles, 9) -- vertices a, b, c -- and the voxelizer
runs on the GPU (``cfdx_voxelize`` in libcfdx_lbm.so; its mask equals the
reference CPU voxelizer's bit for bit).  Readers and transforms are host code.
"""
from __future__ import annotations

import ctypes
import math
import struct
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import bindings as B


@dataclass(frozen=True)
class VoxelGrid3D:
    """nx x ny x nz cells over the box [minimum, maximum] (reference VoxelGrid3D, voxelize.hpp:8)."""

    nx: int
    ny: int
    nz: int
    minimum: tuple = (0.0, 0.0, 0.0)
    maximum: tuple = (1.0, 1.0, 1.0)

    def c_struct(self) -> B.cfdx_voxel_grid:
        g = B.cfdx_voxel_grid()
        g.nx, g.ny, g.nz = int(self.nx), int(self.ny), int(self.nz)
        for k in range(3):
            g.minimum[k] = float(self.minimum[k])
            g.maximum[k] = float(self.maximum[k])
        return g


def as_surface(triangles) -> np.ndarray:
    """(count, 9) float64 C-contiguous view of a triangle array ((count, 3, 3) or flat)."""
    t = np.ascontiguousarray(triangles, dtype=np.float64)
    if t.size % 9:
        raise ValueError("a surface is a multiple of 9 coordinates (triangles a, b, c)")
    return t.reshape(-1, 9)


# ------------------------------------------------------------------ readers
def read_ascii_stl(path) -> np.ndarray:
    """Triangles of an ASCII STL: every three ``vertex x y z`` form one (reference mesh_io.cpp:18).

    Raises ValueError when the vertex count is not a multiple of three (the reference's
    "malformed ASCII STL").
    """
    tokens = Path(path).read_text().split()
    verts = []
    i = 0
    while i < len(tokens):
        if tokens[i] == "vertex":
            verts.append(tuple(float(v) for v in tokens[i + 1:i + 4]))
            i += 4
        else:
            i += 1
    if len(verts) % 3:
        raise ValueError(f"malformed ASCII STL: {path}")
    return np.asarray(verts, np.float64).reshape(-1, 9)


def read_binary_stl(path) -> np.ndarray:
    """Triangles of a binary STL (80-byte header, u32 count, 50 bytes per facet)."""
    data = Path(path).read_bytes()
    if len(data) < 84:
        raise ValueError(f"truncated binary STL: {path}")
    (count,) = struct.unpack_from("<I", data, 80)
    if len(data) < 84 + 50 * count:
        raise ValueError(f"truncated binary STL: {path}")
    rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("attr", "<u2")]),
                        count=count, offset=84)
    return rec["v"].astype(np.float64)


def read_stl(path) -> np.ndarray:
    """ASCII or binary STL (binary when the size matches its facet count)."""
    data = Path(path).read_bytes()
    if len(data) >= 84:
        (count,) = struct.unpack_from("<I", data, 80)
        if len(data) == 84 + 50 * count:
            return read_binary_stl(path)
    return read_ascii_stl(path)


def read_obj_triangles(path) -> np.ndarray:
    """Triangles of an OBJ file's ``v`` / ``f`` records (first three indices of a face; reference mesh_io.cpp:17)."""
    verts = []
    tris = []
    for line in Path(path).read_text().splitlines():
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "v":
            verts.append(tuple(float(v) for v in parts[1:4]))
        elif parts[0] == "f":
            idx = []
            for tok in parts[1:4]:
                i = int(tok.split("/")[0])
                if i <= 0 or i > len(verts):
                    raise ValueError("OBJ index out of range")
                idx.append(i - 1)
            tris.append(verts[idx[0]] + verts[idx[1]] + verts[idx[2]])
    return np.asarray(tris, np.float64).reshape(-1, 9)


def write_ascii_stl(path, triangles, name: str = "surface"):
    """Writes an ASCII STL (facet normals from the vertex order)."""
    t = as_surface(triangles).reshape(-1, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    norm = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.divide(n, norm, out=np.zeros_like(n), where=norm > 0)
    lines = [f"solid {name}"]
    for tri, nn in zip(t, n):
        lines.append(f"  facet normal {nn[0]:.17g} {nn[1]:.17g} {nn[2]:.17g}")
        lines.append("    outer loop")
        for v in tri:
            lines.append(f"      vertex {v[0]:.17g} {v[1]:.17g} {v[2]:.17g}")
        lines.append("    endloop")
        lines.append("  endfacet")
    lines.append(f"endsolid {name}")
    Path(path).write_text("\n".join(lines) + "\n")


# ------------------------------------------------------------------ transforms
def transform_surface(triangles, translation=(0.0, 0.0, 0.0), axis=(0.0, 0.0, 1.0), angle: float = 0.0):
    """Rotation about `axis` (through the origin) by `angle` radians, then translation.

    Reference transform_surface (src/lbm/voxelize.cpp:6): Rodrigues' formula
    p c + (k x p) s + k (k . p)(1 - c) with k = axis/|axis| (a zero axis leaves p),
    evaluated in the reference's operation order.
    """
    p = as_surface(triangles).reshape(-1, 3)
    ax = np.asarray(axis, np.float64)
    tr = np.asarray(translation, np.float64)
    n = math.sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2])
    if n < 1e-30:
        r = p.copy()
    else:
        k = ax * (1.0 / n)
        c, s = math.cos(angle), math.sin(angle)
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        kx, ky, kz = k
        cross = np.stack([ky * z - kz * y, kz * x - kx * z, kx * y - ky * x], axis=1)
        kp = (kx * x + ky * y) + kz * z
        r = (p * c + cross * s) + np.outer(kp * (1.0 - c), np.ones(3)) * k
    return (r + tr).reshape(-1, 9)


def fit_to_box(triangles, minimum=(0.0, 0.0, 0.0), maximum=(1.0, 1.0, 1.0), margin: float = 0.1):
    """Uniformly scales and centres a surface into the box, leaving `margin` of each extent free."""
    t = as_surface(triangles).reshape(-1, 3)
    lo, hi = t.min(axis=0), t.max(axis=0)
    size = np.maximum(hi - lo, 1e-300)
    box_lo, box_hi = np.asarray(minimum, np.float64), np.asarray(maximum, np.float64)
    scale = float(np.min((box_hi - box_lo) * (1.0 - 2.0 * margin) / size))
    centre = (box_lo + box_hi) / 2.0
    return ((t - (lo + hi) / 2.0) * scale + centre).reshape(-1, 9)


# ------------------------------------------------------------------ shapes
def box_surface(lo, hi) -> np.ndarray:
    """Closed axis-aligned box (12 triangles)."""
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x0, y1, z0], [x1, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x0, y1, z1], [x1, y1, z1]], np.float64)
    faces = [(0, 3, 1), (0, 2, 3), (4, 5, 7), (4, 7, 6), (0, 1, 5), (0, 5, 4),
             (2, 6, 7), (2, 7, 3), (0, 4, 6), (0, 6, 2), (1, 3, 7), (1, 7, 5)]
    return np.concatenate([v[list(f)].reshape(1, 9) for f in faces])


def icosphere(centre=(0.5, 0.5, 0.5), radius: float = 0.25, subdivisions: int = 3) -> np.ndarray:
    """Closed sphere: an icosahedron subdivided `subdivisions` times (20 * 4^s triangles)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.asarray(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        new = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new
    v = np.asarray(verts) * radius + np.asarray(centre, np.float64)
    return np.concatenate([v[list(f)].reshape(1, 9) for f in faces])


def torus(centre=(0.5, 0.5, 0.5), major: float = 0.3, minor: float = 0.1, nu: int = 48, nv: int = 24) -> np.ndarray:
    """Closed torus around the z axis (2 nu nv triangles)."""
    u = np.linspace(0, 2 * np.pi, nu, endpoint=False)
    w = np.linspace(0, 2 * np.pi, nv, endpoint=False)
    uu, ww = np.meshgrid(u, w, indexing="ij")
    pts = np.stack([(major + minor * np.cos(ww)) * np.cos(uu), (major + minor * np.cos(ww)) * np.sin(uu),
                    minor * np.sin(ww)], axis=-1) + np.asarray(centre, np.float64)
    tris = []
    for i in range(nu):
        for j in range(nv):
            a, b = pts[i, j], pts[(i + 1) % nu, j]
            c, d = pts[(i + 1) % nu, (j + 1) % nv], pts[i, (j + 1) % nv]
            tris.append(np.concatenate([a, b, c]))
            tris.append(np.concatenate([a, c, d]))
    return np.asarray(tris)


# ------------------------------------------------------------------ voxelizer
def voxelize_surface(triangles, grid: VoxelGrid3D, device: int = 0, z_first: int = 0, z_count: Optional[int] = None,
                     value: int = 1, out=None, library=None):
    """Solid mask of a surface on `grid` (reference voxelize_surface), computed on the GPU.

    Returns a uint8 numpy array of nx*ny*z_count cells (1 or `value` inside, 0
    outside) covering global planes z_first .. z_first + z_count - 1 (mod nz),
    or fills `out` (a uint8 CUDA tensor of that many elements) in place.
    """
    lib = library or B.load()
    t = as_surface(triangles)
    zc = grid.nz if z_count is None else int(z_count)
    n = grid.nx * grid.ny * zc
    g = grid.c_struct()
    if out is not None:
        if not hasattr(out, "data_ptr") or out.device.type != "cuda" or out.numel() != n:
            raise ValueError(f"out must be a CUDA tensor of {n} uint8 cells")
        lib.check(lib.raw.cfdx_voxelize(ctypes.c_void_p(t.ctypes.data), len(t), ctypes.byref(g), int(z_first), zc,
                                        int(value), ctypes.c_void_p(out.data_ptr()), B.DEVICE,
                                        out.device.index or 0), "cfdx_voxelize")
        return out
    mask = np.zeros(n, np.uint8)
    lib.check(lib.raw.cfdx_voxelize(ctypes.c_void_p(t.ctypes.data), len(t), ctypes.byref(g), int(z_first), zc,
                                    int(value), ctypes.c_void_p(mask.ctypes.data), B.HOST, int(device)),
              "cfdx_voxelize")
    return mask


__all__ = [
    "VoxelGrid3D",
    "as_surface",
    "box_surface",
    "fit_to_box",
    "icosphere",
    "read_ascii_stl",
    "read_binary_stl",
    "read_obj_triangles",
    "read_stl",
    "torus",
    "transform_surface",
    "voxelize_surface",
    "write_ascii_stl",
]
