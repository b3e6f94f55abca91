"""Synthetic case builders for the benchmark configurations.

The reference's case surface is ``cfd-solve`` / ``cfd-bench`` (apps/cfd-solve.cpp:163-222,
apps/cfd-bench.cpp:173-233); these helpers build the lattices those cases and
the north-star configurations describe, seeded so every run is reproducible:

* :func:`cavity_flags`           lid-driven cavity (re-exported from :mod:`.lbm`);
* :func:`channel_flags`          periodic in x, no-slip walls on the y and z faces;
* :func:`sphere_pack`            seeded random spheres (radii uniform in [rmin, rmax])
                                 filling a target solid fraction, inside a channel;
* :func:`gray_field`             seeded per-cell gray-LBM solid fraction, uniform in [lo, hi).

All return numpy arrays in the engine's cell order n = (z*ny + y)*nx + x.
"""
from __future__ import annotations

import numpy as np

from .lbm import cavity_flags

__all__ = ["cavity_flags", "channel_flags", "sphere_pack", "gray_field"]


def channel_flags(nx: int, ny: int, nz: int) -> np.ndarray:
    """Stationary walls (flag 1) on y = 0, y = ny-1, z = 0, z = nz-1; periodic in x."""
    f = np.zeros((nz, ny, nx), np.uint8)
    f[:, 0, :] = 1
    f[:, ny - 1, :] = 1
    f[0, :, :] = 1
    f[nz - 1, :, :] = 1
    return f.reshape(-1)


def sphere_pack(nx: int, ny: int, nz: int, fraction: float = 0.10, rmin: float = 4.0, rmax: float = 12.0,
                seed: int = 1, walls: bool = True) -> np.ndarray:
    """Flags of a channel (if `walls`) with seeded random solid spheres.

    Sphere centres are uniform over the box (periodic in x: spheres wrap in x)
    and radii uniform in [rmin, rmax]; spheres are added until the solid
    fraction of the interior reaches `fraction`.
    """
    rng = np.random.default_rng(seed)
    solid = np.zeros((nz, ny, nx), bool)
    target = fraction * nx * ny * nz
    z, y, x = np.ogrid[:nz, :ny, :nx]
    count = 0
    while count < target:
        r = rng.uniform(rmin, rmax)
        cx, cy, cz = rng.uniform(0, nx), rng.uniform(0, ny), rng.uniform(0, nz)
        # bounding box of the sphere (x wraps)
        z0, z1 = max(0, int(cz - r) - 1), min(nz, int(cz + r) + 2)
        y0, y1 = max(0, int(cy - r) - 1), min(ny, int(cy + r) + 2)
        dx = np.abs(x + 0.5 - cx)
        dx = np.minimum(dx, nx - dx)
        d2 = dx ** 2 + (y[:, y0:y1] + 0.5 - cy) ** 2 + (z[z0:z1] + 0.5 - cz) ** 2
        inside = d2 <= r * r
        block = solid[z0:z1, y0:y1, :]
        count += int(np.count_nonzero(inside & ~block))
        block |= inside
    flags = solid.astype(np.uint8).reshape(-1)
    if walls:
        flags = np.maximum(flags, channel_flags(nx, ny, nz))
    return flags


def gray_field(cells: int, seed: int, lo: float = 0.0, hi: float = 0.2) -> np.ndarray:
    """Per-cell gray-LBM solid fraction, uniform in [lo, hi) from `seed` (float32)."""
    return np.random.default_rng(seed).uniform(lo, hi, cells).astype(np.float32)
