"""Generates tests/golden/voxel_fixtures.npz from the REFERENCE voxelizer itself.

Every mask here is the output of the reference's cfd::lbm::voxelize_surface
(src/lbm/voxelize.cpp:4-5), and every transformed surface the output of its
transform_surface (:6), compiled from its sources by oracle/Makefile into
oracle/_ref/libcfdref.so (bit-exact build, -ffp-contract=off).  The fixtures
pin the CPU oracle (tests/test_voxelize_oracle.py) and the CUDA voxelizer
(tests/test_gpu_voxelize.py) where the reference is not present.

Run from the repository root after ``make -C oracle``:
    python tests/golden/make_voxel_fixtures.py

The inputs are synthetic surfaces built by cfd_solvers_b200.geometry:
  cube8            the box [.25, .75]^3 on 8^3 over the unit box (the shape of the
                   reference's own voxelizer test, tests/test_completion.cpp:885-901)
  knife_edge       the box [.125, .875]^3 on 4^3: box faces pass through cell
                   centres, so rays start on the surface (distance 0 is no hit)
  sphere           an icosphere (2 subdivisions) on 24 x 20 x 18 over a skewed box
  torus            a 48 x 24 torus on 32 x 32 x 16
  moved_cube       the cube rotated 0.3 rad about (1, 1, 0.5) and shifted by
                   (0.05, -0.02, 0.03) with the reference's transform_surface
  open_and_flat    one open triangle plus two zero-area triangles (parity of
                   an open surface; degenerate triangles never hit)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cfd_solvers_b200 import geometry as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "voxel_fixtures.npz"


def cases():
    cube = G.box_surface((0.25, 0.25, 0.25), (0.75, 0.75, 0.75))
    yield "cube8", cube, (8, 8, 8), (0, 0, 0), (1, 1, 1)
    yield "knife_edge", G.box_surface((0.125,) * 3, (0.875,) * 3), (4, 4, 4), (0, 0, 0), (1, 1, 1)
    yield ("sphere", G.icosphere((0.41, 0.52, 0.47), 0.33, 2), (24, 20, 18), (0.0, 0.05, -0.1),
           (1.0, 1.02, 0.95))
    yield "torus", G.torus((0.5, 0.5, 0.5), 0.3, 0.12, 48, 24), (32, 32, 16), (0, 0, 0.2), (1, 1, 0.8)
    moved = O.ref_transform_surface(cube, (0.05, -0.02, 0.03), (1.0, 1.0, 0.5), 0.3)
    yield "moved_cube", moved, (16, 16, 16), (0, 0, 0), (1, 1, 1)
    flat = np.array([[0.5, 0.1, 0.1, 0.5, 0.9, 0.2, 0.5, 0.3, 0.9],      # open triangle in the plane x = 0.5
                     [0.2, 0.2, 0.2, 0.4, 0.4, 0.4, 0.6, 0.6, 0.6],      # collinear: zero area
                     [0.3, 0.3, 0.3, 0.3, 0.3, 0.3, 0.7, 0.2, 0.5]], np.float64)  # repeated vertex
    yield "open_and_flat", flat, (10, 9, 8), (0, 0, 0), (1, 1, 1)


def main():
    if not O.reference_available():
        raise SystemExit("oracle/_ref/libcfdref.so is not built (run `make -C oracle` where the reference is present)")
    arrays, meta = {}, {}
    for name, tris, (nx, ny, nz), lo, hi in cases():
        tris = np.ascontiguousarray(tris, np.float64).reshape(-1, 9)
        mask = O.ref_voxelize(tris, nx, ny, nz, lo, hi)
        arrays[f"{name}_tris"] = tris
        arrays[f"{name}_mask"] = mask
        meta[name] = {"grid": [nx, ny, nz], "minimum": list(map(float, lo)), "maximum": list(map(float, hi)),
                      "triangles": int(len(tris)), "solid_cells": int(mask.sum())}
    cube = G.box_surface((0.25, 0.25, 0.25), (0.75, 0.75, 0.75))
    arrays["transform_in"] = cube
    arrays["transform_out"] = O.ref_transform_surface(cube, (0.05, -0.02, 0.03), (1.0, 1.0, 0.5), 0.3)
    arrays["transform_zero_axis"] = O.ref_transform_surface(cube, (0.1, 0.2, 0.3), (0.0, 0.0, 0.0), 1.0)
    arrays["meta"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
