"""The voxelizer oracle, the geometry host code and the voxelizer ABI, without a GPU.

* the C oracle (oracle/voxel_oracle.c) reproduces the reference voxelizer's
  masks and transforms stored in tests/golden/voxel_fixtures.npz bit for bit
  (box, knife-edge box, sphere, torus, transformed box, open and degenerate
  triangles);
* cfd_solvers_b200.geometry.transform_surface (host code of the product)
  reproduces the reference's transform_surface bit for bit;
* STL (ASCII, binary) and OBJ readers; the reference's malformed-STL error;
* with the reference compiled here (oracle/_ref): oracle == reference on random
  rotated surfaces, and the reference's own Ahmed-body model
  (tests/test_real_3d_model.cpp:29-40: 18 triangles, a bounded solid);
* the C ABI rejects the inputs the reference rejects before touching a device.
"""
from __future__ import annotations

import ctypes
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from cfd_solvers_b200 import bindings as B
from cfd_solvers_b200 import geometry as G

GOLDEN = Path(__file__).resolve().parent / "golden" / "voxel_fixtures.npz"
REF_MODEL = Path("/root/reference/examples/models/ahmed_body.stl")


@pytest.fixture(scope="module")
def fixtures():
    data = np.load(GOLDEN)
    return data, json.loads(bytes(data["meta"]).decode())


def test_oracle_matches_reference_masks(oracle_mod, fixtures):
    data, meta = fixtures
    assert set(meta) == {"cube8", "knife_edge", "sphere", "torus", "moved_cube", "open_and_flat"}
    for name, m in meta.items():
        nx, ny, nz = m["grid"]
        got = oracle_mod.voxelize(data[f"{name}_tris"], nx, ny, nz, m["minimum"], m["maximum"])
        assert np.array_equal(got, data[f"{name}_mask"]), name
        assert int(got.sum()) == m["solid_cells"]


def test_reference_cube_facts(fixtures):
    """The reference test's own assertions (tests/test_completion.cpp:896-901)."""
    data, _ = fixtures
    mask = data["cube8_mask"].reshape(8, 8, 8)
    assert mask[4, 4, 4] == 1 and mask[0, 0, 0] == 0
    assert not np.array_equal(data["moved_cube_mask"], np.zeros(16 ** 3, np.uint8))


def test_transforms_match_reference(oracle_mod, fixtures):
    data, _ = fixtures
    cube = data["transform_in"]
    expect = data["transform_out"]
    assert np.array_equal(oracle_mod.transform_surface(cube, (0.05, -0.02, 0.03), (1.0, 1.0, 0.5), 0.3), expect)
    assert np.array_equal(G.transform_surface(cube, (0.05, -0.02, 0.03), (1.0, 1.0, 0.5), 0.3), expect)
    assert np.array_equal(G.transform_surface(cube, (0.1, 0.2, 0.3), (0.0, 0.0, 0.0), 1.0),
                          data["transform_zero_axis"])


def test_shapes_are_closed_and_sized():
    for t in (G.box_surface((0, 0, 0), (1, 2, 3)), G.icosphere(subdivisions=2), G.torus(nu=12, nv=8)):
        tri = t.reshape(-1, 3, 3)
        edges = {}
        for a, b, c in tri:
            for p, q in ((a, b), (b, c), (c, a)):
                key = tuple(sorted((tuple(np.round(p, 12)), tuple(np.round(q, 12)))))
                edges[key] = edges.get(key, 0) + 1
        assert set(edges.values()) == {2}  # every edge shared by two triangles
    assert len(G.icosphere(subdivisions=3)) == 20 * 64
    assert len(G.torus(nu=10, nv=6)) == 120


def test_stl_and_obj_readers(tmp_path):
    t = G.icosphere(subdivisions=1)
    G.write_ascii_stl(tmp_path / "s.stl", t)
    assert np.array_equal(G.read_ascii_stl(tmp_path / "s.stl"), t)
    assert np.array_equal(G.read_stl(tmp_path / "s.stl"), t)
    # binary STL
    rec = np.zeros(len(t), dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("attr", "<u2")]))
    rec["v"] = t.astype(np.float32)
    (tmp_path / "b.stl").write_bytes(b"\0" * 80 + struct.pack("<I", len(t)) + rec.tobytes())
    assert np.array_equal(G.read_stl(tmp_path / "b.stl"), t.astype(np.float32).astype(np.float64))
    # OBJ with v/vt/vn face tokens and a quad (first three indices)
    (tmp_path / "m.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1/1/1 2/2/2 3/3/3\nf 1 2 4 3\n")
    o = G.read_obj_triangles(tmp_path / "m.obj")
    assert o.shape == (2, 9) and list(o[1]) == [0, 0, 0, 1, 0, 0, 0, 0, 1]
    (tmp_path / "bad.obj").write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(ValueError):
        G.read_obj_triangles(tmp_path / "bad.obj")
    (tmp_path / "bad.stl").write_text("solid x\n vertex 0 0 0\n vertex 1 0 0\nendsolid\n")
    with pytest.raises(ValueError):
        G.read_ascii_stl(tmp_path / "bad.stl")


def test_fit_to_box():
    t = G.fit_to_box(G.box_surface((10, 20, 30), (12, 21, 34)), (0, 0, 0), (1, 1, 1), margin=0.1)
    p = t.reshape(-1, 3)
    assert p.min() >= 0.1 - 1e-12 and p.max() <= 0.9 + 1e-12
    assert np.isclose(np.ptp(p[:, 2]), 0.8)


def test_abi_rejects_invalid_inputs():
    lib = B.load()
    t = G.box_surface((0.2,) * 3, (0.8,) * 3)
    g = G.VoxelGrid3D(4, 4, 4).c_struct()
    out = np.zeros(64, np.uint8)

    def call(tris, count, grid, z0=0, zc=4):
        return lib.raw.cfdx_voxelize(ctypes.c_void_p(tris.ctypes.data), count, ctypes.byref(grid), z0, zc, 1,
                                     ctypes.c_void_p(out.ctypes.data), B.HOST, 0)

    assert call(t, 0, g) == B.ERR_INVALID                       # no triangles
    bad = G.VoxelGrid3D(4, 4, 4, (0, 0, 0), (1, 0, 1)).c_struct()
    assert call(t, len(t), bad) == B.ERR_INVALID                # empty box
    nan = t.copy()
    nan[3, 4] = np.nan
    assert call(nan, len(nan), g) == B.ERR_INVALID              # non-finite coordinate
    assert call(t, len(t), g, z0=4) == B.ERR_INVALID            # z_first outside the grid
    assert call(t, len(t), g, zc=0) == B.ERR_INVALID


@pytest.mark.reference
def test_oracle_matches_reference_on_random_surfaces(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(9)
    for k in range(6):
        base = G.icosphere(rng.uniform(0.3, 0.7, 3), rng.uniform(0.15, 0.3), 2) if k % 2 else \
            G.torus(rng.uniform(0.4, 0.6, 3), 0.25, 0.08, 24, 12)
        t = G.transform_surface(base, rng.normal(0, 0.05, 3), rng.normal(size=3), rng.uniform(0, 6.3))
        nx, ny, nz = rng.integers(5, 23, 3)
        lo = rng.uniform(-0.1, 0.1, 3)
        hi = lo + rng.uniform(0.9, 1.2, 3)
        assert np.array_equal(oracle_mod.voxelize(t, nx, ny, nz, lo, hi), oracle_mod.ref_voxelize(t, nx, ny, nz, lo, hi))


@pytest.mark.reference
def test_reference_ahmed_body_model(oracle_mod):
    if not REF_MODEL.exists() or not oracle_mod.reference_available():
        pytest.skip("the reference tree is not present")
    t = G.read_ascii_stl(REF_MODEL)
    assert len(t) == 18
    mask = oracle_mod.voxelize(t, 32, 20, 20, (0, 0, 0), (1, 1, 1))
    assert 0 < mask.sum() < mask.size
    assert np.array_equal(mask, oracle_mod.ref_voxelize(t, 32, 20, 20, (0, 0, 0), (1, 1, 1)))
