"""The CUDA voxelizer against the reference's masks and the oracle (GPU).

* every golden mask of the reference voxelizer (tests/golden/voxel_fixtures.npz)
  is reproduced bit for bit;
* random rotated spheres and tori on odd, non-cubic grids equal the oracle bit
  for bit, also for plane windows (z_first / z_count, wrapping past nz), a
  solid value other than 1 and output straight into device memory;
* ``set_solid_surface`` gives the same flags -- and so the same populations after
  stepping -- as voxelizing on the host and calling ``set_flags``, with and
  without base flags, on whole lattices and on z-slabs.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "voxel_fixtures.npz"


@pytest.fixture(scope="module")
def fixtures():
    data = np.load(GOLDEN)
    return data, json.loads(bytes(data["meta"]).decode())


def test_reference_masks_bitwise(engine, fixtures):
    from cfd_solvers_b200 import geometry as G

    data, meta = fixtures
    for name, m in meta.items():
        nx, ny, nz = m["grid"]
        grid = G.VoxelGrid3D(nx, ny, nz, tuple(m["minimum"]), tuple(m["maximum"]))
        got = G.voxelize_surface(data[f"{name}_tris"], grid)
        assert np.array_equal(got, data[f"{name}_mask"]), name


def random_surfaces(G, rng, count):
    for k in range(count):
        if k % 3 == 0:
            base = G.icosphere(rng.uniform(0.3, 0.7, 3), rng.uniform(0.15, 0.3), int(rng.integers(1, 4)))
        elif k % 3 == 1:
            base = G.torus(rng.uniform(0.4, 0.6, 3), 0.25, 0.08, 30, 14)
        else:
            base = G.box_surface(rng.uniform(0.1, 0.4, 3), rng.uniform(0.6, 0.9, 3))
        yield G.transform_surface(base, rng.normal(0, 0.05, 3), rng.normal(size=3), rng.uniform(0, 6.3))


def test_random_surfaces_match_oracle(engine, oracle_mod):
    from cfd_solvers_b200 import geometry as G

    rng = np.random.default_rng(21)
    for t in random_surfaces(G, rng, 9):
        nx, ny, nz = (int(v) for v in rng.integers(7, 41, 3))
        lo = rng.uniform(-0.1, 0.1, 3)
        hi = lo + rng.uniform(0.9, 1.2, 3)
        grid = G.VoxelGrid3D(nx, ny, nz, tuple(lo), tuple(hi))
        expect = oracle_mod.voxelize(t, nx, ny, nz, lo, hi)
        assert np.array_equal(G.voxelize_surface(t, grid), expect)
        # a window of planes that wraps past nz, with another solid value
        z0, zc = int(rng.integers(0, nz)), int(nz + 3)
        window = G.voxelize_surface(t, grid, z_first=z0, z_count=zc, value=7)
        planes = (z0 + np.arange(zc)) % nz
        ref = expect.reshape(nz, ny * nx)[planes].reshape(-1) * 7
        assert np.array_equal(window, ref)


def test_device_output(engine, oracle_mod):
    import torch

    from cfd_solvers_b200 import geometry as G

    t = G.icosphere((0.5, 0.45, 0.55), 0.3, 3)
    grid = G.VoxelGrid3D(33, 29, 27, (0, 0, 0), (1, 1, 1))
    out = torch.full((33 * 29 * 27,), 9, dtype=torch.uint8, device="cuda:0")
    G.voxelize_surface(t, grid, out=out)
    assert np.array_equal(out.cpu().numpy(), oracle_mod.voxelize(t, 33, 29, 27, (0, 0, 0), (1, 1, 1)))


def test_many_triangles(engine, oracle_mod):
    """A 20480-triangle sphere: bitwise against the oracle on 32 x 30 x 26; on 160^3 the
    plane windows agree with the full mask and the solid fraction is the sphere's volume."""
    from cfd_solvers_b200 import geometry as G

    # rotate about the sphere's own centre (transform_surface rotates about the origin)
    t = G.transform_surface(G.icosphere((0.0, 0.0, 0.0), 0.37, 5), (0.51, 0.5, 0.49), (0.3, 1.0, 0.2), 0.7)
    small = G.VoxelGrid3D(32, 30, 26)
    assert np.array_equal(G.voxelize_surface(t, small), oracle_mod.voxelize(t, 32, 30, 26, (0, 0, 0), (1, 1, 1)))
    n = 160
    grid = G.VoxelGrid3D(n, n, n)
    full = G.voxelize_surface(t, grid)
    band = G.voxelize_surface(t, grid, z_first=70, z_count=5)
    assert np.array_equal(band, full.reshape(n, -1)[70:75].reshape(-1))
    assert abs(full.mean() - 4.0 / 3.0 * np.pi * 0.37 ** 3) < 0.01


def make_channel(cs, n=24, storage="fp32", q=19):
    cfg = cs.InPlaceLbmConfig(nx=n, ny=n - 4, nz=n - 2, tau=0.6, acceleration_x=1e-5, lattice=f"d3q{q}",
                              storage=storage, collision="trt")
    return cfg


def test_set_solid_surface_equals_host_mask(engine):
    from cfd_solvers_b200 import geometry as G
    from cfd_solvers_b200.cases import channel_flags

    cs = engine
    cfg = make_channel(cs)
    t = G.torus((0.45, 0.5, 0.5), 0.28, 0.1, 30, 14)
    lo, hi = (0.0, 0.0, 0.0), (1.0, 0.9, 0.95)
    grid = G.VoxelGrid3D(cfg.nx, cfg.ny, cfg.nz, lo, hi)
    base = channel_flags(cfg.nx, cfg.ny, cfg.nz)
    mask = G.voxelize_surface(t, grid, value=3)
    host_flags = np.where(mask != 0, mask, base).astype(np.uint8)
    with cs.EsotericPullCudaSolver(cfg) as a, cs.EsotericPullCudaSolver(cfg) as b:
        a.set_flags(host_flags)
        b.set_solid_surface(t, lo, hi, solid_id=3, base_flags=base)
        for s in (a, b):
            s.set_wall_velocity(3, 0.0, 0.0, 0.01)
            s.initialize_uniform()
            s.step(6)
        assert np.array_equal(a.logical_populations(), b.logical_populations())
        # without base flags the outside is fluid
        b.set_solid_surface(t, lo, hi, solid_id=1)
        a.set_flags((mask != 0).astype(np.uint8))
        for s in (a, b):
            s.initialize_uniform()
            s.step(3)
        assert np.array_equal(a.logical_populations(), b.logical_populations())
        with pytest.raises(ValueError):
            b.set_solid_surface(t, lo, hi, solid_id=0)
        with pytest.raises(ValueError):
            b.set_solid_surface(t[:0], lo, hi)


def test_slabs_voxelize_their_own_planes(engine):
    from cfd_solvers_b200 import geometry as G
    from cfd_solvers_b200 import slabs as S
    from cfd_solvers_b200.cases import channel_flags

    cs = engine
    cfg = make_channel(cs, storage="fp16s")
    t = G.icosphere((0.5, 0.5, 0.47), 0.3, 3)
    base = channel_flags(cfg.nx, cfg.ny, cfg.nz)
    with cs.EsotericPullCudaSolver(cfg) as w:
        w.set_solid_surface(t, solid_id=1, base_flags=base)
        w.initialize_taylor_green(0.03)
        w.step(5)
        expect = w.logical_populations()
    ss = S.virtual_slabs(cfg, 3)
    try:
        for s in ss:
            s.set_solid_surface(t, solid_id=1, base_flags=s.slab.local(base))
            s.initialize_taylor_green(0.03)
        S.virtual_step(ss, 5)
        assert np.array_equal(S.gather_virtual_logical(ss), expect)
    finally:
        for s in ss:
            s.close()


def test_repeated_calls_reuse_scratch_and_release(engine):
    """The voxelizer's and the Q-criterion's temporary buffers come from the library's per-device
    pool: repeated calls give the same mask, and release_scratch hands the pool's memory back
    without disturbing later calls."""
    from cfd_solvers_b200 import geometry as G

    cs = engine
    t = G.icosphere((0.5, 0.5, 0.5), 0.3, 3)
    grid = G.VoxelGrid3D(48, 40, 32)
    first = G.voxelize_surface(t, grid)
    for _ in range(4):
        assert np.array_equal(G.voxelize_surface(t, grid), first)
    cs.release_scratch(0)
    assert np.array_equal(G.voxelize_surface(t, grid), first)
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=24, ny=20, nz=16, tau=0.7)) as s:
        s.initialize_taylor_green(0.03)
        s.step(3)
        q0 = s.q_criterion()
        cs.release_scratch(0)
        assert np.array_equal(s.q_criterion(), q0)
    with pytest.raises(ValueError):
        cs.release_scratch(1 << 20)
