"""The resident free-surface, particle and Q-criterion restatements (oracle), without a GPU.

The reference's resident solvers are SYCL-only (resident_multiphysics_sycl.hpp:202-405) and cannot
be built here.  Their algorithms are the ones of the reference's CPU free surface
(src/lbm/free_surface.cpp) and point particles (src/lbm/particles.cpp) in FP32 instead of FP64,
with the advection in per-cell rather than per-face form and a per-cell clamp; those CPU
functions compile here (oracle/_ref), so the float32 restatements are pinned against them within
FP32 rounding on inputs where the clamp and the normal threshold do not act.  The reference chain
test's gate (tests/test_v0156_gpu_lbm_multiphysics.cpp:43-49) is checked on the restatement too.
"""
from __future__ import annotations

import numpy as np
import pytest


def smooth_fill(nx, ny, nz, centre=(7.3, 6.6, 5.9), radius=4.5, width=3.0):
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = np.sqrt((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2)
    return (0.5 - 0.4 * np.tanh((r - radius) / width)).reshape(-1)


def velocity(n, scale, seed):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-scale, scale, n).astype(np.float32) for _ in range(3)]


def test_chain_gate_zero_flow_volume(oracle_mod):
    nx, ny, nz = 10, 8, 6
    f = oracle_mod.fill_half_space_x(nx, ny, nz, 3.5)
    row = f[:nx]
    assert list(row) == [1, 1, 1, 0.5, 0, 0, 0, 0, 0, 0]
    zero = [np.zeros(nx * ny * nz, np.float32)] * 3
    f1 = oracle_mod.fill_advect(f, zero, nx, ny, nz, 0.2)
    assert abs(f1.sum(dtype=np.float64) - f.sum(dtype=np.float64)) < 2.0e-4 * nx * ny * nz
    assert np.array_equal(f1, f)  # at rest nothing moves


def test_half_space_edges(oracle_mod):
    assert np.all(oracle_mod.fill_half_space_x(4, 2, 2, -1.0) == 0)
    assert np.all(oracle_mod.fill_half_space_x(4, 2, 2, 9.0) == 1)
    assert list(oracle_mod.fill_half_space_x(4, 2, 2, 2.0)[:4]) == [1, 1, 0, 0]


def test_uniform_velocity_translates_and_conserves(oracle_mod):
    # a uniform u = 1 with dt = 1 moves the fill one cell exactly (upwind is exact at CFL 1)
    nx, ny, nz = 12, 4, 4
    f = oracle_mod.fill_half_space_x(nx, ny, nz, 5.0)
    u = [np.ones(nx * ny * nz, np.float32), np.zeros(nx * ny * nz, np.float32), np.zeros(nx * ny * nz, np.float32)]
    f1 = oracle_mod.fill_advect(f, u, nx, ny, nz, 1.0)
    assert np.array_equal(f1.reshape(nz, ny, nx), np.roll(f.reshape(nz, ny, nx), 1, axis=2))
    # a divergence-free-in-sum random field keeps the total where nothing clamps
    g = smooth_fill(12, 12, 12).astype(np.float32)
    v = velocity(g.size, 0.05, 3)
    g1 = oracle_mod.fill_advect(g, v, 12, 12, 12, 1.0)
    assert abs(g1.sum(dtype=np.float64) - g.sum(dtype=np.float64)) < 1e-4


def test_clamp(oracle_mod):
    nx = ny = nz = 4
    f = np.zeros(nx * ny * nz, np.float32)
    f[0] = 1.0
    u = [np.full(f.size, -0.9, np.float32), np.zeros(f.size, np.float32), np.zeros(f.size, np.float32)]
    f1 = oracle_mod.fill_advect(f, u, nx, ny, nz, 1.0)
    assert f1.min() >= 0 and f1.max() <= 1


@pytest.mark.parametrize("steps", [1, 5])
def test_advection_matches_reference_cpu(oracle_mod, steps):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    nx, ny, nz = 16, 14, 12
    f = smooth_fill(nx, ny, nz)
    u = velocity(f.size, 0.02, 5)
    dt = 0.8
    ref = oracle_mod.ref_free_surface(f, u, nx, ny, nz, dt, steps)
    g = f.astype(np.float32)
    for _ in range(steps):
        g = oracle_mod.fill_advect(g, u, nx, ny, nz, dt)
    assert 0.0 < g.min() and g.max() < 1.0  # the clamp did not act
    assert np.max(np.abs(g - ref["fill"])) < 5e-7
    assert abs(g.sum(dtype=np.float64) - ref["volume"]) < 1e-3


def test_geometry_and_tension_match_reference_cpu(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    nx, ny, nz = 16, 14, 12
    f = smooth_fill(nx, ny, nz)
    sigma, rho = 0.072, 1.3
    ref = oracle_mod.ref_free_surface(f, velocity(f.size, 0.0, 1), nx, ny, nz, 1.0, 0, sigma, rho)
    nxv, nyv, nzv, k = oracle_mod.fill_geometry(f.astype(np.float32), nx, ny, nz)
    assert np.max(np.abs(np.stack([nxv, nyv, nzv]) - ref["normals"])) < 1e-5
    assert np.max(np.abs(k - ref["curvature"])) < 1e-5
    zero = [np.zeros(f.size, np.float32)] * 3
    a = oracle_mod.surface_tension(f.astype(np.float32), k, zero, nx, ny, nz, sigma, rho)
    assert np.max(np.abs(np.stack(a) - ref["tension"])) < 2e-8
    # a sphere of fill 1 inside: curvature is positive at the interface (kappa = -div n, n points inward)
    r = np.abs(f - 0.5) < 0.1
    assert np.median(k[r]) > 0


def test_normals_threshold(oracle_mod):
    f = np.full(4 * 4 * 4, 0.3, np.float32)
    nxv, nyv, nzv, k = oracle_mod.fill_geometry(f, 4, 4, 4)
    assert not np.any(nxv) and not np.any(nyv) and not np.any(nzv) and not np.any(k)


def test_particles_match_reference_cpu(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    nx, ny, nz = 10, 8, 6
    n = nx * ny * nz
    rng = np.random.default_rng(11)
    count = 40
    rec = np.zeros((count, 8))
    rec[:, 0] = rng.uniform(-3, nx + 3, count)  # positions outside the box wrap
    rec[:, 1] = rng.uniform(0, ny, count)
    rec[:, 2] = rng.uniform(-nz, 0, count)
    rec[:, 3:6] = rng.normal(0, 0.05, (count, 3))
    rec[:, 6] = rng.uniform(0.5, 2, count)
    rec[:, 7] = rng.uniform(0.3, 3, count)
    rec = rec.astype(np.float32).astype(np.float64)  # the device state is float32
    u = velocity(n, 0.05, 12)
    g = (0.0, -1e-3, 2e-4)
    ref, ref_a = oracle_mod.ref_particles(rec, u, nx, ny, nz, 0.5, True, g)
    st, acc = oracle_mod.particles_advance(rec.T.astype(np.float32), u, [np.zeros(n, np.float32)] * 3, nx, ny, nz,
                                           0.5, True, g)
    pos_err = np.abs(st[:3].T - ref[:, :3])
    pos_err = np.minimum(pos_err, np.array([nx, ny, nz]) - pos_err)  # periodic distance
    assert pos_err.max() < 1e-5
    assert np.max(np.abs(st[3:6].T - ref[:, 3:6])) < 1e-6
    assert np.max(np.abs(np.stack(acc) - ref_a)) < 1e-6
    # momentum: the spread force sums to minus the total drag
    drag = ((st[3:6] - rec.T[3:6].astype(np.float32)) / 0.5 - np.array(g, np.float32)[:, None]) * rec.T[6]
    assert np.allclose(np.stack(acc).sum(1, dtype=np.float64), -drag.sum(1), atol=1e-6)


def test_particles_at_rest_stay(oracle_mod):
    # the chain test's seed particle in a fluid at rest (test_v0156_gpu_lbm_multiphysics.cpp:52-58)
    nx, ny, nz = 10, 8, 6
    st = np.array([[2.25], [3.5], [2.75], [0], [0], [0], [1.0], [0.5]], np.float32)
    zero = [np.zeros(nx * ny * nz, np.float32)] * 3
    out, acc = oracle_mod.particles_advance(st, zero, zero, nx, ny, nz, 0.05, True)
    assert np.array_equal(out, st)
    assert not any(np.any(a) for a in acc)


def test_resident_q_matches_reference_interior(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    nx, ny, nz = 9, 8, 7
    u = velocity(nx * ny * nz, 0.1, 4)
    q32 = oracle_mod.resident_q(u, nx, ny, nz).reshape(nz, ny, nx)
    q64 = oracle_mod.q_criterion(np.stack(u, 1).astype(np.float64), nx, ny, nz).reshape(nz, ny, nx)
    inner = (slice(1, -1),) * 3
    assert np.max(np.abs(q32[inner] - q64[inner])) < 1e-7
    # solid-body rotation about z: Q = omega^2 away from the periodic seam
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    w = 0.01
    rot = [(-w * (y - 4)).astype(np.float32).reshape(-1), (w * (x - 4)).astype(np.float32).reshape(-1),
           np.zeros(nx * ny * nz, np.float32)]
    q = oracle_mod.resident_q(rot, nx, ny, nz).reshape(nz, ny, nx)
    assert np.allclose(q[:, 1:-1, 1:-1], w * w, rtol=1e-5)
