"""The D3Q7 thermal restatement (oracle), without a GPU.

The reference's resident thermal lattice is SYCL-only (resident_multiphysics_sycl.hpp:51-200) and
cannot be built here, so its restatement is pinned by the physics it must reproduce: a sine mode
decays as exp(-D k^2 t) with D = (tau - 1/2) / 4, a uniform field stays uniform and the total is
conserved, and a uniform velocity carries a profile at that velocity.
"""
from __future__ import annotations

import numpy as np

W = np.array([0.25] + [0.125] * 6, np.float32)


def equilibrium(T):
    return (W[:, None] * np.asarray(T, np.float32).reshape(-1)[None, :]).astype(np.float32)


def test_diffusion_rate(oracle_mod):
    nx, ny, nz, D, steps = 32, 4, 4, 0.05, 200
    x = np.arange(nx)
    T = np.broadcast_to((1 + 0.1 * np.sin(2 * np.pi * x / nx)).astype(np.float32), (nz, ny, nx))
    u = [np.zeros(nx * ny * nz, np.float32)] * 3
    g = oracle_mod.thermal_d3q7_step(equilibrium(T), u, nx, ny, nz, D, steps)
    Tn = g.reshape(7, -1).sum(0).reshape(nz, ny, nx)[0, 0]
    k = 2 * np.pi / nx
    assert abs((Tn.max() - Tn.min()) / 2 / (0.1 * np.exp(-D * k * k * steps)) - 1) < 0.01


def test_uniform_field_and_conservation(oracle_mod):
    nx, ny, nz = 6, 5, 4
    rng = np.random.default_rng(2)
    u = [rng.normal(0, 0.02, nx * ny * nz).astype(np.float32) for _ in range(3)]
    g = oracle_mod.thermal_d3q7_step(equilibrium(np.full(nx * ny * nz, 300.0)), u, nx, ny, nz, 0.02, 3)
    assert np.abs(g.sum(dtype=np.float64) / (300.0 * nx * ny * nz) - 1) < 2e-5  # the reference's gate
    # at rest a uniform field stays uniform (with a non-solenoidal u the conservative form compresses it)
    zero = [np.zeros(nx * ny * nz, np.float32)] * 3
    g = oracle_mod.thermal_d3q7_step(equilibrium(np.full(nx * ny * nz, 300.0)), zero, nx, ny, nz, 0.02, 3)
    assert np.array_equal(g.reshape(7, -1).sum(0), np.full(nx * ny * nz, np.float32(300.0)))
    # a random field conserves its total
    T0 = rng.uniform(0, 1, nx * ny * nz).astype(np.float32)
    g = oracle_mod.thermal_d3q7_step(equilibrium(T0), u, nx, ny, nz, 0.02, 10)
    assert abs(g.sum(dtype=np.float64) / T0.sum(dtype=np.float64) - 1) < 1e-5


def test_advection_speed(oracle_mod):
    nx, ny, nz, steps, ux = 64, 2, 2, 100, 0.05
    x = np.arange(nx)
    T = np.broadcast_to(np.exp(-((x - 20.0) / 4.0) ** 2).astype(np.float32), (nz, ny, nx))
    u = [np.full(nx * ny * nz, ux, np.float32), np.zeros(nx * ny * nz, np.float32), np.zeros(nx * ny * nz, np.float32)]
    g = oracle_mod.thermal_d3q7_step(equilibrium(T), u, nx, ny, nz, 0.01, steps)
    Tn = g.reshape(7, -1).sum(0).reshape(nz, ny, nx)[0, 0]
    centre = (Tn * x).sum() / Tn.sum()
    assert abs(centre - (20.0 + ux * steps)) < 0.05
