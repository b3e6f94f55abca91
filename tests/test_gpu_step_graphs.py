"""Step loops of 8 or more steps replay a captured CUDA graph of 8 steps (cfdx_lbm_step, csrc/capi.cu).

A graph launches the same kernels with the same argument blocks as the step-by-step loop, so a
run of many steps in one call must equal the same steps taken one call at a time, bit for bit,
for every storage the graph path takes (FP32, FP64; FP16 and slabs keep plain launches), with
walls, moving walls, gray cells, per-cell forces and the paired FP32 kernel, from even and odd
time steps, and for step counts that leave a remainder after the whole graphs.  The graph is
kept on the handle between calls (one per starting parity) and must be captured again whenever
a parameter, a buffer or the kernel choice changes.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solver(cs, q, storage, kind, variant=0):
    nx, ny, nz = 18, 14, 12
    lattice = {19: "d3q19", 27: "d3q27"}[q]
    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.62, lattice=lattice, storage=storage,
                                                      collision="trt", acceleration_x=2e-5))
    if variant:
        s.set_launch_shape(0, 0, variant)
    if kind in ("cavity", "gray"):
        s.set_flags(cs.cavity_flags(nx, ny, nz))
        s.set_wall_velocity(2, 0.05, 0.0, 0.0)
    if kind == "gray":
        rng = np.random.default_rng(3)
        s.set_solid_fraction(rng.uniform(0, 0.2, nx * ny * nz).astype(np.float32))
        s.set_local_body_acceleration(*(rng.normal(0, 1e-5, nx * ny * nz).astype(np.float32) for _ in range(3)))
    s.initialize_taylor_green(0.03)
    return s


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["fp32", "fp64"])
@pytest.mark.parametrize("kind", ["periodic", "cavity", "gray"])
def test_graph_steps_equal_single_steps(engine, q, storage, kind):
    cs = engine
    with solver(cs, q, storage, kind) as a, solver(cs, q, storage, kind) as b:
        a.step(1)
        b.step(1)  # start both at an odd time step
        a.step(101)  # 12 graph replays of 8 + 5 plain steps
        for _ in range(101):
            b.step(1)
        assert a.time_step() == b.time_step() == 102
        assert np.array_equal(a.logical_populations(), b.logical_populations())
        a.step(64)
        b.step(32)
        b.step(32)
        assert np.array_equal(a.logical_populations(), b.logical_populations())


def test_graph_steps_paired_fp32_kernel(engine):
    cs = engine
    with solver(cs, 19, "fp32", "cavity", variant=2) as a, solver(cs, 19, "fp32", "cavity", variant=1) as b:
        a.step(70)
        for _ in range(70):
            b.step(1)
        assert np.array_equal(a.logical_populations(), b.logical_populations())


def test_cached_graph_follows_changes(engine):
    """Calls that replay the handle's graph, and calls after changes that must not replay it."""
    cs = engine

    def run(s, steps, single):
        if single:
            for _ in range(steps):
                s.step(1)
        else:
            s.step(steps)

    with solver(cs, 19, "fp32", "cavity") as a, solver(cs, 19, "fp32", "cavity") as b:
        plan = [
            (None, 16), (None, 8), (None, 1), (None, 8), (None, 9),   # replays from even and odd steps
            (lambda s: s.set_tau(0.7), 16),
            (lambda s: s.set_wall_velocity(2, 0.02, 0.01, 0.0), 8),
            (lambda s: s.set_launch_shape(0, 0, 2), 16),              # paired kernel
            (lambda s: s.set_launch_shape(0, 0, 1), 8),
            (lambda s: s.set_flags(cs.cavity_flags(18, 14, 12, lid_id=3)), 8),
            (lambda s: s.set_wall_velocity(3, -0.03, 0.0, 0.0), 24),
        ]
        for change, steps in plan:
            for s, single in ((a, False), (b, True)):
                if change:
                    change(s)
                run(s, steps, single)
            assert a.time_step() == b.time_step()
            assert np.array_equal(a.logical_populations(), b.logical_populations())
