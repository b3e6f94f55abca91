"""The paired-cell step kernel against the one-cell kernel (GPU).

Both variants evaluate the same per-cell collision with the same rounding
(FP16 stores: the same stochastic rounding bits per cell and direction), so
after any number of steps their populations must agree bit for bit.
The cases cover partial warps (nx/2 not a multiple of 32), multi-warp rows,
the x-periodic wrap of shifted word accesses, random walls next to fluid
cells inside one thread's pair, moving walls, gray cells and both parities.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(18, 15, 13), (130, 6, 5), (2, 6, 4), (64, 9, 7)]


def run(cs, variant, q, shape, storage, flags_kind, gray, steps, seed=11, planes=0):
    nx, ny, nz = shape
    n = nx * ny * nz
    rng = np.random.default_rng(seed)
    storage, _, rounding = storage.partition(":")
    cfg = cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.6, lattice={19: "d3q19", 27: "d3q27"}[q],
                              storage=storage, collision="trt", smagorinsky_les=True, smagorinsky_cs=0.1,
                              acceleration_x=1e-5, fp16_rounding=rounding or "stochastic")
    with cs.EsotericPullCudaSolver(cfg) as s:
        s.set_launch_shape(0, 0, variant)
        s.set_step_planes(planes)
        if flags_kind == "random":
            fl = (rng.random(n) < 0.2).astype(np.uint8)
            fl[rng.random(n) < 0.05] = 3
            s.set_flags(fl)
            s.set_wall_velocity(3, 0.02, -0.01, 0.0)
        elif flags_kind == "cavity":
            s.set_flags(cs.cavity_flags(nx, ny, nz))
            s.set_wall_velocity(2, 0.08, 0.0, 0.0)
        if gray:
            s.set_solid_fraction(rng.uniform(0, 0.2, n).astype(np.float32))
        s.initialize_taylor_green(0.05)
        s.step(steps)
        logical = s.logical_populations()
        red = s.reduce()
        return logical, red


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp16s:nearest"])
@pytest.mark.parametrize("shape", SHAPES, ids=[f"{a}x{b}x{c}" for a, b, c in SHAPES])
@pytest.mark.parametrize("flags_kind, gray", [(None, False), ("random", False), ("cavity", True)])
@pytest.mark.parametrize("steps", [5, 6])
def test_paired_matches_single_bitwise(engine, q, storage, shape, flags_kind, gray, steps):
    a_log, a_red = run(engine, 1, q, shape, storage, flags_kind, gray, steps)
    b_log, b_red = run(engine, 2, q, shape, storage, flags_kind, gray, steps)
    assert np.array_equal(a_log.view(np.uint32), b_log.view(np.uint32))
    assert a_red["mass"] == b_red["mass"]


def test_paired_variant_requires_even_nx(engine):
    cs = engine
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=17, ny=4, nz=4)) as s:
        with pytest.raises(ValueError, match="paired"):
            s.set_launch_shape(0, 0, 2)
        s.set_launch_shape(0, 0, 0)  # automatic falls back to one cell per thread
        s.step(3)


# The wall-aware FP16 pair kernel (variants 3 and 4) marches along z; plane
# counts that do not divide nz leave a short last chunk, and rows of 256 cells
# span more than one warp.  The pipelined form (variant 3) reads flags three
# and wall-link masks two planes ahead: runs of 1, 2 and 3 planes per thread
# end its look-ahead at every depth.
W2_SHAPES = SHAPES + [(256, 5, 9)]


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["fp16s", "fp16s:nearest"])
@pytest.mark.parametrize("shape", W2_SHAPES, ids=[f"{a}x{b}x{c}" for a, b, c in W2_SHAPES])
@pytest.mark.parametrize("flags_kind, gray", [(None, False), ("random", False), ("random", True),
                                              ("cavity", False), ("cavity", True)])
@pytest.mark.parametrize("variant, planes", [(3, 0), (3, 1), (3, 2), (3, 3), (4, 1), (4, 5)])
def test_wall_aware_pairs_match_single_bitwise(engine, q, storage, shape, flags_kind, gray, variant, planes):
    steps = 5
    a_log, a_red = run(engine, 1, q, shape, storage, flags_kind, gray, steps)
    b_log, b_red = run(engine, variant, q, shape, storage, flags_kind, gray, steps, planes=planes)
    assert np.array_equal(a_log.view(np.uint32), b_log.view(np.uint32))
    assert a_red["mass"] == b_red["mass"]


def test_wall_aware_pairs_need_fp16_and_even_nx(engine):
    cs = engine
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=16, ny=4, nz=4)) as s:
        with pytest.raises(ValueError, match="wall-aware"):
            s.set_launch_shape(0, 0, 3)
        with pytest.raises(ValueError, match="planes"):
            s.set_step_planes(-1)
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=17, ny=4, nz=4, storage="fp16s")) as s:
        with pytest.raises(ValueError, match="wall-aware"):
            s.set_launch_shape(0, 0, 4)
