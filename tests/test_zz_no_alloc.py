"""cfdx_lbm_reduce_noalloc through the C ABI (GPU).

The entry point serves callers that cannot allocate device memory when they
read the conservation sums (device memory held by another allocator, loops
that must not take cudaMalloc's device-wide synchronisation, FFI callers
without a CUDA allocation API).  It must give the same sums as
cfdx_lbm_reduce(), which allocates its scratch, on consecutive calls, for
every lattice shape: its fixed scratch holds min(ny*nz, 4096) blocks' partial
sums, so tall (nz > 4096) and thin (nz = 4) lattices both reduce.

Kept in a file that sorts last so that a run stopping at the first failure
has run every other test first; it passes alone in a fresh process too.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12  # FP64 sums over a different fixed block decomposition


def noalloc(lib, handle):
    out = (ctypes.c_double * 7)()
    status = lib.raw.cfdx_lbm_reduce_noalloc(handle, out)
    return status, list(out)


def assert_same(got, ref):
    assert got[0] == pytest.approx(ref["mass"], rel=REL)
    for k in range(3):
        assert got[1 + k] == pytest.approx(ref["momentum"][k], rel=1e-9, abs=1e-12)
    assert got[4] == pytest.approx(ref["kinetic_energy"], rel=REL)
    assert got[5] == ref["max_speed"]
    assert got[6] == ref["nonfinite"] == 0


@pytest.mark.parametrize("lattice, storage", [("d3q19", "fp32"), ("d3q27", "fp16s"), ("d3q19", "fp64")])
def test_noalloc_reduce_matches_reduce_on_consecutive_calls(engine, lattice, storage):
    cs = engine
    lib = cs.load()
    cfg = cs.InPlaceLbmConfig(nx=40, ny=36, nz=30, tau=0.56, lattice=lattice, storage=storage, collision="trt",
                              smagorinsky_les=True, smagorinsky_cs=0.1)
    with cs.EsotericPullCudaSolver(cfg) as s:
        s.set_flags(cs.cavity_flags(40, 36, 30))
        s.set_wall_velocity(2, 0.1, 0.0, 0.0)
        s.initialize_uniform()
        s.step(7)
        first_status, first = noalloc(lib, s.handle)
        assert first_status == 0, lib.last_error()
        assert_same(first, s.reduce())
        s.step(4)
        second_status, second = noalloc(lib, s.handle)
        assert second_status == 0, lib.last_error()
        assert_same(second, s.reduce())
        assert second[4] != first[4]  # the state moved between the two calls


@pytest.mark.parametrize("shape", [(2, 2, 4097), (2, 2, 4096), (1024, 1024, 4), (64, 64, 2)],
                         ids=["tall-4097", "tall-4096", "thin-1024x1024x4", "thin-64x64x2"])
def test_noalloc_reduce_any_lattice_shape(engine, shape):
    cs = engine
    lib = cs.load()
    nx, ny, nz = shape
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.7)) as s:
        s.initialize_taylor_green(0.05)
        s.step(3)
        status, out = noalloc(lib, s.handle)
        assert status == 0, lib.last_error()
        assert_same(out, s.reduce())
        status, again = noalloc(lib, s.handle)
        assert status == 0 and again == out
