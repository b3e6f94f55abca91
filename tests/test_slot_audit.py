"""Slot-ownership audit: the stand-in for a race detector on the in-place step.

In-place (Esoteric-Pull) streaming is race-free because each population slot is touched, within
one step, by one cell (the reference states this invariant for its CPU loop).  The audit
(cfdx_lbm_debug_slot_audit, csrc/slot_audit.cu) runs the one-cell step kernel's own addressing
with a storage type that only records the loads, stores and threads per slot.  A link into a wall
cell loads one of the wall cell's two slots of that pair and stores the other (half-way
bounce-back in place; the two swap roles the next step), so each wall link adds one read-only
and one write-only slot, both the fluid cell's alone.

CPU: the per-slot classification, with planted races, through the library's host entry point.
GPU: every lattice, storage and wall kind at odd sizes, both parities, and slabs with ghost
planes: q slots per fluid cell, each read once and written once by the same thread.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

TOUCHED, READ_TWICE, WRITTEN_TWICE, READ_ONLY, WRITE_ONLY, FOREIGN = 1, 2, 4, 8, 16, 32


def classify(lib, reads, writes, lo, hi, writer):
    out = ctypes.c_uint()
    lib.check(lib.raw.cfdx_debug_audit_classify(reads, writes, lo, hi, writer, ctypes.byref(out)))
    return out.value


def test_classification_with_planted_races():
    from cfd_solvers_b200 import bindings as B

    lib = B.load()
    unused = 0xFFFFFFFF
    assert classify(lib, 0, 0, unused, 0, 0) == 0
    assert classify(lib, 1, 1, 7, 7, 7) == TOUCHED  # the invariant
    assert classify(lib, 2, 1, 7, 7, 7) == TOUCHED | READ_TWICE
    assert classify(lib, 1, 2, 7, 7, 7) == TOUCHED | WRITTEN_TWICE  # two stores: a write-write race
    assert classify(lib, 1, 0, 7, 7, 0) == TOUCHED | READ_ONLY
    assert classify(lib, 0, 1, unused, 0, 7) == TOUCHED | WRITE_ONLY
    assert classify(lib, 1, 1, 7, 7, 8) == TOUCHED | FOREIGN  # stored by another thread than the reader
    assert classify(lib, 2, 1, 7, 9, 7) == TOUCHED | READ_TWICE | FOREIGN  # two readers


def flags_of(kind, nx, ny, nz, rng):
    from cfd_solvers_b200.cases import cavity_flags

    if kind == "none":
        return None
    if kind == "cavity":
        return cavity_flags(nx, ny, nz)
    f = (rng.random(nx * ny * nz) < 0.2).astype(np.uint8)  # random walls, some of them moving
    f[f == 1] = rng.choice(np.array([1, 2, 3], np.uint8), int(f.sum()))
    return f


def wall_links(flags, q, nx, ny, nz):
    """Links from fluid cells into wall cells (periodic neighbours), over the q - 1 directions."""
    from oracle import oracle as O

    f = flags.reshape(nz, ny, nx)
    wall = f != 0
    total = 0
    for cx, cy, cz in O.velocity_set(q)[1:]:
        nb = np.roll(wall, shift=(-int(cz), -int(cy), -int(cx)), axis=(0, 1, 2))  # wall at n + c
        total += int(np.count_nonzero(~wall & nb))
    return total


@pytest.mark.gpu
@pytest.mark.parametrize("lattice,q", [("d3q19", 19), ("d3q27", 27)])
@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp64"])
@pytest.mark.parametrize("walls", ["none", "random", "cavity"])
def test_every_slot_has_one_owner(engine, lattice, q, storage, walls):
    cs = engine
    nx, ny, nz = 17, 15, 13
    rng = np.random.default_rng(q + len(storage) + len(walls))
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.7, lattice=lattice,
                                                       storage=storage, collision="trt")) as s:
        f = flags_of(walls, nx, ny, nz, rng)
        fluid, links = nx * ny * nz, 0
        if f is not None:
            s.set_flags(f)
            for wid in (2, 3):
                s.set_wall_velocity(wid, 0.05, -0.02, 0.01)
            fluid, links = int(np.count_nonzero(f == 0)), wall_links(f, q, nx, ny, nz)
        s.initialize_uniform()
        before = s.logical_populations()
        for parity in (0, 1):
            r = s.debug_slot_audit(parity)
            assert r["slots"] == q * nx * ny * nz
            assert r["written_twice"] == 0 and r["foreign"] == 0 and r["read_twice"] == 0, (parity, r)
            assert r["out_of_range"] == 0, (parity, r)
            assert r["touched"] == q * fluid + links, (parity, r)
            assert r["read_only"] == links and r["write_only"] == links, (parity, r)
        assert np.array_equal(s.logical_populations(), before)  # the audit leaves the lattice alone


@pytest.mark.gpu
def test_paired_and_gray_handles_audit_the_one_cell_addressing(engine):
    cs = engine
    n = 16
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=n, ny=n, nz=n, storage="fp16s")) as s:  # paired kernel
        s.set_solid_fraction(np.full(n ** 3, 0.1, np.float32))  # gray
        for parity in (0, 1):
            r = s.debug_slot_audit(parity)
            assert r["touched"] == 19 * n ** 3 and r["foreign"] == r["written_twice"] == r["read_twice"] == 0
            assert r["out_of_range"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("lattice,q", [("d3q19", 19), ("d3q27", 27)])
def test_slab_ghost_planes(engine, lattice, q):
    """A z-slab's ghost planes are walls of its local lattice: the edge cells' links into them keep
    one owner per slot too."""
    from cfd_solvers_b200.slabs import SlabSolver

    cs = engine
    nx, ny, nz = 12, 10, 16
    cfg = cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.7, lattice=lattice)
    with SlabSolver(cfg, 4, 6) as slab:
        slab.initialize_uniform()
        for parity in (0, 1):
            r = slab.debug_slot_audit(parity)
            assert r["slots"] == q * nx * ny * (6 + 2)
            assert r["touched"] == q * nx * ny * 6, r
            assert r["read_twice"] == r["written_twice"] == r["read_only"] == r["write_only"] == r["foreign"] == 0
            assert r["out_of_range"] == 0


@pytest.mark.gpu
def test_audit_size_limit(engine):
    cs = engine
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=8, ny=8, nz=8)) as s:
        with pytest.raises(ValueError):
            s.debug_slot_audit(2)
