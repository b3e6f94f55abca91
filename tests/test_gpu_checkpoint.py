"""CFDCHK3 checkpoints (GPU).

The reference tests its distributed checkpoint for bitwise restart
(tests/test_main.cpp:225-266); the same property is required here: a
lattice restored from a checkpoint continues bit for bit (FP32 storage),
for both parities, walls, moving walls and forces.  Corrupt or mismatched
files raise CheckpointError and leave the lattice untouched.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (18, 14, 12)


def make(cs, q=19, storage="fp32", **kw):
    nx, ny, nz = SHAPE
    return cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, lattice={19: "d3q19", 27: "d3q27"}[q],
                                                         storage=storage, collision="trt", tau=0.7,
                                                         acceleration_x=2e-5, **kw))


def setup(cs, s, seed=3):
    nx, ny, nz = SHAPE
    rng = np.random.default_rng(seed)
    flags = cs.cavity_flags(nx, ny, nz)
    inner = flags == 0
    flags[inner & (rng.random(flags.size) < 0.05)] = 1
    s.set_flags(flags)
    s.set_wall_velocity(2, 0.05, 0.0, 0.01)
    s.initialize_taylor_green(0.03)
    return flags


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("steps", [6, 7])
def test_restart_is_bitwise(engine, tmp_path, q, steps):
    path = tmp_path / "state.chk"
    with make(engine, q) as a, make(engine, q) as b:
        flags = setup(engine, a)
        b.set_flags(flags)
        b.set_wall_velocity(2, 0.05, 0.0, 0.01)
        a.step(steps)
        a.save_checkpoint(path)
        b.load_checkpoint(path)
        assert b.time_step() == steps
        a.step(9)
        b.step(9)
        assert np.array_equal(a.logical_populations().view(np.uint32), b.logical_populations().view(np.uint32))
        assert a.reduce()["mass"] == b.reduce()["mass"]


def test_fp16_restart(engine, tmp_path):
    path = tmp_path / "h.chk"
    with make(engine, 19, "fp16s") as a, make(engine, 19, "fp16s") as b:
        flags = setup(engine, a)
        b.set_flags(flags)
        b.set_wall_velocity(2, 0.05, 0.0, 0.01)
        a.step(5)
        a.save_checkpoint(path)
        b.load_checkpoint(path)
        a.step(4)
        b.step(4)
        assert np.max(np.abs(a.logical_populations() - b.logical_populations())) < 1e-6


def test_file_layout(engine, tmp_path):
    path = tmp_path / "layout.chk"
    nx, ny, nz = SHAPE
    with make(engine, 19) as s:
        s.initialize_taylor_green(0.02)
        s.step(3)
        s.save_checkpoint(path)
        logical = s.logical_populations()
    raw = path.read_bytes()
    assert raw[:8] == b"CFDCHK3\0"
    version, endian, q = struct.unpack_from("<III", raw, 8)
    assert (version, endian, q) == (1, 0x01020304, 19)
    ext = struct.unpack_from("<9Q", raw, 20)
    assert ext == (nx, ny, nz, 0, 0, 0, nx, ny, nz)
    (t,) = struct.unpack_from("<Q", raw, 92)
    tau, ax, ay, az = struct.unpack_from("<4f", raw, 100)
    assert t == 3 and tau == pytest.approx(0.7) and ax == pytest.approx(2e-5)
    pops = np.frombuffer(raw, np.float32, offset=116)
    assert pops.size == 19 * nx * ny * nz
    # no walls, no moving walls: the payload is the logical populations
    assert np.array_equal(pops, logical)


def test_corrupt_and_mismatched_files(engine, tmp_path):
    good = tmp_path / "good.chk"
    with make(engine, 19) as s:
        setup(engine, s)
        s.step(2)
        s.save_checkpoint(good)
        before = s.logical_populations()
        raw = good.read_bytes()
        cases = {
            "magic": b"XFDCHK3\0" + raw[8:],
            "truncated": raw[:-4],
            "trailing": raw + b"\0\0\0\0",
            "q": raw[:16] + struct.pack("<I", 27) + raw[20:],
            "tau": raw[:100] + struct.pack("<f", 0.8) + raw[104:],
        }
        for name, data in cases.items():
            p = tmp_path / f"{name}.chk"
            p.write_bytes(data)
            with pytest.raises(engine.bindings.CheckpointError):
                s.load_checkpoint(p)
            assert np.array_equal(s.logical_populations(), before), name
            assert s.time_step() == 2
        with pytest.raises(engine.bindings.CheckpointError):
            s.load_checkpoint(tmp_path / "missing.chk")
