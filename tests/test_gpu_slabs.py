"""z-slab decomposition on the GPU: slabs of one process against the whole lattice (GPU).

The reference checks its distributed solver by running several blocks in one
process against a serial solver (tests/test_main.cpp:116-149, gate 2e-6) and
the selective halo against the full one bit for bit (:174-215).  Here every
slab runs the same kernels as the whole lattice, hashes global cell indices
for FP16 rounding and takes the global Taylor-Green field, so the gate is
exact: the logical populations of all slabs, put together, equal the whole
lattice's bit for bit, for

* 1 slab (the ring of one, exchanging with itself inside the step), 2, 3 and
  4 slabs, uneven partitions and one-plane slabs;
* D3Q19 / D3Q27; FP32, FP64 and FP16-shifted storage (stochastic and nearest
  rounding); BGK, TRT, Smagorinsky LES; walls and a moving wall across the
  cuts, gray cells, per-cell and uniform forcing;
* the direct cut exchange (one copy kernel per cut) and the pack -> buffer
  -> unpack path that the multi-process NCCL exchange uses.

FP64 reductions agree to 1e-12 (summation order differs).  Checkpoints are
per-slab CFDCHK3 bricks that restart bit for bit.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup(cs, q=19, shape=(12, 10, 13), storage="fp32", coll="trt", les=False, walls=True, gray=False,
          local_force=False, seed=3):
    nx, ny, nz = shape
    n = nx * ny * nz
    rng = np.random.default_rng(seed)
    storage, _, rounding = storage.partition(":")
    cfg = cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.62, lattice={19: "d3q19", 27: "d3q27"}[q],
                              storage=storage, collision=coll, smagorinsky_les=les, smagorinsky_cs=0.12,
                              acceleration_x=2e-5, acceleration_z=-1e-5, fp16_rounding=rounding or "stochastic",
                              rounding_seed=77)
    inputs = {}
    if walls:
        fl = (rng.random(n) < 0.12).astype(np.uint8)
        fl.reshape(nz, ny, nx)[:, 0, :] = 1
        fl.reshape(nz, ny, nx)[[0, nz // 2], ny - 1, :] = 3  # moving rows, one at a cut of the ring
        inputs["flags"] = fl
    if gray:
        inputs["ns"] = rng.uniform(0, 0.2, n).astype(np.float32)
    if local_force:
        inputs["accel"] = (rng.normal(0, 1e-5, (3, n))).astype(np.float32)
    return cfg, inputs


def prepare(s, inputs, local=None):
    pick = local or (lambda a, k=1: a)
    if "flags" in inputs:
        s.set_flags(pick(inputs["flags"]))
        s.set_wall_velocity(3, 0.03, 0.0, -0.01)
    if "ns" in inputs:
        s.set_solid_fraction(pick(inputs["ns"]))
    if "accel" in inputs:
        s.set_local_body_acceleration(*pick(inputs["accel"], 3).reshape(3, -1))
    s.initialize_taylor_green(0.04)


def whole(cs, cfg, inputs, steps, variant=0):
    with cs.EsotericPullCudaSolver(cfg) as s:
        s.set_launch_shape(0, 0, variant)
        prepare(s, inputs)
        s.step(steps)
        return s.logical_populations(), s.reduce(), s.compute_macroscopic()


def sliced(cfg, inputs, ranks, steps, mode="direct", variant=0):
    from cfd_solvers_b200 import slabs as S

    ss = S.virtual_slabs(cfg, ranks)
    try:
        for s in ss:
            s.set_launch_shape(0, 0, variant)
            prepare(s, inputs, local=lambda a, k=1, g=s.slab: g.local(a, k))
        if mode == "direct":
            S.virtual_step(ss, steps)
        elif mode == "phases":
            S.virtual_step(ss, steps, phases=True)
        elif mode == "phases_buffers":
            # the overlapped multi-process order: edges, pack, interior, unpack
            buffers = [(s.message_buffer(), s.message_buffer()) for s in ss]
            for _ in range(steps):
                for s in ss:
                    s.step_phase(S.STEP_EDGES)
                if ranks > 1:
                    for s, (lo, up) in zip(ss, buffers):
                        s.pack(S.SIDE_LOWER, lo)
                        s.pack(S.SIDE_UPPER, up)
                for s in ss:
                    s.step_phase(S.STEP_INTERIOR)
                if ranks == 1:
                    continue
                for s in ss:
                    s.wait()
                for r, s in enumerate(ss):
                    s.unpack(S.SIDE_LOWER, buffers[(r - 1) % ranks][1])
                    s.unpack(S.SIDE_UPPER, buffers[(r + 1) % ranks][0])
                for s in ss:
                    s.wait()
        else:
            buffers = [(s.message_buffer(), s.message_buffer()) for s in ss]
            for _ in range(steps):
                for s in ss:
                    s.step(1)
                if ranks == 1:
                    continue
                for s, (lo, up) in zip(ss, buffers):
                    s.pack(S.SIDE_LOWER, lo)
                    s.pack(S.SIDE_UPPER, up)
                for s in ss:
                    s.wait()
                for r, s in enumerate(ss):
                    s.unpack(S.SIDE_LOWER, buffers[(r - 1) % ranks][1])  # the lower slab's upper message
                    s.unpack(S.SIDE_UPPER, buffers[(r + 1) % ranks][0])  # the upper slab's lower message
                for s in ss:
                    s.wait()
        return S.gather_virtual_logical(ss), S.virtual_reduce(ss), S.gather_virtual_macroscopic(ss)
    finally:
        for s in ss:
            s.close()


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def check(cs, cfg, inputs, ranks, steps, mode="direct", variant=0):
    w_log, w_red, w_mac = whole(cs, cfg, inputs, steps, variant)
    s_log, s_red, s_mac = sliced(cfg, inputs, ranks, steps, mode, variant)
    assert same_bits(s_log, w_log)
    for k in range(4):
        assert same_bits(s_mac[k], w_mac[k])
    assert s_red["mass"] == pytest.approx(w_red["mass"], rel=1e-12)
    assert s_red["kinetic_energy"] == pytest.approx(w_red["kinetic_energy"], rel=1e-12)
    assert s_red["max_speed"] == w_red["max_speed"]
    assert np.allclose(s_red["momentum"], w_red["momentum"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["fp32", "fp64", "fp16s", "fp16s:nearest"])
@pytest.mark.parametrize("ranks", [1, 2, 3, 4])
def test_slabs_match_whole_lattice(engine, q, storage, ranks):
    cfg, inputs = setup(engine, q=q, storage=storage)
    check(engine, cfg, inputs, ranks, steps=7 if ranks % 2 else 6)


@pytest.mark.parametrize("mode", ["direct", "buffers"])
@pytest.mark.parametrize("ranks", [2, 5, 13])
def test_exchange_paths_and_thin_slabs(engine, mode, ranks):
    """13 planes over 5 slabs: slabs of 3 and 2 planes; over 13: one-plane slabs."""
    cfg, inputs = setup(engine, q=27, storage="fp16s", gray=True)
    check(engine, cfg, inputs, ranks, steps=5, mode=mode)


@pytest.mark.parametrize("mode", ["phases", "phases_buffers"])
@pytest.mark.parametrize("q, storage, variant", [(19, "fp32", 0), (27, "fp16s", 0), (19, "fp16s", 0),
                                                 (19, "fp16s", 2), (19, "fp32", 2), (19, "fp16s", 3)])
@pytest.mark.parametrize("ranks", [1, 2, 3, 5])
def test_two_phase_step_matches_whole_lattice(engine, mode, q, storage, variant, ranks):
    """Edge planes, exchange, interior (the overlapped order): the same bits as whole steps, for every
    step kernel, with slabs of 5, 4, 3 and 2 planes (13 planes over up to 5 ranks)."""
    cfg, inputs = setup(engine, q=q, shape=(16, 9, 13), storage=storage, les=True, gray=variant != 3,
                        local_force=True)
    check(engine, cfg, inputs, ranks, steps=5, mode=mode, variant=variant)


def test_two_phase_step_order_is_enforced(engine):
    from cfd_solvers_b200 import slabs as S

    cfg, inputs = setup(engine, q=19, shape=(12, 10, 13))
    ss = S.virtual_slabs(cfg, 2)
    try:
        for s in ss:
            prepare(s, inputs, local=lambda a, k=1, g=s.slab: g.local(a, k))
        with pytest.raises(ValueError, match="EDGES first"):
            ss[0].step_phase(S.STEP_INTERIOR)
        ss[0].step_phase(S.STEP_EDGES)
        with pytest.raises(ValueError, match="half done"):
            ss[0].reduce()
        with pytest.raises(ValueError, match="half done"):
            ss[0].step(1)
        with pytest.raises(ValueError, match="interior phase of the previous step"):
            ss[0].step_phase(S.STEP_EDGES)
        ss[1].step_phase(S.STEP_EDGES)
        ss[0].exchange_with(ss[1])  # halo calls are accepted between the phases
        ss[1].exchange_with(ss[0])
        for s in ss:
            s.step_phase(S.STEP_INTERIOR)
        ss[0].reduce()
    finally:
        for s in ss:
            s.close()
    with engine.EsotericPullCudaSolver(engine.InPlaceLbmConfig(nx=8, ny=8, nz=8)) as s:
        with pytest.raises(ValueError, match="slab handles"):
            s.library.call("cfdx_lbm_step_phase", s.handle, S.STEP_EDGES)


@pytest.mark.parametrize("coll, les", [("bgk", False), ("trt", True)])
@pytest.mark.parametrize("variant", [1, 2])
def test_collisions_forces_and_kernel_variants(engine, coll, les, variant):
    cfg, inputs = setup(engine, q=19, shape=(16, 9, 11), storage="fp16s", coll=coll, les=les, gray=True,
                        local_force=True)
    check(engine, cfg, inputs, 3, steps=6, variant=variant)


def test_periodic_box_without_walls(engine):
    """Slabs always run the flagged kernels (their ghost planes are walls to the kernels).

    So a wall-free slab lattice equals a whole lattice with an all-fluid flag
    field bit for bit, and the flag-free kernels to within FP32 rounding (the
    two instantiations may contract multiply-adds differently).
    """
    cfg, inputs = setup(engine, q=19, shape=(9, 7, 8), storage="fp32", walls=False)
    check(engine, cfg, dict(inputs, flags=np.zeros(9 * 7 * 8, np.uint8)), 4, steps=9, mode="buffers")
    w_log, _, _ = whole(engine, cfg, inputs, 9)
    s_log, _, _ = sliced(cfg, inputs, 4, 9, "buffers")
    assert np.max(np.abs(s_log - w_log)) <= 1e-6


def test_message_size_and_slab_info(engine):
    from cfd_solvers_b200 import slabs as S

    cs = engine
    for storage, es in (("fp32", 4), ("fp16s", 2), ("fp64", 8)):
        for lattice, k in (("d3q19", 5), ("d3q27", 9)):
            cfg = cs.InPlaceLbmConfig(nx=6, ny=5, nz=9, lattice=lattice, storage=storage)
            with S.SlabSolver(cfg, 2, 3) as s:
                assert s.halo_bytes() == k * 6 * 5 * es
                assert s.slab_info() == (2, 3, 9)
                assert s.cells() == 6 * 5 * 5
    with cs.EsotericPullCudaSolver(nx=6, ny=5, nz=9) as s:
        vals = [ctypes.c_uint32() for _ in range(3)]
        s.library.raw.cfdx_lbm_slab_info(s.handle, *[ctypes.byref(v) for v in vals])
        assert [v.value for v in vals] == [0, 9, 9]


def test_exchange_order_is_enforced(engine):
    from cfd_solvers_b200 import slabs as S

    cs = engine
    cfg = cs.InPlaceLbmConfig(nx=6, ny=5, nz=8)
    a, b = S.virtual_slabs(cfg, 2)
    with a, b:
        buf = a.message_buffer()
        with pytest.raises(ValueError):
            a.pack(S.SIDE_UPPER, buf)  # no step yet
        a.step(1)
        with pytest.raises(ValueError):
            a.step(1)  # the previous step's messages are missing
        with pytest.raises(ValueError):
            a.step(2)
        with pytest.raises(ValueError):
            a.exchange_with(b)  # b has not stepped: different time steps
        b.step(1)
        a.exchange_with(b)
        with pytest.raises(ValueError):
            a.exchange_with(b)  # already exchanged
        a.pack(S.SIDE_LOWER, buf)
        b.unpack(S.SIDE_UPPER, buf)
        with pytest.raises(ValueError):
            b.unpack(S.SIDE_UPPER, buf)  # twice
        a.unpack(S.SIDE_LOWER, buf)  # a's own message stands in for b's (order check only)
        a.step(1)
        b.step(1)
        with pytest.raises(ValueError):
            a.pack(S.SIDE_LOWER, buf[:10])  # buffer too small
        with pytest.raises(ValueError):
            a.adjoint_forward(2, 1)
    three = S.virtual_slabs(cfg, 3)
    try:
        for s in three:
            s.step(1)
        with pytest.raises(ValueError):
            three[0].exchange_with(three[2])  # not neighbours in that order
    finally:
        for s in three:
            s.close()


def test_slab_arguments(engine):
    from cfd_solvers_b200 import slabs as S

    cs = engine
    cfg = cs.InPlaceLbmConfig(nx=6, ny=5, nz=8)
    with pytest.raises(ValueError):
        S.SlabSolver(cfg, 6, 3)  # beyond nz
    with pytest.raises(ValueError):
        S.SlabSolver(cfg, 0, 0)


@pytest.mark.parametrize("storage", ["fp32", "fp16s"])
def test_slab_checkpoints_restart(engine, tmp_path, storage):
    """Per-slab CFDCHK3 bricks: FP32 restarts continue bit for bit; an FP16 restart re-encodes
    the stored values exactly as a whole-lattice FP16 restart does, so the two agree bit for bit."""
    from cfd_solvers_b200 import slabs as S

    cs = engine
    cfg, inputs = setup(cs, q=19, storage=storage, gray=True)
    ss = S.virtual_slabs(cfg, 3)
    try:
        for s in ss:
            prepare(s, inputs, local=lambda a, k=1, g=s.slab: g.local(a, k))
        S.virtual_step(ss, 5)
        for r, s in enumerate(ss):
            s.save_checkpoint(tmp_path / f"slab{r}.chk")
        S.virtual_step(ss, 4)
        uninterrupted = S.gather_virtual_logical(ss)
    finally:
        for s in ss:
            s.close()
    with cs.EsotericPullCudaSolver(cfg) as w:
        prepare(w, inputs)
        w.step(5)
        w.save_checkpoint(tmp_path / "whole.chk")
        w.initialize_uniform()
        w.load_checkpoint(tmp_path / "whole.chk")
        w.step(4)
        whole_restart = w.logical_populations()
    ss = S.virtual_slabs(cfg, 3)
    try:
        for s in ss:
            prepare(s, inputs, local=lambda a, k=1, g=s.slab: g.local(a, k))
            s.initialize_uniform()
        for r, s in enumerate(ss):
            s.load_checkpoint(tmp_path / f"slab{r}.chk")
            assert s.time_step() == 5
        S.virtual_step(ss, 4)
        restarted = S.gather_virtual_logical(ss)
        assert same_bits(restarted, whole_restart)
        if storage == "fp32":
            assert same_bits(restarted, uninterrupted)
        else:
            assert np.max(np.abs(restarted - uninterrupted)) < 1e-6
        with pytest.raises(cs.CheckpointError):
            ss[1].load_checkpoint(tmp_path / "slab0.chk")  # another brick
        with pytest.raises(cs.CheckpointError):
            ss[1].load_checkpoint(tmp_path / "whole.chk")
    finally:
        for s in ss:
            s.close()
    # brick header: global extents, begin (0, 0, z_begin), extent (nx, ny, z_extent)
    raw = (tmp_path / "slab1.chk").read_bytes()
    dims = struct.unpack("<9Q", raw[20:92])
    g = S.make_slab(cfg.nx, cfg.ny, cfg.nz, 3, 1)
    assert dims == (cfg.nx, cfg.ny, cfg.nz, 0, 0, g.z_begin, cfg.nx, cfg.ny, g.z_extent)
    assert len(raw) == 92 + 8 + 16 + 19 * cfg.nx * cfg.ny * g.z_extent * 4


def test_distributed_solver_single_rank(engine):
    """Without a process group the per-rank solver is the whole ring on one GPU."""
    from cfd_solvers_b200.slabs import DistributedEsotericPullSolver

    cs = engine
    cfg, inputs = setup(cs, q=27, storage="fp32")
    w_log, w_red, w_mac = whole(cs, cfg, inputs, 6)
    with DistributedEsotericPullSolver(cfg) as d:
        d.set_flags(inputs["flags"])
        d.set_wall_velocity(3, 0.03, 0.0, -0.01)
        d.initialize_taylor_green(0.04)
        d.step(6)
        assert same_bits(d.logical_populations(), w_log)
        g = d.gather_macroscopic()
        for k in range(4):
            assert same_bits(g[k], w_mac[k])
        assert d.mass() == pytest.approx(w_red["mass"], rel=1e-12)
