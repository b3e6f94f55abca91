"""The z-slab decomposition's host logic, without a GPU.

* the partition rule is the reference's (distributed/cartesian.hpp:132-139) and
  slabs form a periodic ring;
* the message layout from the C ABI (host-only ``cfdx_halo_plan``) carries the
  reference's crossing-population count per face cell (5 for D3Q19, 9 for
  D3Q27; tests/test_main.cpp:150-161 of the reference), matches sender and
  receiver chunk by chunk, and never reads a slot the same exchange writes;
* slabs stepped by the CPU oracle with that layout reproduce the whole-lattice
  oracle bit for bit (FP32 and FP64; walls and a moving wall across the cuts,
  TRT with forcing, uneven partitions, one-plane slabs, odd and even step
  counts) -- the reference's virtual-distributed parity test
  (tests/test_main.cpp:116-149) with an exact gate;
* ``DistributedEsotericPullSolver`` over gloo with 2 and 3 ranks (spawned
  processes, the oracle stand-in as each rank's slab) gives the same
  populations, gathered fields and FP64 reductions.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from cfd_solvers_b200 import bindings as B
from cfd_solvers_b200.lbm import InPlaceLbmConfig
from cfd_solvers_b200.slabs import (DistributedEsotericPullSolver, SlabExchanger, halo_plan, make_slab,
                                    partition_axis)

CZ = {19: [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1],
      27: [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1]}


def test_partition_axis_is_the_reference_rule():
    assert [partition_axis(13, r, 3) for r in range(3)] == [(0, 5), (5, 4), (9, 4)]
    assert [partition_axis(8, r, 4) for r in range(4)] == [(0, 2), (2, 2), (4, 2), (6, 2)]
    assert [partition_axis(5, r, 5) for r in range(5)] == [(r, 1) for r in range(5)]
    with pytest.raises(ValueError):
        partition_axis(4, 4, 4)
    with pytest.raises(ValueError):
        make_slab(4, 4, 3, 4, 0)  # more slabs than planes


def test_slab_ring_and_local_planes():
    s = make_slab(3, 2, 7, 3, 0)
    assert (s.z_begin, s.z_extent, s.lower, s.upper) == (0, 3, 2, 1)
    assert list(s.local_planes) == [6, 0, 1, 2, 3]
    g = np.arange(3 * 2 * 7)
    loc = s.local(g)
    assert loc.size == 5 * 6 and list(loc[:6]) == list(range(36, 42))
    assert np.array_equal(s.own(loc), g[:18])
    two = np.arange(2 * 42).reshape(2, 42)
    assert np.array_equal(s.own(s.local(two, 2), 2).reshape(2, -1), two[:, :18])
    last = make_slab(3, 2, 7, 3, 2)
    assert (last.z_begin, last.z_extent, last.upper) == (5, 2, 0)
    assert list(last.local_planes) == [4, 5, 6, 0]


@pytest.mark.parametrize("q, count", [(19, 5), (27, 9)])
def test_plan_counts_match_crossing_populations(q, count):
    for odd in (0, 1):
        for side in (0, 1):
            send, recv = halo_plan(q, odd, side, 4)
            assert len(send) == len(recv) == count


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("ze", [1, 2, 5])
def test_plan_from_first_principles(q, ze):
    """Derives each side's messages from which slots the edge cells touch, and checks the layout."""
    cz = CZ[q]
    for odd in (0, 1):
        pairs = [(2 * p + 1, 2 * p + 2) for p in range((q - 1) // 2)]
        pa = {p: (j if odd else i) for p, (i, j) in enumerate(pairs)}
        pb = {p: (i if odd else j) for p, (i, j) in enumerate(pairs)}
        for side, out in ((0, -1), (1, 1)):
            ghost, edge = (0, 1) if side == 0 else (ze + 1, ze)
            send, recv = halo_plan(q, odd, side, ze)
            # ghost slots the edge cells touched this step (read-modify-write of n + c_j)
            touched = {(ghost, pa[p]) for p, (i, j) in enumerate(pairs) if cz[j] == out}
            # edge slots the neighbour's edge cells read next step (pa_{t+1} = pb_t at n + c_j)
            read_next = {(edge, pb[p]) for p, (i, j) in enumerate(pairs) if cz[j] == -out}
            assert set(send) == touched | read_next and len(send) == len(touched) + len(read_next)
            # what arrives: the neighbour touched our edge slots, and we read its edge next step
            into_edge = {(edge, pa[p]) for p, (i, j) in enumerate(pairs) if cz[j] == -out}
            into_ghost = {(ghost, pb[p]) for p, (i, j) in enumerate(pairs) if cz[j] == out}
            assert set(recv) == into_edge | into_ghost
        # chunk k of an upper send is chunk k of the neighbour's lower receive, and vice versa
        for a, b in ((1, 0), (0, 1)):
            sa, _ = halo_plan(q, odd, a, ze)
            _, rb = halo_plan(q, odd, b, ze)
            assert [d for _, d in sa] == [d for _, d in rb]
        # one exchange never reads a slot it writes (pack and unpack commute; ze = 1 included)
        reads = set(halo_plan(q, odd, 0, ze)[0]) | set(halo_plan(q, odd, 1, ze)[0])
        writes = set(halo_plan(q, odd, 0, ze)[1]) | set(halo_plan(q, odd, 1, ze)[1])
        assert not reads & writes


def test_plan_rejects_bad_arguments():
    lib = B.load()
    import ctypes

    e = (B.cfdx_halo_entry * 9)()
    n = ctypes.c_int()
    assert lib.raw.cfdx_halo_plan(21, 0, 0, 4, e, e, 9, ctypes.byref(n)) == B.ERR_INVALID
    assert lib.raw.cfdx_halo_plan(19, 2, 0, 4, e, e, 9, ctypes.byref(n)) == B.ERR_INVALID
    assert lib.raw.cfdx_halo_plan(19, 0, 2, 4, e, e, 9, ctypes.byref(n)) == B.ERR_INVALID
    assert lib.raw.cfdx_halo_plan(19, 0, 0, 0, e, e, 9, ctypes.byref(n)) == B.ERR_INVALID
    assert lib.raw.cfdx_halo_plan(27, 0, 0, 4, e, e, 5, ctypes.byref(n)) == B.ERR_INVALID


# ----------------------------------------------------------------- oracle slabs
def case(q, nx=6, ny=5, nz=13, coll="trt", seed=5):
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    flags = (rng.random(n) < 0.12).astype(np.uint8)
    flags.reshape(nz, ny, nx)[:, 0, :] = 1          # a wall plane that crosses every cut
    flags.reshape(nz, ny, nx)[3, ny - 1, :] = 2     # a moving wall row inside a slab or at a cut
    cfg = InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, lattice={19: "d3q19", 27: "d3q27"}[q], collision=coll, tau=0.71,
                           trt_tau_minus=0.0, acceleration_x=2e-4, acceleration_y=-1e-4, acceleration_z=3e-4)
    rho = 1.0 + 0.01 * rng.standard_normal(n)
    u = 0.02 * rng.standard_normal((3, n))
    return cfg, flags, np.vstack([rho, u]).astype(np.float32)


def whole_oracle(O, cfg, flags, fields, steps, storage):
    wall = np.zeros((O.MAX_WALL_IDS, 3), np.float32)
    wall[2] = (0.03, 0.0, -0.01)
    L = O.OracleLattice(q=cfg.q, nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, storage=storage, collision=cfg.collision,
                        tau=float(np.float32(cfg.tau)), tau_minus=0.0,
                        accel=tuple(float(np.float32(a)) for a in
                                    (cfg.acceleration_x, cfg.acceleration_y, cfg.acceleration_z)),
                        flags=flags, wall_u=wall)
    L.init_fields(fields.reshape(-1))
    L.step(steps)
    return L


def oracle_slabs(O, cfg, flags, fields, ranks, storage):
    from slab_oracle import OracleSlab

    slabs = []
    for r in range(ranks):
        g = make_slab(cfg.nx, cfg.ny, cfg.nz, ranks, r)
        s = OracleSlab(O, cfg, g.z_begin, g.z_extent, storage)
        s.set_flags(g.local(flags))
        s.set_wall_velocity(2, 0.03, 0.0, -0.01)
        s.initialize_fields(*g.local(fields, 4).reshape(4, -1))
        slabs.append((g, s))
    return slabs


def step_virtual(slabs):
    """One step of every slab, then every cut's two messages (pack -> unpack)."""
    for _, s in slabs:
        s.step(1)
    if len(slabs) == 1:
        return
    msgs = []
    for r, (_, s) in enumerate(slabs):
        up, lo = s.message_buffer(), s.message_buffer()
        s.pack(1, up)
        s.pack(0, lo)
        msgs.append((r, up, lo))
    n = len(slabs)
    for r, up, lo in msgs:
        slabs[(r + 1) % n][1].unpack(0, up)
        slabs[(r - 1) % n][1].unpack(1, lo)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("ranks", [1, 2, 3, 4, 13])
def test_oracle_slabs_match_whole_lattice(oracle_mod, q, ranks):
    O = oracle_mod
    cfg, flags, fields = case(q)
    steps = 7 if ranks % 2 else 6
    whole = whole_oracle(O, cfg, flags, fields, steps, "f32")
    slabs = oracle_slabs(O, cfg, flags, fields, ranks, "f32")
    for _ in range(steps):
        step_virtual(slabs)
    got = np.concatenate([g.own(s.logical_populations(), q).reshape(q, -1) for g, s in slabs], axis=1)
    assert np.array_equal(got.reshape(-1), whole.logical())


def test_oracle_slabs_fp64_and_bgk(oracle_mod):
    O = oracle_mod
    cfg, flags, fields = case(19, nx=5, ny=4, nz=9, coll="bgk", seed=8)
    whole = whole_oracle(O, cfg, flags, fields, 9, "f64")
    slabs = oracle_slabs(O, cfg, flags, fields, 3, "f64")
    for _ in range(9):
        step_virtual(slabs)
    got = np.concatenate([g.own(s.logical_populations(), 19).reshape(19, -1) for g, s in slabs], axis=1)
    assert np.array_equal(got.reshape(-1), whole.logical())


def test_missing_exchange_breaks_parity(oracle_mod):
    """The messages carry real state: dropping one step's exchange changes the result."""
    O = oracle_mod
    cfg, flags, fields = case(19)
    whole = whole_oracle(O, cfg, flags, fields, 4, "f32")
    slabs = oracle_slabs(O, cfg, flags, fields, 2, "f32")
    for k in range(4):
        if k == 2:
            for _, s in slabs:
                s.step(1)
        else:
            step_virtual(slabs)
    got = np.concatenate([g.own(s.logical_populations(), 19).reshape(19, -1) for g, s in slabs], axis=1)
    assert not np.array_equal(got.reshape(-1), whole.logical())


def test_exchanger_single_rank_copies_locally():
    import torch

    ex = SlabExchanger(make_slab(2, 2, 3, 1, 0))
    a, b = torch.arange(4.0), torch.arange(4.0) + 10
    ra, rb = torch.zeros(4), torch.zeros(4)
    ex.exchange(a, b, ra, rb)
    assert torch.equal(ra, b) and torch.equal(rb, a)


# ----------------------------------------------------------------- gloo ranks
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q, steps, out_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from slab_oracle import OracleSlab

        cfg, flags, fields = case(q)
        solver = DistributedEsotericPullSolver(
            cfg, backend=lambda c, z0, ze: OracleSlab(O, c, z0, ze, "f32"))
        assert solver.slab.ranks == world and solver.slab.rank == rank
        solver.set_flags(flags)
        solver.set_wall_velocity(2, 0.03, 0.0, -0.01)
        solver.initialize_fields(*fields)
        solver.step(steps)
        assert solver.time_step() == steps
        assert solver.solver.packs == 2 * steps  # one exchange through both sides per step
        fields_out = solver.gather_macroscopic(dst=0)
        red = solver.reduce()
        pops = solver.logical_populations()
        np.save(os.path.join(out_dir, f"pops{rank}.npy"), pops)
        if rank == 0:
            np.save(os.path.join(out_dir, "fields.npy"), np.stack(fields_out))
            np.save(os.path.join(out_dir, "reduce.npy"),
                    np.array([red["mass"], *red["momentum"], red["kinetic_energy"], red["max_speed"]]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world, q, steps", [(2, 19, 5), (3, 27, 4)])
def test_gloo_ranks_match_whole_lattice(oracle_mod, tmp_path, world, q, steps):
    import torch.multiprocessing as mp

    from slab_oracle import fluid_reduce

    mp.start_processes(_rank_main, args=(world, _free_port(), q, steps, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    O = oracle_mod
    cfg, flags, fields = case(q)
    whole = whole_oracle(O, cfg, flags, fields, steps, "f32")
    pops = np.concatenate([np.load(tmp_path / f"pops{r}.npy").reshape(q, -1) for r in range(world)], axis=1)
    assert np.array_equal(pops.reshape(-1), whole.logical())
    macro = whole.macroscopic()
    got = np.load(tmp_path / "fields.npy")
    for k in range(4):
        assert np.array_equal(got[k], macro[k])
    ref = fluid_reduce(*macro, fluid=flags == 0)
    red = np.load(tmp_path / "reduce.npy")
    assert red[0] == pytest.approx(ref["mass"], rel=1e-12)
    assert red[4] == pytest.approx(ref["kinetic_energy"], rel=1e-12)
    assert red[5] == ref["max_speed"]
    assert np.allclose(red[1:4], ref["momentum"], rtol=1e-10, atol=1e-14)
