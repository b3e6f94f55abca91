"""z-slab decomposition of the in-place lattice: one slab per GPU, one halo exchange per step.

The reference's distributed LBM (include/cfd/solvers/lbm/distributed_pull.hpp) cuts a
two-grid solver into Cartesian bricks (``make_brick`` / ``partition_axis``,
include/cfd/distributed/cartesian.hpp:132-159), runs one ``DistributedPullBlock`` per MPI
rank and, for tests, several blocks in one process (``virtual_step``,
``virtual_exchange``, ``gather_virtual_macroscopic``, distributed_pull.hpp:325-429).
Here the in-place Esoteric-Pull lattice is cut along z only -- planes are contiguous in
the ``[q][z][y][x]`` layout, so every message chunk is one contiguous run -- by the same
partition rule, and the slabs form a periodic ring (the lattice is periodic in z; walls
come from the flags).

* :class:`Slab` / :func:`make_slab` / :func:`partition_axis`  -- geometry (host only).
* :func:`halo_plan`  -- the message layout, from the C ABI (host only, no GPU needed).
* :class:`SlabSolver` -- one slab handle (``cfdx_lbm_create_slab``); its per-cell arrays
  cover the local planes, ghost planes included.
* :class:`SlabExchanger` -- moves the four messages of a step between ranks with
  ``torch.distributed`` point-to-point calls (NCCL over NVLink on GPUs, gloo on CPUs).
* :class:`DistributedEsotericPullSolver` -- the per-rank solver (the reference's
  ``DistributedPullBlock`` role): global arrays in, one step + exchange per step,
  FP64 reductions all-reduced across ranks, per-rank CFDCHK3 checkpoints.
* :func:`virtual_slabs` / :func:`virtual_step` / :func:`virtual_exchange` /
  :func:`gather_virtual_macroscopic` -- several slabs in one process, exchanged slot to
  slot by one copy kernel per cut (``cfdx_lbm_halo_exchange``).
"""
from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import bindings as B
from .lbm import EsotericPullCudaSolver, InPlaceLbmConfig, MacroscopicFields, _LATTICE

SIDE_LOWER = B.SIDE_LOWER
SIDE_UPPER = B.SIDE_UPPER
STEP_EDGES = B.STEP_EDGES
STEP_INTERIOR = B.STEP_INTERIOR


def partition_axis(extent: int, coordinate: int, partitions: int) -> tuple[int, int]:
    """(begin, extent) of part `coordinate` of `partitions` (reference cartesian.hpp:132-139).

    The first ``extent % partitions`` parts get one extra plane.
    """
    if partitions <= 0 or not 0 <= coordinate < partitions:
        raise ValueError("invalid axis partition")
    base, extra = divmod(int(extent), int(partitions))
    return coordinate * base + min(coordinate, extra), base + (1 if coordinate < extra else 0)


@dataclass(frozen=True)
class Slab:
    """Rank `rank`'s slab [z_begin, z_begin + z_extent) of an nx x ny x nz lattice cut into `ranks` slabs."""

    nx: int
    ny: int
    nz: int
    rank: int
    ranks: int
    z_begin: int
    z_extent: int

    @property
    def lower(self) -> int:
        """Rank across the lower side (periodic ring)."""
        return (self.rank - 1) % self.ranks

    @property
    def upper(self) -> int:
        """Rank across the upper side (periodic ring)."""
        return (self.rank + 1) % self.ranks

    @property
    def plane_cells(self) -> int:
        return self.nx * self.ny

    @property
    def local_planes(self) -> np.ndarray:
        """Global z of the local planes 0 .. z_extent + 1 (ghost planes first and last)."""
        return (self.z_begin - 1 + np.arange(self.z_extent + 2)) % self.nz

    @property
    def local_cells(self) -> int:
        return self.plane_cells * (self.z_extent + 2)

    @property
    def own_cells(self) -> int:
        return self.plane_cells * self.z_extent

    def local(self, array, components: int = 1) -> np.ndarray:
        """The local planes (ghosts included) of a global per-cell array of `components` fields."""
        a = np.asarray(array).reshape(components, self.nz, self.plane_cells)
        return np.ascontiguousarray(a[:, self.local_planes, :]).reshape(-1)

    def own(self, local, components: int = 1) -> np.ndarray:
        """The slab's own planes of a local per-cell array of `components` fields."""
        a = np.asarray(local).reshape(components, self.z_extent + 2, self.plane_cells)
        return np.ascontiguousarray(a[:, 1:-1, :]).reshape(-1)


def make_slab(nx: int, ny: int, nz: int, ranks: int, rank: int) -> Slab:
    """Slab of `rank` when nz planes are split over `ranks` ranks (reference make_brick along z)."""
    if ranks <= 0 or not 0 <= rank < ranks:
        raise ValueError("invalid rank / rank count")
    if ranks > nz:
        raise ValueError(f"{ranks} slabs need nz >= {ranks} (nz = {nz})")
    begin, extent = partition_axis(nz, rank, ranks)
    return Slab(int(nx), int(ny), int(nz), int(rank), int(ranks), begin, extent)


def halo_plan(q: int, odd: int, side: int, z_extent: int, library=None):
    """(send, recv) lists of (plane, direction) of one side's messages after a step of parity `odd`.

    Chunk k of the message sent through `side` is the run of direction send[k][1] over
    local plane send[k][0]; chunk k of the message arriving through `side` is written to
    recv[k].  Host-only call into the C ABI (no GPU needed).
    """
    lib = library or B.load()
    send = (B.cfdx_halo_entry * 9)()
    recv = (B.cfdx_halo_entry * 9)()
    count = ctypes.c_int()
    lib.check(lib.raw.cfdx_halo_plan(int(q), int(odd), int(side), int(z_extent), send, recv, 9, ctypes.byref(count)),
              "cfdx_halo_plan")
    return ([(e.plane, e.direction) for e in send[:count.value]],
            [(e.plane, e.direction) for e in recv[:count.value]])


class SlabSolver(EsotericPullCudaSolver):
    """One slab handle; arrays cover its local planes (ghost planes included).

    `config` describes the whole lattice (its nz is the global extent).
    """

    def __init__(self, config: InPlaceLbmConfig, z_begin: int, z_extent: int, library=None):
        self._z = (int(z_begin), int(z_extent))
        super().__init__(config, library=library)
        self._slab = Slab(int(config.nx), int(config.ny), int(config.nz), 0, 1, int(z_begin), int(z_extent))
        size = ctypes.c_size_t()
        self._call("cfdx_lbm_halo_bytes", ctypes.byref(size))
        self._halo_bytes = int(size.value)

    def _create(self, c):
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        self._lib.check(self._lib.raw.cfdx_lbm_create_slab(ctypes.byref(c), self._z[0], self._z[1],
                                                           ctypes.byref(handle), err, len(err)),
                        "cfdx_lbm_create_slab")
        return handle

    def _local_cells(self, c) -> int:
        return c.nx * c.ny * (self._z[1] + 2)

    @property
    def slab(self) -> Slab:
        """Geometry (rank fields are those of a lone slab; DistributedEsotericPullSolver tracks ranks)."""
        return self._slab

    def slab_info(self) -> tuple[int, int, int]:
        vals = [ctypes.c_uint32() for _ in range(3)]
        self._call("cfdx_lbm_slab_info", *[ctypes.byref(v) for v in vals])
        return tuple(int(v.value) for v in vals)

    def halo_bytes(self) -> int:
        """Bytes of one message (5 or 9 plane runs in the storage type)."""
        return self._halo_bytes

    def message_buffer(self):
        """A device buffer for one message (torch uint8 tensor on this slab's device)."""
        import torch

        return torch.empty(self._halo_bytes, dtype=torch.uint8, device=f"cuda:{self._config.device}")

    def step_phase(self, phase: int):
        """One phase of a two-phase step: STEP_EDGES (the edge planes, after which the messages can be
        packed) or STEP_INTERIOR (the rest of that step); equal to step(1) bit for bit."""
        self._call("cfdx_lbm_step_phase", int(phase))

    def pack(self, side: int, buffer):
        """Writes the message of `side` for the step just taken into `buffer` (device, stream-ordered)."""
        self._check_buffer(buffer)
        self._call("cfdx_lbm_halo_pack", int(side), ctypes.c_void_p(buffer.data_ptr()))

    def unpack(self, side: int, buffer):
        """Writes the message that arrived through `side` into the slab (device, stream-ordered)."""
        self._check_buffer(buffer)
        self._call("cfdx_lbm_halo_unpack", int(side), ctypes.c_void_p(buffer.data_ptr()))

    def exchange_with(self, upper: "SlabSolver"):
        """Both messages of the cut between this slab's upper side and `upper`'s lower side."""
        if not upper._h:
            raise RuntimeError("solver is closed")
        self._call("cfdx_lbm_halo_exchange", upper._h)

    def torch_stream(self):
        """This slab's CUDA stream as a torch ExternalStream."""
        import torch

        return torch.cuda.ExternalStream(self.stream(), device=f"cuda:{self._config.device}")

    def _check_buffer(self, buffer):
        if not hasattr(buffer, "data_ptr") or buffer.device.type != "cuda":
            raise ValueError("halo messages live in device memory (a CUDA tensor)")
        if buffer.numel() * buffer.element_size() < self._halo_bytes:
            raise ValueError(f"message buffer holds {buffer.numel() * buffer.element_size()} bytes, "
                             f"needs {self._halo_bytes}")


class SlabExchanger:
    """The four point-to-point messages of one step between ring neighbours.

    Messages going up (this rank's upper side -> the upper rank's lower side) use tag 0,
    messages going down tag 1; every rank posts its sends in the order (upper, lower) and
    its receives in the order (lower, upper), so backends that match by order (NCCL)
    and by tag (gloo) pair them the same way, also on a ring of two where both
    neighbours are one rank.  A ring of one rank copies locally.
    """

    def __init__(self, slab: Slab, group=None):
        self.slab = slab
        self.group = group

    def exchange(self, send_lower, send_upper, recv_lower, recv_upper):
        if self.slab.ranks == 1:
            recv_lower.copy_(send_upper)
            recv_upper.copy_(send_lower)
            return
        import torch.distributed as dist

        g = self.group
        lo = dist.get_global_rank(g, self.slab.lower) if g is not None else self.slab.lower
        up = dist.get_global_rank(g, self.slab.upper) if g is not None else self.slab.upper
        ops = [
            dist.P2POp(dist.isend, send_upper, up, g, 0),
            dist.P2POp(dist.isend, send_lower, lo, g, 1),
            dist.P2POp(dist.irecv, recv_lower, lo, g, 0),
            dist.P2POp(dist.irecv, recv_upper, up, g, 1),
        ]
        for work in dist.batch_isend_irecv(ops):
            work.wait()


def _world(group):
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


class DistributedEsotericPullSolver:
    """This rank's slab of a lattice split along z over the ranks of `group`.

    The reference's per-rank ``DistributedPullBlock`` (distributed_pull.hpp:35-323) with the
    single-GPU solver's method names: inputs are whole-lattice arrays (each rank keeps its
    planes), :meth:`step` runs one step and one halo exchange per time step, reductions are
    FP64 sums (max for the speed) over all ranks, and :meth:`gather_macroscopic` assembles
    the global fields on one rank.  Without an initialised process group it is the whole
    lattice on one rank.  ``backend`` (a factory ``(config, z_begin, z_extent) -> slab``)
    replaces the CUDA slab; the default is :class:`SlabSolver` on ``config.device``.
    """

    def __init__(self, config: InPlaceLbmConfig, group=None, backend=None, library=None):
        rank, ranks = _world(group)
        self.group = group
        self._config = config
        self._slab_geometry = make_slab(config.nx, config.ny, config.nz, ranks, rank)
        g = self._slab_geometry
        make = backend or (lambda cfg, z0, ze: SlabSolver(cfg, z0, ze, library=library))
        self.solver = make(config, g.z_begin, g.z_extent)
        self._exchanger = SlabExchanger(g, group)
        self._buffers = None if ranks == 1 else [self.solver.message_buffer() for _ in range(4)]
        self._stream = self.solver.torch_stream() if hasattr(self.solver, "torch_stream") else None
        # The exchange runs on a stream of its own while the slab's stream steps the interior.
        self._comm_stream = None
        if self._buffers is not None and self._stream is not None and hasattr(self.solver, "step_phase"):
            import torch

            self._comm_stream = torch.cuda.Stream(device=f"cuda:{config.device}")

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if self.solver is not None:
            self.solver.close()
            self.solver = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ geometry
    @property
    def slab(self) -> Slab:
        return self._slab_geometry

    @property
    def config(self) -> InPlaceLbmConfig:
        return self._config

    def time_step(self) -> int:
        return self.solver.time_step()

    # ------------------------------------------------------------ setup
    def initialize_uniform(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        self.solver.initialize_uniform(rho, ux, uy, uz)

    def initialize_taylor_green(self, amplitude=0.03):
        """The whole lattice's Taylor-Green field (global coordinates)."""
        self.solver.initialize_taylor_green(amplitude)

    def initialize_fields(self, rho, ux, uy, uz):
        g = self.slab
        self.solver.initialize_fields(*(g.local(v) for v in (rho, ux, uy, uz)))

    def set_flags(self, flags, local: bool = False):
        """Whole-lattice flags (0 fluid, 1 wall, 2..15 moving wall); ghost planes take the neighbours' flags.

        With ``local=True`` `flags` already covers this rank's local planes
        (``slab.local_planes``, ghost planes included), so no rank needs the whole field.
        """
        self.solver.set_flags(flags if local else self.slab.local(np.asarray(flags, np.uint8)))

    def set_solid_mask(self, mask):
        m = np.asarray(mask).reshape(-1)
        self.set_flags(np.where(m != 0, B.WALL, B.FLUID).astype(np.uint8))

    def set_wall_velocity(self, wall_id: int, ux: float, uy: float, uz: float):
        self.solver.set_wall_velocity(wall_id, ux, uy, uz)

    def set_solid_surface(self, triangles, minimum=(0.0, 0.0, 0.0), maximum=(1.0, 1.0, 1.0), solid_id: int = 1,
                          base_flags=None, local: bool = False):
        """Flags from a surface voxelized over the whole lattice's box; each rank voxelizes its own planes."""
        if base_flags is not None and not local:
            base_flags = self.slab.local(np.asarray(base_flags, np.uint8))
        self.solver.set_solid_surface(triangles, minimum, maximum, solid_id, base_flags)

    def set_solid_fraction(self, ns):
        self.solver.set_solid_fraction(None if ns is None else self.slab.local(np.asarray(ns, np.float32)))

    def set_local_body_acceleration(self, ax, ay, az):
        g = self.slab
        self.solver.set_local_body_acceleration(*(g.local(np.asarray(v, np.float32)) for v in (ax, ay, az)))

    # ------------------------------------------------------------ stepping
    def step(self, count: int = 1):
        """`count` steps, each followed by its halo exchange.

        With a CUDA slab on more than one rank every step runs in two phases
        (reference distributed_pull.hpp:97-116, interior overlapped with the
        boundary exchange): the edge planes, then the messages are packed and
        sent on a communication stream while the slab's stream steps the
        interior planes; the unpacks wait for both.
        """
        for _ in range(int(count)):
            if self._comm_stream is not None:
                self._overlapped_step()
                continue
            self.solver.step(1)
            if self._buffers is not None:
                self._exchange()

    def _overlapped_step(self):
        import torch

        s = self.solver
        send_lo, send_up, recv_lo, recv_up = self._buffers
        s.step_phase(STEP_EDGES)
        s.pack(SIDE_LOWER, send_lo)
        s.pack(SIDE_UPPER, send_up)
        comm = self._comm_stream
        comm.wait_stream(self._stream)
        with torch.cuda.stream(comm):
            self._exchanger.exchange(send_lo, send_up, recv_lo, recv_up)
        s.step_phase(STEP_INTERIOR)
        self._stream.wait_stream(comm)
        s.unpack(SIDE_LOWER, recv_lo)
        s.unpack(SIDE_UPPER, recv_up)

    def _exchange(self):
        s = self.solver
        send_lo, send_up, recv_lo, recv_up = self._buffers
        s.pack(SIDE_LOWER, send_lo)
        s.pack(SIDE_UPPER, send_up)
        stream = self._stream
        if stream is not None:
            import torch

            # NCCL work is queued behind the packs on the slab's stream, and the unpacks
            # behind its completion: no host synchronisation per step.
            with torch.cuda.stream(stream):
                self._exchanger.exchange(send_lo, send_up, recv_lo, recv_up)
        else:
            self._exchanger.exchange(send_lo, send_up, recv_lo, recv_up)
        s.unpack(SIDE_LOWER, recv_lo)
        s.unpack(SIDE_UPPER, recv_up)

    # ------------------------------------------------------------ results
    def compute_macroscopic(self) -> MacroscopicFields:
        """rho, u of this rank's own planes."""
        g = self.slab
        return MacroscopicFields(*(g.own(v) for v in self.solver.compute_macroscopic()))

    def logical_populations(self) -> np.ndarray:
        """[d][own cells] logical populations of this rank's planes."""
        q = _LATTICE[self._config.lattice]
        return self.slab.own(self.solver.logical_populations(), components=q)

    def gather_macroscopic(self, dst: int = 0) -> Optional[MacroscopicFields]:
        """Global rho, u on rank `dst` (None elsewhere); reference gather_virtual_macroscopic."""
        own = self.compute_macroscopic()
        g = self.slab
        if g.ranks == 1:
            return own
        import torch
        import torch.distributed as dist

        dtype = torch.float64 if own.rho.dtype == np.float64 else torch.float32
        sizes = [partition_axis(g.nz, r, g.ranks)[1] * g.plane_cells for r in range(g.ranks)]
        # gather wants equal shapes: pad every slab to the largest (the first)
        local = torch.zeros(4, sizes[0], dtype=dtype)
        local[:, :g.own_cells] = torch.from_numpy(np.stack(own)).to(dtype)
        rank = dist.get_rank(self.group)
        device = self._collective_device()
        parts = [torch.empty(4, sizes[0], dtype=dtype, device=device) for _ in sizes] if rank == dst else None
        dst_global = dist.get_global_rank(self.group, dst) if self.group is not None else dst
        dist.gather(local.to(device), parts, dst=dst_global, group=self.group)
        if rank != dst:
            return None
        full = torch.cat([p[:, :n].cpu() for p, n in zip(parts, sizes)], dim=1).numpy()
        return MacroscopicFields(*(full[k].copy() for k in range(4)))

    def _collective_device(self):
        import torch
        import torch.distributed as dist

        return torch.device(f"cuda:{self._config.device}") if dist.get_backend(self.group) == "nccl" else \
            torch.device("cpu")

    def reduce(self) -> dict:
        """FP64 mass, momentum, kinetic energy, max speed and non-finite count over all ranks."""
        r = self.solver.reduce()
        if self.slab.ranks == 1:
            return r
        import torch
        import torch.distributed as dist

        device = self._collective_device()
        sums = torch.tensor([r["mass"], *r["momentum"], r["kinetic_energy"], float(r["nonfinite"])],
                            dtype=torch.float64, device=device)
        peak = torch.tensor([r["max_speed"]], dtype=torch.float64, device=device)
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=self.group)
        dist.all_reduce(peak, op=dist.ReduceOp.MAX, group=self.group)
        s = sums.cpu().tolist()
        return {"mass": s[0], "momentum": (s[1], s[2], s[3]), "kinetic_energy": s[4],
                "max_speed": float(peak.item()), "nonfinite": int(s[5])}

    def mass(self) -> float:
        return self.reduce()["mass"]

    def kinetic_energy(self) -> float:
        return self.reduce()["kinetic_energy"]

    def max_speed(self) -> float:
        return float(np.float32(self.reduce()["max_speed"]))

    def checksum(self) -> float:
        """mass + kinetic energy over all ranks (examples/phase02_lbm_taylor_green.cpp:3)."""
        r = self.reduce()
        return r["mass"] + r["kinetic_energy"]

    # ------------------------------------------------------------ checkpoints
    def save_checkpoint(self, path):
        """This rank's CFDCHK3 brick (begin = (0, 0, z_begin)); reference save_checkpoint per block."""
        self.solver.save_checkpoint(path)

    def load_checkpoint(self, path):
        """Restores this rank's brick; the file's decomposition must match the slab."""
        self.solver.load_checkpoint(path)


# ------------------------------------------------------------ in-process ranks
def virtual_slabs(config: InPlaceLbmConfig, ranks: int, library=None) -> list[SlabSolver]:
    """`ranks` slab solvers of one lattice in this process, ordered by rank (reference virtual blocks)."""
    out = []
    try:
        for r in range(ranks):
            g = make_slab(config.nx, config.ny, config.nz, ranks, r)
            out.append(SlabSolver(config, g.z_begin, g.z_extent, library=library))
    except Exception:
        for s in out:
            s.close()
        raise
    return out


def virtual_exchange(slabs: Sequence[SlabSolver]):
    """Every cut's two messages, one copy kernel per cut (reference virtual_exchange)."""
    if len(slabs) == 1:
        return  # the ring of one slab exchanges inside its step
    for r, s in enumerate(slabs):
        s.exchange_with(slabs[(r + 1) % len(slabs)])


def virtual_step(slabs: Sequence[SlabSolver], count: int = 1, phases: bool = False):
    """`count` steps of all slabs with an exchange after each (reference virtual_step).

    With `phases` every slab steps its edge planes, the cuts exchange, and then
    the slabs step their interiors (the order of the overlapped multi-process
    step); the results are the same bits."""
    for _ in range(int(count)):
        if phases:
            for s in slabs:
                s.step_phase(STEP_EDGES)
            virtual_exchange(slabs)
            for s in slabs:
                s.step_phase(STEP_INTERIOR)
            continue
        for s in slabs:
            s.step(1)
        virtual_exchange(slabs)


def gather_virtual_macroscopic(slabs: Sequence[SlabSolver]) -> MacroscopicFields:
    """Global rho, u of in-process slabs (reference gather_virtual_macroscopic)."""
    parts = [s.compute_macroscopic() for s in slabs]
    geo = [s.slab for s in slabs]
    return MacroscopicFields(*(np.concatenate([g.own(p[k]) for g, p in zip(geo, parts)]) for k in range(4)))


def gather_virtual_logical(slabs: Sequence[SlabSolver]) -> np.ndarray:
    """Global [d][n] logical populations of in-process slabs."""
    q = slabs[0]._q
    parts = [s.slab.own(s.logical_populations(), components=q).reshape(q, -1) for s in slabs]
    return np.concatenate(parts, axis=1).reshape(-1)


def virtual_reduce(slabs: Sequence[SlabSolver]) -> dict:
    """FP64 reductions of in-process slabs combined (sums, max speed)."""
    rs = [s.reduce() for s in slabs]
    return {"mass": sum(r["mass"] for r in rs),
            "momentum": tuple(sum(r["momentum"][k] for r in rs) for k in range(3)),
            "kinetic_energy": sum(r["kinetic_energy"] for r in rs),
            "max_speed": max(r["max_speed"] for r in rs),
            "nonfinite": sum(r["nonfinite"] for r in rs)}


__all__ = [
    "DistributedEsotericPullSolver",
    "Slab",
    "SlabExchanger",
    "SlabSolver",
    "gather_virtual_logical",
    "gather_virtual_macroscopic",
    "halo_plan",
    "make_slab",
    "partition_axis",
    "virtual_exchange",
    "virtual_reduce",
    "virtual_slabs",
    "virtual_step",
]
