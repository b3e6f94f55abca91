"""An oracle-backed stand-in for the CUDA slab (test infrastructure).

``OracleSlab`` has the interface ``DistributedEsotericPullSolver`` drives
(step / pack / unpack / message_buffer / fields / reductions), with the CPU
oracle (oracle/lbm_oracle.c) as the per-slab stepper: the local lattice has
the two ghost planes, and only the slab's own planes are stepped
(``ora_step_planes``).  Messages follow the product's layout (the C ABI's
host-only ``cfdx_halo_plan``), so the exchange logic and the layout are
checked on CPU against the whole-lattice oracle.
"""
from __future__ import annotations

import numpy as np

from cfd_solvers_b200.lbm import MacroscopicFields
from cfd_solvers_b200.slabs import SIDE_LOWER, SIDE_UPPER, Slab, halo_plan


class OracleSlab:
    def __init__(self, O, config, z_begin: int, z_extent: int, storage: str = "f32"):
        self.O = O
        self.q = config.q
        self.nx, self.ny, self.nz = config.nx, config.ny, config.nz
        self.ze = z_extent
        self.slab = Slab(config.nx, config.ny, config.nz, 0, 1, z_begin, z_extent)
        self.P = config.nx * config.ny
        self.storage = storage
        self.wall_u = np.zeros((O.MAX_WALL_IDS, 3), np.float32)
        self.L = O.OracleLattice(q=self.q, nx=self.nx, ny=self.ny, nz=z_extent + 2, storage=storage,
                                 collision=config.collision, tau=float(np.float32(config.tau)),
                                 tau_minus=float(np.float32(config.trt_tau_minus)),
                                 accel=tuple(float(np.float32(a)) for a in
                                             (config.acceleration_x, config.acceleration_y, config.acceleration_z)),
                                 flags=np.zeros(self.P * (z_extent + 2), np.uint8), wall_u=self.wall_u)
        self.packs = 0

    # --- setup
    def set_flags(self, local_flags):
        self.L.flags = np.asarray(local_flags, np.uint8).copy()

    def set_wall_velocity(self, wall_id, ux, uy, uz):
        self.wall_u[wall_id] = (ux, uy, uz)

    def initialize_fields(self, rho, ux, uy, uz):
        self.L.init_fields(np.concatenate([np.asarray(v, np.float32) for v in (rho, ux, uy, uz)]))

    # --- stepping and messages
    def _slots(self):
        return self.L.f.reshape(self.q, self.ze + 2, self.P)

    def step(self, count: int = 1):
        assert count == 1
        self.L.step_planes(1, self.ze + 1)
        if self.ze == self.nz:  # the whole ring: exchange with itself
            lo, up = self.message_buffer(), self.message_buffer()
            self.pack(SIDE_LOWER, lo)
            self.pack(SIDE_UPPER, up)
            self.unpack(SIDE_LOWER, up)
            self.unpack(SIDE_UPPER, lo)

    def _chunks(self, buffer):
        return buffer.numpy().view(self.L.f.dtype).reshape(-1, self.P)

    def message_buffer(self):
        import torch

        k = len(halo_plan(self.q, 0, 0, self.ze)[0])
        return torch.zeros(k * self.P * self.L.f.itemsize, dtype=torch.uint8)

    def pack(self, side, buffer):
        send, _ = halo_plan(self.q, (self.L.t - 1) & 1, side, self.ze)
        v, f = self._chunks(buffer), self._slots()
        for k, (plane, d) in enumerate(send):
            v[k] = f[d, plane]
        self.packs += 1

    def unpack(self, side, buffer):
        _, recv = halo_plan(self.q, (self.L.t - 1) & 1, side, self.ze)
        v, f = self._chunks(buffer), self._slots()
        for k, (plane, d) in enumerate(recv):
            f[d, plane] = v[k]

    # --- results (local planes, ghost planes included)
    def time_step(self) -> int:
        return self.L.t

    def logical_populations(self):
        return self.L.logical()

    def compute_macroscopic(self):
        return MacroscopicFields(*self.L.macroscopic())

    def reduce(self) -> dict:
        return fluid_reduce(self.slab.own(self.L.macroscopic()[0]), *[self.slab.own(v) for v in
                                                                       self.L.macroscopic()[1:]],
                            fluid=self.slab.own(self.L.flags) == 0)

    def close(self):
        pass


def fluid_reduce(rho, ux, uy, uz, fluid) -> dict:
    """FP64 sums over fluid cells of per-cell values (mass, momentum, KE, max speed)."""
    r, x, y, z = (np.asarray(v, np.float64)[fluid] for v in (rho, ux, uy, uz))
    sp = np.sqrt(x * x + y * y + z * z)
    return {"mass": float(r.sum()), "momentum": (float((r * x).sum()), float((r * y).sum()), float((r * z).sum())),
            "kinetic_energy": float(0.5 * (r * sp * sp).sum()), "max_speed": float(sp.max(initial=0.0)),
            "nonfinite": 0}
