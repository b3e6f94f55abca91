"""ctypes access to the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check in __graft_entry__.py and the CPU-baseline leg
of bench.py import this module.  It wraps

* ``liblbm_oracle.so`` -- the C restatement of the reference's in-place
  Esoteric-Pull step (lbm_oracle.h), and
* ``_ref/libcfdref.so`` / ``_ref/libcfdref_fast.so`` -- the reference's own
  CPU solvers compiled from its sources by oracle/Makefile
  (include/cfd/solvers/lbm/esoteric_pull.hpp, one_step_pull.hpp,
  precision_pull.hpp, compressed_pull.hpp).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liblbm_oracle.so"
REF_SO = HERE / "_ref" / "libcfdref.so"
REF_FAST_SO = HERE / "_ref" / "libcfdref_fast.so"
REF_CLI = HERE / "_ref" / "cfd-bench"

STORE = {"f32": 0, "f64": 1, "f16s": 2}
COLLISION = {"bgk": 0, "trt": 1}
MAX_WALL_IDS = 16

_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
_u8 = ctypes.POINTER(ctypes.c_uint8)


class _OraCfg(ctypes.Structure):
    _fields_ = [
        ("q", ctypes.c_int),
        ("nx", ctypes.c_size_t),
        ("ny", ctypes.c_size_t),
        ("nz", ctypes.c_size_t),
        ("storage", ctypes.c_int),
        ("collision", ctypes.c_int),
        ("tau", ctypes.c_double),
        ("tau_minus", ctypes.c_double),
        ("trt_magic", ctypes.c_double),
        ("les_k", ctypes.c_double),
        ("ax", ctypes.c_double),
        ("ay", ctypes.c_double),
        ("az", ctypes.c_double),
        ("local_a", _f),
        ("flags", _u8),
        ("wall_u", _f),
        ("solid_fraction", _f),
        ("scale", _f),
    ]


_lib = None
_ref = {}


def oracle_lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} is not built; run `make -C oracle oracle`")
        lib = ctypes.CDLL(str(ORACLE_SO))
        P = ctypes.POINTER(_OraCfg)
        lib.ora_init.argtypes = [P, ctypes.c_void_p, ctypes.c_int, _f, _f]
        lib.ora_step.argtypes = [P, ctypes.c_void_p, ctypes.c_uint64]
        lib.ora_step_planes.argtypes = [P, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_size_t]
        lib.ora_macroscopic.argtypes = [P, ctypes.c_void_p, ctypes.c_uint64] + [ctypes.c_void_p] * 4
        lib.ora_reduce.argtypes = [P, ctypes.c_void_p, ctypes.c_uint64, _d]
        lib.ora_logical.argtypes = [P, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        lib.ora_f32_to_f16.argtypes = [ctypes.c_float]
        lib.ora_f32_to_f16.restype = ctypes.c_uint16
        lib.ora_f16_to_f32.argtypes = [ctypes.c_uint16]
        lib.ora_f16_to_f32.restype = ctypes.c_float
        lib.ora_reference_les_k.restype = ctypes.c_float
        lib.ora_adjoint_forward.argtypes = [P, _d, ctypes.c_uint64, _d]
        lib.ora_adjoint.argtypes = [P, _d, ctypes.c_uint64, _d, _d, _d, _d]
        sz = ctypes.c_size_t
        lib.ora_voxelize.argtypes = [_d, sz, sz, sz, sz, _d, _d, _u8]
        lib.ora_transform_surface.argtypes = [_d, sz, _d, _d, ctypes.c_double, _d]
        for name in ("ora_voxelize", "ora_transform_surface", "ora_init", "ora_step", "ora_step_planes",
                     "ora_macroscopic", "ora_reduce", "ora_logical", "ora_adjoint_forward",
                     "ora_adjoint"):
            getattr(lib, name).restype = ctypes.c_int
        _lib = lib
    return _lib


def reference_les_k() -> float:
    """The reference's fixed Smagorinsky coefficient 16*sqrt(2)/(3*pi^2) in float."""
    return float(oracle_lib().ora_reference_les_k())


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


@dataclass
class OracleLattice:
    """An oracle lattice with its own population array (numpy, host)."""

    q: int
    nx: int
    ny: int
    nz: int
    storage: str = "f32"
    collision: str = "bgk"
    tau: float = 0.6
    tau_minus: float = 0.0
    trt_magic: float = 3.0 / 16.0
    les_k: float = 0.0
    accel: tuple = (0.0, 0.0, 0.0)
    local_a: Optional[np.ndarray] = None
    flags: Optional[np.ndarray] = None
    wall_u: Optional[np.ndarray] = None
    solid_fraction: Optional[np.ndarray] = None
    scale: Optional[np.ndarray] = None
    t: int = 0
    f: np.ndarray = field(init=False)

    def __post_init__(self):
        n = self.cells
        dt = {"f32": np.float32, "f64": np.float64, "f16s": np.uint16}[self.storage]
        self.f = np.zeros(self.q * n, dtype=dt)
        self._keep = {}
        self._cfg = _OraCfg()
        self._refresh()

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def _arr(self, name, value, dtype):
        if value is None:
            self._keep[name] = None
            return None
        a = np.ascontiguousarray(value, dtype=dtype)
        self._keep[name] = a
        return a

    def _refresh(self):
        c = self._cfg
        c.q, c.nx, c.ny, c.nz = self.q, self.nx, self.ny, self.nz
        c.storage = STORE[self.storage]
        c.collision = COLLISION[self.collision]
        c.tau, c.tau_minus, c.trt_magic, c.les_k = self.tau, self.tau_minus, self.trt_magic, self.les_k
        c.ax, c.ay, c.az = self.accel
        c.local_a = _ptr(self._arr("local_a", self.local_a, np.float32), _f)
        c.flags = _ptr(self._arr("flags", self.flags, np.uint8), _u8)
        wall = self.wall_u
        if wall is None and self.flags is not None:
            wall = np.zeros((MAX_WALL_IDS, 3), np.float32)
        c.wall_u = _ptr(self._arr("wall_u", wall, np.float32), _f)
        c.solid_fraction = _ptr(self._arr("sf", self.solid_fraction, np.float32), _f)
        c.scale = _ptr(self._arr("scale", self.scale, np.float32), _f)

    def _call(self, rc):
        if rc != 0:
            raise ValueError("oracle rejected the configuration")

    def init_uniform(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        self._refresh()
        p = np.array([rho, ux, uy, uz], np.float32)
        self._call(oracle_lib().ora_init(ctypes.byref(self._cfg), self.f.ctypes.data, 0, _ptr(p, _f), None))
        self.t = 0

    def init_taylor_green(self, amplitude=0.03):
        self._refresh()
        p = np.array([amplitude, 0, 0, 0], np.float32)
        self._call(oracle_lib().ora_init(ctypes.byref(self._cfg), self.f.ctypes.data, 1, _ptr(p, _f), None))
        self.t = 0

    def init_fields(self, fields: np.ndarray):
        self._refresh()
        fl = np.ascontiguousarray(fields, np.float32).reshape(4 * self.cells)
        self._call(oracle_lib().ora_init(ctypes.byref(self._cfg), self.f.ctypes.data, 2, None, _ptr(fl, _f)))
        self.t = 0

    def step(self, count=1):
        self._refresh()
        lib = oracle_lib()
        for _ in range(count):
            self._call(lib.ora_step(ctypes.byref(self._cfg), self.f.ctypes.data, self.t))
            self.t += 1

    def step_planes(self, z_begin: int, z_end: int):
        """One step of the cells of planes [z_begin, z_end) only (ora_step_planes)."""
        self._refresh()
        self._call(oracle_lib().ora_step_planes(ctypes.byref(self._cfg), self.f.ctypes.data, self.t, z_begin, z_end))
        self.t += 1

    def macroscopic(self):
        self._refresh()
        dt = np.float64 if self.storage == "f64" else np.float32
        out = [np.zeros(self.cells, dt) for _ in range(4)]
        self._call(oracle_lib().ora_macroscopic(ctypes.byref(self._cfg), self.f.ctypes.data, self.t,
                                                *[o.ctypes.data for o in out]))
        return out

    def reduce(self):
        self._refresh()
        out = np.zeros(7, np.float64)
        self._call(oracle_lib().ora_reduce(ctypes.byref(self._cfg), self.f.ctypes.data, self.t, _ptr(out, _d)))
        return {"mass": out[0], "momentum": out[1:4].copy(), "kinetic_energy": out[4], "max_speed": out[5],
                "nonfinite": int(out[6])}

    def logical(self):
        self._refresh()
        dt = np.float64 if self.storage == "f64" else np.float32
        out = np.zeros(self.q * self.cells, dt)
        self._call(oracle_lib().ora_logical(ctypes.byref(self._cfg), self.f.ctypes.data, self.t, out.ctypes.data))
        return out


    # ------------------------------------------------ FP64 discrete adjoint
    def adjoint_forward(self, x0: np.ndarray, steps: int) -> np.ndarray:
        """Logical FP64 forward (lbm_adjoint_oracle.c): x after `steps` steps."""
        self._refresh()
        x0 = np.ascontiguousarray(x0, np.float64)
        out = np.zeros_like(x0)
        self._call(oracle_lib().ora_adjoint_forward(ctypes.byref(self._cfg), _ptr(x0, _d), steps, _ptr(out, _d)))
        return out

    def adjoint(self, x0: np.ndarray, steps: int, g_u: np.ndarray, g_rho: Optional[np.ndarray] = None):
        """dJ/dn_s (per cell) and dJ/dtau for dJ/du = g_u (3, N) and dJ/drho = g_rho at the final state."""
        self._refresh()
        x0 = np.ascontiguousarray(x0, np.float64)
        gu = np.ascontiguousarray(g_u, np.float64).reshape(3 * self.cells)
        gr = None if g_rho is None else np.ascontiguousarray(g_rho, np.float64)
        gns = np.zeros(self.cells, np.float64)
        gtau = np.zeros(1, np.float64)
        self._call(oracle_lib().ora_adjoint(ctypes.byref(self._cfg), _ptr(x0, _d), steps, _ptr(gr, _d), _ptr(gu, _d),
                                            _ptr(gns, _d), _ptr(gtau, _d)))
        return gns, float(gtau[0])


def logical_velocity(x: np.ndarray, q: int, cells: int, accel=(0.0, 0.0, 0.0)):
    """rho and u + a/2 of logical populations x ([d][n], float64)."""
    cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])[:q]
    cy = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1])[:q]
    cz = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1])[:q]
    f = x.reshape(q, cells)
    rho = f.sum(0)
    safe = np.where(rho > 0, rho, 1.0)
    u = np.stack([cx @ f, cy @ f, cz @ f]) / safe + 0.5 * np.asarray(accel, np.float64)[:, None]
    return rho, np.where(rho > 0, u, 0.0)


def voxelize(tris, nx: int, ny: int, nz: int, lo, hi) -> np.ndarray:
    """Oracle voxel mask (uint8, n = (k*ny + j)*nx + i) of triangles (count x 9 doubles)."""
    t = np.ascontiguousarray(tris, np.float64).reshape(-1, 9)
    lo_, hi_ = np.ascontiguousarray(lo, np.float64), np.ascontiguousarray(hi, np.float64)
    mask = np.zeros(nx * ny * nz, np.uint8)
    if oracle_lib().ora_voxelize(_ptr(t, _d), len(t), nx, ny, nz, _ptr(lo_, _d), _ptr(hi_, _d), _ptr(mask, _u8)):
        raise ValueError("invalid voxelization inputs")
    return mask


def transform_surface(tris, translation, axis, angle: float) -> np.ndarray:
    t = np.ascontiguousarray(tris, np.float64).reshape(-1, 9)
    tr, ax = np.ascontiguousarray(translation, np.float64), np.ascontiguousarray(axis, np.float64)
    out = np.empty_like(t)
    oracle_lib().ora_transform_surface(_ptr(t, _d), len(t), _ptr(tr, _d), _ptr(ax, _d), float(angle), _ptr(out, _d))
    return out


def q_criterion(velocity, nx: int, ny: int, nz: int, dx: float = 1.0, dy: float = 1.0, dz: float = 1.0):
    """Q-criterion restated in numpy, operand for operand as the reference's q_criterion_3d
    (src/lbm/visualization.cpp:122-148): central differences (p - m) / (2 d), then
    s2, o2 accumulated over (i, j) in row order; 0 on the outer layer."""
    u = np.asarray(velocity, np.float64).reshape(nz, ny, nx, 3)
    q = np.zeros((nz, ny, nx), np.float64)
    c = (slice(1, -1),) * 3

    def d(axis, comp, h):
        sl_p = [slice(1, -1)] * 3
        sl_m = [slice(1, -1)] * 3
        sl_p[axis] = slice(2, None)
        sl_m[axis] = slice(0, -2)
        return (u[tuple(sl_p) + (comp,)] - u[tuple(sl_m) + (comp,)]) / (2 * h)

    # axes of the array: 0 = z, 1 = y, 2 = x
    g = [[d(2, i, dx), d(1, i, dy), d(0, i, dz)] for i in range(3)]
    s2 = np.zeros(q[c].shape)
    o2 = np.zeros(q[c].shape)
    for i in range(3):
        for j in range(3):
            sij = 0.5 * (g[i][j] + g[j][i])
            oij = 0.5 * (g[i][j] - g[j][i])
            s2 = s2 + sij * sij
            o2 = o2 + oij * oij
    q[c] = 0.5 * (o2 - s2)
    return q.reshape(-1)


def thermal_d3q7_step(g, u, nx: int, ny: int, nz: int, diffusivity: float, steps: int = 1):
    """The reference's resident D3Q7 thermal step (resident_multiphysics_sycl.hpp:94-130) restated in
    float32 numpy, operand for operand: pull from the periodic neighbours, T = sum in direction order,
    geq = (w T)(1 + 4 c.u) with c.u = (cx ux + cy uy) + cz uz, out = g - omega (g - geq),
    tau = 0.5 + 4 D, omega = 1 / tau.  g is [7][nz][ny][nx], u = (ux, uy, uz) per cell."""
    f32 = np.float32
    cx, cy, cz = [0, 1, -1, 0, 0, 0, 0], [0, 0, 0, 1, -1, 0, 0], [0, 0, 0, 0, 0, 1, -1]
    w = [f32(0.25)] + [f32(0.125)] * 6
    tau = f32(f32(0.5) + f32(f32(4.0) * f32(diffusivity)))
    omega = f32(f32(1.0) / tau)
    g = np.asarray(g, f32).reshape(7, nz, ny, nx).copy()
    ux, uy, uz = (np.asarray(c, f32).reshape(nz, ny, nx) for c in u)
    for _ in range(steps):
        local = [np.roll(g[d], shift=(cz[d], cy[d], cx[d]), axis=(0, 1, 2)) for d in range(7)]
        t = np.zeros((nz, ny, nx), f32)
        for d in range(7):
            t = t + local[d]
        out = np.empty_like(g)
        for d in range(7):
            cu = (f32(cx[d]) * ux + f32(cy[d]) * uy) + f32(cz[d]) * uz
            geq = (w[d] * t) * (f32(1.0) + f32(4.0) * cu)
            out[d] = local[d] - omega * (local[d] - geq)
        g = out
    return g.reshape(-1)


# The velocity sets in the reference's direction order (descriptors.hpp:59-146): D3Q19 is the first
# 19 directions of D3Q27; pairs (i, i+1) for odd i are opposites.
_CX = (0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1)
_CY = (0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1)
_CZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1)


def velocity_set(q: int) -> np.ndarray:
    """(q, 3) integer lattice velocities of D3Q19 or D3Q27."""
    if q not in (19, 27):
        raise ValueError("q must be 19 or 27")
    return np.stack([_CX[:q], _CY[:q], _CZ[:q]], 1).astype(np.int64)


def f32_to_f16_bits(v: float) -> int:
    return int(oracle_lib().ora_f32_to_f16(v))


def f16_bits_to_f32(h: int) -> float:
    return float(oracle_lib().ora_f16_to_f32(h))


# ----------------------------------------------------------------- reference
def reference_available(fast: bool = False) -> bool:
    return (REF_FAST_SO if fast else REF_SO).exists()


def ref_lib(fast: bool = False):
    key = "fast" if fast else "exact"
    if key not in _ref:
        path = REF_FAST_SO if fast else REF_SO
        if not path.exists():
            raise RuntimeError(f"{path} is not built; run `make -C oracle ref` where the reference is present")
        lib = ctypes.CDLL(str(path))
        sz = ctypes.c_size_t
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_thread_capacity.restype = ctypes.c_uint
        lib.ref_esoteric_run.argtypes = [ctypes.c_int, sz, sz, sz, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_int, ctypes.c_int, _f, _u8, _f, sz, _f, _f, _f, _f,
                                         _f, _d]
        lib.ref_twogrid_run.argtypes = [ctypes.c_int, sz, sz, sz, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_float, ctypes.c_int, _f, sz, _f, _f, _f, _f, _d]
        lib.ref_precision_run.argtypes = [ctypes.c_int, sz, sz, sz, ctypes.c_double, ctypes.c_int, _d, sz, _d, _d,
                                          _d, _d, _d]
        lib.ref_compressed_run.argtypes = [ctypes.c_int, sz, sz, sz, ctypes.c_float, ctypes.c_int, _f, sz, _f, _f,
                                           _f, _f, _d]
        lib.ref_bench.argtypes = [ctypes.c_int, sz, sz, sz, ctypes.c_float, ctypes.c_int, _u8, sz, sz, ctypes.c_uint,
                                  _d, _d]
        lib.ref_bench.restype = ctypes.c_double
        lib.ref_voxelize.argtypes = [_d, sz, sz, sz, sz, _d, _d, _u8]
        lib.ref_transform_surface.argtypes = [_d, sz, _d, _d, ctypes.c_double, _d]
        lib.ref_free_surface.argtypes = [sz, sz, sz, _d, _f, _f, _f, ctypes.c_double, sz, ctypes.c_double,
                                         ctypes.c_double, _d, _d, _d, _d]
        lib.ref_particles.argtypes = [sz, sz, sz, _f, _f, _f, _d, sz, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, _f]
        _ref[key] = lib
    return _ref[key]


def ref_voxelize(tris, nx: int, ny: int, nz: int, lo, hi) -> np.ndarray:
    """The reference's voxelize_surface (src/lbm/voxelize.cpp) on the same inputs."""
    lib = ref_lib()
    t = np.ascontiguousarray(tris, np.float64).reshape(-1, 9)
    lo_, hi_ = np.ascontiguousarray(lo, np.float64), np.ascontiguousarray(hi, np.float64)
    mask = np.zeros(nx * ny * nz, np.uint8)
    _check(lib, lib.ref_voxelize(_ptr(t, _d), len(t), nx, ny, nz, _ptr(lo_, _d), _ptr(hi_, _d), _ptr(mask, _u8)))
    return mask


def ref_transform_surface(tris, translation, axis, angle: float) -> np.ndarray:
    lib = ref_lib()
    t = np.ascontiguousarray(tris, np.float64).reshape(-1, 9)
    tr, ax = np.ascontiguousarray(translation, np.float64), np.ascontiguousarray(axis, np.float64)
    out = np.empty_like(t)
    _check(lib, lib.ref_transform_surface(_ptr(t, _d), len(t), _ptr(tr, _d), _ptr(ax, _d), float(angle),
                                          _ptr(out, _d)))
    return out


def ref_free_surface(fill, u, nx: int, ny: int, nz: int, dt: float, steps: int, sigma: float = 0.0,
                     density: float = 1.0) -> dict:
    """The reference's CPU free surface (src/lbm/free_surface.cpp): `steps` advect_free_surface_vof
    calls (interface epsilon 0), then normals, curvature, surface-tension acceleration and volume."""
    lib = ref_lib()
    n = nx * ny * nz
    f = np.ascontiguousarray(fill, np.float64).reshape(-1).copy()
    ux, uy, uz = (np.ascontiguousarray(c, np.float32).reshape(-1) for c in u)
    normals, tension = np.zeros(3 * n), np.zeros(3 * n)
    curvature, volume = np.zeros(n), np.zeros(1)
    _check(lib, lib.ref_free_surface(nx, ny, nz, _ptr(f, _d), _ptr(ux, _f), _ptr(uy, _f), _ptr(uz, _f), float(dt),
                                     int(steps), float(sigma), float(density), _ptr(normals, _d),
                                     _ptr(curvature, _d), _ptr(tension, _d), _ptr(volume, _d)))
    return {"fill": f, "normals": normals.reshape(n, 3).T.copy(), "curvature": curvature,
            "tension": tension.reshape(n, 3).T.copy(), "volume": float(volume[0])}


def ref_particles(records, u, nx: int, ny: int, nz: int, dt: float, two_way: bool, gravity=(0.0, 0.0, 0.0)):
    """The reference's CPU advance_immersed_boundary_particles (src/lbm/particles.cpp:86-140), once:
    (records after the step, count x 8 doubles; acceleration 3 x N floats or None)."""
    lib = ref_lib()
    n = nx * ny * nz
    r = np.ascontiguousarray(records, np.float64).reshape(-1, 8).copy()
    ux, uy, uz = (np.ascontiguousarray(c, np.float32).reshape(-1) for c in u)
    acc = np.zeros(3 * n, np.float32)
    _check(lib, lib.ref_particles(nx, ny, nz, _ptr(ux, _f), _ptr(uy, _f), _ptr(uz, _f), _ptr(r, _d), len(r), float(dt),
                                  int(bool(two_way)), *(float(g) for g in gravity), _ptr(acc, _f)))
    return r, (acc.reshape(3, n) if two_way else None)


# ------------------------------------------------ resident free surface, particles, Q
# Restatements of the reference's resident SYCL solvers (resident_multiphysics_sycl.hpp:202-405)
# in float32 numpy, one rounding per operation in the reference's operand order.  Fields are
# flat arrays of nx*ny*nz cells, x fastest; every axis is periodic.

def _shifts(v, nx: int, ny: int, nz: int):
    """(xp, xm, yp, ym, zp, zm): the periodic neighbour values of every cell."""
    a = np.asarray(v).reshape(nz, ny, nx)
    return tuple(np.roll(a, s, axis=ax).reshape(-1) for ax in (2, 1, 0) for s in (-1, 1))


def fill_half_space_x(nx: int, ny: int, nz: int, interface_x: float) -> np.ndarray:
    """initialize_half_space_x (resident_multiphysics_sycl.hpp:227-236)."""
    f32 = np.float32
    left = (np.arange(nx * ny * nz) % nx).astype(f32)
    right = left + f32(1.0)
    i = f32(interface_x)
    return np.where(i <= left, f32(0.0), np.where(i >= right, f32(1.0), i - left)).astype(f32)


def fill_advect(phi, u, nx: int, ny: int, nz: int, dt: float) -> np.ndarray:
    """advect (resident_multiphysics_sycl.hpp:238-264): face velocity 0.5 (u_n + u_nb), upwind
    flux u_face * phi_upwind, phi - dt ((fxp - fxm) + (fyp - fym) + (fzp - fzm)), clamped to [0, 1]."""
    f32 = np.float32
    half, dt = f32(0.5), f32(dt)
    p = np.asarray(phi, f32).reshape(-1)
    ux, uy, uz = (np.asarray(c, f32).reshape(-1) for c in u)
    pxp, pxm, pyp, pym, pzp, pzm = _shifts(p, nx, ny, nz)
    uxp_, uxm_, _, _, _, _ = _shifts(ux, nx, ny, nz)
    _, _, uyp_, uym_, _, _ = _shifts(uy, nx, ny, nz)
    _, _, _, _, uzp_, uzm_ = _shifts(uz, nx, ny, nz)

    def up(v, here, there):
        return np.where(v >= 0, v * here, v * there)

    uxp, uxm = half * (ux + uxp_), half * (uxm_ + ux)
    uyp, uym = half * (uy + uyp_), half * (uym_ + uy)
    uzp, uzm = half * (uz + uzp_), half * (uzm_ + uz)
    div = ((up(uxp, p, pxp) - up(uxm, pxm, p)) + (up(uyp, p, pyp) - up(uym, pym, p))) + (up(uzp, p, pzp) -
                                                                                       up(uzm, pzm, p))
    v = p - dt * div
    return np.where(v < 0, f32(0.0), np.where(v > 1, f32(1.0), v)).astype(f32)


def _half_gradient(p, nx, ny, nz):
    f32 = np.float32
    pxp, pxm, pyp, pym, pzp, pzm = _shifts(p, nx, ny, nz)
    return f32(0.5) * (pxp - pxm), f32(0.5) * (pyp - pym), f32(0.5) * (pzp - pzm)


def fill_geometry(phi, nx: int, ny: int, nz: int):
    """refresh_geometry (resident_multiphysics_sycl.hpp:269-298): normals grad/|grad| (0 where
    |grad| <= 1e-12) and curvature -0.5 ((nx_xp - nx_xm) + (ny_yp - ny_ym) + (nz_zp - nz_zm))."""
    f32 = np.float32
    p = np.asarray(phi, f32).reshape(-1)
    gx, gy, gz = _half_gradient(p, nx, ny, nz)
    mag = np.sqrt((gx * gx + gy * gy) + gz * gz)
    ok = mag > f32(1.0e-12)
    safe = np.where(ok, mag, f32(1.0))
    nrm = [np.where(ok, g / safe, f32(0.0)).astype(f32) for g in (gx, gy, gz)]
    sx = _shifts(nrm[0], nx, ny, nz)
    sy = _shifts(nrm[1], nx, ny, nz)
    sz = _shifts(nrm[2], nx, ny, nz)
    curvature = f32(-0.5) * (((sx[0] - sx[1]) + (sy[2] - sy[3])) + (sz[4] - sz[5]))
    return nrm[0], nrm[1], nrm[2], curvature.astype(f32)


def surface_tension(phi, curvature, acceleration, nx: int, ny: int, nz: int, sigma: float, density: float = 1.0):
    """add_surface_tension_acceleration (resident_multiphysics_sycl.hpp:300-318) on (ax, ay, az):
    c = sigma * kappa / rho; a += c * 0.5 (phi_p - phi_m) per axis."""
    f32 = np.float32
    p = np.asarray(phi, f32).reshape(-1)
    c = (f32(sigma) * np.asarray(curvature, f32)) / f32(density)
    return tuple((np.asarray(a, f32) + c * g).astype(f32) for a, g in zip(acceleration, _half_gradient(p, nx, ny, nz)))


def _periodic32(v, extent: int):
    f32 = np.float32
    e = f32(extent)
    turns = np.floor(v / e).astype(f32)
    v = v - turns * e
    v = np.where(v >= e, v - e, v)
    return np.where(v < 0, v + e, v).astype(f32)


def particles_advance(state, u, acceleration, nx: int, ny: int, nz: int, dt: float, two_way: bool,
                      gravity=(0.0, 0.0, 0.0)):
    """ResidentParticlesSycl3D::advance (resident_multiphysics_sycl.hpp:348-369) on the float32
    state [8][count] (x, y, z, vx, vy, vz, mass, response): trilinear velocity in (dz, dy, dx)
    order, drag = mass (u - v) / response, two-way spreading of -drag * w (added here in particle
    order; the device adds atomically), v += dt (drag / mass + g), x = periodic(x + dt v)."""
    f32 = np.float32
    st = np.asarray(state, f32).reshape(8, -1).copy()
    dt = f32(dt)
    g = [f32(v) for v in gravity]
    ux, uy, uz = (np.asarray(c, f32).reshape(-1) for c in u)
    acc = None if acceleration is None else [np.asarray(a, f32).reshape(-1).copy() for a in acceleration]
    pos = [_periodic32(st[k], e) for k, e in enumerate((nx, ny, nz))]
    vel = [st[3], st[4], st[5]]
    mass, response = st[6], st[7]
    base = [np.floor(p).astype(np.int64) for p in pos]
    t = [p - b.astype(f32) for p, b in zip(pos, base)]
    fu = [np.zeros_like(mass) for _ in range(3)]
    corners = []
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = [t[k] if d else f32(1.0) - t[k] for k, d in enumerate((dx, dy, dz))]
                ix = (base[0] + dx) % nx
                iy = (base[1] + dy) % ny
                iz = (base[2] + dz) % nz
                n = (iz * ny + iy) * nx + ix
                wt = (w[0] * w[1]) * w[2]
                corners.append((n, wt))
                fu = [f + wt * c[n] for f, c in zip(fu, (ux, uy, uz))]
    drag = [(mass * (f - v)) / response for f, v in zip(fu, vel)]
    if two_way:
        for p_ in range(mass.size):
            for n, wt in corners:
                for k in range(3):
                    acc[k][n[p_]] = f32(acc[k][n[p_]] + f32(-drag[k][p_]) * wt[p_])
    vel = [v + dt * (d / mass + gk) for v, d, gk in zip(vel, drag, g)]
    pos = [_periodic32(p + dt * v, e) for p, v, e in zip(pos, vel, (nx, ny, nz))]
    for k in range(3):
        st[k] = pos[k]
        st[3 + k] = vel[k]
    return st, (None if acc is None else tuple(acc))


def resident_q(u, nx: int, ny: int, nz: int) -> np.ndarray:
    """ResidentFlowDiagnosticsSycl3D::q_criterion (resident_multiphysics_sycl.hpp:394-402): periodic
    g[i][axis] = 0.5 (u_i(+) - u_i(-)), s2 and o2 over (i, j) in row order, Q = 0.5 (o2 - s2)."""
    f32 = np.float32
    half = f32(0.5)
    comps = [_shifts(np.asarray(c, f32).reshape(-1), nx, ny, nz) for c in u]
    g = [[half * (comps[i][2 * a] - comps[i][2 * a + 1]) for a in range(3)] for i in range(3)]
    s2 = np.zeros_like(g[0][0])
    o2 = np.zeros_like(g[0][0])
    for i in range(3):
        for j in range(3):
            sij, oij = half * (g[i][j] + g[j][i]), half * (g[i][j] - g[j][i])
            s2 = s2 + sij * sij
            o2 = o2 + oij * oij
    return (half * (o2 - s2)).astype(f32)


def _init_args(init):
    kind, *vals = init
    if kind == "uniform":
        p = np.array((list(vals) + [1.0, 0.0, 0.0, 0.0])[:4] if vals else [1.0, 0, 0, 0], np.float32)
        return 0, p
    p = np.array([vals[0] if vals else 0.03, 0, 0, 0], np.float32)
    return 1, p


def _check(lib, rc):
    if rc != 0:
        raise ValueError(lib.ref_last_error().decode())


def ref_esoteric(q, nx, ny, nz, tau, steps, init=("tg", 0.03), accel=(0.0, 0.0, 0.0), les=False, mask=None,
                 local_a=None, logical=False, fast=False):
    """Run the reference EsotericPullSolver<D> (esoteric_pull.hpp:104-515)."""
    lib = ref_lib(fast)
    n = nx * ny * nz
    kind, p = _init_args(init)
    rho, ux, uy, uz = (np.zeros(n, np.float32) for _ in range(4))
    pops = np.zeros(q * n, np.float32) if logical else None
    out = np.zeros(3, np.float64)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    la = None if local_a is None else np.ascontiguousarray(local_a, np.float32)
    _check(lib, lib.ref_esoteric_run(q, nx, ny, nz, tau, *accel, int(les), kind, _ptr(p, _f), _ptr(m, _u8),
                                     _ptr(la, _f), steps, _ptr(rho, _f), _ptr(ux, _f), _ptr(uy, _f), _ptr(uz, _f),
                                     _ptr(pops, _f), _ptr(out, _d)))
    return {"rho": rho, "ux": ux, "uy": uy, "uz": uz, "logical": pops, "mass": out[0], "kinetic_energy": out[1],
            "max_speed": out[2]}


def ref_twogrid(q, nx, ny, nz, tau, odd_tau, steps, init=("tg", 0.03), accel=(0.0, 0.0, 0.0)):
    """Run the reference two-grid OneStepPullSolver<D>(config, odd_tau) (one_step_pull.hpp:16-215)."""
    lib = ref_lib()
    n = nx * ny * nz
    kind, p = _init_args(init)
    rho, ux, uy, uz = (np.zeros(n, np.float32) for _ in range(4))
    mass = np.zeros(1, np.float64)
    _check(lib, lib.ref_twogrid_run(q, nx, ny, nz, tau, odd_tau, *accel, kind, _ptr(p, _f), steps, _ptr(rho, _f),
                                    _ptr(ux, _f), _ptr(uy, _f), _ptr(uz, _f), _ptr(mass, _d)))
    return {"rho": rho, "ux": ux, "uy": uy, "uz": uz, "mass": mass[0]}


def ref_precision(q, nx, ny, nz, tau, steps, init=("tg", 0.03)):
    """Run the reference FP64 two-grid PrecisionPullSolver<D,double> (precision_pull.hpp:49-213)."""
    lib = ref_lib()
    n = nx * ny * nz
    kind, p32 = _init_args(init)
    p = np.array([init[1] if len(init) > 1 else 0.03, 0, 0, 0], np.float64) if kind == 1 else p32.astype(np.float64)
    rho, ux, uy, uz = (np.zeros(n, np.float64) for _ in range(4))
    mass = np.zeros(1, np.float64)
    _check(lib, lib.ref_precision_run(q, nx, ny, nz, tau, kind, _ptr(p, _d), steps, _ptr(rho, _d), _ptr(ux, _d),
                                      _ptr(uy, _d), _ptr(uz, _d), _ptr(mass, _d)))
    return {"rho": rho, "ux": ux, "uy": uy, "uz": uz, "mass": mass[0]}


def ref_compressed(q, nx, ny, nz, tau, steps, init=("tg", 0.03)):
    """Run the reference shifted-FP16 two-grid solver (compressed_pull.hpp:72-147)."""
    lib = ref_lib()
    n = nx * ny * nz
    kind, p = _init_args(init)
    rho, ux, uy, uz = (np.zeros(n, np.float32) for _ in range(4))
    mass = np.zeros(1, np.float64)
    _check(lib, lib.ref_compressed_run(q, nx, ny, nz, tau, kind, _ptr(p, _f), steps, _ptr(rho, _f), _ptr(ux, _f),
                                       _ptr(uy, _f), _ptr(uz, _f), _ptr(mass, _d)))
    return {"rho": rho, "ux": ux, "uy": uy, "uz": uz, "mass": mass[0]}


def ref_bench(q, nx, ny, nz, tau, warmup, steps, threads=0, les=False, mask=None):
    """Time the reference in-place CPU step (optimised build).  Returns (MLUPS, seconds, mass_rel)."""
    lib = ref_lib(fast=True)
    sec = np.zeros(1, np.float64)
    rel = np.zeros(1, np.float64)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    mlups = lib.ref_bench(q, nx, ny, nz, tau, int(les), _ptr(m, _u8), warmup, steps, threads, _ptr(sec, _d),
                          _ptr(rel, _d))
    if mlups < 0:
        raise ValueError(lib.ref_last_error().decode())
    return mlups, float(sec[0]), float(rel[0])


def ref_threads() -> int:
    return int(ref_lib(fast=True).ref_thread_capacity())


def cavity_flags(nx, ny, nz, lid_id=2):
    """Lid-driven cavity flags: walls on x=0, x=nx-1, y=0, z=0, z=nz-1; moving lid on y=ny-1."""
    fl = np.zeros((nz, ny, nx), np.uint8)
    fl[:, :, 0] = 1
    fl[:, :, nx - 1] = 1
    fl[:, 0, :] = 1
    fl[0, :, :] = 1
    fl[nz - 1, :, :] = 1
    fl[:, ny - 1, :] = lid_id
    return fl.reshape(-1)


if os.environ.get("CFDX_ORACLE_SELFTEST"):
    print(reference_les_k())
