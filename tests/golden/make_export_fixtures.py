"""Generates tests/golden/export_fixtures.npz from the REFERENCE field writers.

The files are the output of the reference's write_vtk_structured_3d and
write_json_state_3d (src/lbm/visualization.cpp:39-109) and the arrays the
output of its q_criterion_3d (:122-148), compiled from its sources by
oracle/Makefile into oracle/_ref/libcfdref.so.  They pin the engine's writers
(tests/test_export_host.py, byte for byte) and its device Q-criterion
(tests/test_gpu_export.py, bit for bit) where the reference is not present.

Run from the repository root after ``make -C oracle``:
    python tests/golden/make_export_fixtures.py

Inputs (seeded, synthetic): a 5 x 4 x 3 field whose values include integers,
negative numbers, tiny and huge magnitudes and signed zeros; a 7 x 6 x 5
random velocity field with spacings (1, 0.5, 2) for the Q-criterion.
"""
from __future__ import annotations

import ctypes
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "export_fixtures.npz"


def field_inputs():
    rng = np.random.default_rng(4)
    n = 5 * 4 * 3
    s = rng.normal(0, 1, n)
    s[:8] = [1.0, -2.0, 0.0, -0.0, 1e-300, 3.5e200, 1.0 / 3.0, 123456789.0]
    u = rng.normal(0, 0.05, (n, 3))
    u[0] = (0.0, -0.0, 1.0)
    solid = (rng.random(n) < 0.3).astype(np.uint8)
    solid[1] = 7
    return s, u, solid


def main():
    if not O.reference_available():
        raise SystemExit("oracle/_ref/libcfdref.so is not built (run `make -C oracle` where the reference is present)")
    lib = O.ref_lib()
    dp = ctypes.POINTER(ctypes.c_double)
    u8 = ctypes.POINTER(ctypes.c_uint8)
    sz = ctypes.c_size_t
    lib.ref_write_vtk_3d.argtypes = [ctypes.c_char_p, sz, sz, sz, dp, dp, u8, ctypes.c_char_p]
    lib.ref_write_json_3d.argtypes = [ctypes.c_char_p, sz, sz, sz, ctypes.c_uint64, dp, u8, ctypes.c_char_p]
    lib.ref_q_criterion.argtypes = [sz, sz, sz, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
    s, u, solid = field_inputs()
    arrays = {"scalar": s, "velocity": u, "solid": solid}
    with tempfile.TemporaryDirectory() as d:
        for key, vel, sol in (("vtk_full", u, solid), ("vtk_scalar", None, None)):
            path = f"{d}/{key}.vtk".encode()
            rc = lib.ref_write_vtk_3d(path, 5, 4, 3, s.ctypes.data_as(dp),
                                      None if vel is None else np.ascontiguousarray(vel).ctypes.data_as(dp),
                                      None if sol is None else sol.ctypes.data_as(u8), b"speed")
            assert rc == 0, lib.ref_last_error()
            arrays[key] = np.frombuffer(Path(path.decode()).read_bytes(), np.uint8)
        for key, sol in (("json_full", solid), ("json_scalar", None)):
            path = f"{d}/{key}.json".encode()
            rc = lib.ref_write_json_3d(path, 5, 4, 3, 1234, s.ctypes.data_as(dp),
                                       None if sol is None else sol.ctypes.data_as(u8), b"speed")
            assert rc == 0, lib.ref_last_error()
            arrays[key] = np.frombuffer(Path(path.decode()).read_bytes(), np.uint8)
    rng = np.random.default_rng(5)
    vel = np.ascontiguousarray(rng.normal(0, 0.1, (7 * 6 * 5, 3)))
    q = np.zeros(7 * 6 * 5)
    assert lib.ref_q_criterion(7, 6, 5, vel.ctypes.data_as(dp), 1.0, 0.5, 2.0, q.ctypes.data_as(dp)) == 0
    arrays["q_velocity"] = vel
    arrays["q_reference"] = q
    np.savez_compressed(OUT, **arrays)
    print({k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
