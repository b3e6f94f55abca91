"""Generates the golden fixtures in this directory from the REFERENCE itself.

Every array here is produced by the reference's own CPU solvers, compiled
from its sources by oracle/Makefile into oracle/_ref/libcfdref.so (bit-exact
build, -ffp-contract=off).  The fixtures pin the CPU oracle (tests/test_oracle_golden.py)
and the CUDA path (tests/test_gpu_parity.py) on machines where the reference
is not present.

Run from the repository root after ``make -C oracle``:
    python tests/golden/make_golden.py

Cases (reference files and tests they restate):
  c1_d3q19_tg64      64^3 D3Q19 BGK, tau 0.6, Taylor-Green A = 0.05, 10 + 100 steps
                     (the plain-method config; esoteric_pull.hpp:104-515).  Fields are
                     stored on every 4th cell of a fixed stride to keep the file small.
  sycl_parity_q19/q27  16x14x12, tau 0.72, a = (1e-6, -0.5e-6, 0.25e-6), A = 0.018, 12 steps
                     (the CPU/SYCL parity template, tests/test_main.cpp:587-615)
  les_q19            20x18x16, tau 0.56, Smagorinsky, A = 0.05, 24 steps
                     (tests/test_v0141_lbm_les_qcriterion.cpp:50-61)
  solid_first_q19/q27  12x10x8 random 15% mask (seed 1), tau 0.8, a = (2e-5,-1e-5,5e-6),
                     A = 0.02, one step: logical populations (esoteric_pull.hpp:434-492)
  trt_q19/q27_s7/s8  two-grid TRT 18x14x10, tau 0.73, tau- 1.1, a = (2e-6,-1e-6,5e-7), A = 0.017
                     (one_step_pull.hpp:187-204; tests/test_main.cpp:340-434)
  bgk_q19/q27_s7/s8  two-grid BGK OneStepPullSolver(config) 18x14x10, tau 0.73, A = 0.017
                     (tests/test_main.cpp:340-372, odd and even step counts)
  bgk_forced_q19/q27 the same from rest with a = (2e-6, -1e-6, 5e-7), 60 steps
                     (tests/test_main.cpp:403-434)
  f64_q19            two-grid FP64 18x14x10, tau 0.73, A = 0.017, 8 steps (precision_pull.hpp)
  f16_q19            two-grid shifted-FP16 16x14x12, tau 0.72, A = 0.025, 16 steps
                     (compressed_pull.hpp; tests/test_v0141_lbm_les_qcriterion.cpp:143-180)
  phase02            published checksum of examples/phase02_lbm_taylor_green.cpp
                     (examples/results/v0.19.0_reference.json:62-75)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

C1_STRIDE = 4


def fields(r):
    return {k: r[k] for k in ("rho", "ux", "uy", "uz")}


def main():
    out = {}
    meta = {}

    # C1: plain method, small
    r = O.ref_esoteric(19, 64, 64, 64, 0.6, 110, init=("tg", 0.05), logical=False)
    for k, v in fields(r).items():
        out[f"c1_d3q19_tg64_{k}"] = v[::C1_STRIDE].copy()
    meta["c1_d3q19_tg64"] = {"mass": r["mass"], "kinetic_energy": r["kinetic_energy"],
                             "max_speed": r["max_speed"], "checksum": r["mass"] + r["kinetic_energy"],
                             "stride": C1_STRIDE, "steps": 110, "tau": 0.6, "amplitude": 0.05}

    # CPU/SYCL parity template
    for q in (19, 27):
        r = O.ref_esoteric(q, 16, 14, 12, 0.72, 12, init=("tg", 0.018), accel=(1e-6, -0.5e-6, 0.25e-6), logical=True)
        for k, v in fields(r).items():
            out[f"sycl_parity_q{q}_{k}"] = v
        out[f"sycl_parity_q{q}_logical"] = r["logical"]
        meta[f"sycl_parity_q{q}"] = {"mass": r["mass"], "kinetic_energy": r["kinetic_energy"],
                                     "max_speed": r["max_speed"]}

    # Smagorinsky LES
    r = O.ref_esoteric(19, 20, 18, 16, 0.56, 24, init=("tg", 0.05), les=True, logical=True)
    for k, v in fields(r).items():
        out[f"les_q19_{k}"] = v
    out["les_q19_logical"] = r["logical"]
    meta["les_q19"] = {"mass": r["mass"], "kinetic_energy": r["kinetic_energy"], "max_speed": r["max_speed"]}

    # first solid step
    rng = np.random.default_rng(1)
    mask = (rng.random((8, 10, 12)) < 0.15).astype(np.uint8).reshape(-1)
    out["solid_first_mask"] = mask
    for q in (19, 27):
        r = O.ref_esoteric(q, 12, 10, 8, 0.8, 1, init=("tg", 0.02), accel=(2e-5, -1e-5, 0.5e-5), mask=mask,
                           logical=True)
        out[f"solid_first_q{q}_logical"] = r["logical"]

    # TRT two-grid
    for q in (19, 27):
        for s in (7, 8):
            r = O.ref_twogrid(q, 18, 14, 10, 0.73, 1.1, s, init=("tg", 0.017), accel=(2e-6, -1e-6, 0.5e-6))
            for k, v in fields(r).items():
                out[f"trt_q{q}_s{s}_{k}"] = v

    # BGK two-grid: the in-place/two-grid gates of tests/test_main.cpp:340-434
    for q in (19, 27):
        for s in (7, 8):
            r = O.ref_twogrid(q, 18, 14, 10, 0.73, 0.0, s, init=("tg", 0.017))
            for k, v in fields(r).items():
                out[f"bgk_q{q}_s{s}_{k}"] = v
        r = O.ref_twogrid(q, 18, 14, 10, 0.73, 0.0, 60, init=("uniform",), accel=(2e-6, -1e-6, 0.5e-6))
        for k, v in fields(r).items():
            out[f"bgk_forced_q{q}_{k}"] = v

    # FP64 two-grid
    r = O.ref_precision(19, 18, 14, 10, 0.73, 8, init=("tg", 0.017))
    for k, v in fields(r).items():
        out[f"f64_q19_{k}"] = v

    # shifted FP16 two-grid
    r = O.ref_compressed(19, 16, 14, 12, 0.72, 16, init=("tg", 0.025))
    for k, v in fields(r).items():
        out[f"f16_q19_{k}"] = v
    meta["f16_q19"] = {"mass": r["mass"]}

    # published phase02 checksum (examples/results/v0.19.0_reference.json:62-75)
    meta["phase02"] = {"n": 48, "tau": 0.58, "les": True, "amplitude": 0.04, "steps": 80,
                       "checksum": 110609.77375653926,
                       "source": "examples/results/v0.19.0_reference.json:73"}

    np.savez_compressed(HERE / "reference_fixtures.npz", **out)
    (HERE / "reference_fixtures.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    size = (HERE / "reference_fixtures.npz").stat().st_size
    print(f"wrote {len(out)} arrays ({size / 1e6:.2f} MB) and {len(meta)} metadata entries")


if __name__ == "__main__":
    main()
