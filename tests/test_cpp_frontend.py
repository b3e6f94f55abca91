"""C++20 front end and the cfd-bench CLI (compile on CPU; run on the GPU).

The C++ header must give reference-style drivers the reference's method
names and exception types; the CLI must keep cfd-bench's options and record
schema (apps/cfd-bench.cpp:100-170) with --backend cuda.
"""
from __future__ import annotations

import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "cfd_solvers_b200"
CLI = PKG / "cfd-bench-cuda"


def cxx():
    for c in ("/usr/bin/g++", "g++"):
        if shutil.which(c) or Path(c).exists():
            return c
    pytest.skip("no C++ compiler")


@pytest.fixture(scope="module")
def frontend(tmp_path_factory):
    lib = PKG / "libcfdx_lbm.so"
    if not lib.exists():
        pytest.skip("libcfdx_lbm.so not built")
    exe = tmp_path_factory.mktemp("cpp") / "frontend_check"
    subprocess.run([cxx(), "-std=c++20", "-O1", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "frontend_check.cpp"),
                    "-o", str(exe), f"-L{PKG}", "-lcfdx_lbm", f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def test_header_compiles_and_maps_errors_without_device(frontend):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    out = subprocess.run([str(frontend), "nodevice"], capture_output=True, text=True, check=True).stdout
    assert out.startswith("runtime_error") and "no CUDA device" in out


def test_cli_help_and_argument_errors():
    if not CLI.exists():
        pytest.skip("cfd-bench-cuda not built")
    assert "--backend cuda" in subprocess.run([str(CLI), "--help"], capture_output=True, text=True).stdout
    r = subprocess.run([str(CLI), "--backend", "cpu"], capture_output=True, text=True)
    assert r.returncode == 1 and "--backend cuda" in r.stderr
    r = subprocess.run([str(CLI), "--tau", "0.4"], capture_output=True, text=True)
    assert r.returncode == 1 and "must be > 0.5" in r.stderr


@pytest.mark.gpu
def test_frontend_on_gpu_matches_python_api(frontend, tmp_path, engine):
    out = subprocess.run([str(frontend), "gpu", str(tmp_path)], capture_output=True, text=True, check=True).stdout
    vals = dict(line.split(" ", 1) for line in out.strip().splitlines())
    import numpy as np

    cfg = engine.InPlaceLbmConfig(nx=24, ny=20, nz=16, tau=0.62, acceleration_x=1e-5)
    with engine.EsotericPullCudaSolver(cfg) as s:
        mask = np.zeros(24 * 20 * 16, np.uint8)
        mask[::17] = 1
        s.set_solid_mask(mask)
        s.initialize_taylor_green(0.04)
        s.step(13)
        assert int(vals["time_step"]) == 13
        assert float(vals["checksum"]) == s.checksum()
        assert float(vals["mass"]) == s.mass()
    assert vals["restart_bitwise"] == "1"
    assert vals["download_equal"] == "1"
    # slab class, device voxelizer, Q-criterion and writers through the C++ front end
    assert vals["slab_info"] == "0 16 16" and vals["slab_equals_whole"] == "1"
    assert int(vals["halo_bytes"]) == 5 * 24 * 20 * 4
    assert vals["voxel_cube"] == "1 0 64"  # the reference cube test's facts; 4^3 cells inside
    assert vals["q_criterion_equal"] == "1" and vals["exported"] == "1"
    assert (tmp_path / "frame.vtk").read_text().startswith("# vtk DataFile Version 3.0\ncfd_solvers LBM 3-D\nASCII")
    assert '"dimensions": [24, 20, 16]' in (tmp_path / "state.json").read_text()
    # the reference's resident chain through ResidentThermalD3Q7Cuda, ResidentFreeSurfaceCuda3D,
    # ResidentParticlesCuda3D and ResidentFlowDiagnosticsCuda3D
    for key in ("chain_thermal", "chain_volume", "chain_particles", "chain_q", "chain_flow"):
        assert vals[key] == "1", key
    assert vals["chain_grid"] == "invalid_argument"
    assert vals["size_mismatch"] == "invalid_argument"
    assert vals["wall_id"] == "out_of_range"


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["taylor-green", "cavity"])
def test_cli_json_record(case):
    r = subprocess.run([str(CLI), "--nx", "32", "--ny", "24", "--nz", "16", "--steps", "20", "--warmup", "3",
                        "--case", case, "--collision", "trt", "--storage", "fp16s", "--json"],
                       capture_output=True, text=True, check=True)
    rec = json.loads(r.stdout)
    for key in ("schema", "lattice", "backend", "streaming", "device", "nx", "ny", "nz", "q", "steps", "seconds",
                "mlups", "estimated_ddf_gbps", "allocated_ddf_mib", "single_grid_ddf_mib", "mass_error_abs",
                "mass_error_rel", "glups", "algorithmic_bytes_per_update", "storage_precision", "checksum"):
        assert key in rec
    assert rec["schema"] == "cfd_solvers.benchmark.v1" and rec["backend"] == "cuda" and rec["q"] == 19
    assert rec["mlups"] > 0 and rec["mass_error_rel"] < 1e-3


def test_release_scratch_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import cfd_solvers_b200 as cs
    from cfd_solvers_b200.bindings import CudaError

    with pytest.raises(CudaError):
        cs.release_scratch(0)
