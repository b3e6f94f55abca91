"""The cfd-solve-cuda case runner (cfd_solvers_b200/apps/cfd_solve.cpp).

It carries the reference's in-place LBM cases of apps/cfd-solve.cpp (`lbm-d3q19-*`,
`lbm-d3q27-*`: 64^3 / 56^3 periodic BGK, Taylor-Green 0.02, tau 0.6, 100 steps; the
reference's key=value output line) with the CUDA backend, and the 3-D cases of the engine:
lid-driven cavity, sphere-pack channel and the gray-LBM adjoint with a finite-difference check.
The CPU tests cover the listing and argument errors; the GPU tests run every case and check
its numbers against the Python API or physics.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SOLVE = ROOT / "cfd_solvers_b200" / "cfd-solve-cuda"
CASES = ("lbm-d3q19-cuda", "lbm-d3q27-cuda", "lbm-cavity3d-cuda", "lbm-channel-spheres-cuda", "lbm-gray-adjoint-cuda")


def run(*args, check=True):
    if not SOLVE.exists():
        pytest.skip("cfd-solve-cuda not built")
    r = subprocess.run([str(SOLVE), *args], capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError(f"rc={r.returncode}\n{r.stdout}\n{r.stderr}")
    return r


def values(line: str) -> dict:
    out = {}
    for tok in line.split():
        if "=" in tok:
            k, v = tok.split("=", 1)
            out[k] = v.strip('"')
    return out


def test_list_and_errors():
    listing = run("--list").stdout
    for case in CASES:
        assert case in listing
    r = run("lbm-d2q9-cuda", check=False)
    assert r.returncode == 1 and "Unknown solver: lbm-d2q9-cuda" in r.stderr and "lbm-d3q19-cuda" in r.stdout
    r = run("lbm-d3q19-cuda", "--steps", "0", check=False)
    assert r.returncode == 1 and "--steps must be a positive integer" in r.stderr
    r = run("lbm-d3q19-cuda", "--storage", "fp8", check=False)
    assert r.returncode == 1 and "--storage" in r.stderr
    r = run("lbm-d3q19-cuda", "--tau", "0.5", check=False)
    assert r.returncode == 1 and "--tau" in r.stderr


def test_no_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = run("lbm-d3q19-cuda", check=False)
    assert r.returncode == 1 and "no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case,edge,lattice", [("lbm-d3q19-cuda", 64, "d3q19"), ("lbm-d3q27-cuda", 56, "d3q27")])
def test_inplace_cases_match_python_api(engine, case, edge, lattice):
    v = values(run(case).stdout)
    assert v["backend"] == "cuda" and v["streaming"] == "in-place" and int(v["cells"]) == edge ** 3
    assert float(v["mass_error_rel"]) < 1e-5 and float(v["MLUPS"]) > 0
    with engine.EsotericPullCudaSolver(engine.InPlaceLbmConfig(nx=edge, ny=edge, nz=edge, tau=0.6,
                                                               lattice=lattice)) as s:
        s.initialize_taylor_green(0.02)
        s.step(100)
        assert float(v["kinetic_energy"]) == pytest.approx(s.kinetic_energy(), rel=1e-5)
        assert float(v["max_speed"]) == pytest.approx(s.max_speed(), rel=1e-5)


@pytest.mark.gpu
def test_cavity3d_case_and_export(tmp_path):
    vtk, js = tmp_path / "cavity.vtk", tmp_path / "cavity.json"
    v = values(run("lbm-cavity3d-cuda", "--n", "32", "--steps", "400", "--vtk", str(vtk), "--json", str(js)).stdout)
    assert v["case"] == "lid-driven-cavity-3d" and int(v["cells"]) == 32 ** 3
    assert 0.0 < float(v["max_speed"]) < 0.2 and float(v["mass_error_rel"]) < 1e-3
    assert np.isfinite(float(v["center_ux"])) and abs(float(v["center_ux"])) < 0.1
    assert vtk.read_text().startswith("# vtk DataFile Version 3.0")
    assert '"dimensions": [32, 32, 32]' in js.read_text()


@pytest.mark.gpu
def test_channel_spheres_fp16_tracks_fp32():
    args = ("lbm-channel-spheres-cuda", "--nx", "64", "--ny", "32", "--nz", "32", "--steps", "600", "--seed", "3")
    a = values(run(*args).stdout)
    b = values(run(*args, "--storage", "fp16s").stdout)
    assert a["sphere_fraction"] == b["sphere_fraction"] and float(a["sphere_fraction"]) >= 0.10
    ua, ub = float(a["mean_ux"]), float(b["mean_ux"])
    assert ua > 0 and abs(ub - ua) / ua < 2e-2
    assert float(b["mass_error_rel"]) < 1e-3


@pytest.mark.gpu
def test_gray_adjoint_case_fd_check():
    v = values(run("lbm-gray-adjoint-cuda", "--n", "16", "--steps", "60", "--interval", "8", "--storage", "fp64",
                   "--fd-check", "4").stdout)
    assert v["case"] == "gray-adjoint" and int(v["fd_cells"]) == 4
    assert float(v["J"]) > 0 and float(v["grad_ns_l2"]) > 0
    assert float(v["fd_max_abs_err_over_max_fd"]) < 1e-4
    w = values(run("lbm-gray-adjoint-cuda", "--n", "16", "--steps", "60", "--interval", "8").stdout)
    assert float(w["J"]) == pytest.approx(float(v["J"]), rel=1e-2)  # FP32 storage: same objective
    assert float(w["adjoint_over_forward"]) > 0
