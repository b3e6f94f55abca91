"""Device Q-criterion and solver export (GPU).

* cfdx_q_criterion equals the reference's q_criterion_3d bit for bit on the
  golden velocity field (tests/golden/export_fixtures.npz), from host and from
  device memory;
* a solver's q_criterion (macroscopic velocity -> Q without leaving the
  device) equals the oracle's Q of the downloaded velocity, FP32 and FP64
  storage, D3Q19 and D3Q27;
* write_vtk / write_json_state write the same bytes as the host writers given
  the downloaded fields; slabs refuse the Q-criterion.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "export_fixtures.npz"


def test_q_matches_reference(engine):
    import torch

    from cfd_solvers_b200 import export as E

    fx = np.load(GOLDEN)
    q = E.q_criterion_3d(7, 6, 5, fx["q_velocity"], 1.0, 0.5, 2.0)
    assert np.array_equal(q, fx["q_reference"])
    dev = torch.tensor(fx["q_velocity"], device="cuda:0")
    qd = E.q_criterion_3d(7, 6, 5, dev, 1.0, 0.5, 2.0)
    assert np.array_equal(qd.cpu().numpy(), fx["q_reference"])
    with pytest.raises(ValueError):
        E.q_criterion_3d(2, 6, 5, np.zeros((60, 3)))


@pytest.mark.parametrize("spacing", [(1.0, 0.5, 2.0), (0.3, 0.7, 1.1), (1.0, 0.3, 0.125)])
def test_q_spacings_match_oracle(engine, oracle_mod, spacing):
    """Power-of-two spacings take the multiply path, others the division path (mixed in the last
    case); both equal the FP64 restatement of the reference's q_criterion_3d bit for bit."""
    from cfd_solvers_b200 import export as E

    nx, ny, nz = 11, 9, 8
    v = np.random.default_rng(4).normal(0, 0.05, (nx * ny * nz, 3))
    q = E.q_criterion_3d(nx, ny, nz, v, *spacing)
    assert np.array_equal(q, oracle_mod.q_criterion(v, nx, ny, nz, *spacing))


def run_solver(cs, storage, lattice):
    cfg = cs.InPlaceLbmConfig(nx=14, ny=12, nz=10, tau=0.6, storage=storage, lattice=lattice, collision="trt",
                              acceleration_x=1e-4)
    s = cs.EsotericPullCudaSolver(cfg)
    s.set_flags(cs.cavity_flags(14, 12, 10))
    s.set_wall_velocity(2, 0.05, 0.0, 0.0)
    s.initialize_taylor_green(0.03)
    s.step(7)
    return s


@pytest.mark.parametrize("storage", ["fp32", "fp64"])
@pytest.mark.parametrize("lattice", ["d3q19", "d3q27"])
def test_solver_q_equals_oracle_of_downloaded_velocity(engine, oracle_mod, storage, lattice):
    import torch

    with run_solver(engine, storage, lattice) as s:
        f = s.compute_macroscopic()
        vel = np.stack([np.asarray(c, np.float64) for c in (f.ux, f.uy, f.uz)], axis=1)
        expect = oracle_mod.q_criterion(vel, 14, 12, 10, 1.0, 2.0, 0.5)
        assert np.array_equal(s.q_criterion(1.0, 2.0, 0.5), expect)
        out = torch.empty(14 * 12 * 10, dtype=torch.float64, device="cuda:0")
        s.q_criterion(1.0, 2.0, 0.5, out=out)
        assert np.array_equal(out.cpu().numpy(), expect)


def test_solver_writers(engine, tmp_path):
    from cfd_solvers_b200 import export as E

    with run_solver(engine, "fp32", "d3q19") as s:
        s.write_vtk(tmp_path / "frame.vtk")
        s.write_json_state(tmp_path / "live" / "state.json", field="q_criterion")
        s.write_vtk(tmp_path / "frame_b.vtk", field="rho", binary=True)
        f = s.compute_macroscopic()
        solid = (np.asarray(f.rho) == 0).astype(np.uint8)
        E.write_vtk_structured_3d(tmp_path / "host.vtk", 14, 12, 10, E.speed(f), (f.ux, f.uy, f.uz), solid, "speed")
        E.write_json_state_3d(tmp_path / "host.json", 14, 12, 10, s.time_step(), s.q_criterion(), solid,
                              "q_criterion")
        E.write_vtk_structured_3d(tmp_path / "host_b.vtk", 14, 12, 10, np.asarray(f.rho, np.float64),
                                  (f.ux, f.uy, f.uz), solid, "rho", binary=True)
    assert (tmp_path / "frame.vtk").read_bytes() == (tmp_path / "host.vtk").read_bytes()
    assert (tmp_path / "live" / "state.json").read_bytes() == (tmp_path / "host.json").read_bytes()
    assert (tmp_path / "frame_b.vtk").read_bytes() == (tmp_path / "host_b.vtk").read_bytes()
    assert solid.sum() > 0


def test_slab_refuses_q(engine):
    from cfd_solvers_b200 import slabs as S

    cfg = engine.InPlaceLbmConfig(nx=8, ny=8, nz=8)
    with S.SlabSolver(cfg, 0, 4) as s:
        with pytest.raises(ValueError):
            s.q_criterion()
