"""Field writers and the Q-criterion oracle, without a GPU.

* the engine's native writers (cfdx_write_vtk_3d / cfdx_write_json_state_3d)
  produce the reference writers' files byte for byte
  (tests/golden/export_fixtures.npz, made by the reference's
  src/lbm/visualization.cpp:39-109), with and without velocity and solid
  data, and publish the JSON state through a temporary file;
* the binary legacy-VTK form reads back to the same values;
* the numpy Q-criterion restatement (oracle) equals the reference's
  q_criterion_3d bit for bit;
* size and path errors surface as ValueError / the I/O error.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from cfd_solvers_b200 import CfdxError
from cfd_solvers_b200 import export as E

GOLDEN = Path(__file__).resolve().parent / "golden" / "export_fixtures.npz"


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN)


def test_vtk_ascii_matches_reference_bytes(fx, tmp_path):
    s, u, solid = fx["scalar"], fx["velocity"], fx["solid"]
    E.write_vtk_structured_3d(tmp_path / "a.vtk", 5, 4, 3, s, u, solid, "speed")
    assert (tmp_path / "a.vtk").read_bytes() == bytes(fx["vtk_full"])
    E.write_vtk_structured_3d(tmp_path / "sub" / "b.vtk", 5, 4, 3, s, scalar_name="speed")
    assert (tmp_path / "sub" / "b.vtk").read_bytes() == bytes(fx["vtk_scalar"])
    # velocity as three component arrays gives the same file
    E.write_vtk_structured_3d(tmp_path / "c.vtk", 5, 4, 3, s, (u[:, 0], u[:, 1], u[:, 2]), solid, "speed")
    assert (tmp_path / "c.vtk").read_bytes() == bytes(fx["vtk_full"])


def test_json_matches_reference_bytes(fx, tmp_path):
    s, solid = fx["scalar"], fx["solid"]
    E.write_json_state_3d(tmp_path / "live" / "state.json", 5, 4, 3, 1234, s, solid, "speed")
    assert (tmp_path / "live" / "state.json").read_bytes() == bytes(fx["json_full"])
    assert not (tmp_path / "live" / "state.json.tmp").exists()
    E.write_json_state_3d(tmp_path / "live" / "state.json", 5, 4, 3, 1234, s, scalar_name="speed")  # replaces
    assert (tmp_path / "live" / "state.json").read_bytes() == bytes(fx["json_scalar"])


def read_binary_vtk(path):
    data = Path(path).read_bytes()
    out = {}
    pos = 0

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        text = data[pos:end].decode()
        pos = end + 1
        return text

    header = [line() for _ in range(10)]
    cells = int(header[7].split()[1])
    out["header"] = header
    out["scalar"] = np.frombuffer(data, ">f8", cells, pos)
    pos += 8 * cells + 1
    if pos < len(data) and data[pos:].startswith(b"VECTORS"):
        line()
        out["velocity"] = np.frombuffer(data, ">f8", 3 * cells, pos).reshape(-1, 3)
        pos += 24 * cells + 1
    if pos < len(data) and data[pos:].startswith(b"SCALARS solid"):
        line()
        line()
        out["solid"] = np.frombuffer(data, np.uint8, cells, pos)
        pos += cells + 1
    assert pos == len(data)
    return out


def test_vtk_binary_reads_back(fx, tmp_path):
    s, u, solid = fx["scalar"], fx["velocity"], fx["solid"]
    E.write_vtk_structured_3d(tmp_path / "b.vtk", 5, 4, 3, s, u, solid, "speed", binary=True)
    r = read_binary_vtk(tmp_path / "b.vtk")
    assert r["header"][2] == "BINARY" and r["header"][4] == "DIMENSIONS 5 4 3"
    assert np.array_equal(r["scalar"], s) and np.array_equal(r["velocity"], u) and np.array_equal(r["solid"], solid)


def test_writer_errors(fx, tmp_path):
    s = fx["scalar"]
    with pytest.raises(ValueError):
        E.write_vtk_structured_3d(tmp_path / "x.vtk", 5, 4, 4, s)
    with pytest.raises(ValueError):
        E.write_json_state_3d(tmp_path / "x.json", 5, 4, 3, 0, s, np.zeros(7, np.uint8))
    (tmp_path / "dir.vtk").mkdir()
    with pytest.raises(CfdxError):
        E.write_vtk_structured_3d(tmp_path / "dir.vtk", 5, 4, 3, s)


def test_q_oracle_matches_reference(oracle_mod, fx):
    q = oracle_mod.q_criterion(fx["q_velocity"], 7, 6, 5, 1.0, 0.5, 2.0)
    assert np.array_equal(q, fx["q_reference"])
    assert np.all(q.reshape(5, 6, 7)[0] == 0.0) and np.all(q.reshape(5, 6, 7)[:, :, -1] == 0.0)
