"""The C ABI library and its host-side logic, without a GPU.

* the library loads and exports every symbol include/*.h declares;
* the ctypes binding declares exactly those symbols;
* configuration errors surface as the reference's exception types before any
  device work (esoteric_pull.hpp:111-113,292-301);
* with no CUDA device the engine fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        names.update(re.findall(r"CFDX_API\s+[\w\s\*]+?\b(cfdx_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"cfdx_lbm_create", "cfdx_lbm_step", "cfdx_lbm_reduce", "cfdx_lbm_macroscopic"} <= names


def test_library_exports_every_declared_symbol():
    from cfd_solvers_b200 import bindings

    lib = ctypes.CDLL(str(bindings.DEFAULT_LIBRARY))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from cfd_solvers_b200 import bindings

    assert set(bindings.SIGNATURES) == declared_symbols()


def test_version_and_defaults():
    import cfd_solvers_b200 as cs

    lib = cs.load()
    assert "sm_100a" in lib.version
    c = cs.bindings.cfdx_lbm_config()
    assert lib.raw.cfdx_lbm_config_default(ctypes.byref(c)) == 0
    assert (c.nx, c.ny, c.nz, c.lattice, c.storage) == (128, 128, 128, 19, 0)
    assert c.tau == pytest.approx(0.6)
    assert c.trt_magic == pytest.approx(3 / 16)


@pytest.mark.parametrize("kwargs, message", [
    (dict(tau=0.5), "tau must be > 0.5"),
    (dict(nx=1), "nx, ny >= 2"),
    (dict(nz=1), "nz >= 2"),
    (dict(lattice="d2q9"), "lattice"),
    (dict(storage="bf16"), "storage"),
    (dict(collision="mrt"), "collision"),
    (dict(acceleration_x=float("nan")), "finite"),
])
def test_invalid_configuration_raises_value_error(kwargs, message):
    import cfd_solvers_b200 as cs

    base = dict(nx=8, ny=8, nz=8)
    base.update(kwargs)
    with pytest.raises(ValueError, match=message):
        cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(**base))


def test_null_handle_is_rejected():
    import cfd_solvers_b200 as cs

    lib = cs.load()
    assert lib.raw.cfdx_lbm_step(None, 1) == cs.bindings.ERR_INVALID
    status, message = lib.last_error()
    assert status == cs.bindings.ERR_INVALID and "null" in message


def test_no_device_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import cfd_solvers_b200 as cs

    with pytest.raises(cs.CudaError, match="no CUDA device"):
        cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=8, ny=8, nz=8))


def test_missing_library_fails_loudly(tmp_path):
    import cfd_solvers_b200 as cs

    with pytest.raises(RuntimeError, match="not built"):
        cs.load(tmp_path / "libmissing.so")


def test_cavity_flags_layout():
    import numpy as np

    import cfd_solvers_b200 as cs

    fl = cs.cavity_flags(6, 5, 4).reshape(4, 5, 6)
    assert (fl[:, 4, :] == 2).all()          # lid
    assert (fl[1:-1, 0, :] == 1).all()       # floor
    assert (fl[0, :4, :] == 1).all() and (fl[-1, :4, :] == 1).all()
    assert (fl[1:-1, 1:4, 1:-1] == 0).all()  # interior fluid
    assert int(np.count_nonzero(fl == 0)) == 2 * 3 * 4


def test_trt_and_les_helpers():
    import cfd_solvers_b200 as cs

    assert cs.trt_tau_minus(0.51) == pytest.approx(19.25)
    assert cs.trt_tau_minus(0.55) == pytest.approx(4.25)
    assert cs.trt_tau_minus(0.6) == pytest.approx(2.375)
    # K(Cs) reproduces the reference's fixed coefficient at Cs = sqrt(8/27)/pi
    import math

    from oracle import oracle as O

    assert cs.smagorinsky_k(math.sqrt(8 / 27) / math.pi) == pytest.approx(O.reference_les_k(), rel=1e-6)
