"""The FP64 CPU adjoint (oracle/lbm_adjoint_oracle.c) against finite differences (CPU).

The reference has no adjoint, so the adjoint is pinned (a) through its
forward, which must reproduce the oracle's in-place step on logical
populations, and (b) against central finite differences of the FP64 oracle
forward for the misfit J = 1/2 sum |u(T) - u*|^2 over fluid cells.
"""
from __future__ import annotations

import numpy as np
import pytest

CASES = [("trt", 0.0), ("bgk", 0.0), ("trt", 0.9)]


def problem(O, q, coll, tau_minus, seed=5):
    rng = np.random.default_rng(seed)
    nx, ny, nz = 7, 6, 5
    n = nx * ny * nz
    flags = (rng.random(n) < 0.1).astype(np.uint8)
    ns = rng.uniform(0.0, 0.2, n).astype(np.float32)
    ustar = rng.normal(0.0, 0.01, (3, n))
    kw = dict(q=q, nx=nx, ny=ny, nz=nz, storage="f64", collision=coll, tau=0.63, tau_minus=tau_minus,
              accel=(1e-3, -2e-4, 3e-4), flags=flags, solid_fraction=ns)
    return kw, ustar, flags == 0


def misfit(O, kw, ustar, fluid, steps, **over):
    k = dict(kw, **over)
    L = O.OracleLattice(**k)
    L.init_taylor_green(0.04)
    L.step(steps)
    _, u = O.logical_velocity(L.logical(), k["q"], L.cells, k["accel"])
    r = (u - ustar) * fluid
    return 0.5 * float(np.sum(r * r))


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("coll,tau_minus", CASES)
def test_adjoint_oracle_vs_finite_differences(oracle_mod, q, coll, tau_minus):
    O = oracle_mod
    steps = 9
    kw, ustar, fluid = problem(O, q, coll, tau_minus)
    L = O.OracleLattice(**kw)
    L.init_taylor_green(0.04)
    x0 = L.logical().astype(np.float64)
    ref = O.OracleLattice(**kw)
    ref.init_taylor_green(0.04)
    ref.step(steps)
    xe = L.adjoint_forward(x0, steps)
    assert np.max(np.abs(xe - ref.logical())) < 1e-14
    _, u = O.logical_velocity(xe, q, L.cells, kw["accel"])
    gns, gtau = L.adjoint(x0, steps, (u - ustar) * fluid)
    ns = kw["solid_fraction"]
    for c in np.flatnonzero(fluid)[:4]:
        p, m = ns.copy(), ns.copy()
        p[c] += np.float32(1e-5)
        m[c] -= np.float32(1e-5)
        fd = (misfit(O, kw, ustar, fluid, steps, solid_fraction=p) -
              misfit(O, kw, ustar, fluid, steps, solid_fraction=m)) / (float(p[c]) - float(m[c]))
        assert gns[c] == pytest.approx(fd, rel=1e-5, abs=1e-12)
    fd = (misfit(O, kw, ustar, fluid, steps, tau=0.63 + 1e-6) - misfit(O, kw, ustar, fluid, steps, tau=0.63 - 1e-6)) / 2e-6
    assert gtau == pytest.approx(fd, rel=1e-6)
    assert np.all(gns[~fluid] == 0.0)


def test_adjoint_oracle_rejects_out_of_scope(oracle_mod):
    O = oracle_mod
    L = O.OracleLattice(q=19, nx=4, ny=4, nz=4, storage="f64", les_k=0.1)
    with pytest.raises(ValueError):
        L.adjoint(np.zeros(19 * 64), 2, np.zeros((3, 64)))
    flags = np.zeros(64, np.uint8)
    flags[5] = 2
    L = O.OracleLattice(q=19, nx=4, ny=4, nz=4, storage="f64", flags=flags)
    with pytest.raises(ValueError):
        L.adjoint(np.zeros(19 * 64), 2, np.zeros((3, 64)))
