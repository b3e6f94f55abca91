"""The CPU oracle against the reference's own outputs (CPU, no GPU).

The fixtures in tests/golden/ were produced by the reference's solvers
compiled from its sources (tests/golden/make_golden.py).  The FP32 oracle
evaluates the reference's arithmetic in the reference's order, so on the
features the reference has it must match bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

KCX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1]
KCY = [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1]
KCZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def maxabs(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


@pytest.mark.parametrize("q", [19, 27])
def test_sycl_parity_template_bitwise(oracle_mod, golden, q):
    """tests/test_main.cpp:587-615 configuration; oracle == reference bit for bit."""
    data, meta = golden
    L = oracle_mod.OracleLattice(q, 16, 14, 12, tau=0.72, accel=(1e-6, -0.5e-6, 0.25e-6))
    L.init_taylor_green(0.018)
    L.step(12)
    assert np.array_equal(bits(L.logical()), bits(data[f"sycl_parity_q{q}_logical"]))
    for name, arr in zip(("rho", "ux", "uy", "uz"), L.macroscopic()):
        assert np.array_equal(bits(arr), bits(data[f"sycl_parity_q{q}_{name}"])), name
    red = L.reduce()
    m = meta[f"sycl_parity_q{q}"]
    assert red["mass"] == pytest.approx(m["mass"], rel=1e-14)
    assert red["kinetic_energy"] == pytest.approx(m["kinetic_energy"], rel=1e-12)
    assert red["max_speed"] == m["max_speed"]


def test_smagorinsky_bitwise(oracle_mod, golden):
    """Reference LES at its fixed coefficient (esoteric_pull.hpp:72-97), 24 steps."""
    data, meta = golden
    L = oracle_mod.OracleLattice(19, 20, 18, 16, tau=0.56, les_k=oracle_mod.reference_les_k())
    L.init_taylor_green(0.05)
    L.step(24)
    assert np.array_equal(bits(L.logical()), bits(data["les_q19_logical"]))
    red = L.reduce()
    assert red["kinetic_energy"] == pytest.approx(meta["les_q19"]["kinetic_energy"], rel=1e-12)


def test_plain_method_64cubed(oracle_mod, golden):
    """Plain-method config: 64^3 D3Q19 BGK, tau 0.6, Taylor-Green A = 0.05, 110 steps."""
    data, meta = golden
    m = meta["c1_d3q19_tg64"]
    L = oracle_mod.OracleLattice(19, 64, 64, 64, tau=0.6)
    L.init_taylor_green(0.05)
    L.step(110)
    s = m["stride"]
    for name, arr in zip(("rho", "ux", "uy", "uz"), L.macroscopic()):
        assert np.array_equal(bits(arr[::s]), bits(data[f"c1_d3q19_tg64_{name}"])), name
    red = L.reduce()
    assert red["mass"] + red["kinetic_energy"] == pytest.approx(m["checksum"], rel=1e-13)


@pytest.mark.parametrize("q", [19, 27])
def test_bounce_back_first_step_pin(oracle_mod, golden, q):
    """In-place half-way bounce-back vs the reference's 3-pass solid step.

    The reference re-encodes the odd-parity layout of direction 2p+2 from the
    cell n + c_{2p+1} (esoteric_pull.hpp:481-484), so its logical population
    2p+2 at n equals the physically streamed value at n + c_{2p+1}; all other
    populations compare at the same cell.  Bit-exact after one step.
    """
    data, _ = golden
    mask = data["solid_first_mask"]
    nx, ny, nz = 12, 10, 8
    L = oracle_mod.OracleLattice(q, nx, ny, nz, tau=0.8, accel=(2e-5, -1e-5, 0.5e-5), flags=mask)
    L.init_taylor_green(0.02)
    L.step(1)
    lo = L.logical().reshape(q, nz, ny, nx)
    rl = data[f"solid_first_q{q}_logical"].reshape(q, nz, ny, nx)
    fluid = mask.reshape(nz, ny, nx) == 0
    for d in range(q):
        if d == 0 or d % 2 == 1:
            a, b = lo[d][fluid], rl[d][fluid]
        else:
            i = d - 1
            shift = (-KCZ[i], -KCY[i], -KCX[i])
            sh = np.roll(lo[d], shift=shift, axis=(0, 1, 2))
            sel = fluid & np.roll(fluid, shift=shift, axis=(0, 1, 2))
            a, b = sh[sel], rl[d][sel]
        assert np.array_equal(bits(a), bits(b)), d


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("steps", [7, 8])
def test_trt_against_reference_two_grid(oracle_mod, golden, q, steps):
    """In-place TRT vs the reference's two-grid TRT (one_step_pull.hpp:187-204).

    In-place and two-grid states differ by one collision's rounding; gate of
    the reference's in-place/two-grid parity test (tests/test_main.cpp:423).
    """
    data, _ = golden
    L = oracle_mod.OracleLattice(q, 18, 14, 10, collision="trt", tau=0.73, tau_minus=1.1,
                                 accel=(2e-6, -1e-6, 0.5e-6))
    L.init_taylor_green(0.017)
    L.step(steps)
    for name, arr in zip(("rho", "ux", "uy", "uz"), L.macroscopic()):
        assert maxabs(arr, data[f"trt_q{q}_s{steps}_{name}"]) < 7e-6, name


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("steps", [7, 8])
def test_bgk_inplace_against_reference_two_grid(oracle_mod, golden, q, steps):
    """tests/test_main.cpp:340-372: in-place vs the reference's two-grid pull, Taylor-Green
    A = 0.017 on 18x14x10, tau 0.73, odd and even step counts; gate 5e-6."""
    data, _ = golden
    L = oracle_mod.OracleLattice(q, 18, 14, 10, tau=0.73)
    L.init_taylor_green(0.017)
    L.step(steps)
    for name, arr in zip(("rho", "ux", "uy", "uz"), L.macroscopic()):
        assert maxabs(arr, data[f"bgk_q{q}_s{steps}_{name}"]) < 5e-6, name


@pytest.mark.parametrize("q", [19, 27])
def test_forced_inplace_against_reference_two_grid(oracle_mod, golden, q):
    """tests/test_main.cpp:403-434: from rest with a = (2e-6, -1e-6, 5e-7), 60 steps; gate 7e-6."""
    data, _ = golden
    L = oracle_mod.OracleLattice(q, 18, 14, 10, tau=0.73, accel=(2e-6, -1e-6, 0.5e-6))
    L.init_uniform()
    L.step(60)
    got = L.macroscopic()
    for name, arr in zip(("rho", "ux", "uy", "uz"), got):
        assert maxabs(arr, data[f"bgk_forced_q{q}_{name}"]) < 7e-6, name
    assert got[1][got[1].size // 2] > 0


def test_fp64_against_reference_precision_solver(oracle_mod, golden):
    """FP64 oracle vs PrecisionPullSolver<D3Q19,double> (precision_pull.hpp:49-213).

    The reference's FP64 solver multiplies by the FP32 lattice weights cast to
    double (precision_pull.hpp:43); the oracle uses exact double weights, so
    the two agree to the float rounding of the weights (~3e-8 per step), not
    to double rounding.
    """
    data, _ = golden
    L = oracle_mod.OracleLattice(19, 18, 14, 10, storage="f64", tau=0.73)
    L.init_taylor_green(0.017)
    L.step(8)
    for name, arr in zip(("rho", "ux", "uy", "uz"), L.macroscopic()):
        assert maxabs(arr, data[f"f64_q19_{name}"]) < 1e-6, name


def test_fp16_shifted_against_reference_codec(oracle_mod, golden):
    """Shifted FP16 storage (s_d = 1) vs the reference's shifted-half two-grid solver.

    The reference codec rounds half away from zero in software
    (compressed_pull.hpp:27,35); the oracle rounds to nearest even like the
    hardware conversion, so the gate is statistical: the reference's own
    shifted-FP16 gates (tests/test_v0141_lbm_les_qcriterion.cpp:175-176).
    """
    data, meta = golden
    L = oracle_mod.OracleLattice(19, 16, 14, 12, storage="f16s", tau=0.72)
    L.init_taylor_green(0.025)
    L.step(16)
    for name, arr in zip(("rho", "ux", "uy", "uz"), L.macroscopic()):
        assert maxabs(arr, data[f"f16_q19_{name}"]) < 4e-4, name
    assert abs(L.reduce()["mass"] - meta["f16_q19"]["mass"]) / meta["f16_q19"]["mass"] < 2e-4


def test_phase02_published_checksum(oracle_mod, golden):
    """Known-answer test: phase02 Taylor-Green + Smagorinsky checksum published by the reference.

    examples/phase02_lbm_taylor_green.cpp:3: 48^3 D3Q19, tau 0.58, LES, A = 0.04,
    80 steps, checksum = mass() + kinetic_energy() = 110609.77375653926
    (examples/results/v0.19.0_reference.json:73, built with -O3 and contraction
    on another CPU).
    """
    _, meta = golden
    m = meta["phase02"]
    L = oracle_mod.OracleLattice(19, 48, 48, 48, tau=0.58, les_k=oracle_mod.reference_les_k())
    L.init_taylor_green(0.04)
    L.step(80)
    red = L.reduce()
    assert red["mass"] + red["kinetic_energy"] == pytest.approx(m["checksum"], rel=1e-9)


def test_poiseuille_channel_profile(oracle_mod):
    """Half-way bounce-back reproduces the analytic Poiseuille profile.

    Gate of the reference's D2Q9 Poiseuille test (tests/test_main.cpp:449-477):
    relative L2 error < 1 %.  (The reference's 3-D 3-pass solid path misses
    this gate by a wide margin because of the odd-parity re-encoding offset
    pinned in test_bounce_back_first_step_pin.)
    """
    q, nx, ny, nz, tau, g = 19, 4, 14, 4, 0.8, 1e-5
    mask = np.zeros((nz, ny, nx), np.uint8)
    mask[:, 0, :] = 1
    mask[:, ny - 1, :] = 1
    L = oracle_mod.OracleLattice(q, nx, ny, nz, tau=tau, accel=(g, 0, 0), flags=mask.reshape(-1))
    L.init_uniform()
    L.step(5000)
    ux = L.macroscopic()[1].reshape(nz, ny, nx)
    nu = (tau - 0.5) / 3
    h = ny - 2
    num, den = 0.0, 0.0
    for y in range(1, ny - 1):
        wy = y - 0.5
        exact = g * wy * (h - wy) / (2 * nu)
        num += (ux[:, y, :].mean() - exact) ** 2
        den += exact ** 2
    assert np.sqrt(num / den) < 0.01


def test_fp16_conversion_round_to_nearest_even(oracle_mod):
    """The oracle's binary16 conversion equals IEEE RNE (numpy float16) on 2^20 values."""
    rng = np.random.default_rng(0)
    vals = np.concatenate([
        rng.normal(0, 1e-3, 1 << 18), rng.normal(0, 1.0, 1 << 18), rng.uniform(-7e4, 7e4, 1 << 18),
        rng.normal(0, 1e-6, 1 << 18), np.array([0.0, -0.0, 65504.0, 65520.0, 6.1e-5, 5.96e-8, 2.98e-8])]).astype(np.float32)
    ref = vals.astype(np.float16).view(np.uint16)
    lib = oracle_mod.oracle_lib()
    sample = np.arange(0, vals.size, 97)
    got = np.array([lib.ora_f32_to_f16(float(v)) for v in vals[sample]], np.uint16)
    assert np.array_equal(got, ref[sample])
    back = np.array([lib.ora_f16_to_f32(int(h)) for h in ref[sample]], np.float32)
    assert np.array_equal(back, ref[sample].view(np.float16).astype(np.float32))


@pytest.mark.reference
@pytest.mark.parametrize("q", [19, 27])
def test_live_reference_forced_parity(oracle_mod, q):
    """Live reference run (when oracle/_ref is built): forced BGK+LES, odd size, bitwise."""
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    acc = (2e-6, -1e-6, 0.5e-6)
    k = oracle_mod.reference_les_k()
    L = oracle_mod.OracleLattice(q, 17, 15, 13, tau=0.66, les_k=k, accel=acc)
    L.init_taylor_green(0.03)
    L.step(9)
    r = oracle_mod.ref_esoteric(q, 17, 15, 13, 0.66, 9, init=("tg", 0.03), accel=acc, les=True, logical=True)
    assert np.array_equal(bits(L.logical()), bits(r["logical"]))


@pytest.mark.parametrize("q", [19, 27])
def test_velocity_set_moments(oracle_mod, q):
    """tests/test_main.cpp:278-310 on the oracle's velocity set with the reference's weights
    (descriptors.hpp:59-146): sum w = 1, isotropic second moments, opposite pairs (i, i+1)."""
    c = oracle_mod.velocity_set(q).astype(np.float64)
    speed2 = (c * c).sum(1)
    table = {19: {0: 1 / 3, 1: 1 / 18, 2: 1 / 36}, 27: {0: 8 / 27, 1: 2 / 27, 2: 1 / 54, 3: 1 / 216}}[q]
    w = np.array([table[int(s)] for s in speed2])
    assert abs(w.sum() - 1) < 2e-7
    for a in range(3):
        assert abs((w * c[:, a] ** 2).sum() - 1 / 3) < 2e-7
    assert abs((w * c[:, 0] * c[:, 1]).sum()) < 2e-7
    for i in range(1, q, 2):
        assert np.array_equal(c[i], -c[i + 1])
