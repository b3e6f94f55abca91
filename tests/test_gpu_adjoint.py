"""The discrete adjoint on the GPU (GPU).

Gates:
* FP64 storage (FP64 adjoint arithmetic) vs the FP64 CPU adjoint of the
  oracle (oracle/lbm_adjoint_oracle.c, itself checked against finite
  differences): 1e-10 relative to max |dJ/dn_s|, 1e-10 on dJ/dtau;
* FP32 storage (FP32 adjoint) vs the FP64 CPU adjoint: 1e-3 relative to
  max |dJ/dn_s| and on dJ/dtau (the north-star gradient gate);
* FP16-shifted storage: 2e-2 (the forward states themselves carry FP16
  quantisation);
* checkpoint interval: gradients bitwise identical for intervals 1, 3 and
  more than the step count (the forward pass and the segment recompute run
  the same out-of-place kernel, so the recomputed states are the forward's
  bit for bit);
* the autograd Function returns the same gradients, and on FP64 storage they
  match central finite differences of the GPU forward to 1e-6.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ = 12, 10, 9


def problem(q, coll="trt", tau_minus=0.0, seed=11):
    rng = np.random.default_rng(seed)
    n = NX * NY * NZ
    flags = (rng.random(n) < 0.1).astype(np.uint8)
    ns = rng.uniform(0.0, 0.2, n).astype(np.float32)
    ustar = rng.normal(0.0, 0.01, (3, n))
    kw = dict(collision=coll, tau=0.63, trt_tau_minus=tau_minus, acceleration_x=1e-3, acceleration_y=-2e-4,
              acceleration_z=3e-4)
    return kw, flags, ns, ustar


def oracle_gradient(O, q, kw, flags, ns, ustar, steps):
    accel = (kw["acceleration_x"], kw["acceleration_y"], kw["acceleration_z"])
    f32 = lambda v: float(np.float32(v))  # noqa: E731  (the C ABI's config fields are float)
    L = O.OracleLattice(q=q, nx=NX, ny=NY, nz=NZ, storage="f64", collision=kw["collision"], tau=f32(kw["tau"]),
                        tau_minus=f32(kw["trt_tau_minus"]), accel=tuple(f32(a) for a in accel), flags=flags,
                        solid_fraction=ns)
    L.init_taylor_green(0.04)
    x0 = L.logical().astype(np.float64)
    xe = L.adjoint_forward(x0, steps)
    _, u = O.logical_velocity(xe, q, L.cells, tuple(f32(a) for a in accel))
    fluid = flags == 0
    gu = (u - ustar) * fluid
    gns, gtau = L.adjoint(x0, steps, gu)
    return gu, gns, gtau


def solver(cs, q, storage, kw, flags, ns):
    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=NX, ny=NY, nz=NZ, lattice={19: "d3q19", 27: "d3q27"}[q],
                                                      storage=storage, **kw))
    s.set_flags(flags)
    s.set_solid_fraction(ns)
    s.initialize_taylor_green(0.04)
    return s


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("coll,tau_minus", [("trt", 0.0), ("bgk", 0.0), ("trt", 0.9)])
def test_adjoint_fp64_matches_oracle(engine, oracle_mod, q, coll, tau_minus):
    steps = 10
    kw, flags, ns, ustar = problem(q, coll, tau_minus)
    gu, gns_ref, gtau_ref = oracle_gradient(oracle_mod, q, kw, flags, ns, ustar, steps)
    with solver(engine, q, "fp64", kw, flags, ns) as s:
        s.adjoint_forward(steps, 4)
        g = gu.astype(np.float32)
        gns, gtau = s.adjoint_backward(g[0], g[1], g[2])
    # the seed went through float32; compare against the oracle fed the same seed
    _, gns_ref32, gtau_ref32 = oracle_gradient_seed(oracle_mod, q, kw, flags, ns, steps, g)
    assert rel(gns, gns_ref32) < 1e-10
    assert gtau == pytest.approx(gtau_ref32, rel=1e-10)
    assert np.all(gns[flags != 0] == 0.0)
    assert rel(gns_ref32, gns_ref) < 1e-5  # float32 seed rounding only


def oracle_gradient_seed(O, q, kw, flags, ns, steps, seed):
    accel = tuple(float(np.float32(kw[k])) for k in ("acceleration_x", "acceleration_y", "acceleration_z"))
    L = O.OracleLattice(q=q, nx=NX, ny=NY, nz=NZ, storage="f64", collision=kw["collision"],
                        tau=float(np.float32(kw["tau"])), tau_minus=float(np.float32(kw["trt_tau_minus"])),
                        accel=accel, flags=flags, solid_fraction=ns)
    L.init_taylor_green(0.04)
    x0 = L.logical().astype(np.float64)
    gns, gtau = L.adjoint(x0, steps, np.asarray(seed, np.float64))
    return None, gns, gtau


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage,gate", [("fp32", 1e-3), ("fp16s", 2e-2)])
def test_adjoint_reduced_precision_vs_oracle(engine, oracle_mod, q, storage, gate):
    steps = 10
    kw, flags, ns, ustar = problem(q)
    gu, gns_ref, gtau_ref = oracle_gradient(oracle_mod, q, kw, flags, ns, ustar, steps)
    g = gu.astype(np.float32)
    with solver(engine, q, storage, kw, flags, ns) as s:
        s.adjoint_forward(steps, 4)
        gns, gtau = s.adjoint_backward(g[0], g[1], g[2])
    assert rel(gns, gns_ref) < gate
    assert gtau == pytest.approx(gtau_ref, rel=gate)


@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp64"])
def test_adjoint_interval_invariance(engine, storage):
    steps = 9
    kw, flags, ns, ustar = problem(19)
    g = np.random.default_rng(3).normal(0, 1e-3, (3, NX * NY * NZ)).astype(np.float32)
    out = []
    for interval in (1, 3, 64):
        with solver(engine, 19, storage, kw, flags, ns) as s:
            s.adjoint_forward(steps, interval)
            out.append(s.adjoint_backward(g[0], g[1], g[2]))
    for gns, gtau in out[1:]:
        assert np.array_equal(gns, out[0][0])
        assert gtau == out[0][1]


@pytest.mark.parametrize("storage", ["fp32", "fp16s"])
def test_adjoint_two_level_recompute_is_bitwise_equal(engine, storage):
    """Sub-checkpoint intervals 2, 3, 5 and 7 under segments of 8 steps (the last one 7 steps: two
    levels, and one level for m = 7) give the one-level gradients bit for bit, with fewer frames
    (m = 7 holds 1 + 6, as many as one level)."""
    steps, interval = 23, 8
    kw, flags, ns, ustar = problem(19)
    g = np.random.default_rng(5).normal(0, 1e-3, (3, NX * NY * NZ)).astype(np.float32)

    def run(sub):
        with solver(engine, 19, storage, kw, flags, ns) as s:
            s.adjoint_forward(steps, interval, sub)
            mem = s.adjoint_memory()
            return s.adjoint_backward(g[0], g[1], g[2]), mem

    (gns0, gtau0), mem0 = run(0)
    for sub in (2, 3, 5, 7):
        (gns, gtau), mem = run(sub)
        assert np.array_equal(gns, gns0), sub
        assert gtau == gtau0, sub
        assert mem < mem0 if sub < 7 else mem == mem0, sub


def test_adjoint_rejects_subinterval_one(engine):
    kw, flags, ns, _ = problem(19)
    with solver(engine, 19, "fp32", kw, flags, ns) as s:
        with pytest.raises(ValueError):
            s.adjoint_forward(4, 2, 1)


def test_adjoint_keeps_forward_state_and_reuses_seed(engine):
    kw, flags, ns, _ = problem(19)
    g = np.random.default_rng(4).normal(0, 1e-3, (3, NX * NY * NZ)).astype(np.float32)
    with solver(engine, 19, "fp32", kw, flags, ns) as s:
        s.adjoint_forward(7, 3)
        before = s.compute_macroscopic()
        a = s.adjoint_backward(g[0], g[1], g[2])
        after = s.compute_macroscopic()
        b = s.adjoint_backward(g[0], g[1], g[2])
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
        assert np.array_equal(a[0], b[0]) and a[1] == b[1]
        assert s.adjoint_memory() > 0
        s.adjoint_release()
        assert s.adjoint_memory() == 0


def test_adjoint_of_total_mass_is_zero(engine):
    """Every part of the step conserves mass, so J = sum of fluid rho has zero gradient (FP64)."""
    kw, flags, ns, _ = problem(27)
    zero = np.zeros(NX * NY * NZ, np.float32)
    with solver(engine, 27, "fp64", kw, flags, ns) as s:
        s.adjoint_forward(7, 3)
        gm, gt = s.adjoint_backward(zero, zero, zero, g_rho=(flags == 0).astype(np.float32))
        assert np.max(np.abs(gm)) < 1e-12 and abs(gt) < 1e-10


def test_adjoint_same_as_plain_steps(engine):
    kw, flags, ns, _ = problem(27)
    with solver(engine, 27, "fp32", kw, flags, ns) as a, solver(engine, 27, "fp32", kw, flags, ns) as b:
        a.adjoint_forward(11, 4)
        b.step(11)
        # same step, out-of-place kernel: equal to a few ulp of FP32
        assert np.max(np.abs(a.logical_populations() - b.logical_populations())) < 1e-6
        assert a.time_step() == b.time_step() == 11


def test_adjoint_errors(engine):
    kw, flags, ns, _ = problem(19)
    z = np.zeros(NX * NY * NZ, np.float32)
    with solver(engine, 19, "fp32", kw, flags, ns) as s:
        with pytest.raises(ValueError):
            s.adjoint_backward(z, z, z)  # no forward yet
        s.adjoint_forward(3, 2)
        s.step(1)
        with pytest.raises(ValueError):
            s.adjoint_backward(z, z, z)  # the lattice moved on
        s.adjoint_forward(3, 2)
        s.set_tau(0.7)
        with pytest.raises(ValueError):
            s.adjoint_backward(z, z, z)  # a parameter changed
        with pytest.raises(ValueError):
            s.adjoint_forward(0, 2)
    les = dict(kw, smagorinsky_les=True, smagorinsky_cs=0.1)
    with solver(engine, 19, "fp32", les, flags, ns) as s:
        with pytest.raises(ValueError):
            s.adjoint_forward(3, 2)
    moving = flags.copy()
    moving[0] = 2
    with solver(engine, 19, "fp32", kw, moving, ns) as s:
        with pytest.raises(ValueError):
            s.adjoint_forward(3, 2)


def test_autograd_matches_adjoint_and_finite_differences(engine):
    torch = pytest.importorskip("torch")
    from cfd_solvers_b200.autograd import gray_lbm

    steps = 12
    kw, flags, ns, ustar = problem(19)
    dev = torch.device("cuda:0")
    fluid = torch.tensor(flags == 0, device=dev)
    target = torch.tensor(ustar, dtype=torch.float32, device=dev)

    def objective(s, ns_t, tau_t):
        _, u = gray_lbm(ns_t, tau_t, s, steps, interval=5, init=lambda sv: sv.initialize_taylor_green(0.04))
        r = (u.double() - target.double()) * fluid
        return 0.5 * (r * r).sum()

    with solver(engine, 19, "fp64", kw, flags, ns) as s:
        ns_t = torch.tensor(ns, dtype=torch.float64, device=dev, requires_grad=True)
        tau_t = torch.tensor(0.63, dtype=torch.float64, device=dev, requires_grad=True)
        J = objective(s, ns_t, tau_t)
        J.backward()
        g = ns_t.grad.cpu().numpy()
        gt = float(tau_t.grad)
        cells = np.flatnonzero(flags == 0)[:6]
        h = 1e-4
        for c in cells:
            p = ns_t.detach().clone()
            m = ns_t.detach().clone()
            p[c] += h
            m[c] -= h
            fd = (float(objective(s, p, tau_t.detach())) - float(objective(s, m, tau_t.detach()))) / (2 * h)
            # the forward sees n_s through float32 storage of the field
            hh = float(np.float32(ns[c] + h)) - float(np.float32(ns[c] - h))
            fd *= 2 * h / hh
            assert g[c] == pytest.approx(fd, rel=1e-6, abs=1e-12)
        ht = 1e-5
        fdt = (float(objective(s, ns_t.detach(), torch.tensor(0.63 + ht, dtype=torch.float64, device=dev))) -
               float(objective(s, ns_t.detach(), torch.tensor(0.63 - ht, dtype=torch.float64, device=dev)))) / (2 * ht)
        # tau reaches the device as float32
        tp, tm = float(np.float32(0.63 + ht)), float(np.float32(0.63 - ht))
        fdt *= 2 * ht / (tp - tm)
        assert gt == pytest.approx(fdt, rel=1e-5)


def test_autograd_two_level_recompute_same_gradients(engine):
    torch = pytest.importorskip("torch")
    from cfd_solvers_b200.autograd import gray_lbm

    kw, flags, ns, ustar = problem(19)
    dev = torch.device("cuda:0")
    target = torch.tensor(ustar, dtype=torch.float32, device=dev)
    grads = []
    with solver(engine, 19, "fp32", kw, flags, ns) as s:
        for sub in (0, 2):
            ns_t = torch.tensor(ns, dtype=torch.float32, device=dev, requires_grad=True)
            _, u = gray_lbm(ns_t, 0.63, s, 13, interval=6, subinterval=sub)
            (0.5 * ((u - target) ** 2).sum()).backward()
            grads.append(ns_t.grad.cpu().numpy())
    assert np.array_equal(grads[0], grads[1])
