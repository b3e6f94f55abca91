"""The resident D3Q7 thermal lattice on the GPU.

* it equals the oracle restatement bit for bit when driven by a real flow's
  device velocity (cavity with walls and a moving lid, several coupled steps);
* the reference's resident chain test (tests/test_v0156_gpu_lbm_multiphysics.cpp:26-40):
  a uniform 300 K field keeps its total to 2e-5 through step(macro, 3) and the
  Boussinesq coupling, and neither the thermal lattice nor the coupled flow
  step moves a field through the host;
* the Boussinesq term lands in the flow's acceleration field exactly and drives
  the flow the next step.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cavity(cs, nx=12, ny=10, nz=8):
    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.7, collision="trt"))
    s.set_flags(cs.cavity_flags(nx, ny, nz))
    s.set_wall_velocity(2, 0.05, 0.0, 0.0)
    s.initialize_uniform()
    s.step(30)
    return s


def test_thermal_matches_oracle_bitwise(engine, oracle_mod):
    from cfd_solvers_b200.multiphysics import ResidentThermalD3Q7

    cs = engine
    nx, ny, nz = 12, 10, 8
    with cavity(cs, nx, ny, nz) as flow:
        rng = np.random.default_rng(7)
        T0 = rng.uniform(290, 310, nx * ny * nz).astype(np.float32)
        with ResidentThermalD3Q7(flow, 0.03) as th:
            th.initialize_field(T0)
            g = (np.array([0.25] + [0.125] * 6, np.float32)[:, None] * T0[None, :]).astype(np.float32)
            for _ in range(3):
                macro = flow.refresh_device_macroscopic()
                f = flow.compute_macroscopic()
                th.step(macro, 4)
                g = oracle_mod.thermal_d3q7_step(g, (f.ux, f.uy, f.uz), nx, ny, nz, 0.03, 4)
                flow.step(2)
            T = g.reshape(7, -1)
            expect = np.zeros(nx * ny * nz, np.float32)
            for d in range(7):
                expect = expect + T[d]
            assert np.array_equal(th.temperature(), expect)


def test_reference_resident_chain(engine):
    from cfd_solvers_b200.multiphysics import ParticleVector3, ResidentThermalD3Q7

    cs = engine
    nx, ny, nz = 10, 8, 6
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.72)) as flow:
        flow.initialize_uniform(1.0, 0.0, 0.0, 0.0)
        force = flow.device_local_acceleration(clear=True)
        macro = flow.refresh_device_macroscopic()
        with ResidentThermalD3Q7(flow, 0.02) as th:
            th.initialize_uniform(300.0)
            heat0 = th.total_scalar()
            stats0 = th.transfer_stats()
            th.step(macro, 3)
            th.add_boussinesq_acceleration(force, 300.0, 3.0e-3, ParticleVector3(0.0, -1.0, 0.0))
            heat1 = th.total_scalar()
            assert abs(heat1 - heat0) / heat0 < 2.0e-5
            assert th.transfer_stats() == stats0  # no field through the host
            assert th.resident_bytes() >= 14 * nx * ny * nz * 4
            f0 = flow.transfer_stats()
            flow.step(2)
            for _ in range(3):  # the coupled loop: velocity view, thermal step, cleared force, buoyancy, flow step
                th.step(flow.refresh_device_macroscopic(), 1)
                force = flow.device_local_acceleration(clear=True)
                th.add_boussinesq_acceleration(force, 300.0, 3.0e-3, (0.0, -1.0, 0.0))
                flow.step(1)
            flow.wait()
            f1 = flow.transfer_stats()
            assert (f1.host_to_device_bytes, f1.device_to_host_bytes) == (f0.host_to_device_bytes,
                                                                          f0.device_to_host_bytes)


def test_boussinesq_term_and_coupling(engine):
    import ctypes

    from cfd_solvers_b200.multiphysics import ResidentThermalD3Q7

    cs = engine
    nx, ny, nz = 8, 16, 6
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.8)) as flow:
        flow.initialize_uniform()
        force = flow.device_local_acceleration(clear=True)
        y = np.repeat(np.arange(ny), nx)[None, :].repeat(nz, 0).reshape(-1)
        T0 = (300.0 + 2.0 * np.sin(2 * np.pi * y / ny)).astype(np.float32)
        with ResidentThermalD3Q7(flow, 0.02) as th:
            th.initialize_field(T0)
            T = th.temperature()
            th.add_boussinesq_acceleration(force, 300.0, 1e-3, (0.0, -1.0, 0.0))
            n = nx * ny * nz
            flow.wait()
            # the flow's acceleration field, read back through its device pointer
            got = np.zeros(n, np.float32)
            rt = ctypes.CDLL("libcudart.so.12")
            rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
            assert rt.cudaMemcpy(got.ctypes.data, force.ay, n * 4, 2) == 0  # device to host
            scale = (np.float32(-1e-3) * (T - np.float32(300.0))).astype(np.float32)
            expect = (np.float32(0.0) + scale * np.float32(-1.0)).astype(np.float32)
            assert np.array_equal(got, expect)
            flow.step(5)
            f = flow.compute_macroscopic()
            # warm rows (T > 300) are pushed up (+y), cold rows down
            warm = T0.reshape(nz, ny, nx)[:, :, 0].mean(0) > 300.0
            uy = np.asarray(f.uy).reshape(nz, ny, nx).mean((0, 2))
            assert np.all(uy[warm] > 0) and np.all(uy[~warm & (np.abs(T0.reshape(nz, ny, nx)[0, :, 0] - 300) > 0.1)] < 0)


def test_thermal_arguments(engine):
    from cfd_solvers_b200.multiphysics import ResidentThermalD3Q7
    from cfd_solvers_b200.slabs import SlabSolver

    cs = engine
    with cs.EsotericPullCudaSolver(nx=6, ny=5, nz=4) as flow:
        with pytest.raises(ValueError):
            ResidentThermalD3Q7(flow, 0.0)
        with ResidentThermalD3Q7(flow, 0.01) as th:
            with pytest.raises(ValueError):
                th.initialize_uniform(float("nan"))
            with pytest.raises(ValueError):
                th.initialize_field(np.zeros(5, np.float32))
    with SlabSolver(cs.InPlaceLbmConfig(nx=6, ny=5, nz=8), 0, 4) as slab:
        with pytest.raises(ValueError):
            ResidentThermalD3Q7(slab, 0.01)
