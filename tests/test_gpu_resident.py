"""The resident free surface, point particles and FP32 Q-criterion on the GPU.

* each kernel equals its float32 restatement (oracle) bit for bit when driven by
  a real flow's device velocity (a lid-driven cavity after some steps), except
  the atomically spread particle force, whose order of additions is not fixed
  (checked to 1e-6 relative there, bit for bit where particles do not share cells);
* the reference's resident chain test (tests/test_v0156_gpu_lbm_multiphysics.cpp:43-61):
  the zero-flow advection keeps the volume to 2e-4 per cell, surface tension and
  the two-way particle push touch the flow's acceleration field without any host
  transfer, and the Q-criterion returns a device field;
* argument checks follow the reference's exceptions.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cavity(cs, nx=12, ny=10, nz=8, steps=40):
    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.7, collision="trt"))
    s.set_flags(cs.cavity_flags(nx, ny, nz))
    s.set_wall_velocity(2, 0.08, 0.0, 0.0)
    s.initialize_uniform()
    s.step(steps)
    return s


def device_read(ptr, count):
    out = np.zeros(count, np.float32)
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert rt.cudaMemcpy(out.ctypes.data, ptr, count * 4, 2) == 0  # device to host
    return out


def device_write(ptr, values):
    v = np.ascontiguousarray(values, np.float32)
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert rt.cudaMemcpy(ptr, v.ctypes.data, v.nbytes, 1) == 0  # host to device


@pytest.mark.parametrize("nx", [12, 14])  # four-cell kernels (nx % 4 == 0) and the one-cell fallback
def test_free_surface_matches_oracle_bitwise(engine, oracle_mod, nx):
    from cfd_solvers_b200.multiphysics import ResidentFreeSurface3D

    cs = engine
    ny, nz = 10, 8
    n = nx * ny * nz
    with cavity(cs, nx, ny, nz) as flow:
        with ResidentFreeSurface3D(flow) as fs:
            fs.initialize_half_space_x(5.25)
            phi = oracle_mod.fill_half_space_x(nx, ny, nz, 5.25)
            assert np.array_equal(fs.fill(), phi)
            for _ in range(3):
                macro = flow.refresh_device_macroscopic()
                f = flow.compute_macroscopic()
                for _ in range(4):
                    fs.advect(macro, 1.5)
                    phi = oracle_mod.fill_advect(phi, (f.ux, f.uy, f.uz), nx, ny, nz, 1.5)
                flow.step(3)
            assert np.array_equal(fs.fill(), phi)
            assert abs(fs.volume() - phi.sum(dtype=np.float64)) < 1e-9 * n
            # geometry and surface tension into a known acceleration field
            force = flow.device_local_acceleration(clear=True)
            flow.wait()  # the clear is ordered on the flow's stream; the writes below are not
            a0 = [np.linspace(-1e-4, 1e-4, n, dtype=np.float32) * (k + 1) for k in range(3)]
            for ptr, v in zip((force.ax, force.ay, force.az), a0):
                device_write(ptr, v)
            fs.add_surface_tension_acceleration(force, 0.072, 1.25)
            flow.wait()
            g = fs.geometry()
            nxv, nyv, nzv, k = oracle_mod.fill_geometry(phi, nx, ny, nz)
            assert np.array_equal(g["normal_x"], nxv) and np.array_equal(g["normal_y"], nyv)
            assert np.array_equal(g["normal_z"], nzv) and np.array_equal(g["curvature"], k)
            expect = oracle_mod.surface_tension(phi, k, a0, nx, ny, nz, 0.072, 1.25)
            for ptr, e in zip((force.ax, force.ay, force.az), expect):
                assert np.array_equal(device_read(ptr, n), e)


def test_particles_match_oracle(engine, oracle_mod):
    from cfd_solvers_b200.multiphysics import ImmersedBoundaryParticle, ParticleVector3, ResidentParticles3D

    cs = engine
    nx, ny, nz = 12, 10, 8
    n = nx * ny * nz
    rng = np.random.default_rng(21)
    count = 300
    ps = [ImmersedBoundaryParticle(ParticleVector3(*rng.uniform(-4, 16, 3)), ParticleVector3(*rng.normal(0, 0.02, 3)),
                                   float(rng.uniform(0.5, 2)), float(rng.uniform(0.3, 3))) for _ in range(count)]
    with cavity(cs, nx, ny, nz) as flow, ResidentParticles3D(flow, count) as parts:
        parts.upload(ps)
        st = ResidentParticles3D._records(ps).T.astype(np.float32)
        force = flow.device_local_acceleration(clear=True)
        acc = [np.zeros(n, np.float32)] * 3
        parts.reset_transfer_stats()
        gravity = ParticleVector3(0.0, -2e-4, 0.0)
        for _ in range(3):
            macro = flow.refresh_device_macroscopic()
            f = flow.compute_macroscopic()
            parts.advance(macro, force, 0.5, True, gravity)
            st, acc = oracle_mod.particles_advance(st, (f.ux, f.uy, f.uz), acc, nx, ny, nz, 0.5, True, gravity)
        assert parts.transfer_stats().host_to_device_bytes == 0
        assert parts.transfer_stats().device_to_host_bytes == 0
        got = parts.download_records()
        assert np.array_equal(got[:, :6].T.astype(np.float32), st[:6])  # the particle state, bit for bit
        flow.wait()
        for ptr, e in zip((force.ax, force.ay, force.az), acc):
            got_a = device_read(ptr, n)  # atomics: the order of additions is not fixed
            assert np.all(np.abs(got_a - e) <= 1e-6 * (1.0 + np.abs(e)))
        # one-way coupling leaves the field untouched
        before = [device_read(p, n) for p in (force.ax, force.ay, force.az)]
        parts.advance(flow.refresh_device_macroscopic(), force, 0.5, False)
        flow.wait()
        assert all(np.array_equal(device_read(p, n), b) for p, b in zip((force.ax, force.ay, force.az), before))


def test_single_particle_spread_bitwise(engine, oracle_mod):
    from cfd_solvers_b200.multiphysics import ImmersedBoundaryParticle, ParticleVector3, ResidentParticles3D

    cs = engine
    nx, ny, nz = 12, 10, 8
    n = nx * ny * nz
    p = ImmersedBoundaryParticle(ParticleVector3(11.6, 0.3, 7.9), ParticleVector3(0.01, -0.02, 0.005), 1.5, 0.7)
    with cavity(cs, nx, ny, nz) as flow, ResidentParticles3D(flow, 1) as parts:
        parts.upload([p])
        force = flow.device_local_acceleration(clear=True)
        macro = flow.refresh_device_macroscopic()
        f = flow.compute_macroscopic()
        parts.advance(macro, force, 0.25, True)
        st, acc = oracle_mod.particles_advance(ResidentParticles3D._records([p]).T.astype(np.float32),
                                               (f.ux, f.uy, f.uz), [np.zeros(n, np.float32)] * 3, nx, ny, nz, 0.25,
                                               True)
        flow.wait()
        for ptr, e in zip((force.ax, force.ay, force.az), acc):
            assert np.array_equal(device_read(ptr, n), e)  # the wrapped corner cells, one add each
        assert np.array_equal(parts.download_records()[0, :6].astype(np.float32), st[:6, 0])


@pytest.mark.parametrize("nx", [12, 14])
def test_resident_q_matches_oracle(engine, oracle_mod, nx):
    from cfd_solvers_b200.multiphysics import ResidentFlowDiagnostics3D

    cs = engine
    ny, nz = 10, 19  # z-marching kernel: chunks of 8 planes, the last one partial
    with cavity(cs, nx, ny, nz) as flow, ResidentFlowDiagnostics3D(flow) as diag:
        macro = flow.refresh_device_macroscopic()
        f = flow.compute_macroscopic()
        q = diag.q_criterion(macro)
        assert q
        flow.wait()
        assert np.array_equal(device_read(q, nx * ny * nz), oracle_mod.resident_q((f.ux, f.uy, f.uz), nx, ny, nz))
        assert diag.resident_bytes() == nx * ny * nz * 4


def test_reference_resident_chain(engine):
    from cfd_solvers_b200.multiphysics import (ImmersedBoundaryParticle, ParticleVector3, ResidentFlowDiagnostics3D,
                                               ResidentFreeSurface3D, ResidentParticles3D)

    cs = engine
    nx, ny, nz = 10, 8, 6
    cells = nx * ny * nz
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.72)) as flow:
        flow.initialize_uniform(1.0, 0.0, 0.0, 0.0)
        force = flow.device_local_acceleration(clear=True)
        macro = flow.refresh_device_macroscopic()
        with ResidentFreeSurface3D(flow) as surface:
            surface.initialize_half_space_x(3.5)
            v0 = surface.volume()
            s0 = surface.transfer_stats()
            surface.advect(macro, 0.2)
            v1 = surface.volume()
            assert abs(v1 - v0) < 2.0e-4 * cells
            surface.add_surface_tension_acceleration(force, 0.072, 1.0)
            assert surface.transfer_stats() == s0
            assert surface.resident_bytes() >= 6 * cells * 4
        seed = ImmersedBoundaryParticle(ParticleVector3(2.25, 3.5, 2.75), ParticleVector3(0, 0, 0), 1.0, 0.5)
        with ResidentParticles3D(flow, 1) as particles:
            particles.upload([seed])
            particles.reset_transfer_stats()
            particles.advance(macro, force, 0.05, True)
            assert particles.transfer_stats() == (0, 0, 0)
            assert particles.resident_bytes() == 32
            out = particles.download()[0]
            assert out.position == pytest.approx((2.25, 3.5, 2.75)) and out.mass == 1.0 and out.response_time == 0.5
        with ResidentFlowDiagnostics3D(flow) as diagnostics:
            assert diagnostics.q_criterion(macro)
        f0 = flow.transfer_stats()
        flow.step(2)
        flow.wait()
        f1 = flow.transfer_stats()
        assert (f1.host_to_device_bytes, f1.device_to_host_bytes) == (f0.host_to_device_bytes, f0.device_to_host_bytes)


def test_surface_tension_drives_flow(engine):
    """A fill slab's two interfaces pull with opposite signs: the force field is antisymmetric
    about the slab centre and the flow moves after coupled steps."""
    from cfd_solvers_b200.multiphysics import ResidentFreeSurface3D

    cs = engine
    nx, ny, nz = 16, 8, 8
    with cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=nx, ny=ny, nz=nz, tau=0.8)) as flow:
        flow.initialize_uniform()
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        bump = (0.5 + 0.4 * np.cos(2 * np.pi * x / nx) * np.cos(2 * np.pi * y / ny)).astype(np.float32)
        with ResidentFreeSurface3D(flow) as fs:
            fs.initialize_field(bump.reshape(-1))
            for _ in range(5):
                force = flow.device_local_acceleration(clear=True)
                fs.add_surface_tension_acceleration(force, 0.05)
                flow.step(1)
            f = flow.compute_macroscopic()
            assert np.max(np.abs(f.ux)) > 1e-7 and np.all(np.isfinite(f.ux))


def test_resident_arguments(engine):
    from cfd_solvers_b200.multiphysics import (ImmersedBoundaryParticle, ResidentFlowDiagnostics3D,
                                               ResidentFreeSurface3D, ResidentParticles3D)
    from cfd_solvers_b200.slabs import SlabSolver

    cs = engine
    with cs.EsotericPullCudaSolver(nx=6, ny=5, nz=4) as flow:
        macro = flow.refresh_device_macroscopic()
        force = flow.device_local_acceleration(clear=True)
        with ResidentFreeSurface3D(flow) as fs:
            for bad in (-0.1, 1.5, float("nan")):
                with pytest.raises(ValueError):
                    fs.initialize_uniform(bad)
            with pytest.raises(ValueError):
                fs.initialize_half_space_x(float("inf"))
            with pytest.raises(ValueError):
                fs.initialize_field(np.full(6 * 5 * 4, 2.0, np.float32))
            with pytest.raises(ValueError):
                fs.advect(macro, 0.0)
            with pytest.raises(ValueError):
                fs.add_surface_tension_acceleration(force, -1.0)
            with pytest.raises(ValueError):
                fs.add_surface_tension_acceleration(force, 0.1, 0.0)
        with ResidentParticles3D(flow, 2) as parts:
            with pytest.raises(ValueError):
                parts.upload([ImmersedBoundaryParticle()])  # count mismatch
            with pytest.raises(ValueError):
                parts.upload([ImmersedBoundaryParticle(mass=0.0), ImmersedBoundaryParticle()])
            with pytest.raises(ValueError):
                parts.advance(macro, force, -0.1, True)
        with ResidentParticles3D(flow, 0) as empty:
            empty.upload([])
            empty.advance(macro, force, 0.1, True)
            assert empty.download() == []
    with cs.EsotericPullCudaSolver(nx=2, ny=5, nz=4) as thin:
        with pytest.raises(ValueError):
            ResidentFlowDiagnostics3D(thin)  # Q needs 3 cells per axis
        ResidentFreeSurface3D(thin).close()
    with SlabSolver(cs.InPlaceLbmConfig(nx=6, ny=5, nz=8), 0, 4) as slab:
        for make in (ResidentFreeSurface3D, ResidentFlowDiagnostics3D, lambda s: ResidentParticles3D(s, 1)):
            with pytest.raises(ValueError):
                make(slab)
