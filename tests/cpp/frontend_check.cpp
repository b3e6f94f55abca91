// Exercises the C++20 front end (include/cfd/solvers/lbm/esoteric_pull_cuda.hpp)
// the way a reference driver uses cfd::lbm::EsotericPullSolver<D>.
//   frontend_check nodevice        -> expects std::runtime_error from the constructor (no CUDA device)
//   frontend_check gpu <dir>       -> runs a small case, prints "key value" lines for the test to check
#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"
#include "cfd/solvers/lbm/resident_multiphysics_cuda.hpp"

#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "nodevice";
    cfd::lbm::cuda::InPlaceLbmConfig config;
    config.nx = 24;
    config.ny = 20;
    config.nz = 16;
    config.tau = 0.62F;
    config.acceleration_x = 1e-5F;
    if (mode == "nodevice") {
        try {
            cfd::lbm::EsotericPullCudaSolver<cfd::lbm::cuda::D3Q19> solver(config);
            std::cout << "unexpected: constructed without a device\n";
            return 1;
        } catch (const std::runtime_error& e) {
            std::cout << "runtime_error " << e.what() << '\n';
        }
        try {
            config.tau = 0.4F;
            cfd::lbm::EsotericPullCudaSolver<cfd::lbm::cuda::D3Q19> solver(config);
            return 1;
        } catch (const std::invalid_argument& e) {
            std::cout << "invalid_argument " << e.what() << '\n';
        }
        return 0;
    }
    const std::string dir = argc > 2 ? argv[2] : ".";
    cfd::lbm::EsotericPullCudaSolver<cfd::lbm::cuda::D3Q19> solver(config);
    std::vector<std::uint8_t> mask(solver.cells(), 0);
    for (std::size_t n = 0; n < mask.size(); n += 17) mask[n] = 1;
    solver.set_solid_mask(mask);
    solver.initialize_taylor_green(0.04F);
    solver.step(13);
    std::printf("time_step %llu\n", static_cast<unsigned long long>(solver.time_step()));
    std::printf("checksum %.17g\n", solver.checksum());
    std::printf("mass %.17g\n", solver.mass());
    std::printf("kinetic_energy %.17g\n", solver.kinetic_energy());
    const auto fields = solver.compute_macroscopic();
    std::printf("download_equal %d\n", solver.download_macroscopic().ux == fields.ux ? 1 : 0);
    double sum_ux = 0.0;
    for (const float v : fields.ux) sum_ux += v;
    std::printf("sum_ux %.17g\n", sum_ux);
    solver.save_checkpoint(dir + "/frontend.chk");
    cfd::lbm::EsotericPullCudaSolver<cfd::lbm::cuda::D3Q19> restored(config);
    restored.set_solid_mask(mask);
    restored.load_checkpoint(dir + "/frontend.chk");
    solver.step(7);
    restored.step(7);
    std::printf("restart_bitwise %d\n", solver.logical_populations() == restored.logical_populations() ? 1 : 0);
    // a whole-ring slab steps like the whole lattice
    {
        cfd::lbm::EsotericPullCudaSlab<cfd::lbm::cuda::D3Q19> slab(config, 0U, static_cast<std::uint32_t>(config.nz));
        cfd::lbm::EsotericPullCudaSolver<cfd::lbm::cuda::D3Q19> whole(config);
        const auto info = slab.slab_info();
        std::vector<std::uint8_t> local(slab.cells(), 0);
        const std::size_t plane = config.nx * config.ny;
        for (std::size_t k = 0; k < config.nz + 2; ++k) // local plane k = global (k - 1) mod nz
            for (std::size_t i = 0; i < plane; ++i)
                local[k * plane + i] = mask[((k + config.nz - 1) % config.nz) * plane + i];
        slab.set_solid_mask(local);
        whole.set_solid_mask(mask);
        slab.initialize_taylor_green(0.04F);
        whole.initialize_taylor_green(0.04F);
        slab.step(9);
        whole.step(9);
        const auto a = slab.compute_macroscopic();
        const auto b = whole.compute_macroscopic();
        bool same = true;
        for (std::size_t n = 0; n < b.ux.size(); ++n) same = same && a.ux[n + plane] == b.ux[n] && a.rho[n + plane] == b.rho[n];
        std::printf("slab_info %u %u %u\n", info[0], info[1], info[2]);
        std::printf("slab_equals_whole %d\n", same ? 1 : 0);
        std::printf("halo_bytes %zu\n", slab.halo_bytes());
    }
    // the reference's cube test (tests/test_completion.cpp:885-901) through the device voxelizer
    {
        struct P { double x, y, z; };
        struct T { P a, b, c; };
        struct S { std::vector<T> triangles; } cube;
        struct G { std::size_t nx, ny, nz; P minimum, maximum; } grid{8, 8, 8, {0, 0, 0}, {1, 1, 1}};
        const P p000{.25, .25, .25}, p100{.75, .25, .25}, p010{.25, .75, .25}, p110{.75, .75, .25};
        const P p001{.25, .25, .75}, p101{.75, .25, .75}, p011{.25, .75, .75}, p111{.75, .75, .75};
        for (const T& t : {T{p000, p110, p100}, T{p000, p010, p110}, T{p001, p101, p111}, T{p001, p111, p011},
                           T{p000, p100, p101}, T{p000, p101, p001}, T{p010, p011, p111}, T{p010, p111, p110},
                           T{p000, p001, p011}, T{p000, p011, p010}, T{p100, p110, p111}, T{p100, p111, p101}})
            cube.triangles.push_back(t);
        const auto m = cfd::lbm::cuda::voxelize_surface(cube, grid);
        auto idx = [](std::size_t i, std::size_t j, std::size_t k) { return (k * 8 + j) * 8 + i; };
        std::size_t solid = 0;
        for (auto v : m) solid += v;
        std::printf("voxel_cube %d %d %zu\n", m[idx(4, 4, 4)], m[idx(0, 0, 0)], solid);
        cfd::lbm::EsotericPullCudaSolver<cfd::lbm::cuda::D3Q19> body(config);
        body.set_solid_surface(cube, P{0, 0, 0}, P{1, 1, 1});
        body.initialize_uniform();
        body.step(2);
        const auto q = body.q_criterion();
        const auto f = body.compute_macroscopic();
        std::vector<P> vel(f.ux.size());
        std::vector<double> speed(f.ux.size());
        for (std::size_t n = 0; n < vel.size(); ++n) {
            vel[n] = {f.ux[n], f.uy[n], f.uz[n]};
            speed[n] = std::sqrt(double(f.ux[n]) * f.ux[n] + double(f.uy[n]) * f.uy[n] + double(f.uz[n]) * f.uz[n]);
        }
        const auto q2 = cfd::lbm::cuda::q_criterion_3d(config.nx, config.ny, config.nz, std::span<const P>(vel));
        std::printf("q_criterion_equal %d\n", q == q2 ? 1 : 0);
        cfd::lbm::cuda::write_vtk_structured_3d(dir + "/frame.vtk", config.nx, config.ny, config.nz,
                                                std::span<const double>(speed), std::span<const P>(vel), {}, "speed");
        cfd::lbm::cuda::write_json_state_3d(dir + "/state.json", config.nx, config.ny, config.nz, body.time_step(),
                                            std::span<const double>(speed));
        std::printf("exported 1\n");
    }
    // the reference's resident chain (tests/test_v0156_gpu_lbm_multiphysics.cpp:26-67) through the C++ classes
    {
        namespace lc = cfd::lbm::cuda;
        lc::InPlaceLbmConfig c;
        c.nx = 10;
        c.ny = 8;
        c.nz = 6;
        c.tau = 0.72F;
        const std::size_t cells = 480;
        cfd::lbm::EsotericPullCudaSolver<lc::D3Q19> flow(c);
        flow.initialize_uniform(1.0F, 0.0F, 0.0F, 0.0F);
        auto force = flow.device_local_acceleration(true);
        auto macro = flow.refresh_device_macroscopic();
        cfd::lbm::ResidentThermalD3Q7Cuda thermal(flow, lc::ResidentThermalConfig{10, 8, 6, 0.02F});
        thermal.initialize_uniform(300.0F);
        const double heat0 = thermal.total_scalar();
        thermal.reset_transfer_stats();
        thermal.step(macro, 3U);
        thermal.add_boussinesq_acceleration(force, 300.0F, 3.0e-3F, lc::ParticleVector3{0.0, -1.0, 0.0});
        const double heat1 = thermal.total_scalar();
        std::printf("chain_thermal %d\n",
                    std::abs(heat1 - heat0) / heat0 < 2.0e-5 && thermal.transfer_stats().host_transfer_bytes() == 0U);
        cfd::lbm::ResidentFreeSurfaceCuda3D surface(flow, 10, 8, 6);
        surface.initialize_half_space_x(3.5F);
        const double volume0 = surface.volume();
        surface.advect(macro, 0.2F);
        const double volume1 = surface.volume();
        std::printf("chain_volume %d\n", std::abs(volume1 - volume0) < 2.0e-4 * static_cast<double>(cells));
        surface.add_surface_tension_acceleration(force, 0.072F, 1.0F);
        lc::ImmersedBoundaryParticle seed{{2.25, 3.5, 2.75}, {}, 1.0, 0.5};
        cfd::lbm::ResidentParticlesCuda3D particles(flow, 10, 8, 6, 1U);
        particles.upload(std::span<const lc::ImmersedBoundaryParticle>(&seed, 1U));
        particles.reset_transfer_stats();
        particles.advance(macro, force, 0.05F, true);
        std::printf("chain_particles %d\n", particles.transfer_stats().host_transfer_bytes() == 0U);
        cfd::lbm::ResidentFlowDiagnosticsCuda3D diagnostics(flow, 10, 8, 6);
        std::printf("chain_q %d\n", diagnostics.q_criterion(macro) != nullptr);
        flow.reset_transfer_stats();
        flow.step(2U);
        flow.wait();
        std::printf("chain_flow %d\n", flow.transfer_stats().host_transfer_bytes() == 0U);
        try {
            cfd::lbm::ResidentFreeSurfaceCuda3D wrong(flow, 10, 8, 7);
        } catch (const std::invalid_argument&) {
            std::printf("chain_grid invalid_argument\n");
        }
    }
    try {
        solver.set_solid_mask(std::vector<std::uint8_t>(3));
    } catch (const std::invalid_argument&) {
        std::printf("size_mismatch invalid_argument\n");
    }
    try {
        solver.set_wall_velocity(1, 0.1F, 0.0F, 0.0F);
    } catch (const std::out_of_range&) {
        std::printf("wall_id out_of_range\n");
    }
    return 0;
}
