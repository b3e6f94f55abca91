// Exercises the C++20 front end (include/cfd/solvers/lbm/esoteric_pull_cuda.hpp)
// the way a reference driver uses cfd::lbm::EsotericPullSolver<D>.
//   frontend_check nodevice        -> expects std::runtime_error from the constructor (no CUDA device)
//   frontend_check gpu <dir>       -> runs a small case, prints "key value" lines for the test to check
#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"

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
