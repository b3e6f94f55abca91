// Exercises the C++20 front end (include/cfd/solvers/lbm/esoteric_pull_cuda.hpp)
// the way a reference driver uses cfd::lbm::EsotericPullSolver<D>.
//   frontend_check nodevice        -> expects std::runtime_error from the constructor (no CUDA device)
//   frontend_check gpu <dir>       -> runs a small case, prints "key value" lines for the test to check
#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"

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
