// cfd-bench for the B200 engine: the reference's benchmark CLI
// (apps/cfd-bench.cpp) with the `--backend cuda` branch its dispatch_backend
// (apps/cfd-bench.cpp:236-261) would gain, written against the C++20 front
// end include/cfd/solvers/lbm/esoteric_pull_cuda.hpp.
//
// Same options, case and output records as the reference: D3Q19/D3Q27
// in-place Esoteric-Pull, Taylor-Green start (amplitude 0.02), `--warmup`
// untimed then `--steps` timed steps (host steady clock around step() +
// wait(), like the reference's SYCL branch), text / --csv / --json
// (schema cfd_solvers.benchmark.v1).  Added keys: glups,
// algorithmic_bytes_per_update, roofline_fraction (given --hbm-peak-gbs),
// storage_precision, collision, checksum.  Extensions: --storage
// fp32|fp16s|fp64, --collision bgk|trt, --les, --case taylor-green|cavity.
#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"

#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace {

struct Options {
    std::string lattice{"d3q19"};
    std::string backend{"cuda"};
    std::string streaming{"in-place"};
    std::string storage{"fp32"};
    std::string collision{"bgk"};
    std::string case_name{"taylor-green"};
    std::size_t nx{64};
    std::size_t ny{64};
    std::size_t nz{64};
    std::size_t warmup{10};
    std::size_t steps{100};
    float tau{0.6F};
    bool les{false};
    double hbm_peak_gbs{0.0};
    bool csv{false};
    bool json{false};
};

std::size_t parse_size(const char* text, std::string_view option) {
    const auto value = std::strtoull(text, nullptr, 10);
    if (value == 0ULL) throw std::invalid_argument(std::string(option) + " must be > 0");
    return static_cast<std::size_t>(value);
}

float parse_tau(const char* text, std::string_view option) {
    const float value = std::strtof(text, nullptr);
    if (!(value > 0.5F)) throw std::invalid_argument(std::string(option) + " must be > 0.5");
    return value;
}

void usage() {
    std::cout << "usage: cfd-bench-cuda [--lattice d3q19|d3q27] [--backend cuda] [--streaming in-place]\n"
                 "                      [--nx N] [--ny N] [--nz N] [--warmup N] [--steps N] [--tau T]\n"
                 "                      [--storage fp32|fp16s|fp64] [--collision bgk|trt] [--les]\n"
                 "                      [--case taylor-green|cavity] [--hbm-peak-gbs G] [--csv|--json]\n";
}

Options parse_options(int argc, char** argv) {
    Options o;
    for (int i = 1; i < argc; ++i) {
        const std::string_view arg = argv[i];
        const auto value = [&](std::string_view name) -> const char* {
            if (i + 1 >= argc) throw std::invalid_argument(std::string(name) + " requires a value");
            return argv[++i];
        };
        if (arg == "--lattice") o.lattice = value(arg);
        else if (arg == "--backend") o.backend = value(arg);
        else if (arg == "--streaming") o.streaming = value(arg);
        else if (arg == "--nx") o.nx = parse_size(value(arg), arg);
        else if (arg == "--ny") o.ny = parse_size(value(arg), arg);
        else if (arg == "--nz") o.nz = parse_size(value(arg), arg);
        else if (arg == "--warmup") o.warmup = parse_size(value(arg), arg);
        else if (arg == "--steps") o.steps = parse_size(value(arg), arg);
        else if (arg == "--tau") o.tau = parse_tau(value(arg), arg);
        else if (arg == "--storage") o.storage = value(arg);
        else if (arg == "--collision") o.collision = value(arg);
        else if (arg == "--case") o.case_name = value(arg);
        else if (arg == "--les") o.les = true;
        else if (arg == "--hbm-peak-gbs") o.hbm_peak_gbs = std::strtod(value(arg), nullptr);
        else if (arg == "--csv") o.csv = true;
        else if (arg == "--json") o.json = true;
        else if (arg == "--help" || arg == "-h") {
            usage();
            std::exit(0);
        } else {
            throw std::invalid_argument("unknown option " + std::string(arg));
        }
    }
    if (o.backend != "cuda") throw std::invalid_argument("this build provides --backend cuda");
    if (o.streaming != "in-place") throw std::invalid_argument("the CUDA backend runs --streaming in-place");
    return o;
}

std::string json_escape(std::string_view text) {
    std::string out;
    for (const char c : text) {
        if (c == '"' || c == '\\') out.push_back('\\');
        out.push_back(c);
    }
    return out;
}

std::vector<std::uint8_t> cavity_flags(std::size_t nx, std::size_t ny, std::size_t nz) {
    // walls on x = 0, nx-1, y = 0, z = 0, nz-1; moving lid (id 2) on y = ny-1
    std::vector<std::uint8_t> f(nx * ny * nz, 0);
    for (std::size_t z = 0; z < nz; ++z)
        for (std::size_t y = 0; y < ny; ++y)
            for (std::size_t x = 0; x < nx; ++x) {
                const std::size_t n = (z * ny + y) * nx + x;
                if (x == 0 || x + 1 == nx || y == 0 || z == 0 || z + 1 == nz) f[n] = 1;
                if (y + 1 == ny && !(x == 0 || x + 1 == nx || z == 0 || z + 1 == nz)) f[n] = 2;
            }
    return f;
}

template <class Descriptor> int run_cuda(const Options& o) {
    namespace cu = cfd::lbm::cuda;
    cu::InPlaceLbmConfig config;
    config.nx = o.nx;
    config.ny = o.ny;
    config.nz = o.nz;
    config.tau = o.tau;
    config.smagorinsky_les = o.les;
    config.smagorinsky_cs = o.les ? 0.1F : 0.0F;
    if (o.collision == "trt") config.collision = cu::Collision::trt;
    else if (o.collision != "bgk") throw std::invalid_argument("collision must be bgk or trt");
    if (o.storage == "fp16s") config.storage = cu::Storage::fp16s;
    else if (o.storage == "fp64") config.storage = cu::Storage::fp64;
    else if (o.storage != "fp32") throw std::invalid_argument("storage must be fp32, fp16s or fp64");

    cfd::lbm::EsotericPullCudaSolver<Descriptor> solver(config);
    std::size_t fluid = solver.cells();
    if (o.case_name == "cavity") {
        const auto flags = cavity_flags(o.nx, o.ny, o.nz);
        solver.set_flags(flags);
        solver.set_wall_velocity(2, 0.1F, 0.0F, 0.0F);
        solver.initialize_uniform();
        fluid = 0;
        for (const auto v : flags) fluid += v == 0 ? 1U : 0U;
    } else if (o.case_name == "taylor-green") {
        solver.initialize_taylor_green(0.02F);
    } else {
        throw std::invalid_argument("case must be taylor-green or cavity");
    }
    const double mass0 = solver.total_mass();
    solver.step(o.warmup);
    solver.wait();
    const auto begin = std::chrono::steady_clock::now();
    solver.step(o.steps);
    solver.wait();
    const auto end = std::chrono::steady_clock::now();
    const double seconds = std::chrono::duration<double>(end - begin).count();
    const double mass1 = solver.total_mass();
    const double checksum = solver.checksum();

    const std::size_t cells = solver.cells();
    const double updates = static_cast<double>(cells) * static_cast<double>(o.steps);
    const double mlups = updates / seconds / 1.0e6;
    const double value_bytes = o.storage == "fp16s" ? 2.0 : (o.storage == "fp64" ? 8.0 : 4.0);
    // populations read and written once per fluid cell, plus the flag byte of every cell
    const double alg_bytes_per_update =
        (2.0 * Descriptor::q * value_bytes * static_cast<double>(fluid) + (fluid == cells ? 0.0 : cells)) /
        static_cast<double>(cells);
    const double estimated_gbps = mlups * 2.0 * Descriptor::q * sizeof(float) / 1000.0;
    const double achieved_gbs = mlups * alg_bytes_per_update / 1000.0;
    const double allocated_mib = static_cast<double>(solver.population_bytes()) / (1024.0 * 1024.0);
    const double single_grid_mib = static_cast<double>(Descriptor::q) * cells * sizeof(float) / (1024.0 * 1024.0);
    const double mass_error_abs = std::abs(mass1 - mass0);
    const double mass_error_rel = mass0 != 0.0 ? mass_error_abs / std::abs(mass0) : 0.0;
    const std::string device = solver.device_name();
    const double roofline = o.hbm_peak_gbs > 0.0 ? achieved_gbs / o.hbm_peak_gbs : -1.0;

    if (o.csv) {
        std::cout << "lattice,backend,streaming,device,nx,ny,nz,q,steps,seconds,mlups,estimated_ddf_gbps,"
                     "allocated_ddf_mib,single_grid_ddf_mib,mass_error_abs,mass_error_rel,glups,"
                     "algorithmic_bytes_per_update,roofline_fraction,storage_precision,collision,checksum\n";
        std::cout << o.lattice << ",cuda,in-place,\"" << device << "\"," << o.nx << ',' << o.ny << ',' << o.nz << ','
                  << Descriptor::q << ',' << o.steps << ',' << std::setprecision(9) << seconds << ',' << mlups << ','
                  << estimated_gbps << ',' << allocated_mib << ',' << single_grid_mib << ',' << mass_error_abs << ','
                  << mass_error_rel << ',' << mlups / 1000.0 << ',' << alg_bytes_per_update << ',' << roofline << ','
                  << o.storage << ',' << o.collision << (o.les ? "+les" : "") << ',' << std::setprecision(17)
                  << checksum << '\n';
        return 0;
    }
    if (o.json) {
        std::cout << std::setprecision(12) << "{\"schema\":\"cfd_solvers.benchmark.v1\","
                  << "\"lattice\":\"" << json_escape(o.lattice) << "\",\"backend\":\"cuda\",\"streaming\":\"in-place\","
                  << "\"device\":\"" << json_escape(device) << "\",\"nx\":" << o.nx << ",\"ny\":" << o.ny
                  << ",\"nz\":" << o.nz << ",\"q\":" << Descriptor::q << ",\"steps\":" << o.steps
                  << ",\"seconds\":" << seconds << ",\"mlups\":" << mlups << ",\"estimated_ddf_gbps\":" << estimated_gbps
                  << ",\"allocated_ddf_mib\":" << allocated_mib << ",\"single_grid_ddf_mib\":" << single_grid_mib
                  << ",\"mass_error_abs\":" << mass_error_abs << ",\"mass_error_rel\":" << mass_error_rel
                  << ",\"glups\":" << mlups / 1000.0 << ",\"algorithmic_bytes_per_update\":" << alg_bytes_per_update
                  << ",\"roofline_fraction\":";
        if (roofline >= 0.0) std::cout << roofline; else std::cout << "null";
        std::cout << ",\"storage_precision\":\"" << o.storage << "\",\"collision\":\"" << o.collision
                  << (o.les ? "+les" : "") << "\",\"case\":\"" << o.case_name << "\",\"checksum\":"
                  << std::setprecision(17) << checksum << "}\n";
        return 0;
    }
    std::cout << "lattice=" << o.lattice << " backend=cuda streaming=in-place device=\"" << device << "\"\n"
              << "grid=" << o.nx << 'x' << o.ny << 'x' << o.nz << " q=" << Descriptor::q << " steps=" << o.steps
              << " storage=" << o.storage << " collision=" << o.collision << (o.les ? "+les" : "")
              << " case=" << o.case_name << '\n'
              << std::fixed << std::setprecision(3) << "time_s=" << seconds << " MLUPS=" << mlups
              << " GLUPS=" << mlups / 1000.0 << " estimated_DDF_GB/s=" << estimated_gbps
              << " algorithmic_GB/s=" << achieved_gbs << '\n'
              << "allocated_DDF_MiB=" << allocated_mib << " single_grid_DDF_MiB=" << single_grid_mib << '\n'
              << std::scientific << "mass_error_abs=" << mass_error_abs << " mass_error_rel=" << mass_error_rel
              << std::setprecision(17) << " checksum=" << checksum << '\n';
    return 0;
}

} // namespace

int main(int argc, char** argv) {
    try {
        const Options options = parse_options(argc, argv);
        if (options.lattice == "d3q19") return run_cuda<cfd::lbm::cuda::D3Q19>(options);
        if (options.lattice == "d3q27") return run_cuda<cfd::lbm::cuda::D3Q27>(options);
        throw std::invalid_argument("lattice must be d3q19 or d3q27 (the CUDA engine has no D2Q9)");
    } catch (const std::exception& error) {
        std::cerr << "cfd-bench: " << error.what() << '\n';
        return 1;
    }
}
