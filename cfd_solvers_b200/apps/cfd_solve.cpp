// cfd-solve for the B200 engine: the in-place LBM cases of the reference's
// case runner (apps/cfd-solve.cpp:163-222, dispatch at :960-988), with the
// `-cuda` cases its SYCL branch has as `-sycl`, plus the 3-D cases the CUDA
// engine adds (lid-driven cavity, sphere-pack channel, gray-LBM adjoint).
// Written against the C++20 front end include/cfd/solvers/lbm/esoteric_pull_cuda.hpp.
//
//   cfd-solve-cuda --list
//   cfd-solve-cuda <case> [--nx N] [--ny N] [--nz N] [--n N] [--steps N] [--tau T]
//                         [--storage fp32|fp16s|fp64] [--seed S] [--interval K] [--fd-check K]
//                         [--vtk PATH] [--json PATH]
//
// Each case prints one line of key=value pairs, as the reference's cases do.
#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace {

namespace cu = cfd::lbm::cuda;
using Clock = std::chrono::steady_clock;

struct Options {
    std::string case_name;
    std::size_t nx{0}, ny{0}, nz{0}; // 0: the case's default
    std::size_t steps{0};
    float tau{0.0F};
    std::string storage{"fp32"};
    std::uint64_t seed{1};
    std::uint32_t interval{16};
    std::size_t fd_check{0};
    std::string vtk, json;
};

void print_list() {
    std::cout << "Available solvers (CUDA, sm_100a):\n"
                 "  lbm-d3q19-cuda            single-grid periodic BGK D3Q19, Taylor-Green start\n"
                 "  lbm-d3q27-cuda            single-grid periodic BGK D3Q27, Taylor-Green start\n"
                 "  lbm-cavity3d-cuda         3-D lid-driven cavity, TRT + Smagorinsky, moving-wall lid\n"
                 "  lbm-channel-spheres-cuda  force-driven channel through a seeded sphere pack, TRT\n"
                 "  lbm-gray-adjoint-cuda     gray-LBM channel: misfit gradient by the discrete adjoint\n";
}

std::size_t parse_size(const char* text, std::string_view option) {
    char* end = nullptr;
    const auto value = std::strtoull(text, &end, 10);
    if (end == text || *end != '\0' || value == 0ULL)
        throw std::invalid_argument(std::string(option) + " must be a positive integer");
    return static_cast<std::size_t>(value);
}

Options parse_options(int argc, char** argv) {
    Options o;
    o.case_name = argv[1];
    for (int i = 2; i < argc; ++i) {
        const std::string_view arg = argv[i];
        const auto value = [&](std::string_view name) -> const char* {
            if (i + 1 >= argc) throw std::invalid_argument(std::string(name) + " requires a value");
            return argv[++i];
        };
        if (arg == "--nx") o.nx = parse_size(value(arg), arg);
        else if (arg == "--ny") o.ny = parse_size(value(arg), arg);
        else if (arg == "--nz") o.nz = parse_size(value(arg), arg);
        else if (arg == "--n") o.nx = o.ny = o.nz = parse_size(value(arg), arg);
        else if (arg == "--steps") o.steps = parse_size(value(arg), arg);
        else if (arg == "--tau") {
            o.tau = std::strtof(value(arg), nullptr);
            if (!(o.tau > 0.5F)) throw std::invalid_argument("--tau must be > 0.5");
        } else if (arg == "--storage") o.storage = value(arg);
        else if (arg == "--seed") o.seed = parse_size(value(arg), arg);
        else if (arg == "--interval") o.interval = static_cast<std::uint32_t>(parse_size(value(arg), arg));
        else if (arg == "--fd-check") o.fd_check = parse_size(value(arg), arg);
        else if (arg == "--vtk") o.vtk = value(arg);
        else if (arg == "--json") o.json = value(arg);
        else throw std::invalid_argument("unknown option " + std::string(arg));
    }
    if (o.storage != "fp32" && o.storage != "fp16s" && o.storage != "fp64")
        throw std::invalid_argument("--storage must be fp32, fp16s or fp64");
    return o;
}

void apply_defaults(Options& o, std::size_t nx, std::size_t ny, std::size_t nz, std::size_t steps, float tau) {
    if (!o.nx) o.nx = nx;
    if (!o.ny) o.ny = ny;
    if (!o.nz) o.nz = nz;
    if (!o.steps) o.steps = steps;
    if (!(o.tau > 0.0F)) o.tau = tau;
}

cu::InPlaceLbmConfig base_config(const Options& o) {
    cu::InPlaceLbmConfig c;
    c.nx = o.nx;
    c.ny = o.ny;
    c.nz = o.nz;
    c.tau = o.tau;
    c.storage = o.storage == "fp16s" ? cu::Storage::fp16s : (o.storage == "fp64" ? cu::Storage::fp64 : cu::Storage::fp32);
    return c;
}

template <class Solver> double seconds_of(Solver& solver, std::size_t steps) {
    solver.wait();
    const auto t0 = Clock::now();
    solver.step(steps);
    solver.wait();
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

double mlups(std::size_t cells, std::size_t steps, double seconds) {
    return static_cast<double>(cells) * static_cast<double>(steps) / (seconds * 1.0e6);
}

// lbm-d3q19-cuda / lbm-d3q27-cuda: the reference's run_lbm_inplace_sycl (apps/cfd-solve.cpp:191-212).
template <class D> int run_inplace(Options o, std::size_t edge) {
    apply_defaults(o, edge, edge, edge, 100, 0.60F);
    cfd::lbm::EsotericPullCudaSolver<D> solver(base_config(o));
    solver.initialize_taylor_green(0.02F);
    const double mass0 = solver.total_mass();
    const double seconds = seconds_of(solver, o.steps);
    const double mass1 = solver.total_mass();
    std::cout << "backend=cuda streaming=in-place device=\"" << solver.device_name() << "\""
              << " cells=" << solver.cells()
              << " population_MiB=" << static_cast<double>(solver.population_bytes()) / (1024.0 * 1024.0)
              << " storage=" << o.storage << " mass_error_abs=" << std::abs(mass1 - mass0)
              << " mass_error_rel=" << std::abs(mass1 - mass0) / std::abs(mass0)
              << " kinetic_energy=" << solver.kinetic_energy() << " max_speed=" << solver.max_speed()
              << " MLUPS=" << mlups(solver.cells(), o.steps, seconds) << '\n';
    return 0;
}

std::size_t at(std::size_t x, std::size_t y, std::size_t z, std::size_t nx, std::size_t ny) {
    return (z * ny + y) * nx + x;
}

// walls on x = 0, nx-1, y = 0, z = 0, nz-1; moving lid (id 2) on y = ny-1
std::vector<std::uint8_t> cavity_flags(std::size_t nx, std::size_t ny, std::size_t nz) {
    std::vector<std::uint8_t> f(nx * ny * nz, 0);
    for (std::size_t z = 0; z < nz; ++z)
        for (std::size_t y = 0; y < ny; ++y)
            for (std::size_t x = 0; x < nx; ++x) {
                const bool side = x == 0 || x + 1 == nx || z == 0 || z + 1 == nz;
                f[at(x, y, z, nx, ny)] = side || y == 0 ? 1 : (y + 1 == ny ? 2 : 0);
            }
    return f;
}

void export_fields(const Options& o, const cu::MacroscopicFields& f, const std::vector<std::uint8_t>& flags,
                   std::uint64_t step) {
    if (o.vtk.empty() && o.json.empty()) return;
    struct V {
        double x, y, z;
    };
    std::vector<double> speed(f.ux.size());
    std::vector<V> velocity(f.ux.size());
    std::vector<std::uint8_t> solid(flags.size());
    for (std::size_t n = 0; n < speed.size(); ++n) {
        velocity[n] = {f.ux[n], f.uy[n], f.uz[n]};
        speed[n] = std::sqrt(velocity[n].x * velocity[n].x + velocity[n].y * velocity[n].y +
                             velocity[n].z * velocity[n].z);
        solid[n] = flags.empty() ? 0 : (flags[n] != 0 ? 1 : 0);
    }
    if (!o.vtk.empty())
        cu::write_vtk_structured_3d(o.vtk, o.nx, o.ny, o.nz, std::span<const double>(speed),
                                    std::span<const V>(velocity), std::span<const std::uint8_t>(solid), "speed",
                                    speed.size() > (1U << 20));
    if (!o.json.empty())
        cu::write_json_state_3d(o.json, o.nx, o.ny, o.nz, step, std::span<const double>(speed),
                                std::span<const std::uint8_t>(solid), "speed");
}

// lbm-cavity3d-cuda: the 3-D form of the reference's lbm-cavity case (apps/cfd-solve.cpp:255-273):
// TRT (magic 3/16) + Smagorinsky Cs 0.1, lid velocity (0.1, 0, 0), from rest.
int run_cavity3d(Options o) {
    apply_defaults(o, 128, 128, 128, 2000, 0.51F);
    cu::InPlaceLbmConfig c = base_config(o);
    c.collision = cu::Collision::trt;
    c.smagorinsky_les = true;
    c.smagorinsky_cs = 0.1F;
    cfd::lbm::EsotericPullCudaSolver<cu::D3Q19> solver(c);
    const auto flags = cavity_flags(o.nx, o.ny, o.nz);
    solver.set_flags(flags);
    solver.set_wall_velocity(2, 0.1F, 0.0F, 0.0F);
    solver.initialize_uniform();
    const double mass0 = solver.total_mass();
    const double seconds = seconds_of(solver, o.steps);
    const auto f = solver.compute_macroscopic();
    const std::size_t centre = at(o.nx / 2, o.ny / 2, o.nz / 2, o.nx, o.ny);
    const double mass1 = solver.total_mass();
    std::cout << "case=lid-driven-cavity-3d cells=" << solver.cells() << " steps=" << o.steps
              << " storage=" << o.storage << " center_ux=" << f.ux[centre] << " center_uy=" << f.uy[centre]
              << " max_speed=" << solver.max_speed() << " mass_error_rel=" << std::abs(mass1 - mass0) / mass0
              << " MLUPS=" << mlups(solver.cells(), o.steps, seconds) << '\n';
    export_fields(o, f, flags, solver.time_step());
    return 0;
}

// Channel walls on y = 0, ny-1, z = 0, nz-1 (periodic in x) plus seeded random
// spheres (radii uniform in [4, 12], centres uniform, x periodic) added until
// they cover 10 % of the cells; std::mt19937_64(seed).
std::vector<std::uint8_t> sphere_channel(std::size_t nx, std::size_t ny, std::size_t nz, std::uint64_t seed,
                                         double* solid_fraction) {
    std::vector<std::uint8_t> f(nx * ny * nz, 0);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> radius(4.0, 12.0), ux(0.0, double(nx)), uy(0.0, double(ny)),
        uz(0.0, double(nz));
    const double target = 0.10 * static_cast<double>(f.size());
    std::size_t count = 0;
    while (static_cast<double>(count) < target) {
        const double r = radius(rng), cx = ux(rng), cy = uy(rng), cz = uz(rng);
        const auto lo = [](double c, double rr) { return static_cast<std::size_t>(std::max(0.0, std::floor(c - rr))); };
        const std::size_t z1 = std::min(nz, static_cast<std::size_t>(cz + r) + 2U),
                          y1 = std::min(ny, static_cast<std::size_t>(cy + r) + 2U);
        for (std::size_t z = lo(cz, r); z < z1; ++z)
            for (std::size_t y = lo(cy, r); y < y1; ++y)
                for (std::size_t x = 0; x < nx; ++x) {
                    double dx = std::abs(double(x) + 0.5 - cx);
                    dx = std::min(dx, double(nx) - dx);
                    const double dy = double(y) + 0.5 - cy, dz = double(z) + 0.5 - cz;
                    std::uint8_t& cell = f[at(x, y, z, nx, ny)];
                    if (!cell && dx * dx + dy * dy + dz * dz <= r * r) {
                        cell = 1;
                        ++count;
                    }
                }
    }
    *solid_fraction = static_cast<double>(count) / static_cast<double>(f.size());
    for (std::size_t z = 0; z < nz; ++z)
        for (std::size_t y = 0; y < ny; ++y)
            for (std::size_t x = 0; x < nx; ++x)
                if (y == 0 || y + 1 == ny || z == 0 || z + 1 == nz) f[at(x, y, z, nx, ny)] = 1;
    return f;
}

// lbm-channel-spheres-cuda: TRT (magic 3/16), tau 0.55, body force gx = 1e-6.
int run_channel_spheres(Options o) {
    apply_defaults(o, 128, 64, 64, 2000, 0.55F);
    cu::InPlaceLbmConfig c = base_config(o);
    c.collision = cu::Collision::trt;
    c.acceleration_x = 1.0e-6F;
    cfd::lbm::EsotericPullCudaSolver<cu::D3Q19> solver(c);
    double spheres = 0.0;
    const auto flags = sphere_channel(o.nx, o.ny, o.nz, o.seed, &spheres);
    solver.set_flags(flags);
    solver.initialize_uniform();
    const double mass0 = solver.total_mass();
    const double seconds = seconds_of(solver, o.steps);
    const auto f = solver.compute_macroscopic();
    double sum_ux = 0.0;
    std::size_t fluid = 0;
    for (std::size_t n = 0; n < flags.size(); ++n)
        if (!flags[n]) {
            sum_ux += f.ux[n];
            ++fluid;
        }
    const double mass1 = solver.total_mass();
    std::cout << "case=channel-spheres cells=" << solver.cells() << " steps=" << o.steps << " storage=" << o.storage
              << " sphere_fraction=" << spheres << " mean_ux=" << sum_ux / static_cast<double>(fluid)
              << " max_speed=" << solver.max_speed() << " mass_error_rel=" << std::abs(mass1 - mass0) / mass0
              << " MLUPS=" << mlups(solver.cells(), o.steps, seconds) << '\n';
    export_fields(o, f, flags, solver.time_step());
    return 0;
}

// u (FP64 fields) of the final state after `steps` steps from rest with solid fraction ns.
std::vector<double> run_velocity(cfd::lbm::EsotericPullCudaSolver<cu::D3Q19>& s, const std::vector<float>& ns,
                                 std::size_t steps) {
    const std::size_t n = s.cells();
    s.set_solid_fraction(ns);
    s.initialize_uniform();
    s.step(steps);
    std::vector<double> rho(n), u(3 * n);
    cu::check(cfdx_lbm_macroscopic_f64(s.native_handle(), rho.data(), u.data(), u.data() + n, u.data() + 2 * n,
                                       CFDX_HOST),
              "macroscopic_f64");
    return u;
}

double misfit(const std::vector<double>& u, const std::vector<double>& target, const std::vector<std::uint8_t>& flags) {
    const std::size_t n = flags.size();
    double j = 0.0;
    for (std::size_t k = 0; k < 3; ++k)
        for (std::size_t c = 0; c < n; ++c)
            if (!flags[c]) {
                const double r = u[k * n + c] - target[k * n + c];
                j += 0.5 * r * r;
            }
    return j;
}

// lbm-gray-adjoint-cuda: gray-LBM TRT channel (partial bounce-back n_s), J = 1/2 sum over fluid
// cells |u(steps) - u*|^2 with u* from a hidden n_s*, dJ/dn_s by the discrete adjoint; with
// --fd-check K, central differences of J on K random fluid cells.  adjoint_over_forward is the
// reverse sweep's time over the plain forward's (the checkpointed forward is reported apart).
int run_gray_adjoint(Options o) {
    apply_defaults(o, 32, 32, 32, 200, 0.6F);
    cu::InPlaceLbmConfig c = base_config(o);
    c.collision = cu::Collision::trt;
    c.acceleration_x = 1.0e-5F;
    cfd::lbm::EsotericPullCudaSolver<cu::D3Q19> s(c);
    const std::size_t n = s.cells();
    std::vector<std::uint8_t> flags(n, 0);
    for (std::size_t z = 0; z < o.nz; ++z)
        for (std::size_t y = 0; y < o.ny; ++y)
            for (std::size_t x = 0; x < o.nx; ++x)
                if (y == 0 || y + 1 == o.ny || z == 0 || z + 1 == o.nz) flags[at(x, y, z, o.nx, o.ny)] = 1;
    s.set_flags(flags);
    std::mt19937_64 rng(o.seed);
    std::uniform_real_distribution<float> gray(0.0F, 0.2F);
    std::vector<float> ns(n, 0.0F), hidden(n, 0.0F);
    for (std::size_t k = 0; k < n; ++k) {
        const float a = gray(rng), b = gray(rng);
        if (!flags[k]) {
            ns[k] = a;
            hidden[k] = b;
        }
    }
    const std::vector<double> target = run_velocity(s, hidden, o.steps);

    s.set_solid_fraction(ns);
    s.initialize_uniform();
    s.wait();
    const auto t0 = Clock::now();
    s.step(o.steps);
    s.wait();
    const double forward = std::chrono::duration<double>(Clock::now() - t0).count();

    s.initialize_uniform();
    s.wait();
    const auto t1 = Clock::now();
    s.adjoint_forward(o.steps, o.interval);
    s.wait();
    const double checkpointed = std::chrono::duration<double>(Clock::now() - t1).count();
    std::vector<double> rho(n), u(3 * n);
    cu::check(cfdx_lbm_macroscopic_f64(s.native_handle(), rho.data(), u.data(), u.data() + n, u.data() + 2 * n,
                                       CFDX_HOST),
              "macroscopic_f64");
    std::vector<float> gx(n, 0.0F), gy(n, 0.0F), gz(n, 0.0F);
    for (std::size_t k = 0; k < n; ++k)
        if (!flags[k]) {
            gx[k] = static_cast<float>(u[k] - target[k]);
            gy[k] = static_cast<float>(u[n + k] - target[n + k]);
            gz[k] = static_cast<float>(u[2 * n + k] - target[2 * n + k]);
        }
    const auto t2 = Clock::now();
    const auto grad = s.adjoint_backward(gx, gy, gz);
    const double adjoint = std::chrono::duration<double>(Clock::now() - t2).count();
    const std::size_t adjoint_bytes = s.adjoint_memory();
    s.adjoint_release();
    const double j = misfit(u, target, flags);
    double norm = 0.0;
    for (const double g : grad.solid_fraction) norm += g * g;
    std::cout << "case=gray-adjoint cells=" << n << " steps=" << o.steps << " interval=" << o.interval
              << " storage=" << o.storage << " J=" << j << " grad_ns_l2=" << std::sqrt(norm)
              << " grad_tau=" << grad.tau << " forward_s=" << forward << " checkpointed_forward_s=" << checkpointed
              << " adjoint_s=" << adjoint << " adjoint_over_forward=" << adjoint / forward
              << " adjoint_MiB=" << static_cast<double>(adjoint_bytes) / (1024.0 * 1024.0);
    if (o.fd_check) {
        std::vector<std::size_t> fluid;
        for (std::size_t k = 0; k < n; ++k)
            if (!flags[k]) fluid.push_back(k);
        std::shuffle(fluid.begin(), fluid.end(), rng);
        fluid.resize(std::min(o.fd_check, fluid.size()));
        const float eps = o.storage == "fp64" ? 1.0e-3F : 1.0e-2F;
        double worst = 0.0, scale = 0.0;
        for (const std::size_t k : fluid) {
            std::vector<float> p = ns, m = ns;
            p[k] += eps;
            m[k] -= eps;
            const double fd = (misfit(run_velocity(s, p, o.steps), target, flags) -
                               misfit(run_velocity(s, m, o.steps), target, flags)) /
                              (static_cast<double>(p[k]) - static_cast<double>(m[k]));
            worst = std::max(worst, std::abs(fd - grad.solid_fraction[k]));
            scale = std::max(scale, std::abs(fd));
        }
        std::cout << " fd_cells=" << fluid.size() << " fd_max_abs_err_over_max_fd=" << (scale > 0 ? worst / scale : 0.0);
    }
    std::cout << '\n';
    return 0;
}

} // namespace

int main(int argc, char** argv) {
    if (argc < 2 || std::string_view(argv[1]) == "--list") {
        print_list();
        return 0;
    }
    try {
        const Options o = parse_options(argc, argv);
        if (o.case_name == "lbm-d3q19-cuda") return run_inplace<cu::D3Q19>(o, 64);
        if (o.case_name == "lbm-d3q27-cuda") return run_inplace<cu::D3Q27>(o, 56);
        if (o.case_name == "lbm-cavity3d-cuda") return run_cavity3d(o);
        if (o.case_name == "lbm-channel-spheres-cuda") return run_channel_spheres(o);
        if (o.case_name == "lbm-gray-adjoint-cuda") return run_gray_adjoint(o);
        std::cerr << "Unknown solver: " << o.case_name << "\n";
        print_list();
        return 1;
    } catch (const std::exception& e) {
        std::cerr << "cfd-solve-cuda: " << e.what() << '\n';
        return 1;
    }
}
