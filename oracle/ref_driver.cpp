// Driver around the reference's own CPU solvers -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile directly against the reference's headers and its
// one instantiation unit (src/lbm/esoteric_pull.cpp) where they lie; no
// reference source is copied into this repository.  Output goes to
// oracle/_ref/ only.  It exposes a small C interface so the tests can run the
// reference on the same seeded inputs as the CUDA path, and so bench.py can
// time the reference's CPU path on the GPU box's host cores.
//
// Reference classes driven here:
//   cfd::lbm::EsotericPullSolver<D>            include/cfd/solvers/lbm/esoteric_pull.hpp:104-515
//   cfd::lbm::OneStepPullSolver<D> (TRT)       include/cfd/solvers/lbm/one_step_pull.hpp:16-215
//   cfd::lbm::PrecisionPullSolver<D,double>    include/cfd/solvers/lbm/precision_pull.hpp:49-213
//   cfd::lbm::CompressedPopulationPullSolver<D, ShiftedHalfCodec<D>>
//                                              include/cfd/solvers/lbm/compressed_pull.hpp:95-147
//   the CPU free surface and point particles   src/lbm/free_surface.cpp, src/lbm/particles.cpp
#include "cfd/core/parallel.hpp"
#include "cfd/solvers/lbm/compressed_pull.hpp"
#include "cfd/solvers/lbm/esoteric_pull.hpp"
#include "cfd/solvers/lbm/free_surface.hpp"
#include "cfd/solvers/lbm/one_step_pull.hpp"
#include "cfd/solvers/lbm/particles.hpp"
#include "cfd/solvers/lbm/precision_pull.hpp"
#include "cfd/solvers/lbm/visualization.hpp"
#include "cfd/solvers/lbm/voxelize.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>

namespace {

thread_local char g_error[512];

void set_error(const char* text) {
    std::strncpy(g_error, text, sizeof g_error - 1U);
    g_error[sizeof g_error - 1U] = '\0';
}

template <class F> int guarded(F&& body) {
    try {
        body();
        return 0;
    } catch (const std::exception& e) {
        set_error(e.what());
        return 1;
    } catch (...) {
        set_error("unknown exception");
        return 2;
    }
}

template <class Solver> void apply_init(Solver& s, int kind, const float* p) {
    if (kind == 0)
        s.initialize_uniform(p[0], p[1], p[2], p[3]);
    else
        s.initialize_taylor_green(p[0]);
}

template <class D>
void esoteric_run(std::size_t nx, std::size_t ny, std::size_t nz, float tau, float ax, float ay, float az, int les,
                  int init_kind, const float* init_p, const std::uint8_t* mask, const float* local_a,
                  std::size_t steps, float* rho, float* ux, float* uy, float* uz, float* logical, double* out) {
    cfd::lbm::InPlaceLbmConfig cfg{nx, ny, nz, tau, ax, ay, az};
    cfg.smagorinsky_les = les != 0;
    cfd::lbm::EsotericPullSolver<D> solver(cfg);
    const std::size_t n = solver.cells();
    if (mask) solver.set_solid_mask(std::span<const std::uint8_t>(mask, n));
    if (local_a)
        solver.set_local_body_acceleration(std::span<const float>(local_a, n), std::span<const float>(local_a + n, n),
                                           std::span<const float>(local_a + 2 * n, n));
    apply_init(solver, init_kind, init_p);
    solver.step(steps);
    const auto m = solver.compute_macroscopic();
    std::memcpy(rho, m.rho.data(), n * sizeof(float));
    std::memcpy(ux, m.ux.data(), n * sizeof(float));
    std::memcpy(uy, m.uy.data(), n * sizeof(float));
    std::memcpy(uz, m.uz.data(), n * sizeof(float));
    if (logical) {
        const auto pops = solver.logical_populations();
        std::memcpy(logical, pops.data(), pops.size() * sizeof(float));
    }
    out[0] = solver.mass();
    out[1] = solver.kinetic_energy();
    out[2] = static_cast<double>(solver.max_speed());
}

template <class D>
void twogrid_run(std::size_t nx, std::size_t ny, std::size_t nz, float tau, float odd_tau, float ax, float ay, float az,
                 int init_kind, const float* init_p, std::size_t steps, float* rho, float* ux, float* uy, float* uz,
                 double* mass) {
    cfd::lbm::InPlaceLbmConfig cfg{nx, ny, nz, tau, ax, ay, az};
    cfd::lbm::OneStepPullSolver<D> solver(cfg, odd_tau);
    apply_init(solver, init_kind, init_p);
    solver.step(steps);
    const auto m = solver.compute_macroscopic();
    const std::size_t n = solver.cells();
    std::memcpy(rho, m.rho.data(), n * sizeof(float));
    std::memcpy(ux, m.ux.data(), n * sizeof(float));
    std::memcpy(uy, m.uy.data(), n * sizeof(float));
    std::memcpy(uz, m.uz.data(), n * sizeof(float));
    *mass = solver.mass();
}

template <class D>
void precision_run(std::size_t nx, std::size_t ny, std::size_t nz, double tau, int init_kind, const double* init_p,
                   std::size_t steps, double* rho, double* ux, double* uy, double* uz, double* mass) {
    cfd::lbm::PrecisionPullSolver<D, double> solver(cfd::lbm::TypedLbmConfig<double>{nx, ny, nz, tau});
    if (init_kind == 0)
        solver.initialize_uniform(init_p[0], init_p[1], init_p[2], init_p[3]);
    else
        solver.initialize_taylor_green(init_p[0]);
    solver.step(steps);
    const auto m = solver.compute_macroscopic();
    const std::size_t n = nx * ny * nz;
    std::memcpy(rho, m.rho.data(), n * sizeof(double));
    std::memcpy(ux, m.ux.data(), n * sizeof(double));
    std::memcpy(uy, m.uy.data(), n * sizeof(double));
    std::memcpy(uz, m.uz.data(), n * sizeof(double));
    *mass = static_cast<double>(solver.mass());
}

template <class D>
void compressed_run(std::size_t nx, std::size_t ny, std::size_t nz, float tau, int init_kind, const float* init_p,
                    std::size_t steps, float* rho, float* ux, float* uy, float* uz, double* mass) {
    using Solver = cfd::lbm::CompressedPopulationPullSolver<D, cfd::lbm::ShiftedHalfCodec<D>>;
    Solver solver(typename Solver::Config{nx, ny, nz, tau});
    apply_init(solver, init_kind, init_p);
    solver.step(steps);
    const auto m = solver.compute_macroscopic();
    const std::size_t n = nx * ny * nz;
    std::memcpy(rho, m.rho.data(), n * sizeof(float));
    std::memcpy(ux, m.ux.data(), n * sizeof(float));
    std::memcpy(uy, m.uy.data(), n * sizeof(float));
    std::memcpy(uz, m.uz.data(), n * sizeof(float));
    *mass = solver.mass();
}

// Times solver.step(steps) after solver.step(warmup), the way apps/cfd-bench.cpp:173-191 does.
template <class D>
double bench_run(std::size_t nx, std::size_t ny, std::size_t nz, float tau, int les, const std::uint8_t* mask,
                 std::size_t warmup, std::size_t steps, unsigned threads, double* seconds, double* mass_rel) {
    if (threads > 0U) cfd::core::set_cpu_threads(threads);
    cfd::lbm::InPlaceLbmConfig cfg{nx, ny, nz, tau};
    cfg.smagorinsky_les = les != 0;
    cfd::lbm::EsotericPullSolver<D> solver(cfg);
    if (mask) solver.set_solid_mask(std::span<const std::uint8_t>(mask, solver.cells()));
    solver.initialize_uniform();
    const double mass0 = solver.mass();
    solver.step(warmup);
    const auto begin = std::chrono::steady_clock::now();
    solver.step(steps);
    const auto end = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(end - begin).count();
    *mass_rel = std::abs(solver.mass() - mass0) / mass0;
    return static_cast<double>(solver.cells()) * static_cast<double>(steps) / *seconds / 1.0e6;
}

} // namespace

extern "C" {

const char* ref_last_error(void) { return g_error; }

unsigned ref_thread_capacity(void) { return cfd::core::cpu_thread_capacity(); }

int ref_esoteric_run(int q, std::size_t nx, std::size_t ny, std::size_t nz, float tau, float ax, float ay, float az,
                     int les, int init_kind, const float* init_p, const std::uint8_t* mask, const float* local_a,
                     std::size_t steps, float* rho, float* ux, float* uy, float* uz, float* logical, double* out) {
    return guarded([&] {
        if (q == 19)
            esoteric_run<cfd::lbm::D3Q19Descriptor>(nx, ny, nz, tau, ax, ay, az, les, init_kind, init_p, mask,
                                                    local_a, steps, rho, ux, uy, uz, logical, out);
        else if (q == 27)
            esoteric_run<cfd::lbm::D3Q27Descriptor>(nx, ny, nz, tau, ax, ay, az, les, init_kind, init_p, mask,
                                                    local_a, steps, rho, ux, uy, uz, logical, out);
        else
            throw std::invalid_argument("q must be 19 or 27");
    });
}

int ref_twogrid_run(int q, std::size_t nx, std::size_t ny, std::size_t nz, float tau, float odd_tau, float ax,
                    float ay, float az, int init_kind, const float* init_p, std::size_t steps, float* rho, float* ux,
                    float* uy, float* uz, double* mass) {
    return guarded([&] {
        if (q == 19)
            twogrid_run<cfd::lbm::D3Q19Descriptor>(nx, ny, nz, tau, odd_tau, ax, ay, az, init_kind, init_p, steps, rho,
                                                   ux, uy, uz, mass);
        else if (q == 27)
            twogrid_run<cfd::lbm::D3Q27Descriptor>(nx, ny, nz, tau, odd_tau, ax, ay, az, init_kind, init_p, steps, rho,
                                                   ux, uy, uz, mass);
        else
            throw std::invalid_argument("q must be 19 or 27");
    });
}

int ref_precision_run(int q, std::size_t nx, std::size_t ny, std::size_t nz, double tau, int init_kind,
                      const double* init_p, std::size_t steps, double* rho, double* ux, double* uy, double* uz,
                      double* mass) {
    return guarded([&] {
        if (q == 19)
            precision_run<cfd::lbm::D3Q19Descriptor>(nx, ny, nz, tau, init_kind, init_p, steps, rho, ux, uy, uz, mass);
        else if (q == 27)
            precision_run<cfd::lbm::D3Q27Descriptor>(nx, ny, nz, tau, init_kind, init_p, steps, rho, ux, uy, uz, mass);
        else
            throw std::invalid_argument("q must be 19 or 27");
    });
}

int ref_compressed_run(int q, std::size_t nx, std::size_t ny, std::size_t nz, float tau, int init_kind,
                       const float* init_p, std::size_t steps, float* rho, float* ux, float* uy, float* uz,
                       double* mass) {
    return guarded([&] {
        if (q == 19)
            compressed_run<cfd::lbm::D3Q19Descriptor>(nx, ny, nz, tau, init_kind, init_p, steps, rho, ux, uy, uz, mass);
        else if (q == 27)
            compressed_run<cfd::lbm::D3Q27Descriptor>(nx, ny, nz, tau, init_kind, init_p, steps, rho, ux, uy, uz, mass);
        else
            throw std::invalid_argument("q must be 19 or 27");
    });
}

// The reference's triangle-surface voxelizer (src/lbm/voxelize.cpp):
// triangles are 9 doubles each (a, b, c), the grid spans [lo, hi].
int ref_voxelize(const double* tris, std::size_t count, std::size_t nx, std::size_t ny, std::size_t nz,
                 const double* lo, const double* hi, std::uint8_t* mask) {
    return guarded([&] {
        cfd::io::TriangleSurface s;
        for (std::size_t t = 0; t < count; ++t) {
            const double* v = tris + 9 * t;
            s.triangles.push_back({{v[0], v[1], v[2]}, {v[3], v[4], v[5]}, {v[6], v[7], v[8]}});
        }
        const cfd::lbm::VoxelGrid3D g{nx, ny, nz, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
        const auto m = cfd::lbm::voxelize_surface(s, g);
        std::memcpy(mask, m.data(), m.size());
    });
}

// The reference's rigid transform of a surface (rotation about `axis` by `angle`, then translation).
int ref_transform_surface(const double* tris, std::size_t count, const double* translation, const double* axis,
                          double angle, double* out) {
    return guarded([&] {
        cfd::io::TriangleSurface s;
        for (std::size_t t = 0; t < count; ++t) {
            const double* v = tris + 9 * t;
            s.triangles.push_back({{v[0], v[1], v[2]}, {v[3], v[4], v[5]}, {v[6], v[7], v[8]}});
        }
        const auto r = cfd::lbm::transform_surface(s, {translation[0], translation[1], translation[2]},
                                                   {axis[0], axis[1], axis[2]}, angle);
        for (std::size_t t = 0; t < count; ++t) {
            const auto& q = r.triangles[t];
            const double v[9] = {q.a.x, q.a.y, q.a.z, q.b.x, q.b.y, q.b.z, q.c.x, q.c.y, q.c.z};
            std::memcpy(out + 9 * t, v, sizeof v);
        }
    });
}

// The reference's field writers and Q-criterion (src/lbm/visualization.cpp:39-148);
// velocity is 3 doubles per cell (x, y, z), solid may be null.
int ref_write_vtk_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, const double* scalar,
                     const double* velocity, const std::uint8_t* solid, const char* name) {
    return guarded([&] {
        const std::size_t n = nx * ny * nz;
        std::vector<cfd::lbm::Vector3> u;
        if (velocity)
            for (std::size_t i = 0; i < n; ++i) u.push_back({velocity[3 * i], velocity[3 * i + 1], velocity[3 * i + 2]});
        cfd::lbm::write_vtk_structured_3d(path, nx, ny, nz, std::span<const double>(scalar, n), u,
                                          solid ? std::span<const std::uint8_t>(solid, n)
                                                : std::span<const std::uint8_t>(),
                                          name);
    });
}

int ref_write_json_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, std::uint64_t step,
                      const double* scalar, const std::uint8_t* solid, const char* name) {
    return guarded([&] {
        const std::size_t n = nx * ny * nz;
        cfd::lbm::write_json_state_3d(path, nx, ny, nz, step, std::span<const double>(scalar, n),
                                      solid ? std::span<const std::uint8_t>(solid, n)
                                            : std::span<const std::uint8_t>(),
                                      name);
    });
}

int ref_q_criterion(std::size_t nx, std::size_t ny, std::size_t nz, const double* velocity, double dx, double dy,
                    double dz, double* q) {
    return guarded([&] {
        const std::size_t n = nx * ny * nz;
        std::vector<cfd::lbm::Vector3> u;
        for (std::size_t i = 0; i < n; ++i) u.push_back({velocity[3 * i], velocity[3 * i + 1], velocity[3 * i + 2]});
        const auto r = cfd::lbm::q_criterion_3d(nx, ny, nz, u, dx, dy, dz);
        std::memcpy(q, r.data(), n * sizeof(double));
    });
}

// advect_free_surface_vof `steps` times (eps 0) on fill (N doubles, in place), then the
// normals (3N, xyz interleaved), curvature (N) and surface-tension acceleration (3N) of the result.
int ref_free_surface(std::size_t nx, std::size_t ny, std::size_t nz, double* fill, const float* ux, const float* uy,
                     const float* uz, double dt, std::size_t steps, double sigma, double density, double* normals,
                     double* curvature, double* tension, double* volume) {
    return guarded([&] {
        const std::size_t n = nx * ny * nz;
        auto s = cfd::lbm::make_free_surface_field(nx, ny, nz, std::span<const double>(fill, n), 0.0);
        for (std::size_t k = 0; k < steps; ++k)
            cfd::lbm::advect_free_surface_vof(s, std::span<const float>(ux, n), std::span<const float>(uy, n),
                                              std::span<const float>(uz, n), dt, 0.0);
        std::memcpy(fill, s.fill.data(), n * sizeof(double));
        const auto nrm = cfd::lbm::free_surface_normals(s);
        const auto k = cfd::lbm::free_surface_curvature(s);
        const auto a = cfd::lbm::free_surface_surface_tension_acceleration(s, sigma, density);
        for (std::size_t i = 0; i < n; ++i) {
            normals[3 * i] = nrm[i].x;
            normals[3 * i + 1] = nrm[i].y;
            normals[3 * i + 2] = nrm[i].z;
            tension[3 * i] = a[i].x;
            tension[3 * i + 1] = a[i].y;
            tension[3 * i + 2] = a[i].z;
        }
        std::memcpy(curvature, k.data(), n * sizeof(double));
        *volume = cfd::lbm::free_surface_volume(s);
    });
}

// advance_immersed_boundary_particles once: records = count x 8 doubles (position, velocity, mass,
// response time; updated in place); with two_way, acceleration = 3N floats (x | y | z planes).
int ref_particles(std::size_t nx, std::size_t ny, std::size_t nz, const float* ux, const float* uy, const float* uz,
                  double* records, std::size_t count, double dt, int two_way, double gx, double gy, double gz,
                  float* acceleration) {
    return guarded([&] {
        const std::size_t n = nx * ny * nz;
        std::vector<cfd::lbm::ImmersedBoundaryParticle> ps(count);
        for (std::size_t i = 0; i < count; ++i) {
            const double* r = records + 8 * i;
            ps[i] = {{r[0], r[1], r[2]}, {r[3], r[4], r[5]}, r[6], r[7]};
        }
        const auto out = cfd::lbm::advance_immersed_boundary_particles(
            nx, ny, nz, std::span<const float>(ux, n), std::span<const float>(uy, n), std::span<const float>(uz, n),
            ps, dt, two_way != 0, {gx, gy, gz});
        for (std::size_t i = 0; i < count; ++i) {
            double* r = records + 8 * i;
            const auto& p = ps[i];
            const double v[8] = {p.position.x, p.position.y, p.position.z, p.velocity.x,
                                 p.velocity.y, p.velocity.z, p.mass,       p.response_time};
            std::memcpy(r, v, sizeof(v));
        }
        if (two_way) {
            std::memcpy(acceleration, out.acceleration_x.data(), n * sizeof(float));
            std::memcpy(acceleration + n, out.acceleration_y.data(), n * sizeof(float));
            std::memcpy(acceleration + 2 * n, out.acceleration_z.data(), n * sizeof(float));
        }
    });
}

// Returns MLUPS of the reference in-place CPU path (negative on error).
double ref_bench(int q, std::size_t nx, std::size_t ny, std::size_t nz, float tau, int les, const std::uint8_t* mask,
                 std::size_t warmup, std::size_t steps, unsigned threads, double* seconds, double* mass_rel) {
    double mlups = -1.0;
    const int rc = guarded([&] {
        if (q == 19)
            mlups = bench_run<cfd::lbm::D3Q19Descriptor>(nx, ny, nz, tau, les, mask, warmup, steps, threads, seconds,
                                                         mass_rel);
        else if (q == 27)
            mlups = bench_run<cfd::lbm::D3Q27Descriptor>(nx, ny, nz, tau, les, mask, warmup, steps, threads, seconds,
                                                         mass_rel);
        else
            throw std::invalid_argument("q must be 19 or 27");
    });
    return rc == 0 ? mlups : -1.0;
}

} // extern "C"
