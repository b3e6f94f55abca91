// C++20 front end of the resident solvers coupled to an EsotericPullCudaSolver
// through its device views: the reference's ResidentThermalD3Q7Sycl,
// ResidentFreeSurfaceSycl3D, ResidentParticlesSycl3D and
// ResidentFlowDiagnosticsSycl3D (include/cfd/solvers/lbm/resident_multiphysics_sycl.hpp:51-405)
// with the same method names, arguments and exceptions.  Where the reference
// takes the flow's sycl::queue, these take the flow solver itself: they run on
// its device and CUDA stream.  Each must be destroyed before its flow solver.
#pragma once

#include <cstddef>
#include <cstdint>
#include <span>
#include <stdexcept>
#include <utility>
#include <vector>

#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"

namespace cfd::lbm {

namespace cuda {

// The reference's ResidentThermalConfig (resident_multiphysics_sycl.hpp:51-54).
struct ResidentThermalConfig {
    std::size_t nx{64U}, ny{64U}, nz{64U};
    float diffusivity{0.01F};
};

// The reference's ParticleVector3 / ImmersedBoundaryParticle (particles.hpp:9-18).
struct ParticleVector3 {
    double x{}, y{}, z{};
};
struct ImmersedBoundaryParticle {
    ParticleVector3 position{};
    ParticleVector3 velocity{};
    double mass{1.0};
    double response_time{1.0};
};

template <class Flow> void require_grid(const Flow& flow, std::size_t nx, std::size_t ny, std::size_t nz,
                                        const char* what) {
    const auto& c = flow.config();
    if (c.nx != nx || c.ny != ny || c.nz != nz) throw std::invalid_argument(what);
}

} // namespace cuda

class ResidentThermalD3Q7Cuda {
public:
    template <class Flow, class Config = cuda::ResidentThermalConfig>
    ResidentThermalD3Q7Cuda(Flow& flow, const Config& config) {
        cuda::require_grid(flow, config.nx, config.ny, config.nz, "invalid resident thermal lattice");
        char error[1024] = {0};
        cuda::check(cfdx_thermal_create(flow.native_handle(), config.diffusivity, &h_, error, sizeof error),
                    "ResidentThermalD3Q7Cuda");
    }
    ~ResidentThermalD3Q7Cuda() {
        if (h_) cfdx_thermal_destroy(h_);
    }
    ResidentThermalD3Q7Cuda(const ResidentThermalD3Q7Cuda&) = delete;
    ResidentThermalD3Q7Cuda& operator=(const ResidentThermalD3Q7Cuda&) = delete;

    void initialize_uniform(float temperature) {
        cuda::check(cfdx_thermal_init_uniform(h_, temperature), "initialize_uniform");
    }
    template <class View> void step(const View& flow, std::size_t count = 1U) {
        cuda::check(cfdx_thermal_step(h_, flow.ux, flow.uy, flow.uz, count), "step");
    }
    [[nodiscard]] float* refresh_device_scalar() {
        float* t = nullptr;
        cuda::check(cfdx_thermal_refresh_device_scalar(h_, &t), "refresh_device_scalar");
        return t;
    }
    template <class View, class Vector>
    void add_boussinesq_acceleration(View force, float reference_temperature, float beta, Vector gravity) {
        cuda::check(cfdx_thermal_add_boussinesq(h_, force.ax, force.ay, force.az, reference_temperature, beta,
                                                static_cast<float>(gravity.x), static_cast<float>(gravity.y),
                                                static_cast<float>(gravity.z)),
                    "add_boussinesq_acceleration");
    }
    [[nodiscard]] double total_scalar() const {
        double t = 0.0;
        cuda::check(cfdx_thermal_total(h_, &t), "total_scalar");
        return t;
    }
    [[nodiscard]] std::size_t resident_bytes() const { return info().first; }
    [[nodiscard]] cuda::TransferStats transfer_stats() const {
        cuda::TransferStats s = info().second;
        s.host_to_device_bytes -= base_.host_to_device_bytes;
        s.device_to_host_bytes -= base_.device_to_host_bytes;
        return s;
    }
    void reset_transfer_stats() { base_ = info().second; }

private:
    [[nodiscard]] std::pair<std::size_t, cuda::TransferStats> info() const {
        std::size_t r = 0;
        cuda::TransferStats s;
        cuda::check(cfdx_thermal_info(h_, &r, &s.host_to_device_bytes, &s.device_to_host_bytes), "transfer_stats");
        return {r, s};
    }
    cfdx_thermal* h_{nullptr};
    cuda::TransferStats base_{};
};

class ResidentFreeSurfaceCuda3D {
public:
    template <class Flow> ResidentFreeSurfaceCuda3D(Flow& flow, std::size_t nx, std::size_t ny, std::size_t nz) {
        cuda::require_grid(flow, nx, ny, nz, "invalid resident free-surface lattice");
        char error[1024] = {0};
        cuda::check(cfdx_surface_create(flow.native_handle(), &h_, error, sizeof error), "ResidentFreeSurfaceCuda3D");
        cells_ = nx * ny * nz;
    }
    ~ResidentFreeSurfaceCuda3D() {
        if (h_) cfdx_surface_destroy(h_);
    }
    ResidentFreeSurfaceCuda3D(const ResidentFreeSurfaceCuda3D&) = delete;
    ResidentFreeSurfaceCuda3D& operator=(const ResidentFreeSurfaceCuda3D&) = delete;

    void initialize_uniform(float fill) { cuda::check(cfdx_surface_init_uniform(h_, fill), "initialize_uniform"); }
    void initialize_half_space_x(float interface_x) {
        cuda::check(cfdx_surface_init_half_space_x(h_, interface_x), "initialize_half_space_x");
    }
    template <class View> void advect(const View& flow, float dt) {
        if (flow.cells != cells_) throw std::invalid_argument("invalid resident free-surface advection");
        cuda::check(cfdx_surface_advect(h_, flow.ux, flow.uy, flow.uz, dt), "advect");
    }
    [[nodiscard]] float* fill_device() {
        float* f = nullptr;
        cuda::check(cfdx_surface_device_fill(h_, &f), "fill_device");
        return f;
    }
    // device [normal x | y | z | curvature], 4 * cells floats
    float* refresh_geometry() {
        float* g = nullptr;
        cuda::check(cfdx_surface_refresh_geometry(h_, &g), "refresh_geometry");
        return g;
    }
    template <class View> void add_surface_tension_acceleration(View force, float surface_tension, float density = 1.0F) {
        if (force.cells != cells_) throw std::invalid_argument("invalid resident surface-tension coupling");
        cuda::check(cfdx_surface_add_tension(h_, force.ax, force.ay, force.az, surface_tension, density),
                    "add_surface_tension_acceleration");
    }
    [[nodiscard]] double volume() const {
        double v = 0.0;
        cuda::check(cfdx_surface_volume(h_, &v), "volume");
        return v;
    }
    [[nodiscard]] std::vector<float> fill() const {
        std::vector<float> out(cells_);
        cuda::check(cfdx_surface_fill(h_, out.data(), 0, CFDX_HOST), "fill");
        return out;
    }
    [[nodiscard]] std::size_t resident_bytes() const {
        std::size_t r = 0;
        std::uint64_t a = 0, b = 0;
        cuda::check(cfdx_surface_info(h_, &r, &a, &b), "resident_bytes");
        return r;
    }

private:
    cfdx_surface* h_{nullptr};
    std::size_t cells_{0};
};

class ResidentParticlesCuda3D {
public:
    template <class Flow>
    ResidentParticlesCuda3D(Flow& flow, std::size_t nx, std::size_t ny, std::size_t nz, std::size_t count)
        : count_(count), cells_(nx * ny * nz) {
        cuda::require_grid(flow, nx, ny, nz, "invalid resident particle lattice");
        char error[1024] = {0};
        cuda::check(cfdx_particles_create(flow.native_handle(), count, &h_, error, sizeof error),
                    "ResidentParticlesCuda3D");
    }
    ~ResidentParticlesCuda3D() {
        if (h_) cfdx_particles_destroy(h_);
    }
    ResidentParticlesCuda3D(const ResidentParticlesCuda3D&) = delete;
    ResidentParticlesCuda3D& operator=(const ResidentParticlesCuda3D&) = delete;

    // P: any type with .position / .velocity (.x .y .z), .mass, .response_time
    // (the reference's ImmersedBoundaryParticle).
    template <class P> void upload(std::span<const P> particles) {
        std::vector<double> rec;
        rec.reserve(8U * particles.size());
        for (const P& p : particles)
            for (double v : {double(p.position.x), double(p.position.y), double(p.position.z), double(p.velocity.x),
                             double(p.velocity.y), double(p.velocity.z), double(p.mass), double(p.response_time)})
                rec.push_back(v);
        cuda::check(cfdx_particles_upload(h_, rec.data(), particles.size()), "upload");
    }
    template <class P = cuda::ImmersedBoundaryParticle> [[nodiscard]] std::vector<P> download() const {
        std::vector<double> rec(8U * count_);
        cuda::check(cfdx_particles_download(h_, rec.data(), count_), "download");
        std::vector<P> out(count_);
        for (std::size_t i = 0; i < count_; ++i) {
            const double* r = rec.data() + 8U * i;
            out[i].position = {r[0], r[1], r[2]};
            out[i].velocity = {r[3], r[4], r[5]};
            out[i].mass = r[6];
            out[i].response_time = r[7];
        }
        return out;
    }
    template <class View, class Force, class Vector = cuda::ParticleVector3>
    void advance(const View& flow, Force force, float dt, bool two_way, Vector gravity = {}) {
        if (flow.cells != cells_ || force.cells != flow.cells)
            throw std::invalid_argument("invalid resident particle coupling");
        cuda::check(cfdx_particles_advance(h_, flow.ux, flow.uy, flow.uz, force.ax, force.ay, force.az, dt,
                                           two_way ? 1 : 0, static_cast<float>(gravity.x),
                                           static_cast<float>(gravity.y), static_cast<float>(gravity.z)),
                    "advance");
    }
    [[nodiscard]] std::size_t resident_bytes() const { return info().first; }
    [[nodiscard]] std::size_t size() const noexcept { return count_; }
    [[nodiscard]] cuda::TransferStats transfer_stats() const {
        cuda::TransferStats s = info().second;
        s.host_to_device_bytes -= base_.host_to_device_bytes;
        s.device_to_host_bytes -= base_.device_to_host_bytes;
        return s;
    }
    void reset_transfer_stats() { base_ = info().second; }

private:
    [[nodiscard]] std::pair<std::size_t, cuda::TransferStats> info() const {
        std::size_t r = 0;
        cuda::TransferStats s;
        cuda::check(cfdx_particles_info(h_, &r, &s.host_to_device_bytes, &s.device_to_host_bytes), "transfer_stats");
        return {r, s};
    }
    cfdx_particles* h_{nullptr};
    std::size_t count_{0}, cells_{0};
    cuda::TransferStats base_{};
};

class ResidentFlowDiagnosticsCuda3D {
public:
    template <class Flow>
    ResidentFlowDiagnosticsCuda3D(Flow& flow, std::size_t nx, std::size_t ny, std::size_t nz) : cells_(nx * ny * nz) {
        cuda::require_grid(flow, nx, ny, nz, "diagnostic/flow lattice size mismatch");
        char error[1024] = {0};
        cuda::check(cfdx_diagnostics_create(flow.native_handle(), &h_, error, sizeof error),
                    "ResidentFlowDiagnosticsCuda3D");
    }
    ~ResidentFlowDiagnosticsCuda3D() {
        if (h_) cfdx_diagnostics_destroy(h_);
    }
    ResidentFlowDiagnosticsCuda3D(const ResidentFlowDiagnosticsCuda3D&) = delete;
    ResidentFlowDiagnosticsCuda3D& operator=(const ResidentFlowDiagnosticsCuda3D&) = delete;

    // device Q field (cells floats, owned here, overwritten by the next call)
    template <class View> [[nodiscard]] float* q_criterion(const View& flow) {
        if (flow.cells != cells_) throw std::invalid_argument("diagnostic/flow lattice size mismatch");
        float* q = nullptr;
        cuda::check(cfdx_diagnostics_q_criterion(h_, flow.ux, flow.uy, flow.uz, &q), "q_criterion");
        return q;
    }
    [[nodiscard]] std::size_t resident_bytes() const noexcept { return cells_ * sizeof(float); }

private:
    cfdx_diagnostics* h_{nullptr};
    std::size_t cells_{0};
};

} // namespace cfd::lbm
