// C++20 front end of the B200 in-place Esoteric-Pull engine.
//
// cfd::lbm::EsotericPullCudaSolver<Descriptor> has the interface of the
// reference's CPU solver cfd::lbm::EsotericPullSolver<Descriptor>
// (include/cfd/solvers/lbm/esoteric_pull.hpp:104-515) and of its SYCL twin
// (esoteric_pull_sycl.hpp:18-475): same constructor argument, method names,
// argument meaning and exception types, so a driver switches by changing the
// class name.  Every call goes through the C ABI of libcfdx_lbm.so
// (include/cfdx_lbm.h); the step runs as sm_100a CUDA kernels, with no CPU
// fallback.
//
// Descriptor: any type with `static constexpr int q` equal to 19 or 27 --
// the reference's D3Q19Descriptor / D3Q27Descriptor, or the tags
// cfd::lbm::cuda::D3Q19 / D3Q27 below when the reference headers are absent.
// Config: any type with the members of the reference's InPlaceLbmConfig
// (nx, ny, nz, tau, acceleration_x/y/z, smagorinsky_les), e.g.
// cfd::lbm::cuda::InPlaceLbmConfig, which adds the engine's extensions.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <new>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "cfdx_lbm.h"

namespace cfd::lbm {

namespace cuda {

struct D3Q19 {
    static constexpr int q = 19;
};
struct D3Q27 {
    static constexpr int q = 27;
};

enum class Collision { bgk = CFDX_BGK, trt = CFDX_TRT };
enum class Storage { fp32 = CFDX_STORE_F32, fp16s = CFDX_STORE_F16S, fp64 = CFDX_STORE_F64 };
enum class Fp16Rounding { nearest = CFDX_ROUND_NEAREST, stochastic = CFDX_ROUND_STOCHASTIC };

// The reference's InPlaceLbmConfig (esoteric_pull.hpp:20-29) plus the engine's extensions.
struct InPlaceLbmConfig {
    std::size_t nx{128};
    std::size_t ny{128};
    std::size_t nz{128};
    float tau{0.6F};
    float acceleration_x{0.0F};
    float acceleration_y{0.0F};
    float acceleration_z{0.0F};
    bool smagorinsky_les{false};
    // extensions
    Collision collision{Collision::bgk};
    Storage storage{Storage::fp32};
    float smagorinsky_cs{0.0F}; // <= 0: the reference's fixed coefficient
    float trt_magic{3.0F / 16.0F};
    float trt_tau_minus{0.0F}; // > 0: fixed antisymmetric relaxation time
    int device{0};
    Fp16Rounding fp16_rounding{Fp16Rounding::stochastic};
    std::uint32_t rounding_seed{0};
};

// rho and u + a/2 per cell (reference MacroscopicFields, esoteric_pull.hpp:31-36).
struct MacroscopicFields {
    std::vector<float> rho;
    std::vector<float> ux;
    std::vector<float> uy;
    std::vector<float> uz;
};

// Host-transfer counters (reference cfd::core::DeviceTransferStats, core/device_residency.hpp:11-42).
struct TransferStats {
    std::uint64_t host_to_device_bytes{0};
    std::uint64_t device_to_host_bytes{0};
    [[nodiscard]] std::uint64_t host_transfer_bytes() const noexcept {
        return host_to_device_bytes + device_to_host_bytes;
    }
};

// Converts a C ABI status into the reference's exception types.
inline void check(int status, const char* what) {
    if (status == CFDX_OK) return;
    char buffer[1024] = {0};
    cfdx_last_error(buffer, sizeof buffer);
    const std::string message = std::string(what) + ": " + buffer;
    switch (status) {
    case CFDX_ERR_INVALID: throw std::invalid_argument(message);
    case CFDX_ERR_RANGE: throw std::out_of_range(message);
    case CFDX_ERR_OOM: throw std::bad_alloc();
    default: throw std::runtime_error(message);
    }
}

// 9 doubles (a, b, c) per triangle of any surface whose .triangles hold .a .b .c points.
template <class Surface> std::vector<double> pack_triangles(const Surface& surface) {
    std::vector<double> out;
    out.reserve(9 * surface.triangles.size());
    for (const auto& t : surface.triangles)
        for (const auto* p : {&t.a, &t.b, &t.c}) {
            out.push_back(p->x);
            out.push_back(p->y);
            out.push_back(p->z);
        }
    return out;
}

template <class C, class = void> struct has_extensions : std::false_type {};
template <class C> struct has_extensions<C, std::void_t<decltype(std::declval<C>().storage)>> : std::true_type {};

} // namespace cuda

template <class Descriptor> class EsotericPullCudaSolver {
public:
    static constexpr int q = Descriptor::q;
    static constexpr std::size_t pair_count = static_cast<std::size_t>((q - 1) / 2);
    static_assert(q == 19 || q == 27, "the B200 engine implements D3Q19 and D3Q27");

    template <class Config = cuda::InPlaceLbmConfig>
    explicit EsotericPullCudaSolver(const Config& config = Config{}) {
        const cfdx_lbm_config c = native_config(config);
        char error[1024] = {0};
        const int status = cfdx_lbm_create(&c, &handle_, error, sizeof error);
        if (status != CFDX_OK) {
            handle_ = nullptr;
            cuda::check(status, "cfdx_lbm_create");
        }
        config_ = c;
        cells_ = c.nx * c.ny * c.nz;
    }

protected:
    // A z-slab [z_begin, z_begin + z_extent) of the lattice `config` describes
    // (EsotericPullCudaSlab): nx*ny*(z_extent + 2) local cells.
    template <class Config>
    EsotericPullCudaSolver(const Config& config, std::uint32_t z_begin, std::uint32_t z_extent) {
        const cfdx_lbm_config c = native_config(config);
        char error[1024] = {0};
        const int status = cfdx_lbm_create_slab(&c, z_begin, z_extent, &handle_, error, sizeof error);
        if (status != CFDX_OK) {
            handle_ = nullptr;
            cuda::check(status, "cfdx_lbm_create_slab");
        }
        config_ = c;
        cells_ = c.nx * c.ny * (static_cast<std::size_t>(z_extent) + 2U);
    }

    template <class Config> static cfdx_lbm_config native_config(const Config& config) {
        cfdx_lbm_config c;
        cuda::check(cfdx_lbm_config_default(&c), "cfdx_lbm_config_default");
        c.nx = config.nx;
        c.ny = config.ny;
        c.nz = config.nz;
        c.tau = config.tau;
        c.acceleration_x = config.acceleration_x;
        c.acceleration_y = config.acceleration_y;
        c.acceleration_z = config.acceleration_z;
        c.smagorinsky_les = config.smagorinsky_les ? 1 : 0;
        c.lattice = q;
        if constexpr (cuda::has_extensions<Config>::value) {
            c.collision = static_cast<int>(config.collision);
            c.storage = static_cast<int>(config.storage);
            c.smagorinsky_cs = config.smagorinsky_cs;
            c.trt_magic = config.trt_magic;
            c.trt_tau_minus = config.trt_tau_minus;
            c.device = config.device;
            c.fp16_rounding = static_cast<int>(config.fp16_rounding);
            c.rounding_seed = config.rounding_seed;
        }
        return c;
    }

public:

    ~EsotericPullCudaSolver() {
        if (handle_) cfdx_lbm_destroy(handle_);
    }
    EsotericPullCudaSolver(const EsotericPullCudaSolver&) = delete;
    EsotericPullCudaSolver& operator=(const EsotericPullCudaSolver&) = delete;
    EsotericPullCudaSolver(EsotericPullCudaSolver&& other) noexcept
        : handle_(std::exchange(other.handle_, nullptr)), config_(other.config_), cells_(other.cells_),
          mask_(std::move(other.mask_)), local_(other.local_), transfer_base_(other.transfer_base_) {}

    // ------------------------------------------------ reference API (CPU class)
    void initialize_uniform(float rho = 1.0F, float ux = 0.0F, float uy = 0.0F, float uz = 0.0F) {
        cuda::check(cfdx_lbm_init_uniform(handle_, rho, ux, uy, uz), "initialize_uniform");
    }
    void initialize_taylor_green(float amplitude = 0.03F) {
        cuda::check(cfdx_lbm_init_taylor_green(handle_, amplitude), "initialize_taylor_green");
    }
    void step(std::size_t count = 1) { cuda::check(cfdx_lbm_step(handle_, count), "step"); }

    void set_local_body_acceleration(std::span<const float> ax, std::span<const float> ay, std::span<const float> az) {
        if (ax.size() != cells_ || ay.size() != cells_ || az.size() != cells_)
            throw std::invalid_argument("local body acceleration size mismatch");
        std::vector<float> packed;
        packed.reserve(3 * cells_);
        packed.insert(packed.end(), ax.begin(), ax.end());
        packed.insert(packed.end(), ay.begin(), ay.end());
        packed.insert(packed.end(), az.begin(), az.end());
        cuda::check(cfdx_lbm_set_local_acceleration(handle_, packed.data(), CFDX_HOST), "set_local_body_acceleration");
        local_ = true;
    }
    void clear_local_body_acceleration() noexcept {
        cfdx_lbm_set_local_acceleration(handle_, nullptr, CFDX_HOST);
        local_ = false;
    }
    [[nodiscard]] bool has_local_body_acceleration() const noexcept { return local_; }

    // mask != 0 => solid (stationary half-way bounce-back wall)
    void set_solid_mask(std::span<const std::uint8_t> mask) {
        if (mask.size() != cells_) throw std::invalid_argument("LBM solid mask size mismatch");
        std::vector<std::uint8_t> flags(mask.size());
        for (std::size_t n = 0; n < mask.size(); ++n) flags[n] = mask[n] != 0U ? 1U : 0U;
        cuda::check(cfdx_lbm_set_flags(handle_, flags.data(), CFDX_HOST), "set_solid_mask");
        mask_ = std::move(flags);
    }
    void clear_solid_mask() noexcept {
        cfdx_lbm_set_flags(handle_, nullptr, CFDX_HOST);
        mask_.clear();
    }
    [[nodiscard]] bool has_solid_mask() const noexcept { return !mask_.empty(); }
    [[nodiscard]] const std::vector<std::uint8_t>& solid_mask() const noexcept { return mask_; }

    [[nodiscard]] cuda::MacroscopicFields compute_macroscopic() const {
        cuda::MacroscopicFields f;
        f.rho.resize(cells_);
        f.ux.resize(cells_);
        f.uy.resize(cells_);
        f.uz.resize(cells_);
        cuda::check(cfdx_lbm_macroscopic(handle_, f.rho.data(), f.ux.data(), f.uy.data(), f.uz.data(), CFDX_HOST),
                    "compute_macroscopic");
        return f;
    }
    [[nodiscard]] double mass() const { return reduce()[0]; }
    [[nodiscard]] double kinetic_energy() const { return reduce()[4]; }
    [[nodiscard]] float max_speed() const { return static_cast<float>(reduce()[5]); }
    [[nodiscard]] std::vector<float> logical_populations() const {
        std::vector<float> out(static_cast<std::size_t>(q) * cells_);
        cuda::check(cfdx_lbm_logical_populations(handle_, out.data(), CFDX_HOST), "logical_populations");
        return out;
    }
    [[nodiscard]] const cfdx_lbm_config& config() const noexcept { return config_; }
    [[nodiscard]] std::size_t cells() const noexcept { return cells_; }
    [[nodiscard]] std::uint64_t time_step() const { return info().time_step; }
    [[nodiscard]] std::size_t population_bytes() const { return info().population_bytes; }
    [[nodiscard]] std::size_t two_lattice_population_bytes() const noexcept { return 2U * population_bytes(); }

    // ------------------------------------------------ reference API (SYCL class)
    void wait() { cuda::check(cfdx_lbm_synchronize(handle_), "wait"); }
    // Reference download_macroscopic (esoteric_pull_sycl.hpp:309-325): the device fields copied to the host.
    [[nodiscard]] cuda::MacroscopicFields download_macroscopic() const { return compute_macroscopic(); }
    [[nodiscard]] double total_mass() const { return mass(); }
    [[nodiscard]] std::size_t resident_bytes() const { return info().resident_bytes; }
    [[nodiscard]] std::string device_name() const { return "CUDA device " + std::to_string(config_.device); }

    // Bytes moved through the host since construction or reset_transfer_stats().
    [[nodiscard]] cuda::TransferStats transfer_stats() const {
        const cfdx_lbm_info i = info();
        return {i.host_to_device_bytes - transfer_base_.host_to_device_bytes,
                i.device_to_host_bytes - transfer_base_.device_to_host_bytes};
    }
    void reset_transfer_stats() {
        const cfdx_lbm_info i = info();
        transfer_base_ = {i.host_to_device_bytes, i.device_to_host_bytes};
    }

    // Device views for resident coupling (reference esoteric_pull_sycl.hpp:218-372):
    // the step's macroscopic fields and the per-cell acceleration it consumes.
    struct DeviceMacroscopicView {
        float* rho;
        float* ux;
        float* uy;
        float* uz;
        std::size_t cells;
    };
    struct DeviceAccelerationView {
        float* ax;
        float* ay;
        float* az;
        std::size_t cells;
    };
    // rho and u + a/2 of the current state in device memory owned by the solver.
    [[nodiscard]] DeviceMacroscopicView refresh_device_macroscopic() {
        DeviceMacroscopicView v{nullptr, nullptr, nullptr, nullptr, cells_};
        cuda::check(cfdx_lbm_refresh_device_macroscopic(handle_, &v.rho, &v.ux, &v.uy, &v.uz),
                    "refresh_device_macroscopic");
        return v;
    }
    // The per-cell acceleration the step reads (zeroed on the device with clear).
    [[nodiscard]] DeviceAccelerationView device_local_acceleration(bool clear = false) {
        float* a = nullptr;
        cuda::check(cfdx_lbm_device_local_acceleration(handle_, &a), "device_local_acceleration");
        if (clear) cuda::check(cfdx_lbm_clear_device_acceleration(handle_), "device_local_acceleration");
        local_ = true;
        return {a, a + cells_, a + 2U * cells_, cells_};
    }

    // ------------------------------------------------------------ extensions
    // Cell flags: 0 fluid, 1 wall, 2..15 moving wall (velocity from set_wall_velocity).
    void set_flags(std::span<const std::uint8_t> flags) {
        if (flags.size() != cells_) throw std::invalid_argument("LBM flag field size mismatch");
        cuda::check(cfdx_lbm_set_flags(handle_, flags.data(), CFDX_HOST), "set_flags");
        mask_.assign(flags.begin(), flags.end());
    }
    void set_wall_velocity(int wall_id, float ux, float uy, float uz) {
        cuda::check(cfdx_lbm_set_wall_velocity(handle_, wall_id, ux, uy, uz), "set_wall_velocity");
    }
    void set_solid_fraction(std::span<const float> ns) {
        if (ns.size() != cells_) throw std::invalid_argument("solid fraction size mismatch");
        cuda::check(cfdx_lbm_set_solid_fraction(handle_, ns.data(), CFDX_HOST), "set_solid_fraction");
    }
    // mass, momentum xyz, kinetic energy, max |u|, non-finite cells (FP64 sums)
    [[nodiscard]] std::vector<double> reduce() const {
        std::vector<double> out(CFDX_REDUCE_COUNT);
        cuda::check(cfdx_lbm_reduce(handle_, out.data()), "reduce");
        return out;
    }
    [[nodiscard]] double checksum() const {
        double c = 0.0;
        cuda::check(cfdx_lbm_checksum(handle_, &c), "checksum");
        return c;
    }
    void save_checkpoint(const std::string& path) const {
        cuda::check(cfdx_lbm_checkpoint_save(handle_, path.c_str()), "save_checkpoint");
    }
    void load_checkpoint(const std::string& path) {
        cuda::check(cfdx_lbm_checkpoint_load(handle_, path.c_str()), "load_checkpoint");
    }
    // Flags from a closed triangle surface voxelized on the device over the box
    // [minimum, maximum] (reference voxelize_surface + set_solid_mask,
    // examples/real_lbm3d_model.cpp:146-150): `solid_id` inside, the base flags
    // (or fluid) elsewhere.  Surface: any type whose .triangles hold .a .b .c
    // points with .x .y .z (the reference's cfd::io::TriangleSurface).
    template <class Surface, class Point>
    void set_solid_surface(const Surface& surface, const Point& minimum, const Point& maximum,
                           std::uint8_t solid_id = 1, std::span<const std::uint8_t> base_flags = {}) {
        const std::vector<double> tris = cuda::pack_triangles(surface);
        const double lo[3] = {minimum.x, minimum.y, minimum.z}, hi[3] = {maximum.x, maximum.y, maximum.z};
        if (!base_flags.empty() && base_flags.size() != cells_)
            throw std::invalid_argument("LBM flag field size mismatch");
        cuda::check(cfdx_lbm_set_flags_surface(handle_, tris.data(), tris.size() / 9, lo, hi, solid_id,
                                               base_flags.empty() ? nullptr : base_flags.data(), CFDX_HOST),
                    "set_solid_surface");
    }
    // Q-criterion of the current velocity, computed on the device (reference q_criterion_3d).
    [[nodiscard]] std::vector<double> q_criterion(double dx = 1.0, double dy = 1.0, double dz = 1.0) const {
        std::vector<double> q(cells_);
        cuda::check(cfdx_lbm_q_criterion(handle_, dx, dy, dz, q.data(), CFDX_HOST), "q_criterion");
        return q;
    }
    // Symmetric relaxation time for the following steps (the adjoint's dJ/dtau is taken with respect to it).
    void set_tau(float tau) {
        cuda::check(cfdx_lbm_set_tau(handle_, tau), "set_tau");
        config_.tau = tau;
    }

    // ------------------------------------------------ discrete adjoint (gray LBM)
    // `steps` steps from the current state keeping a checkpoint every `interval` steps;
    // `subinterval` 2 <= m < interval reverses each segment in two levels of recompute
    // (fewer frames held, about twice the recompute steps), 0 in one.
    void adjoint_forward(std::uint64_t steps, std::uint32_t interval, std::uint32_t subinterval = 0) {
        cuda::check(cfdx_lbm_adjoint_set_subinterval(handle_, subinterval), "adjoint_forward");
        cuda::check(cfdx_lbm_adjoint_forward(handle_, steps, interval), "adjoint_forward");
    }
    struct AdjointGradient {
        std::vector<double> solid_fraction; // dJ/dn_s per cell (0 on walls)
        double tau{0.0};                    // dJ/dtau
    };
    // Reverse sweep for J(final state) given dJ/du (and optionally dJ/drho) of the
    // fields compute_macroscopic reports (u includes +a/2).
    [[nodiscard]] AdjointGradient adjoint_backward(std::span<const float> g_ux, std::span<const float> g_uy,
                                                   std::span<const float> g_uz, std::span<const float> g_rho = {}) {
        if (g_ux.size() != cells_ || g_uy.size() != cells_ || g_uz.size() != cells_ ||
            (!g_rho.empty() && g_rho.size() != cells_))
            throw std::invalid_argument("adjoint seed size mismatch");
        AdjointGradient g;
        g.solid_fraction.resize(cells_);
        cuda::check(cfdx_lbm_adjoint_backward(handle_, g_rho.empty() ? nullptr : g_rho.data(), g_ux.data(),
                                              g_uy.data(), g_uz.data(), CFDX_HOST, g.solid_fraction.data(), CFDX_HOST,
                                              &g.tau),
                    "adjoint_backward");
        return g;
    }
    [[nodiscard]] std::size_t adjoint_memory() const {
        std::size_t b = 0;
        cuda::check(cfdx_lbm_adjoint_memory(handle_, &b), "adjoint_memory");
        return b;
    }
    void adjoint_release() { cuda::check(cfdx_lbm_adjoint_release(handle_), "adjoint_release"); }

    [[nodiscard]] cfdx_lbm* native_handle() const noexcept { return handle_; }

private:
    [[nodiscard]] cfdx_lbm_info info() const {
        cfdx_lbm_info i{};
        cuda::check(cfdx_lbm_get_info(handle_, &i), "get_info");
        return i;
    }

    cfdx_lbm* handle_{nullptr};
    cfdx_lbm_config config_{};
    std::size_t cells_{0};
    std::vector<std::uint8_t> mask_;
    bool local_{false};
    cuda::TransferStats transfer_base_{};
};

// One z-slab of a lattice cut along z (the reference's DistributedPullBlock
// brick, distributed_pull.hpp:35-60, cut along z only).  Per-cell arrays
// cover the local planes, ghost planes first and last; after every step the
// slab exchanges one message through each side (pack -> transport -> unpack,
// or exchange_with for two slabs of one process).  See cfdx_lbm_create_slab.
template <class Descriptor> class EsotericPullCudaSlab : public EsotericPullCudaSolver<Descriptor> {
public:
    template <class Config>
    EsotericPullCudaSlab(const Config& config, std::uint32_t z_begin, std::uint32_t z_extent)
        : EsotericPullCudaSolver<Descriptor>(config, z_begin, z_extent) {}

    // (z_begin, z_extent, nz of the whole lattice)
    [[nodiscard]] std::array<std::uint32_t, 3> slab_info() const {
        std::array<std::uint32_t, 3> v{};
        cuda::check(cfdx_lbm_slab_info(this->native_handle(), &v[0], &v[1], &v[2]), "slab_info");
        return v;
    }
    [[nodiscard]] std::size_t halo_bytes() const {
        std::size_t b = 0;
        cuda::check(cfdx_lbm_halo_bytes(this->native_handle(), &b), "halo_bytes");
        return b;
    }
    // side: CFDX_SIDE_LOWER / CFDX_SIDE_UPPER; buffers are device memory of halo_bytes()
    void pack(int side, void* device_buffer) {
        cuda::check(cfdx_lbm_halo_pack(this->native_handle(), side, device_buffer), "halo_pack");
    }
    void unpack(int side, const void* device_buffer) {
        cuda::check(cfdx_lbm_halo_unpack(this->native_handle(), side, device_buffer), "halo_unpack");
    }
    // both messages of the cut between this slab's upper side and `upper`'s lower side
    void exchange_with(EsotericPullCudaSlab& upper) {
        cuda::check(cfdx_lbm_halo_exchange(this->native_handle(), upper.native_handle()), "halo_exchange");
    }
};

namespace cuda {

// Reference voxelize_surface (src/lbm/voxelize.cpp:5) on the device: the
// same mask bit for bit.  Grid: any type with nx, ny, nz and .minimum /
// .maximum points (the reference's VoxelGrid3D).
template <class Surface, class Grid>
[[nodiscard]] std::vector<unsigned char> voxelize_surface(const Surface& surface, const Grid& grid, int device = 0) {
    const std::vector<double> tris = pack_triangles(surface);
    cfdx_voxel_grid g{grid.nx, grid.ny, grid.nz, {grid.minimum.x, grid.minimum.y, grid.minimum.z},
                      {grid.maximum.x, grid.maximum.y, grid.maximum.z}};
    std::vector<unsigned char> mask(grid.nx * grid.ny * grid.nz);
    check(cfdx_voxelize(tris.data(), tris.size() / 9, &g, 0U, static_cast<std::uint32_t>(grid.nz), 1U, mask.data(),
                        CFDX_HOST, device),
          "voxelize_surface");
    return mask;
}

// The velocity type of a scalar-only VTK file.
struct NoVector {
    double x, y, z;
};

// 3 doubles per cell from any vector type with .x .y .z (the reference's Vector3).
template <class V> std::vector<double> pack_vectors(std::span<const V> v) {
    std::vector<double> out;
    out.reserve(3 * v.size());
    for (const auto& e : v) {
        out.push_back(e.x);
        out.push_back(e.y);
        out.push_back(e.z);
    }
    return out;
}

// Reference write_vtk_structured_3d (visualization.cpp:39-67): the same ASCII
// text; binary = true writes the big-endian binary legacy format.
template <class V = NoVector>
void write_vtk_structured_3d(const std::string& path, std::size_t nx, std::size_t ny, std::size_t nz,
                             std::span<const double> scalar, std::span<const V> velocity = {},
                             std::span<const std::uint8_t> solid = {}, const char* scalar_name = "field",
                             bool binary = false) {
    const std::size_t cells = nx * ny * nz;
    if (scalar.size() != cells || (!velocity.empty() && velocity.size() != cells) ||
        (!solid.empty() && solid.size() != cells))
        throw std::invalid_argument("LBM 3-D VTK field size mismatch");
    std::vector<double> u;
    if constexpr (!std::is_same_v<V, NoVector>) u = pack_vectors(velocity);
    check(cfdx_write_vtk_3d(path.c_str(), nx, ny, nz, scalar.data(), u.empty() ? nullptr : u.data(),
                            solid.empty() ? nullptr : solid.data(), scalar_name, binary ? 1 : 0),
          "write_vtk_structured_3d");
}

// Reference write_json_state_3d (visualization.cpp:68-109).
inline void write_json_state_3d(const std::string& path, std::size_t nx, std::size_t ny, std::size_t nz,
                                std::uint64_t step, std::span<const double> scalar,
                                std::span<const std::uint8_t> solid = {}, const char* scalar_name = "field") {
    if (scalar.size() != nx * ny * nz || (!solid.empty() && solid.size() != scalar.size()))
        throw std::invalid_argument("LBM 3-D live state size mismatch");
    check(cfdx_write_json_state_3d(path.c_str(), nx, ny, nz, step, scalar.data(), solid.empty() ? nullptr : solid.data(),
                                   scalar_name),
          "write_json_state_3d");
}

// Reference q_criterion_3d (visualization.cpp:122-148) on the device: the same values bit for bit.
template <class V>
[[nodiscard]] std::vector<double> q_criterion_3d(std::size_t nx, std::size_t ny, std::size_t nz,
                                                 std::span<const V> velocity, double dx = 1.0, double dy = 1.0,
                                                 double dz = 1.0, int device = 0) {
    if (velocity.size() != nx * ny * nz) throw std::invalid_argument("invalid LBM Q-criterion grid");
    const std::vector<double> u = pack_vectors(velocity);
    std::vector<double> q(velocity.size());
    check(cfdx_q_criterion(u.data(), nx, ny, nz, dx, dy, dz, q.data(), CFDX_HOST, device), "q_criterion_3d");
    return q;
}

} // namespace cuda

} // namespace cfd::lbm
