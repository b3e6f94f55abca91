// C ABI of the B200 in-place Esoteric-Pull engine (declared in include/cfdx_lbm.h).
//
// The handle owns the single population lattice, the optional flag /
// acceleration / solid-fraction fields, the reduction scratch and one CUDA
// stream.  Every entry point converts C++ and CUDA failures into a status
// code and a thread-local message; nothing here throws across the ABI or
// aborts.  There is no CPU fallback: without a CUDA device every call that
// needs one returns CFDX_ERR_CUDA.
#include "cfdx_lbm.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "halo.h"
#include "handle_access.h"
#include "lbm_launch.h"
#include "voxelize.h"
#include "export.h"
#include "resident.h"
#include "scratch_pool.h"
#include "slot_audit.h"
#include "thermal.h"

namespace {

using namespace cfdx;

thread_local std::string g_error;
thread_local int g_error_status = CFDX_OK;
std::atomic<int> g_fail_allocations{0};
std::atomic<int> g_retry_allocations{0};           // test hook: first attempts that report out-of-memory
std::atomic<unsigned long long> g_allocation_retries{0};

struct CfdxError : std::runtime_error {
    int status;
    CfdxError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void fail(int status, const std::string& message) { throw CfdxError(status, message); }

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) fail(CFDX_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    fail(CFDX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Allocation wrapper with the test hook of cfdx_debug_fail_allocations().
void* device_alloc(std::size_t bytes, const char* what) {
    if (g_fail_allocations.load() > 0) {
        g_fail_allocations.fetch_sub(1);
        fail(CFDX_ERR_OOM, std::string(what) + ": injected allocation failure (cudaErrorMemoryAllocation)");
    }
    void* p = nullptr;
    cudaError_t e;
    if (g_retry_allocations.load() > 0) {
        g_retry_allocations.fetch_sub(1);
        e = cudaErrorMemoryAllocation; // test hook: the first attempt reports out-of-memory
    } else {
        e = cudaMalloc(&p, bytes);
    }
    if (e == cudaErrorMemoryAllocation) {
        // The scratch pool may hold idle memory from earlier voxelizer / Q-criterion
        // calls: return it to the driver and try once more.  No synchronisation:
        // the trim releases what the pool holds idle now, and pool memory whose
        // stream-ordered free has not run yet stays mapped (waiting for every
        // stream of the device would stall other handles and other libraries).
        cudaGetLastError();
        ++g_allocation_retries;
        int device = 0;
        if (cudaGetDevice(&device) == cudaSuccess && scratch_release(device) == cudaSuccess)
            e = cudaMalloc(&p, bytes);
    }
    check_cuda(e, what);
    return p;
}

void device_free(void* p) {
    if (p) cudaFree(p);
}

template <class F> int guarded(F&& body) {
    try {
        body();
        return CFDX_OK;
    } catch (const CfdxError& e) {
        g_error = e.what();
        g_error_status = e.status;
        return e.status;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        g_error_status = CFDX_ERR_INVALID;
        return CFDX_ERR_INVALID;
    } catch (const std::out_of_range& e) {
        g_error = e.what();
        g_error_status = CFDX_ERR_RANGE;
        return CFDX_ERR_RANGE;
    } catch (const std::bad_alloc& e) {
        g_error = e.what();
        g_error_status = CFDX_ERR_OOM;
        return CFDX_ERR_OOM;
    } catch (const std::exception& e) {
        g_error = e.what();
        g_error_status = CFDX_ERR_UNKNOWN;
        return CFDX_ERR_UNKNOWN;
    } catch (...) {
        g_error = "unknown C++ exception";
        g_error_status = CFDX_ERR_UNKNOWN;
        return CFDX_ERR_UNKNOWN;
    }
}

void copy_error(char* out, std::size_t cap, const std::string& text) {
    if (!out || cap == 0U) return;
    const std::size_t n = std::min(cap - 1U, text.size());
    std::memcpy(out, text.data(), n);
    out[n] = '\0';
}

int storage_bytes(int storage) { return storage == kStoreF64 ? 8 : (storage == kStoreF16S ? 2 : 4); }

// lowbias32 integer hash (C. Wellons, "hash-prospector", public domain).
std::uint32_t lowbias32(std::uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Reference Smagorinsky coefficient 16 sqrt(2) / (3 pi^2), evaluated in float
// as include/cfd/solvers/lbm/esoteric_pull.hpp:94-95 does.
float reference_les_k() {
    const float pi = 3.14159265358979323846F;
    return 16.0F * 1.4142135623730950488F / (3.0F * pi * pi);
}

double lattice_weight(int q, int d) {
    static const int cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
    static const int cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
    static const int cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};
    const int len2 = cx[d] * cx[d] + cy[d] * cy[d] + cz[d] * cz[d];
    if (q == 19) return len2 == 0 ? 1.0 / 3.0 : (len2 == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
    return len2 == 0 ? 8.0 / 27.0 : (len2 == 1 ? 2.0 / 27.0 : (len2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
}

} // namespace

struct cfdx_lbm {
    cfdx_lbm_config cfg{};
    KernelKey key{};
    std::size_t N = 0;
    void* f = nullptr;
    std::size_t f_bytes = 0;
    std::uint8_t* flags = nullptr; // internal flag bytes
    std::uint32_t* wall_mask = nullptr; // wall-link bits of near-wall fluid cells
    std::uint32_t* near_list = nullptr; // two-cell FP16 step with flags: cells of the pairs with walls (k_step_list)
    std::uint32_t near_count = 0;
    bool near_built = false;            // near_list matches the current flags
    float* local_a = nullptr;
    float* ns = nullptr;
    float* macro_scratch = nullptr; // 4*N floats, lazily allocated
    double* reduce_partials = nullptr;
    double* reduce_out = nullptr;
    double* host_reduce = nullptr; // pinned
    int reduce_blocks = 0;
    cudaStream_t stream = nullptr;
    std::uint64_t t = 0;
    // Instantiated graph of kGraphSteps step launches, one per parity of its
    // first step, with what it was captured from; replayed by later calls
    // whose launches match it byte for byte (cfdx_lbm_step).
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        LbmArgs first{};
        KernelKey key{};
        dim3 grid, block;
    } step_graph[2];
    float wall_u[kMaxWallIds][3]{};
    float scale[27]{};
    LaunchShape shape{};
    // step kernel: 0 auto, 1 one cell per thread, 2 paired cells, 3 / 4 the
    // wall-aware z-marching FP16 pair kernel with / without its cp.async pipeline
    int variant = 0;
    std::uint32_t planes = 0; // z-planes per thread of that kernel (0: kDefaultPlanes)
    static constexpr std::uint32_t kDefaultPlanes = 4; // measured: 4 > 8 > 16 on the 512^3 cavity
    // Automatic choice between the one-cell and the paired-cell kernel, from
    // B200 measurements (GLUPS, FP16 D3Q19, one-cell vs two-cell): pairs win
    // only on lattices without flags (BGK periodic 512^3: 64.3 vs 55.6).  With
    // flags the one-cell kernel, whose wall links cost no divergence, wins:
    // LES cavity 48.7 vs 44.6, TRT cavity 52.0 vs 43.8, 512x256x256 sphere
    // pack 45.5 vs 34.4 (the two-cell kernel then leaves the pairs with walls
    // to a list kernel whose scattered cells coalesce poorly).  Pairs lose for
    // FP32 storage and for D3Q27 (the 26 neighbour words of a pair need more
    // registers than the kernel can hold).
    static bool paired_default(int storage, int q, bool flags) {
        return storage == kStoreF16S && q == 19 && !flags;
    }
    // The wall-aware z-marching pair kernel (k_step_w2, cp.async pipeline, 4
    // planes per thread, wall links resolved three planes ahead) against the
    // one-cell kernel, B200, FP16, GLUPS: D3Q19 TRT + Smagorinsky cavity 512^3
    // 52.2 vs 47.8; without Smagorinsky 53.3 vs 51.4; 512x256x256 sphere pack
    // 46.2 vs 45.6; D3Q27 Smagorinsky cavity 384^3 28.1 vs 34.7; gray channels
    // (D3Q19 128^3, D3Q27 256^3) 23.8 vs 37.5 and 12.8 vs 30.3 (the gray and
    // D3Q27 forms spill); periodic BGK 57.1 vs 63.7 for the flag-free paired
    // kernel.  Automatic choice: where it wins.
    static bool w2_default(int storage, int q, bool flags, bool gray) {
        return storage == kStoreF16S && q == 19 && flags && !gray;
    }
    double les_k = 0.0;
    std::uint64_t h2d = 0, d2h = 0, syncs = 0;
    bool moving_walls = false; // some flag is a moving-wall id (2..15)

    // z-slab of a decomposed lattice (cfdx_lbm_create_slab): nz = z_extent + 2
    // local planes, planes 0 and nz-1 being ghost copies of the neighbours'
    // edge planes.  Off for a plain handle.
    struct Slab {
        bool on = false;
        std::uint32_t z_begin = 0, z_extent = 0, nz_global = 0;
        std::uint8_t due = 0; // sides (bit 0 lower, bit 1 upper) whose message of the last step is not yet in
        bool fresh = false;   // a step ran since the last initialisation or checkpoint load
        bool interior_due = false; // a two-phase step ran its edge planes; its interior is still to run
        bool whole_ring() const { return on && z_extent == nz_global; }
    } slab;
    cudaEvent_t event = nullptr; // ordering point between two slabs' streams (cfdx_lbm_halo_exchange)

    // Discrete adjoint (cfdx_lbm_adjoint_*): forward checkpoints every
    // `interval` steps, recompute frames for one segment, the adjoint lattice
    // and the gradient accumulators.  Buffers are kept for reuse until
    // cfdx_lbm_adjoint_release or destroy.
    std::uint32_t adjoint_sub = 0; // cfdx_lbm_adjoint_set_subinterval, for the next forward pass
    struct Adjoint {
        std::uint64_t t0 = 0, steps = 0, t_end = 0;
        std::uint32_t interval = 0;
        std::uint32_t sub = 0;  // sub-checkpoint interval of the reverse sweep (0: one level)
        bool ready = false;     // a forward pass has run and nothing has changed since
        void* checkpoints = nullptr;
        std::size_t checkpoint_bytes = 0;
        void* frames = nullptr;
        std::size_t frame_bytes = 0;
        void* lam = nullptr;
        std::size_t lam_bytes = 0;
        double* grad_ns = nullptr;
        double* tau_partials = nullptr;
        std::size_t tau_blocks = 0;
        double* tau_out = nullptr;
        float* seed = nullptr; // 4*N staging for host-side seeds
    } adj;

    LbmArgs args() const {
        LbmArgs a = args_at(f, storage_bytes(key.storage), static_cast<int>(t & 1U));
        a.round_seed = round_seed(t);
        return a;
    }
    // Seed of the FP16 rounding bits of the step that starts at time step ts.
    std::uint32_t round_seed(std::uint64_t ts) const {
        return lowbias32(static_cast<std::uint32_t>(ts) * 0x9E3779B9U +
                         lowbias32(cfg.rounding_seed ^ static_cast<std::uint32_t>(ts >> 32)));
    }
    // Slot tables and rounding seed of the step that starts at time step ts.
    void set_step(LbmArgs& a, std::uint64_t ts) const {
        set_parity(a, static_cast<int>(ts & 1U));
        a.round_seed = round_seed(ts);
    }
    // Arguments for a lattice of this handle's shape at `lattice` (element
    // size `es` bytes), with the slot tables of parity `odd`.
    LbmArgs args_at(void* lattice, int elem_bytes, int odd) const {
        LbmArgs a;
        std::memset(&a, 0, sizeof a); // padding too: cached step graphs compare arguments byte for byte
        char* base = static_cast<char*>(lattice);
        const std::size_t es = static_cast<std::size_t>(elem_bytes);
        for (int d = 0; d < 27; ++d) a.fd[d] = d < key.q ? base + static_cast<std::size_t>(d) * N * es : nullptr;
        a.rest = a.fd[0];
        a.base = lattice;
        a.rest_off = 0U;
        set_parity(a, odd);
        a.flags = key.flags ? flags : nullptr;
        a.wall_mask = key.flags ? wall_mask : nullptr;
        a.near_list = key.flags ? near_list : nullptr;
        a.near_count = key.flags ? near_count : 0U;
        a.planes = planes == 0U ? kDefaultPlanes : planes;
        a.ax_field = local_a;
        a.ay_field = local_a ? local_a + N : nullptr;
        a.az_field = local_a ? local_a + 2 * N : nullptr;
        a.ns = key.gray ? ns : nullptr;
        a.nx = static_cast<std::uint32_t>(cfg.nx);
        a.ny = static_cast<std::uint32_t>(cfg.ny);
        a.nz = static_cast<std::uint32_t>(cfg.nz);
        a.N = static_cast<std::uint32_t>(N);
        a.z_first = 0U; // step launches cover every plane unless a two-phase step narrows them
        a.z_end = a.nz;
        a.has_force = (cfg.acceleration_x != 0.0F || cfg.acceleration_y != 0.0F || cfg.acceleration_z != 0.0F ||
                       local_a != nullptr)
                          ? 1
                          : 0;
        a.tau = cfg.tau;
        // > 0: fixed TRT antisymmetric rate; 0: from the magic parameter; < 0: BGK
        a.omega_minus = key.collision == kBGK
                            ? -1.0
                            : (cfg.trt_tau_minus > 0.0F ? 1.0 / static_cast<double>(cfg.trt_tau_minus) : 0.0);
        a.trt_magic = cfg.trt_magic;
        a.les_k = les_k;
        a.ax = cfg.acceleration_x;
        a.ay = cfg.acceleration_y;
        a.az = cfg.acceleration_z;
        a.tau_f = static_cast<float>(a.tau);
        a.omega_minus_f = static_cast<float>(a.omega_minus);
        a.trt_magic_f = static_cast<float>(a.trt_magic);
        a.les_k_f = static_cast<float>(a.les_k);
        a.ax_f = static_cast<float>(a.ax);
        a.ay_f = static_cast<float>(a.ay);
        a.az_f = static_cast<float>(a.az);
        a.minus_mode = a.omega_minus > 0.0 ? 1 : (a.omega_minus < 0.0 ? -1 : 0);
        std::memcpy(a.wall_u, wall_u, sizeof wall_u);
        const bool stochastic = key.storage == kStoreF16S && cfg.fp16_rounding == CFDX_ROUND_STOCHASTIC;
        a.round_mask = stochastic ? 0xffffffffU : 0U;
        a.round_add = stochastic ? 0U : 0x10001000U; // nearest: half a step in both 13-bit fields
        a.round_seed = 0U;
        // global index of local cell n: n + (z_begin - 1) * nx * ny (mod 2^32)
        a.hash_base = slab.on ? (slab.z_begin - 1U) * static_cast<std::uint32_t>(cfg.nx * cfg.ny) : 0U;
        for (int d = 0; d < 27; ++d) {
            a.scale[d] = scale[d] == 0.0F ? 1.0F : scale[d];
            a.inv_scale[d] = 1.0F / a.scale[d];
        }
        return a;
    }
    // Slot tables of the given parity: pa[p] is read at the neighbour
    // n + c_{2p+2}, pb[p] at the cell itself (see LbmArgs).
    void set_parity(LbmArgs& a, int odd) const {
        a.odd = odd;
        const bool offsets = static_cast<unsigned long long>(key.q) * N < (1ULL << 32);
        for (int p = 0; p < 13; ++p) {
            const int i = 2 * p + 1, j = i + 1;
            if (j < key.q) {
                a.pa[p] = a.fd[odd ? j : i];
                a.pb[p] = a.fd[odd ? i : j];
                a.pa_off[p] = offsets ? static_cast<std::uint32_t>((odd ? j : i) * N) : 0U;
                a.pb_off[p] = offsets ? static_cast<std::uint32_t>((odd ? i : j) * N) : 0U;
            } else {
                a.pa[p] = a.pb[p] = nullptr;
                a.pa_off[p] = a.pb_off[p] = 0U;
            }
        }
    }
    // The paired-cell step kernel needs FP32/FP16 storage, an even nx and
    // element offsets that fit 32 bits.
    bool paired_eligible() const {
        return key.storage != kStoreF64 && cfg.nx % 2U == 0U && offsets_fit() &&
               (shape.block_x == 0 || shape.block_x % 32 == 0);
    }
    // Element offsets of every slot fit 32 bits (q * cells < 2^32), unless the
    // test hook cfdx_debug_force_wide_slots sends a small lattice through the
    // 64-bit slot-pointer kernels that larger lattices use.
    bool force_wide = false;
    bool offsets_fit() const { return !force_wide && static_cast<unsigned long long>(key.q) * N < (1ULL << 32); }
    // The wall-aware FP16 pair kernel needs FP16 storage, an even nx and
    // element offsets that fit 32 bits.
    bool w2_eligible() const {
        return key.storage == kStoreF16S && cfg.nx % 2U == 0U && offsets_fit() &&
               (shape.block_x == 0 || shape.block_x * shape.block_y == 128);
    }
    void choose_variant() {
        key.narrow = offsets_fit();
        key.w2 = (variant == 3 || variant == 4 ||
                  (variant == 0 && w2_default(key.storage, key.q, key.flags, key.gray))) &&
                 w2_eligible();
        key.w2_pipe = variant != 4;
        key.paired = !key.w2 && (variant == 2 || (variant == 0 && paired_eligible() &&
                                                  paired_default(key.storage, key.q, key.flags)));
    }
    dim3 step_block() const {
        if (key.w2) {
            // 128 threads as one warp along x in each of four rows: the warps of
            // a block cover the same x-segment, so a block's warps meet the same
            // walls (a row's end pairs hold its x-walls) and finish together
            if (shape.block_x > 0 && shape.block_y > 0)
                return dim3(static_cast<unsigned>(shape.block_x), static_cast<unsigned>(shape.block_y), 1U);
            return dim3(32U, 4U, 1U);
        }
        if (!key.paired) return block();
        int bx = shape.block_x, by = shape.block_y;
        if (bx <= 0 || by <= 0) {
            const long long pairs = static_cast<long long>(cfg.nx / 2U);
            bx = static_cast<int>(std::min<long long>(64, ((pairs + 31) / 32) * 32));
            by = std::max(1, 128 / bx);
        }
        return dim3(static_cast<unsigned>(bx), static_cast<unsigned>(by), 1U);
    }
    dim3 block() const { return cell_block(static_cast<long long>(cfg.nx), static_cast<long long>(cfg.ny), shape); }
    dim3 grid() const {
        return cell_grid(static_cast<long long>(cfg.nx), static_cast<long long>(cfg.ny),
                         static_cast<long long>(cfg.nz), block());
    }
    void set_device() const { check_cuda(cudaSetDevice(cfg.device), "cudaSetDevice"); }
    void sync() {
        check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        ++syncs;
    }
};

namespace {

void require(bool ok, const char* message) {
    if (!ok) throw std::invalid_argument(message);
}

// mid_step: the call may come between the two phases of a slab's step
// (cfdx_lbm_step_phase); every other call needs whole steps.
cfdx_lbm* checked(cfdx_lbm* h, bool mid_step = false) {
    if (!h) throw std::invalid_argument("null cfdx_lbm handle");
    if (!mid_step && h->slab.interior_due)
        throw std::invalid_argument("the slab's two-phase step is half done: run its CFDX_STEP_INTERIOR phase first");
    h->set_device();
    return h;
}

void default_scales(cfdx_lbm* h) {
    // Power of two nearest 1/w_d: (f - w_d) * s_d is then the relative
    // deviation from the rest weight, which keeps small deviations out of the
    // FP16 subnormal range; powers of two make the scaling exact.
    for (int d = 0; d < 27; ++d) {
        if (d >= h->key.q) {
            h->scale[d] = 1.0F;
            continue;
        }
        const double w = lattice_weight(h->key.q, d);
        h->scale[d] = static_cast<float>(std::ldexp(1.0, static_cast<int>(std::lround(std::log2(1.0 / w)))));
    }
}

// Copies a caller buffer (host or device) into device memory `dst`.
void upload(cfdx_lbm* h, void* dst, const void* src, std::size_t bytes, int where) {
    require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
    const cudaMemcpyKind kind = where == CFDX_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    check_cuda(cudaMemcpyAsync(dst, src, bytes, kind, h->stream), "cudaMemcpyAsync (upload)");
    if (where == CFDX_HOST) {
        h->h2d += bytes;
        h->sync(); // the caller may release its host buffer on return
    }
}

void download(cfdx_lbm* h, void* dst, const void* src, std::size_t bytes, int where) {
    require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
    const cudaMemcpyKind kind = where == CFDX_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    check_cuda(cudaMemcpyAsync(dst, src, bytes, kind, h->stream), "cudaMemcpyAsync (download)");
    if (where == CFDX_HOST) h->d2h += bytes;
    h->sync();
}

void init_state(cfdx_lbm* h, const InitSpec& in) {
    InitSpec spec = in;
    if (h->slab.on) {
        spec.nz_total = h->slab.nz_global;
        spec.z_origin = (h->slab.z_begin + h->slab.nz_global - 1U) % h->slab.nz_global;
    } else {
        spec.nz_total = static_cast<std::uint32_t>(h->cfg.nz);
        spec.z_origin = 0U;
    }
    // Zero first: wall cells and wall-only slots are never written by the init
    // kernel and must not hold stale or non-finite data.
    check_cuda(cudaMemsetAsync(h->f, 0, h->f_bytes, h->stream), "cudaMemsetAsync");
    check_cuda(launch_init(h->key, h->args(), spec, h->grid(), h->block(), h->stream), "init kernel");
    h->t = 0;
    h->adj.ready = false;
    // Every slot a step reads now holds its own cell's state: no message is due.
    h->slab.due = 0;
    h->slab.fresh = false;
    h->slab.interior_due = false;
}

void ensure_reduce(cfdx_lbm* h) {
    if (h->reduce_partials) return;
    int sms = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->cfg.device), "device attribute");
    const long long rows = static_cast<long long>(h->cfg.ny * h->cfg.nz);
    h->reduce_blocks = static_cast<int>(std::max(1LL, std::min<long long>(4LL * sms, rows)));
    h->reduce_partials = static_cast<double*>(
        device_alloc(sizeof(double) * kReduceFields * static_cast<std::size_t>(h->reduce_blocks), "reduction scratch"));
    h->reduce_out = static_cast<double*>(device_alloc(sizeof(double) * kReduceFields, "reduction output"));
    check_cuda(cudaMallocHost(&h->host_reduce, sizeof(double) * kReduceFields), "cudaMallocHost");
}

void release_adjoint(cfdx_lbm* h) {
    auto& A = h->adj;
    device_free(A.checkpoints);
    device_free(A.frames);
    device_free(A.lam);
    device_free(A.grad_ns);
    device_free(A.tau_partials);
    device_free(A.tau_out);
    device_free(A.seed);
    A = cfdx_lbm::Adjoint{};
}

void release(cfdx_lbm* h) {
    if (!h) return;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    device_free(h->f);
    device_free(h->flags);
    device_free(h->wall_mask);
    device_free(h->near_list);
    device_free(h->local_a);
    device_free(h->ns);
    device_free(h->macro_scratch);
    device_free(h->reduce_partials);
    device_free(h->reduce_out);
    release_adjoint(h);
    for (auto& sg : h->step_graph)
        if (sg.exec) cudaGraphExecDestroy(sg.exec);
    if (h->host_reduce) cudaFreeHost(h->host_reduce);
    if (h->event) cudaEventDestroy(h->event);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

} // namespace

namespace cfdx {

dim3 cell_block(long long nx, long long ny, const LaunchShape& s) {
    int bx = s.block_x, by = s.block_y;
    if (bx <= 0 || by <= 0) {
        bx = static_cast<int>(std::min<long long>(128, ((nx + 31) / 32) * 32));
        by = std::max(1, 128 / bx);
        by = static_cast<int>(std::min<long long>(by, ny));
    }
    return dim3(static_cast<unsigned>(bx), static_cast<unsigned>(by), 1U);
}

dim3 cell_grid(long long nx, long long ny, long long nz, dim3 block) {
    return dim3(static_cast<unsigned>((nx + block.x - 1) / block.x), static_cast<unsigned>((ny + block.y - 1) / block.y),
                static_cast<unsigned>(nz));
}

cudaError_t launch_step(const KernelKey& k, const LbmArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::step(k, a, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::step(k, a, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::step(k, a, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_init(const KernelKey& k, const LbmArgs& a, const InitSpec& spec, dim3 g, dim3 b, cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::init(k, a, spec, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::init(k, a, spec, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::init(k, a, spec, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_macro(const KernelKey& k, const LbmArgs& a, void* rho, void* ux, void* uy, void* uz, bool f64,
                         dim3 g, dim3 b, cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::macro(k, a, rho, ux, uy, uz, f64, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::macro(k, a, rho, ux, uy, uz, f64, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::macro(k, a, rho, ux, uy, uz, f64, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_logical(const KernelKey& k, const LbmArgs& a, float* out, dim3 g, dim3 b, cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::logical(k, a, out, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::logical(k, a, out, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::logical(k, a, out, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_reduce(const KernelKey& k, const LbmArgs& a, double* partials, int blocks, double* out,
                          cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::reduce(k, a, partials, blocks, out, s);
    case kStoreF64: return Launcher<kStoreF64>::reduce(k, a, partials, blocks, out, s);
    case kStoreF16S: return Launcher<kStoreF16S>::reduce(k, a, partials, blocks, out, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_step_oop(const KernelKey& k, const LbmArgs& src, const LbmArgs& dst, dim3 g, dim3 b,
                            cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::step_oop(k, src, dst, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::step_oop(k, src, dst, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::step_oop(k, src, dst, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_adjoint_seed(const KernelKey& k, const AdjointArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::adjoint_seed(k, a, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::adjoint_seed(k, a, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::adjoint_seed(k, a, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_slot_io(const KernelKey& k, const LbmArgs& a, int d, float* buf, bool in, dim3 g, dim3 b,
                           cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::slot_io(k, a, d, buf, in, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::slot_io(k, a, d, buf, in, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::slot_io(k, a, d, buf, in, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_adjoint_step(const KernelKey& k, const AdjointArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    switch (k.storage) {
    case kStoreF32: return Launcher<kStoreF32>::adjoint_step(k, a, g, b, s);
    case kStoreF64: return Launcher<kStoreF64>::adjoint_step(k, a, g, b, s);
    case kStoreF16S: return Launcher<kStoreF16S>::adjoint_step(k, a, g, b, s);
    default: return cudaErrorInvalidValue;
    }
}

int handle_reduce_view(cfdx_lbm* h, ReduceView* view) {
    return guarded([&] {
        checked(h);
        require(view != nullptr, "null view");
        view->key = h->key;
        view->args = h->args();
        view->stream = h->stream;
        view->device = h->cfg.device;
    });
}

int record_error(int status, const char* message) {
    g_error = message ? message : "";
    g_error_status = status;
    return status;
}

void record_download(cfdx_lbm* h, std::uint64_t bytes) {
    h->d2h += bytes;
    ++h->syncs;
}

} // namespace cfdx

extern "C" {

CFDX_API const char* cfdx_version(void) { return "cfd_solvers_b200 0.1.0 (sm_100a)"; }

CFDX_API int cfdx_last_error(char* buffer, std::size_t capacity) {
    copy_error(buffer, capacity, g_error);
    return g_error_status;
}

CFDX_API int cfdx_lbm_config_default(cfdx_lbm_config* c) {
    return guarded([&] {
        require(c != nullptr, "null config");
        *c = cfdx_lbm_config{};
        c->nx = c->ny = c->nz = 128;
        c->tau = 0.6F;
        c->lattice = CFDX_D3Q19;
        c->collision = CFDX_BGK;
        c->storage = CFDX_STORE_F32;
        c->smagorinsky_cs = 0.0F;
        c->trt_magic = 3.0F / 16.0F;
        c->trt_tau_minus = 0.0F;
        c->device = 0;
        c->fp16_rounding = CFDX_ROUND_STOCHASTIC;
        c->rounding_seed = 0U;
    });
}

namespace {

void validate_config(const cfdx_lbm_config& c) {
    // reference esoteric_pull.hpp:111-113,292-301
    require(c.nx >= 2 && c.ny >= 2, "LBM grid requires nx, ny >= 2");
    require(c.nz >= 2, "3-D LBM grid requires nz >= 2");
    require(c.tau > 0.5F && std::isfinite(c.tau), "LBM tau must be > 0.5 for positive viscosity");
    require(c.lattice == CFDX_D3Q19 || c.lattice == CFDX_D3Q27, "lattice must be CFDX_D3Q19 or CFDX_D3Q27");
    require(c.collision == CFDX_BGK || c.collision == CFDX_TRT, "collision must be CFDX_BGK or CFDX_TRT");
    require(c.storage == CFDX_STORE_F32 || c.storage == CFDX_STORE_F64 || c.storage == CFDX_STORE_F16S,
            "unknown storage");
    require(c.fp16_rounding == CFDX_ROUND_NEAREST || c.fp16_rounding == CFDX_ROUND_STOCHASTIC,
            "fp16_rounding must be CFDX_ROUND_NEAREST or CFDX_ROUND_STOCHASTIC");
    require(std::isfinite(c.acceleration_x) && std::isfinite(c.acceleration_y) && std::isfinite(c.acceleration_z),
            "acceleration must be finite");
    if (c.collision == CFDX_TRT)
        require(c.trt_tau_minus > 0.5F || (c.trt_tau_minus <= 0.0F && c.trt_magic > 0.0F),
                "TRT needs trt_tau_minus > 0.5 or trt_magic > 0");
    require(c.nx <= (1U << 30) && c.ny <= 65535U && c.nz <= 65535U, "grid extent exceeds launch limits");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        fail(CFDX_ERR_CUDA, "no CUDA device is available (the B200 engine has no CPU fallback)");
    require(c.device >= 0 && c.device < count, "device ordinal out of range");
}

void apply_flags(cfdx_lbm* h, const std::uint8_t* flags, int where);

// Sets up a new handle for the validated local configuration c.
void build_handle(cfdx_lbm* h, const cfdx_lbm_config& c, const cfdx_lbm::Slab& slab) {
    h->cfg = c;
    h->slab = slab;
    h->set_device();
    h->N = c.nx * c.ny * c.nz;
    require(h->N <= 0xffffffffULL, "lattice exceeds 2^32 - 1 cells");
    h->key = KernelKey{c.storage, c.lattice, c.collision, c.smagorinsky_les != 0, false, false, 0, false, false};
    h->choose_variant();
    h->les_k = c.smagorinsky_les ? (c.smagorinsky_cs > 0.0F
                                        ? 18.0 * std::sqrt(2.0) * double(c.smagorinsky_cs) * double(c.smagorinsky_cs)
                                        : double(reference_les_k()))
                                 : 0.0;
    default_scales(h);
    check_cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreateWithFlags(&h->event, cudaEventDisableTiming), "cudaEventCreate");
    h->f_bytes = static_cast<std::size_t>(c.lattice) * h->N * static_cast<std::size_t>(storage_bytes(c.storage));
    h->f = device_alloc(h->f_bytes, "population lattice");
    InitSpec spec{};
    spec.kind = 0;
    spec.rho = 1.0F;
    init_state(h, spec); // reference constructor calls initialize_uniform()
    // A slab always carries flags: they keep its ghost planes out of every kernel.
    if (slab.on) apply_flags(h, nullptr, CFDX_HOST);
    h->sync();
}

} // namespace

CFDX_API int cfdx_lbm_create(const cfdx_lbm_config* config, cfdx_lbm** out, char* error, std::size_t cap) {
    cfdx_lbm* h = nullptr;
    const int rc = guarded([&] {
        require(config != nullptr && out != nullptr, "null config or output handle");
        *out = nullptr;
        validate_config(*config);
        h = new cfdx_lbm();
        build_handle(h, *config, cfdx_lbm::Slab{});
        *out = h;
    });
    if (rc != CFDX_OK) {
        release(h);
        copy_error(error, cap, g_error);
    }
    return rc;
}

CFDX_API int cfdx_lbm_create_slab(const cfdx_lbm_config* global, std::uint32_t z_begin, std::uint32_t z_extent,
                                  cfdx_lbm** out, char* error, std::size_t cap) {
    cfdx_lbm* h = nullptr;
    const int rc = guarded([&] {
        require(global != nullptr && out != nullptr, "null config or output handle");
        *out = nullptr;
        validate_config(*global);
        require(z_extent >= 1U, "a slab needs at least one plane");
        require(static_cast<std::uint64_t>(z_begin) + z_extent <= global->nz, "slab exceeds the lattice's z extent");
        cfdx_lbm_config local = *global;
        local.nz = static_cast<std::size_t>(z_extent) + 2U;
        require(local.nz <= 65535U, "grid extent exceeds launch limits");
        cfdx_lbm::Slab slab;
        slab.on = true;
        slab.z_begin = z_begin;
        slab.z_extent = z_extent;
        slab.nz_global = static_cast<std::uint32_t>(global->nz);
        h = new cfdx_lbm();
        build_handle(h, local, slab);
        *out = h;
    });
    if (rc != CFDX_OK) {
        release(h);
        copy_error(error, cap, g_error);
    }
    return rc;
}

CFDX_API int cfdx_lbm_destroy(cfdx_lbm* h) {
    return guarded([&] { release(h); });
}

CFDX_API int cfdx_lbm_init_uniform(cfdx_lbm* h, float rho, float ux, float uy, float uz) {
    return guarded([&] {
        checked(h);
        // reference esoteric_pull_sycl.hpp:53-56
        require(rho > 0.0F && std::isfinite(rho) && std::isfinite(ux) && std::isfinite(uy) && std::isfinite(uz),
                "LBM uniform state must be finite with positive density");
        InitSpec s{};
        s.kind = 0;
        s.rho = rho;
        s.ux = ux;
        s.uy = uy;
        s.uz = uz;
        init_state(h, s);
    });
}

CFDX_API int cfdx_lbm_init_taylor_green(cfdx_lbm* h, float amplitude) {
    return guarded([&] {
        checked(h);
        require(std::isfinite(amplitude), "Taylor-Green amplitude must be finite");
        InitSpec s{};
        s.kind = 1;
        s.amplitude = amplitude;
        init_state(h, s);
    });
}

CFDX_API int cfdx_lbm_init_fields(cfdx_lbm* h, const float* fields, int where) {
    return guarded([&] {
        checked(h);
        require(fields != nullptr, "null fields");
        float* tmp = static_cast<float*>(device_alloc(4U * h->N * sizeof(float), "init staging"));
        try {
            upload(h, tmp, fields, 4U * h->N * sizeof(float), where);
            InitSpec s{};
            s.kind = 2;
            s.fields = tmp;
            init_state(h, s);
            h->sync();
        } catch (...) {
            device_free(tmp);
            throw;
        }
        device_free(tmp);
    });
}

namespace {

// FP16 storage with even nx (the two-cell step): the list of fluid cells of
// the x-pairs that are not interior, selected on the device from the
// internal flags, kept at its exact size.
void build_near_list(cfdx_lbm* h) {
    device_free(h->near_list);
    h->near_list = nullptr;
    h->near_count = 0;
    h->near_built = false;
    if (h->key.storage != kStoreF16S || h->cfg.nx % 2U != 0U) return;
    const auto cells = static_cast<std::uint32_t>(h->N);
    std::size_t temp_bytes = 0;
    check_cuda(select_near_cells(h->flags, cells, nullptr, nullptr, nullptr, &temp_bytes, h->stream),
               "near-cell selection (size)");
    const std::size_t list_bytes = ((h->N * sizeof(std::uint32_t)) + 255U) / 256U * 256U;
    char* scratch = static_cast<char*>(device_alloc(list_bytes + 256U + temp_bytes, "near-cell selection scratch"));
    try {
        auto* all = reinterpret_cast<std::uint32_t*>(scratch);
        auto* count = reinterpret_cast<std::uint32_t*>(scratch + list_bytes);
        check_cuda(select_near_cells(h->flags, cells, all, count, scratch + list_bytes + 256U, &temp_bytes, h->stream),
                   "near-cell selection");
        std::uint32_t host_count = 0;
        check_cuda(cudaMemcpyAsync(&host_count, count, sizeof host_count, cudaMemcpyDeviceToHost, h->stream),
                   "cudaMemcpyAsync (near-cell count)");
        h->sync();
        if (host_count > 0U) {
            h->near_list = static_cast<std::uint32_t*>(device_alloc(host_count * sizeof(std::uint32_t), "near-cell list"));
            check_cuda(cudaMemcpyAsync(h->near_list, all, host_count * sizeof(std::uint32_t), cudaMemcpyDeviceToDevice,
                                       h->stream),
                       "cudaMemcpyAsync (near-cell list)");
            h->sync();
        }
        h->near_count = host_count;
        h->near_built = true;
    } catch (...) {
        device_free(scratch);
        throw;
    }
    device_free(scratch);
}

// Keeps the near-cell list in step with the kernel choice: built when the
// two-cell FP16 step runs with flags, dropped otherwise.  flags_changed: the
// flag field was replaced, so a built list is stale.
void refresh_near_list(cfdx_lbm* h, bool flags_changed) {
    const bool need = h->key.paired && h->key.flags && h->key.storage == kStoreF16S;
    if (flags_changed || !need) {
        device_free(h->near_list);
        h->near_list = nullptr;
        h->near_count = 0;
        h->near_built = false;
    }
    if (need && !h->near_built) build_near_list(h);
}

// Internal flags and wall-link masks from the caller's flags (nullptr: none;
// on a slab, all own cells fluid -- its ghost planes stay marked).
void apply_flags(cfdx_lbm* h, const std::uint8_t* flags, int where) {
    h->adj.ready = false;
    if (!flags && !h->slab.on) {
        h->key.flags = false;
        h->moving_walls = false;
        h->choose_variant();
        refresh_near_list(h, true);
        return;
    }
    if (!h->flags) h->flags = static_cast<std::uint8_t*>(device_alloc(h->N, "flag field"));
    if (!h->wall_mask)
        h->wall_mask = static_cast<std::uint32_t*>(device_alloc(h->N * sizeof(std::uint32_t), "wall-link masks"));
    std::uint8_t* user = static_cast<std::uint8_t*>(device_alloc(h->N, "flag staging"));
    try {
        if (flags) {
            upload(h, user, flags, h->N, where);
            // Record whether any cell is a moving wall (the adjoint does not cover them).
            std::string host_copy;
            const std::uint8_t* scan = flags;
            if (where == CFDX_DEVICE) {
                host_copy.resize(h->N);
                check_cuda(cudaMemcpyAsync(host_copy.data(), user, h->N, cudaMemcpyDeviceToHost, h->stream),
                           "cudaMemcpyAsync (flag scan)");
                h->sync();
                scan = reinterpret_cast<const std::uint8_t*>(host_copy.data());
            }
            h->moving_walls =
                std::any_of(scan, scan + h->N, [](std::uint8_t v) { return v >= CFDX_MOVING_WALL_MIN; });
        } else {
            check_cuda(cudaMemsetAsync(user, 0, h->N, h->stream), "cudaMemsetAsync");
            h->moving_walls = false;
        }
        check_cuda(launch_prepare_flags(h->key.q, h->args(), user, h->flags, h->wall_mask, h->slab.on, h->grid(),
                                        h->block(), h->stream),
                   "flag preparation kernel");
        h->sync();
    } catch (...) {
        device_free(user);
        throw;
    }
    device_free(user);
    h->key.flags = true;
    h->choose_variant();
    refresh_near_list(h, true);
}

} // namespace

CFDX_API int cfdx_lbm_set_flags(cfdx_lbm* h, const std::uint8_t* flags, int where) {
    return guarded([&] {
        checked(h);
        apply_flags(h, flags, where);
    });
}

CFDX_API int cfdx_lbm_set_wall_velocity(cfdx_lbm* h, int id, float ux, float uy, float uz) {
    return guarded([&] {
        checked(h);
        h->adj.ready = false;
        if (id < CFDX_MOVING_WALL_MIN || id >= CFDX_MAX_WALL_IDS)
            throw std::out_of_range("moving-wall id must be in [2, 15]");
        require(std::isfinite(ux) && std::isfinite(uy) && std::isfinite(uz), "wall velocity must be finite");
        h->wall_u[id][0] = ux;
        h->wall_u[id][1] = uy;
        h->wall_u[id][2] = uz;
    });
}

CFDX_API int cfdx_lbm_set_local_acceleration(cfdx_lbm* h, const float* accel, int where) {
    return guarded([&] {
        checked(h);
        h->adj.ready = false;
        if (!accel) {
            device_free(h->local_a);
            h->local_a = nullptr;
            return;
        }
        if (!h->local_a) h->local_a = static_cast<float*>(device_alloc(3U * h->N * sizeof(float), "acceleration field"));
        upload(h, h->local_a, accel, 3U * h->N * sizeof(float), where);
    });
}

CFDX_API int cfdx_lbm_device_local_acceleration(cfdx_lbm* h, float** accel) {
    return guarded([&] {
        checked(h);
        h->adj.ready = false;
        require(accel != nullptr, "null output pointer");
        if (!h->local_a) {
            h->local_a = static_cast<float*>(device_alloc(3U * h->N * sizeof(float), "acceleration field"));
            check_cuda(cudaMemsetAsync(h->local_a, 0, 3U * h->N * sizeof(float), h->stream), "cudaMemsetAsync");
            h->sync();
        }
        *accel = h->local_a;
    });
}

CFDX_API int cfdx_lbm_clear_device_acceleration(cfdx_lbm* h) {
    return guarded([&] {
        checked(h);
        if (!h->local_a) return;
        h->adj.ready = false;
        check_cuda(cudaMemsetAsync(h->local_a, 0, 3U * h->N * sizeof(float), h->stream), "cudaMemsetAsync");
    });
}

CFDX_API int cfdx_lbm_set_solid_fraction(cfdx_lbm* h, const float* ns, int where) {
    return guarded([&] {
        checked(h);
        h->adj.ready = false;
        if (!ns) {
            device_free(h->ns);
            h->ns = nullptr;
            h->key.gray = false;
            h->choose_variant();
            return;
        }
        if (!h->ns) h->ns = static_cast<float*>(device_alloc(h->N * sizeof(float), "solid fraction field"));
        upload(h, h->ns, ns, h->N * sizeof(float), where);
        h->key.gray = true;
        h->choose_variant();
    });
}

CFDX_API int cfdx_lbm_set_storage_scale(cfdx_lbm* h, const float* scale) {
    return guarded([&] {
        checked(h);
        h->adj.ready = false;
        require(h->key.storage == kStoreF16S, "storage scales apply to CFDX_STORE_F16S only");
        if (!scale) {
            default_scales(h);
            return;
        }
        for (int d = 0; d < h->key.q; ++d)
            require(std::isfinite(scale[d]) && scale[d] > 0.0F, "storage scales must be finite and positive");
        // Scales are applied per weight class inside the step kernel.
        for (int d = 0; d < h->key.q; ++d) {
            const double w = lattice_weight(h->key.q, d);
            for (int e = 0; e < d; ++e)
                if (lattice_weight(h->key.q, e) == w)
                    require(scale[d] == scale[e], "directions of equal lattice weight must share a storage scale");
        }
        for (int d = 0; d < h->key.q; ++d) h->scale[d] = scale[d];
    });
}

// ------------------------------------------------------------ slab halos
namespace {

std::size_t plane_cells(const cfdx_lbm* h) { return h->cfg.nx * h->cfg.ny; }

std::size_t halo_chunk_bytes(const cfdx_lbm* h) {
    return plane_cells(h) * static_cast<std::size_t>(storage_bytes(h->key.storage));
}

// Start of the run of direction e.direction over local plane e.plane.
char* plane_run(const cfdx_lbm* h, const HaloEntry& e) {
    const std::size_t element = static_cast<std::size_t>(e.direction) * h->N + static_cast<std::size_t>(e.plane) * plane_cells(h);
    return static_cast<char*>(h->f) + element * static_cast<std::size_t>(storage_bytes(h->key.storage));
}

// Message layout of `side` after the step the slab has just taken.
int last_step_plan(const cfdx_lbm* h, int side, HaloEntry* send, HaloEntry* recv) {
    return halo_plan(h->key.q, static_cast<int>((h->t - 1U) & 1U), side, h->slab.z_extent, send, recv);
}

cfdx_lbm* checked_slab(cfdx_lbm* h) {
    checked(h, true); // halo messages travel while the interior of the step runs
    require(h->slab.on, "not a slab handle (cfdx_lbm_create_slab)");
    return h;
}

// Both messages of the cut between lo's upper side and up's lower side:
// one copy launch on lo's stream, after both slabs' steps and before their
// next ones (lo == up: the ring of one slab).
void exchange_cut(cfdx_lbm* lo, cfdx_lbm* up) {
    HaloEntry ls[kMaxHaloChunks], lr[kMaxHaloChunks], us[kMaxHaloChunks], ur[kMaxHaloChunks];
    const int k = last_step_plan(lo, 1, ls, lr);
    last_step_plan(up, 0, us, ur);
    HaloCopy c{};
    for (int i = 0; i < k; ++i) {
        c.src[i] = plane_run(lo, ls[i]);
        c.dst[i] = plane_run(up, ur[i]);
        c.src[k + i] = plane_run(up, us[i]);
        c.dst[k + i] = plane_run(lo, lr[i]);
    }
    c.chunks = 2 * k;
    if (lo != up) {
        check_cuda(cudaSetDevice(up->cfg.device), "cudaSetDevice");
        check_cuda(cudaEventRecord(up->event, up->stream), "cudaEventRecord");
        lo->set_device();
        check_cuda(cudaStreamWaitEvent(lo->stream, up->event, 0), "cudaStreamWaitEvent");
    }
    check_cuda(launch_halo_copy(c, halo_chunk_bytes(lo), lo->stream), "halo copy kernel");
    if (lo != up) {
        check_cuda(cudaEventRecord(lo->event, lo->stream), "cudaEventRecord");
        check_cuda(cudaSetDevice(up->cfg.device), "cudaSetDevice");
        check_cuda(cudaStreamWaitEvent(up->stream, lo->event, 0), "cudaStreamWaitEvent");
        lo->set_device();
    }
    lo->slab.due = static_cast<std::uint8_t>(lo->slab.due & ~2U);
    up->slab.due = static_cast<std::uint8_t>(up->slab.due & ~1U);
}

} // namespace

namespace {

// Step loops of kGraphSteps or more steps replay a CUDA graph of kGraphSteps
// step launches instead of launching each step: on small lattices a step is
// shorter than its launch (32^3: 5.3 us per launched step), and a graph also
// shortens the gaps between kernels.  The graph is captured from the argument
// blocks the loop would launch, so results are unchanged, and kept on the
// handle (one per parity of the first step): a later call replays it when its
// first step's arguments, kernel key and launch shape equal the captured ones
// byte for byte, and captures a new one otherwise -- any call that changes a
// parameter, a buffer or the kernel choice changes one of them.  The steps of
// a graph differ only in parity (kGraphSteps is even) and in the FP16 rounding
// seed, which FP32 and FP64 kernels do not read (it is zeroed here).
// Excluded: slabs (an exchange follows every step), FP16 storage (its rounding
// seed changes every step) and streams that are already being captured.
constexpr std::uint64_t kGraphSteps = 8;
constexpr std::uint64_t kGraphMinSteps = kGraphSteps;

bool graph_steps_eligible(const cfdx_lbm* h, std::uint64_t count) {
    if (count < kGraphMinSteps || h->slab.on || h->key.storage == kStoreF16S) return false;
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &status) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return status == cudaStreamCaptureStatusNone;
}

// Arguments of the step at time step ts as a step graph holds them.
LbmArgs graph_step_args(const cfdx_lbm* h, const LbmArgs& a, std::uint64_t ts) {
    LbmArgs s = a;
    h->set_step(s, ts);
    s.round_seed = 0U;
    return s;
}

bool same_dim(dim3 x, dim3 y) { return x.x == y.x && x.y == y.y && x.z == y.z; }

// Runs whole replays of a kGraphSteps-step graph from time step h->t; returns the steps run.
std::uint64_t step_graphs(cfdx_lbm* h, const LbmArgs& a, dim3 g, dim3 b, std::uint64_t count) {
    static_assert(kGraphSteps % 2U == 0U, "a replay must end on the parity it starts with");
    const std::uint64_t replays = count / kGraphSteps;
    auto& sg = h->step_graph[h->t & 1U];
    const LbmArgs first = graph_step_args(h, a, h->t);
    const bool cached = sg.exec != nullptr && std::memcmp(&sg.first, &first, sizeof first) == 0 &&
                        std::memcmp(&sg.key, &h->key, sizeof h->key) == 0 && same_dim(sg.grid, g) &&
                        same_dim(sg.block, b);
    if (!cached) {
        if (sg.exec) cudaGraphExecDestroy(sg.exec);
        sg.exec = nullptr;
        check_cuda(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        cudaError_t launched = cudaSuccess;
        for (std::uint64_t i = 0; i < kGraphSteps && launched == cudaSuccess; ++i)
            launched = launch_step(h->key, graph_step_args(h, a, h->t + i), g, b, h->stream);
        cudaGraph_t graph = nullptr;
        const cudaError_t ended = cudaStreamEndCapture(h->stream, &graph);
        cudaGraphExec_t exec = nullptr;
        const cudaError_t made =
            launched == cudaSuccess && ended == cudaSuccess ? cudaGraphInstantiate(&exec, graph, 0) : cudaSuccess;
        if (graph) cudaGraphDestroy(graph);
        check_cuda(launched, "step kernel (graph capture)");
        check_cuda(ended, "cudaStreamEndCapture");
        check_cuda(made, "cudaGraphInstantiate");
        sg.exec = exec;
        sg.first = first;
        std::memcpy(&sg.key, &h->key, sizeof h->key);
        sg.grid = g;
        sg.block = b;
    }
    cudaError_t e = cudaSuccess;
    std::uint64_t run = 0;
    for (; run < replays && e == cudaSuccess; ++run) e = cudaGraphLaunch(sg.exec, h->stream);
    check_cuda(e, "cudaGraphLaunch");
    h->t += run * kGraphSteps;
    return run * kGraphSteps;
}

// Enqueues `launches` (returning the first launch error) on the handle's stream,
// inside one captured CUDA graph when the stream is not already being captured:
// the adjoint's segments are a hundred-odd dependent launches each, and a graph
// shortens the gaps between them.  A capture is always ended before an error
// is reported, so the stream never stays in capture mode.
extern "C++" template <class F> void enqueue_captured(cfdx_lbm* h, const char* what, F&& launches) {
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &status) != cudaSuccess || status != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        check_cuda(launches(), what);
        return;
    }
    check_cuda(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    const cudaError_t launched = launches();
    cudaGraph_t graph = nullptr;
    const cudaError_t ended = cudaStreamEndCapture(h->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t made =
        launched == cudaSuccess && ended == cudaSuccess ? cudaGraphInstantiate(&exec, graph, 0) : cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    check_cuda(launched, what);
    check_cuda(ended, "cudaStreamEndCapture");
    check_cuda(made, "cudaGraphInstantiate");
    const cudaError_t e = cudaGraphLaunch(exec, h->stream);
    cudaGraphExecDestroy(exec);
    check_cuda(e, "cudaGraphLaunch");
}

} // namespace

CFDX_API int cfdx_lbm_step(cfdx_lbm* h, std::uint64_t count) {
    return guarded([&] {
        checked(h);
        if (count == 0) return;
        if (h->slab.on) {
            require(h->slab.due == 0, "the halo messages of the slab's previous step have not all been received");
            require(count == 1 || h->slab.whole_ring(), "a slab takes one step between halo exchanges");
        }
        h->adj.ready = false;
        const dim3 g = h->grid(), b = h->step_block();
        LbmArgs a = h->args();
        std::uint64_t done = 0;
        if (graph_steps_eligible(h, count)) done = step_graphs(h, a, g, b, count);
        for (std::uint64_t i = done; i < count; ++i) {
            h->set_step(a, h->t);
            check_cuda(launch_step(h->key, a, g, b, h->stream), "step kernel");
            ++h->t;
            if (h->slab.on) {
                h->slab.due = 3;
                h->slab.fresh = true;
                if (h->slab.whole_ring()) exchange_cut(h, h);
            }
        }
    });
}

// Planes [z0, z1) of the step that starts at h->t (whole-lattice arguments otherwise).
void launch_planes(cfdx_lbm* h, std::uint64_t ts, std::uint32_t z0, std::uint32_t z1) {
    LbmArgs a = h->args();
    h->set_step(a, ts);
    a.z_first = z0;
    a.z_end = z1;
    dim3 g = h->grid();
    g.z = z1 - z0;
    check_cuda(launch_step(h->key, a, g, h->step_block(), h->stream), "step kernel");
}

CFDX_API int cfdx_lbm_step_phase(cfdx_lbm* h, int phase) {
    return guarded([&] {
        checked(h, true);
        require(h->slab.on, "the two-phase step is for slab handles (cfdx_lbm_create_slab)");
        require(phase == CFDX_STEP_EDGES || phase == CFDX_STEP_INTERIOR,
                "phase must be CFDX_STEP_EDGES or CFDX_STEP_INTERIOR");
        const std::uint32_t ze = h->slab.z_extent; // own planes 1..ze; 0 and ze + 1 are ghosts
        if (phase == CFDX_STEP_EDGES) {
            require(!h->slab.interior_due, "the interior phase of the previous step has not run");
            require(h->slab.due == 0, "the halo messages of the slab's previous step have not all been received");
            h->adj.ready = false;
            launch_planes(h, h->t, 1U, 2U);
            if (ze > 1U) launch_planes(h, h->t, ze, ze + 1U);
            ++h->t;
            h->slab.due = 3;
            h->slab.fresh = true;
            h->slab.interior_due = true;
            if (h->slab.whole_ring()) exchange_cut(h, h);
        } else {
            require(h->slab.interior_due, "no interior is due: run CFDX_STEP_EDGES first");
            if (ze > 2U) launch_planes(h, h->t - 1U, 2U, ze); // slabs of one or two planes are all edges
            h->slab.interior_due = false;
        }
    });
}

CFDX_API int cfdx_lbm_slab_info(cfdx_lbm* h, std::uint32_t* z_begin, std::uint32_t* z_extent, std::uint32_t* nz_global) {
    return guarded([&] {
        require(h != nullptr && z_begin != nullptr && z_extent != nullptr && nz_global != nullptr,
                "null handle or output");
        const auto nz = static_cast<std::uint32_t>(h->cfg.nz);
        *z_begin = h->slab.on ? h->slab.z_begin : 0U;
        *z_extent = h->slab.on ? h->slab.z_extent : nz;
        *nz_global = h->slab.on ? h->slab.nz_global : nz;
    });
}

CFDX_API int cfdx_halo_plan(int lattice, int odd, int side, std::uint32_t z_extent, cfdx_halo_entry* send,
                            cfdx_halo_entry* recv, int capacity, int* count) {
    return guarded([&] {
        require(lattice == CFDX_D3Q19 || lattice == CFDX_D3Q27, "lattice must be CFDX_D3Q19 or CFDX_D3Q27");
        require(odd == 0 || odd == 1, "odd must be 0 or 1");
        require(side == CFDX_SIDE_LOWER || side == CFDX_SIDE_UPPER, "side must be CFDX_SIDE_LOWER or CFDX_SIDE_UPPER");
        require(z_extent >= 1U, "a slab needs at least one plane");
        require(send != nullptr && recv != nullptr && count != nullptr, "null output");
        HaloEntry hs[kMaxHaloChunks], hr[kMaxHaloChunks];
        const int k = halo_plan(lattice, odd, side, z_extent, hs, hr);
        require(capacity >= k, "capacity below the chunk count");
        for (int i = 0; i < k; ++i) {
            send[i] = cfdx_halo_entry{hs[i].plane, hs[i].direction};
            recv[i] = cfdx_halo_entry{hr[i].plane, hr[i].direction};
        }
        *count = k;
    });
}

CFDX_API int cfdx_lbm_halo_bytes(cfdx_lbm* h, std::size_t* bytes) {
    return guarded([&] {
        require(h != nullptr && bytes != nullptr, "null handle or output");
        require(h->slab.on, "not a slab handle (cfdx_lbm_create_slab)");
        HaloEntry hs[kMaxHaloChunks], hr[kMaxHaloChunks];
        *bytes = static_cast<std::size_t>(halo_plan(h->key.q, 0, 0, h->slab.z_extent, hs, hr)) * halo_chunk_bytes(h);
    });
}

CFDX_API int cfdx_lbm_halo_pack(cfdx_lbm* h, int side, void* buffer) {
    return guarded([&] {
        checked_slab(h);
        require(side == CFDX_SIDE_LOWER || side == CFDX_SIDE_UPPER, "side must be CFDX_SIDE_LOWER or CFDX_SIDE_UPPER");
        require(buffer != nullptr, "null message buffer");
        require(h->slab.fresh, "no step since the slab was initialised or loaded: there is no message to send");
        HaloEntry hs[kMaxHaloChunks], hr[kMaxHaloChunks];
        const int k = last_step_plan(h, side, hs, hr);
        const std::size_t chunk = halo_chunk_bytes(h);
        HaloCopy c{};
        for (int i = 0; i < k; ++i) {
            c.src[i] = plane_run(h, hs[i]);
            c.dst[i] = static_cast<char*>(buffer) + static_cast<std::size_t>(i) * chunk;
        }
        c.chunks = k;
        check_cuda(launch_halo_copy(c, chunk, h->stream), "halo pack kernel");
    });
}

CFDX_API int cfdx_lbm_halo_unpack(cfdx_lbm* h, int side, const void* buffer) {
    return guarded([&] {
        checked_slab(h);
        require(side == CFDX_SIDE_LOWER || side == CFDX_SIDE_UPPER, "side must be CFDX_SIDE_LOWER or CFDX_SIDE_UPPER");
        require(buffer != nullptr, "null message buffer");
        require((h->slab.due >> side) & 1U, "no message is due through this side (unpacked already, or no step yet)");
        HaloEntry hs[kMaxHaloChunks], hr[kMaxHaloChunks];
        const int k = last_step_plan(h, side, hs, hr);
        const std::size_t chunk = halo_chunk_bytes(h);
        HaloCopy c{};
        for (int i = 0; i < k; ++i) {
            c.src[i] = static_cast<const char*>(buffer) + static_cast<std::size_t>(i) * chunk;
            c.dst[i] = plane_run(h, hr[i]);
        }
        c.chunks = k;
        check_cuda(launch_halo_copy(c, chunk, h->stream), "halo unpack kernel");
        h->slab.due = static_cast<std::uint8_t>(h->slab.due & ~(1U << side));
    });
}

CFDX_API int cfdx_lbm_halo_exchange(cfdx_lbm* lower, cfdx_lbm* upper) {
    return guarded([&] {
        checked_slab(upper);
        checked_slab(lower);
        const auto& a = lower->slab;
        const auto& b = upper->slab;
        require(lower->key.q == upper->key.q && lower->key.storage == upper->key.storage &&
                    lower->cfg.nx == upper->cfg.nx && lower->cfg.ny == upper->cfg.ny && a.nz_global == b.nz_global,
                "slabs of different lattices");
        require((a.z_begin + a.z_extent) % a.nz_global == b.z_begin, "upper is not the slab above lower");
        require(lower->t == upper->t, "slabs at different time steps");
        require(a.fresh && b.fresh && (a.due & 2U) && (b.due & 1U), "no message of this cut is due");
        if (lower->cfg.device != upper->cfg.device) {
            int ok = 0;
            check_cuda(cudaDeviceCanAccessPeer(&ok, lower->cfg.device, upper->cfg.device), "cudaDeviceCanAccessPeer");
            require(ok != 0, "the slabs' devices have no peer access");
            const cudaError_t e = cudaDeviceEnablePeerAccess(upper->cfg.device, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled)
                (void)cudaGetLastError();
            else
                check_cuda(e, "cudaDeviceEnablePeerAccess");
        }
        exchange_cut(lower, upper);
    });
}

CFDX_API int cfdx_lbm_synchronize(cfdx_lbm* h) {
    return guarded([&] {
        checked(h, true);
        h->sync();
    });
}

CFDX_API int cfdx_lbm_macroscopic(cfdx_lbm* h, float* rho, float* ux, float* uy, float* uz, int where) {
    return guarded([&] {
        checked(h);
        require(rho && ux && uy && uz, "null output buffer");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t bytes = h->N * sizeof(float);
        if (where == CFDX_DEVICE) {
            check_cuda(launch_macro(h->key, h->args(), rho, ux, uy, uz, false, h->grid(), h->block(), h->stream),
                       "macroscopic kernel");
            h->sync();
            return;
        }
        if (!h->macro_scratch)
            h->macro_scratch = static_cast<float*>(device_alloc(4U * bytes, "macroscopic scratch"));
        float* s = h->macro_scratch;
        check_cuda(launch_macro(h->key, h->args(), s, s + h->N, s + 2 * h->N, s + 3 * h->N, false, h->grid(),
                                h->block(), h->stream),
                   "macroscopic kernel");
        float* outs[4] = {rho, ux, uy, uz};
        for (int k = 0; k < 4; ++k)
            check_cuda(cudaMemcpyAsync(outs[k], s + k * h->N, bytes, cudaMemcpyDeviceToHost, h->stream),
                       "cudaMemcpyAsync (macroscopic)");
        h->d2h += 4U * bytes;
        h->sync();
    });
}

CFDX_API int cfdx_lbm_macroscopic_f64(cfdx_lbm* h, double* rho, double* ux, double* uy, double* uz, int where) {
    return guarded([&] {
        checked(h);
        require(rho && ux && uy && uz, "null output buffer");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t bytes = h->N * sizeof(double);
        if (where == CFDX_DEVICE) {
            check_cuda(launch_macro(h->key, h->args(), rho, ux, uy, uz, true, h->grid(), h->block(), h->stream),
                       "macroscopic kernel");
            h->sync();
            return;
        }
        double* s = static_cast<double*>(device_alloc(4U * bytes, "macroscopic staging"));
        try {
            check_cuda(launch_macro(h->key, h->args(), s, s + h->N, s + 2 * h->N, s + 3 * h->N, true, h->grid(),
                                    h->block(), h->stream),
                       "macroscopic kernel");
            double* outs[4] = {rho, ux, uy, uz};
            for (int k = 0; k < 4; ++k)
                check_cuda(cudaMemcpyAsync(outs[k], s + k * h->N, bytes, cudaMemcpyDeviceToHost, h->stream),
                           "cudaMemcpyAsync (macroscopic)");
            h->d2h += 4U * bytes;
            h->sync();
        } catch (...) {
            scratch_free(s, h->stream);
            throw;
        }
        scratch_free(s, h->stream);
    });
}

CFDX_API int cfdx_lbm_refresh_device_macroscopic(cfdx_lbm* h, float** rho, float** ux, float** uy, float** uz) {
    return guarded([&] {
        checked(h);
        require(rho && ux && uy && uz, "null output pointer");
        if (!h->macro_scratch)
            h->macro_scratch = static_cast<float*>(device_alloc(4U * h->N * sizeof(float), "macroscopic scratch"));
        float* s = h->macro_scratch;
        check_cuda(launch_macro(h->key, h->args(), s, s + h->N, s + 2 * h->N, s + 3 * h->N, false, h->grid(),
                                h->block(), h->stream),
                   "macroscopic kernel");
        *rho = s;
        *ux = s + h->N;
        *uy = s + 2 * h->N;
        *uz = s + 3 * h->N;
    });
}

CFDX_API int cfdx_lbm_reduce(cfdx_lbm* h, double* out) {
    int nonfinite = 0;
    const int rc = guarded([&] {
        checked(h);
        require(out != nullptr, "null output");
        ensure_reduce(h);
        check_cuda(launch_reduce(h->key, h->args(), h->reduce_partials, h->reduce_blocks, h->reduce_out, h->stream),
                   "reduction kernel");
        check_cuda(cudaMemcpyAsync(h->host_reduce, h->reduce_out, sizeof(double) * kReduceFields,
                                   cudaMemcpyDeviceToHost, h->stream),
                   "cudaMemcpyAsync (reduction)");
        h->d2h += sizeof(double) * kReduceFields;
        h->sync();
        for (int k = 0; k < kReduceFields; ++k) out[k] = h->host_reduce[k];
        out[CFDX_REDUCE_KINETIC_ENERGY] *= 0.5;
        nonfinite = out[CFDX_REDUCE_NONFINITE] > 0.0;
    });
    if (rc == CFDX_OK && nonfinite) {
        g_error = "non-finite populations in " + std::to_string(static_cast<long long>(out[CFDX_REDUCE_NONFINITE])) +
                  " fluid cells";
        g_error_status = CFDX_ERR_NONFINITE;
        return CFDX_ERR_NONFINITE;
    }
    return rc;
}

CFDX_API int cfdx_lbm_checksum(cfdx_lbm* h, double* checksum) {
    double r[kReduceFields];
    if (!checksum) {
        g_error = "null output";
        g_error_status = CFDX_ERR_INVALID;
        return CFDX_ERR_INVALID;
    }
    const int rc = cfdx_lbm_reduce(h, r);
    if (rc == CFDX_OK || rc == CFDX_ERR_NONFINITE) *checksum = r[CFDX_REDUCE_MASS] + r[CFDX_REDUCE_KINETIC_ENERGY];
    return rc;
}

CFDX_API int cfdx_lbm_logical_populations(cfdx_lbm* h, float* out, int where) {
    return guarded([&] {
        checked(h);
        require(out != nullptr, "null output buffer");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t bytes = static_cast<std::size_t>(h->key.q) * h->N * sizeof(float);
        if (where == CFDX_DEVICE) {
            check_cuda(launch_logical(h->key, h->args(), out, h->grid(), h->block(), h->stream), "logical kernel");
            h->sync();
            return;
        }
        float* tmp = static_cast<float*>(device_alloc(bytes, "logical staging"));
        try {
            check_cuda(launch_logical(h->key, h->args(), tmp, h->grid(), h->block(), h->stream), "logical kernel");
            download(h, out, tmp, bytes, CFDX_HOST);
        } catch (...) {
            device_free(tmp);
            throw;
        }
        device_free(tmp);
    });
}

CFDX_API int cfdx_lbm_get_info(cfdx_lbm* h, cfdx_lbm_info* info) {
    return guarded([&] {
        require(h != nullptr && info != nullptr, "null handle or info");
        info->cells = h->N;
        info->q = h->key.q;
        info->storage = h->key.storage;
        info->time_step = h->t;
        info->population_bytes = h->f_bytes;
        std::size_t r = h->f_bytes;
        if (h->flags) r += h->N;
        if (h->local_a) r += 3U * h->N * sizeof(float);
        if (h->ns) r += h->N * sizeof(float);
        if (h->macro_scratch) r += 4U * h->N * sizeof(float);
        if (h->reduce_partials) r += sizeof(double) * kReduceFields * (static_cast<std::size_t>(h->reduce_blocks) + 1U);
        info->resident_bytes = r;
        info->host_to_device_bytes = h->h2d;
        info->device_to_host_bytes = h->d2h;
        info->synchronizations = h->syncs;
        info->fluid_flags = h->key.flags ? 1 : 0;
    });
}

CFDX_API int cfdx_lbm_stream(cfdx_lbm* h, void** stream) {
    return guarded([&] {
        require(h != nullptr && stream != nullptr, "null handle or output");
        *stream = h->stream;
    });
}

CFDX_API int cfdx_lbm_raw_populations(cfdx_lbm* h, void** ptr, std::size_t* bytes) {
    return guarded([&] {
        require(h != nullptr && ptr != nullptr && bytes != nullptr, "null handle or output");
        *ptr = h->f;
        *bytes = h->f_bytes;
    });
}

CFDX_API int cfdx_lbm_set_launch_shape(cfdx_lbm* h, int bx, int by, int variant) {
    return guarded([&] {
        checked(h);
        require(variant >= 0 && variant <= 4,
                "step kernel variant must be 0 (auto), 1 (one cell), 2 (paired) or 3 / 4 (wall-aware FP16 pairs)");
        if (bx == 0 && by == 0) {
            h->shape = LaunchShape{};
        } else {
            require(bx > 0 && by > 0 && bx * by <= 128 && (bx * by) % 32 == 0,
                    "block shape must have bx*by a multiple of 32 and at most 128");
            h->shape = LaunchShape{bx, by};
        }
        h->variant = variant;
        h->key.cells_per_thread = 1;
        if (variant == 2)
            require(h->paired_eligible(),
                    "the paired-cell kernel needs FP32/FP16 storage, an even nx, q*cells < 2^32 and block_x a "
                    "multiple of 32");
        if (variant == 3 || variant == 4)
            require(h->w2_eligible(),
                    "the wall-aware paired kernel needs FP16 storage, an even nx, q*cells < 2^32 and 128-thread "
                    "blocks");

        h->choose_variant();
        refresh_near_list(h, false);
    });
}

CFDX_API int cfdx_lbm_set_step_planes(cfdx_lbm* h, int planes) {
    return guarded([&] {
        checked(h);
        require(planes >= 0 && planes <= 4096, "planes per thread must be in [0, 4096] (0: default)");
        h->planes = static_cast<std::uint32_t>(planes);
    });
}

// ---------------------------------------------------------- checkpoints
// CFDCHK3 version 1, the layout of the reference's distributed two-grid
// checkpoint (include/cfd/solvers/lbm/distributed_pull.hpp:176-245): 8-byte
// magic "CFDCHK3\0", u32 version 1, u32 endian marker 0x01020304, u32 q, the
// global extent, brick begin and brick extent as 3 x u64 each (one brick:
// begin 0, extent = global), u64 time step, f32 tau and ax/ay/az, then q*N
// f32 populations in [d][z][y][x] order.  The populations are what each fluid
// cell gathers at the stored time step (before any moving-wall correction),
// 0 on walls; the time step's parity places them back into the in-place
// slots, so a restart continues bit for bit (FP32 storage; FP16 restarts
// re-encode the decoded values, FP64 ones keep FP32 precision).
extern "C++" {
namespace {

constexpr char kCheckpointMagic[8] = {'C', 'F', 'D', 'C', 'H', 'K', '3', '\0'};

struct File {
    std::FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

template <class T> void put(std::FILE* f, T v, const char* path) {
    if (std::fwrite(&v, sizeof v, 1, f) != 1) fail(CFDX_ERR_IO, std::string("checkpoint write failed: ") + path);
}
template <class T> T get(std::FILE* f, const char* path) {
    T v{};
    if (std::fread(&v, sizeof v, 1, f) != 1) fail(CFDX_ERR_IO, std::string("truncated checkpoint: ") + path);
    return v;
}

// The CFDCHK3 brick of a handle: global extent, begin and extent (rows of
// v), and the local cells it covers (a slab's own planes).
struct Brick {
    std::uint64_t v[3][3];
    std::size_t first_cell, cells;
};

Brick brick_of(const cfdx_lbm* h) {
    Brick b{};
    const std::uint64_t nz = h->slab.on ? h->slab.nz_global : h->cfg.nz;
    const std::uint64_t z0 = h->slab.on ? h->slab.z_begin : 0U;
    const std::uint64_t ze = h->slab.on ? h->slab.z_extent : h->cfg.nz;
    const std::uint64_t rows[3][3] = {{h->cfg.nx, h->cfg.ny, nz}, {0U, 0U, z0}, {h->cfg.nx, h->cfg.ny, ze}};
    std::memcpy(b.v, rows, sizeof rows);
    const std::size_t plane = h->cfg.nx * h->cfg.ny;
    b.first_cell = h->slab.on ? plane : 0U;
    b.cells = plane * static_cast<std::size_t>(ze);
    return b;
}

float* checkpoint_scratch(cfdx_lbm* h) {
    if (!h->macro_scratch)
        h->macro_scratch = static_cast<float*>(device_alloc(4U * h->N * sizeof(float), "macroscopic scratch"));
    return h->macro_scratch;
}

} // namespace
} // extern "C++"

CFDX_API int cfdx_lbm_checkpoint_save(cfdx_lbm* h, const char* path) {
    return guarded([&] {
        checked(h);
        require(path != nullptr, "null checkpoint path");
        File file;
        file.f = std::fopen(path, "wb");
        if (!file.f) fail(CFDX_ERR_IO, std::string("cannot open checkpoint for writing: ") + path);
        std::FILE* f = file.f;
        if (std::fwrite(kCheckpointMagic, 1, 8, f) != 8) fail(CFDX_ERR_IO, std::string("checkpoint write failed: ") + path);
        put<std::uint32_t>(f, 1U, path);
        put<std::uint32_t>(f, 0x01020304U, path);
        put<std::uint32_t>(f, static_cast<std::uint32_t>(h->key.q), path);
        const Brick brick = brick_of(h);
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) put<std::uint64_t>(f, brick.v[r][k], path);
        put<std::uint64_t>(f, h->t, path);
        put<float>(f, h->cfg.tau, path);
        put<float>(f, h->cfg.acceleration_x, path);
        put<float>(f, h->cfg.acceleration_y, path);
        put<float>(f, h->cfg.acceleration_z, path);
        float* dev = checkpoint_scratch(h);
        const std::size_t first = brick.first_cell, cells = brick.cells;
        std::vector<float> host(cells);
        for (int d = 0; d < h->key.q; ++d) {
            check_cuda(launch_slot_io(h->key, h->args(), d, dev, false, h->grid(), h->block(), h->stream),
                       "checkpoint read kernel");
            check_cuda(cudaMemcpyAsync(host.data(), dev + first, cells * sizeof(float), cudaMemcpyDeviceToHost,
                                       h->stream),
                       "cudaMemcpyAsync (checkpoint)");
            h->sync();
            h->d2h += cells * sizeof(float);
            if (std::fwrite(host.data(), sizeof(float), cells, f) != cells)
                fail(CFDX_ERR_IO, std::string("checkpoint write failed: ") + path);
        }
        if (std::fflush(f) != 0) fail(CFDX_ERR_IO, std::string("checkpoint write failed: ") + path);
    });
}

CFDX_API int cfdx_lbm_checkpoint_load(cfdx_lbm* h, const char* path) {
    return guarded([&] {
        checked(h);
        require(path != nullptr, "null checkpoint path");
        File file;
        file.f = std::fopen(path, "rb");
        if (!file.f) fail(CFDX_ERR_IO, std::string("cannot open checkpoint for reading: ") + path);
        std::FILE* f = file.f;
        char magic[8] = {0};
        if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kCheckpointMagic, 8) != 0)
            fail(CFDX_ERR_IO, "invalid checkpoint magic");
        const auto version = get<std::uint32_t>(f, path);
        const auto endian = get<std::uint32_t>(f, path);
        const auto q = get<std::uint32_t>(f, path);
        if (version != 1U || endian != 0x01020304U || q != static_cast<std::uint32_t>(h->key.q))
            fail(CFDX_ERR_IO, "unsupported checkpoint format/descriptor");
        const Brick brick = brick_of(h);
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                const auto v = get<std::uint64_t>(f, path);
                if (v != brick.v[r][k]) fail(CFDX_ERR_IO, "checkpoint decomposition does not match the lattice");
            }
        const auto t = get<std::uint64_t>(f, path);
        const float tau = get<float>(f, path), ax = get<float>(f, path), ay = get<float>(f, path),
                    az = get<float>(f, path);
        if (tau != h->cfg.tau || ax != h->cfg.acceleration_x || ay != h->cfg.acceleration_y ||
            az != h->cfg.acceleration_z)
            fail(CFDX_ERR_IO, "checkpoint LBM configuration mismatch");
        // The whole payload must be present before the lattice is touched.
        const long header = std::ftell(f);
        if (header < 0 || std::fseek(f, 0, SEEK_END) != 0) fail(CFDX_ERR_IO, std::string("cannot size checkpoint: ") + path);
        const long total = std::ftell(f);
        const unsigned long long payload = static_cast<unsigned long long>(h->key.q) * brick.cells * sizeof(float);
        if (total < 0 || static_cast<unsigned long long>(total - header) != payload)
            fail(CFDX_ERR_IO, std::string("checkpoint payload size mismatch (truncated or trailing data): ") + path);
        if (std::fseek(f, header, SEEK_SET) != 0) fail(CFDX_ERR_IO, std::string("cannot read checkpoint: ") + path);
        float* dev = checkpoint_scratch(h);
        // ghost planes of a slab stay 0: their cells are walls, which the write kernel skips
        std::vector<float> host(h->N, 0.0F);
        float* own = host.data() + brick.first_cell;
        h->adj.ready = false;
        h->t = t;
        const LbmArgs a = h->args(); // slot tables of the stored time step's parity
        for (int d = 0; d < h->key.q; ++d) {
            if (std::fread(own, sizeof(float), brick.cells, f) != brick.cells)
                fail(CFDX_ERR_IO, std::string("truncated checkpoint: ") + path);
            upload(h, dev, host.data(), h->N * sizeof(float), CFDX_HOST);
            check_cuda(launch_slot_io(h->key, a, d, dev, true, h->grid(), h->block(), h->stream),
                       "checkpoint write kernel");
        }
        h->sync();
        // Each own cell's populations now sit where its next step reads them,
        // ghost-plane slots included: no message is due.
        h->slab.due = 0;
        h->slab.fresh = false;
    });
}

CFDX_API int cfdx_lbm_set_tau(cfdx_lbm* h, float tau) {
    return guarded([&] {
        checked(h);
        require(tau > 0.5F && std::isfinite(tau), "LBM tau must be > 0.5 for positive viscosity");
        if (h->key.collision == kTRT && h->cfg.trt_tau_minus <= 0.0F)
            require(h->cfg.trt_magic > 0.0F, "TRT needs trt_magic > 0");
        h->adj.ready = false;
        h->cfg.tau = tau;
    });
}

// ------------------------------------------------------------------ adjoint
namespace {

// Grows an adjoint buffer to at least `bytes` (contents not kept).
void adjoint_buffer(void** p, std::size_t* have, std::size_t bytes, const char* what) {
    if (*have >= bytes && *p) return;
    device_free(*p);
    *p = nullptr;
    *have = 0;
    *p = device_alloc(bytes, what);
    *have = bytes;
}

// A segment of `len` steps is reversed with two levels of recompute when a
// sub-checkpoint interval 2 <= sub < len is set.
bool two_level(std::uint64_t sub, std::uint64_t len) { return sub >= 2U && sub < len; }

// Recompute frames of the reverse sweep.  One level: interval - 1 frames,
// the states inside a segment.  Two levels (sub-checkpoint interval m): the
// ceil(interval / m) - 1 sub-checkpoints of a segment, then the m - 1 states
// inside one sub-segment.  The forward pass, and the first recompute pass of
// two levels, use two of the frames as ping-pong buffers.
std::uint64_t adjoint_frames(std::uint64_t steps, std::uint32_t interval, std::uint32_t sub) {
    const std::uint64_t len = std::min<std::uint64_t>(interval, steps);
    if (!two_level(sub, len)) return std::max<std::uint64_t>(len - 1U, 2U);
    return (len + sub - 1U) / sub - 1U + std::max<std::uint64_t>(sub - 1U, 2U);
}

void adjoint_reserve(cfdx_lbm* h, std::uint64_t steps, std::uint32_t interval, std::uint32_t sub) {
    auto& A = h->adj;
    const std::uint64_t segments = (steps + interval - 1U) / interval;
    const std::uint64_t frames = adjoint_frames(steps, interval, sub);
    const std::size_t lam_es = h->key.storage == kStoreF64 ? 8U : 4U;
    const dim3 g = h->grid();
    const std::size_t blocks = static_cast<std::size_t>(g.x) * g.y * g.z;
    try {
        adjoint_buffer(&A.checkpoints, &A.checkpoint_bytes, segments * h->f_bytes, "adjoint checkpoints");
        adjoint_buffer(&A.frames, &A.frame_bytes, frames * h->f_bytes, "adjoint recompute frames");
        adjoint_buffer(&A.lam, &A.lam_bytes, static_cast<std::size_t>(h->key.q) * h->N * lam_es, "adjoint lattice");
        if (!A.grad_ns) A.grad_ns = static_cast<double*>(device_alloc(h->N * sizeof(double), "n_s gradient"));
        if (A.tau_blocks < blocks) {
            device_free(A.tau_partials);
            A.tau_partials = nullptr;
            A.tau_partials = static_cast<double*>(device_alloc(blocks * sizeof(double), "tau gradient partials"));
            A.tau_blocks = blocks;
        }
        if (!A.tau_out) A.tau_out = static_cast<double*>(device_alloc(sizeof(double), "tau gradient"));
    } catch (...) {
        release_adjoint(h);
        throw;
    }
}

// One level: state k of segment `segment` (0: its checkpoint).
void* adjoint_frame(cfdx_lbm* h, std::uint64_t segment, std::uint64_t k) {
    char* base = k == 0U ? static_cast<char*>(h->adj.checkpoints) + segment * h->f_bytes
                         : static_cast<char*>(h->adj.frames) + (k - 1U) * h->f_bytes;
    return base;
}
// Two levels: sub-checkpoint j >= 1 of the segment being reversed, and state
// r >= 1 inside its sub-segment being reversed (`nsub` sub-checkpoints per
// full segment, the checkpoint included).
void* adjoint_subcheckpoint(cfdx_lbm* h, std::uint64_t j) {
    return static_cast<char*>(h->adj.frames) + (j - 1U) * h->f_bytes;
}
void* adjoint_subframe(cfdx_lbm* h, std::uint64_t nsub, std::uint64_t r) {
    return static_cast<char*>(h->adj.frames) + (nsub - 1U + r - 1U) * h->f_bytes;
}

} // namespace

CFDX_API int cfdx_lbm_adjoint_set_subinterval(cfdx_lbm* h, std::uint32_t subinterval) {
    return guarded([&] {
        checked(h);
        require(subinterval != 1U, "a sub-checkpoint interval is 0 (one level) or at least 2");
        h->adjoint_sub = subinterval;
    });
}

CFDX_API int cfdx_lbm_adjoint_forward(cfdx_lbm* h, std::uint64_t steps, std::uint32_t interval) {
    return guarded([&] {
        checked(h);
        require(steps >= 1U && interval >= 1U, "adjoint forward needs steps >= 1 and a checkpoint interval >= 1");
        require(!h->slab.on, "the adjoint covers whole lattices, not slabs");
        require(!h->key.les, "the adjoint does not cover Smagorinsky LES (its tau depends on the populations)");
        require(!h->moving_walls, "the adjoint does not cover moving walls");
        require(h->key.narrow, "the adjoint needs q * cells < 2^32");
        h->adj.ready = false;
        adjoint_reserve(h, steps, interval, h->adjoint_sub);
        auto& A = h->adj;
        A.t0 = h->t;
        A.steps = steps;
        A.interval = interval;
        A.sub = h->adjoint_sub;
        // The forward runs the out-of-place kernel the reverse sweep
        // recomputes with, so every recomputed frame equals the forward's
        // state bit for bit.  Checkpoints and frames all keep the layout of
        // parity P0 (gather with P0's tables, scatter with P0 ^ 1's); the
        // very last step scatters into the live lattice in the layout its
        // final time step reads.
        const int es = storage_bytes(h->key.storage);
        const int P0 = static_cast<int>(A.t0 & 1U);
        const std::uint64_t t_end = A.t0 + steps;
        const dim3 g = h->grid(), b = h->block();
        check_cuda(cudaMemcpyAsync(adjoint_frame(h, 0, 0), h->f, h->f_bytes, cudaMemcpyDeviceToDevice, h->stream),
                   "cudaMemcpyAsync (adjoint checkpoint)");
        const std::uint64_t segments = (steps + interval - 1U) / interval;
        void* work[2] = {adjoint_frame(h, 0, 1), adjoint_frame(h, 0, 2)};
        void* cur = adjoint_frame(h, 0, 0);
        for (std::uint64_t s = 0; s < segments; ++s) {
            const std::uint64_t len = std::min<std::uint64_t>(interval, steps - s * interval);
            for (std::uint64_t k = 1; k <= len; ++k) {
                const bool last = s + 1U == segments && k == len;
                void* dst = last ? h->f : (k == len ? adjoint_frame(h, s + 1U, 0) : work[k & 1U]);
                const int scatter_parity = last && static_cast<int>(t_end & 1U) != P0 ? P0 : (P0 ^ 1);
                LbmArgs src = h->args_at(cur, es, P0);
                src.round_seed = h->round_seed(h->t);
                check_cuda(launch_step_oop(h->key, src, h->args_at(dst, es, scatter_parity), g, b, h->stream),
                           "adjoint forward kernel");
                cur = dst;
                ++h->t;
            }
        }
        A.t_end = h->t;
        A.ready = true;
    });
}

CFDX_API int cfdx_lbm_adjoint_backward(cfdx_lbm* h, const float* g_rho, const float* g_ux, const float* g_uy,
                                       const float* g_uz, int where, double* grad_ns, int grad_where,
                                       double* grad_tau) {
    return guarded([&] {
        checked(h);
        auto& A = h->adj;
        require(A.ready && h->t == A.t_end,
                "cfdx_lbm_adjoint_backward needs cfdx_lbm_adjoint_forward first, with no call that changes the "
                "lattice or its parameters in between");
        require(g_ux && g_uy && g_uz, "null velocity gradient");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        require(grad_where == CFDX_HOST || grad_where == CFDX_DEVICE, "grad_where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t N = h->N;
        const float *gr = g_rho, *gx = g_ux, *gy = g_uy, *gz = g_uz;
        if (where == CFDX_HOST) {
            if (!A.seed) A.seed = static_cast<float*>(device_alloc(4U * N * sizeof(float), "adjoint seed staging"));
            const float* src[4] = {g_rho, g_ux, g_uy, g_uz};
            for (int k = 0; k < 4; ++k)
                if (src[k]) upload(h, A.seed + k * N, src[k], N * sizeof(float), CFDX_HOST);
            gr = g_rho ? A.seed : nullptr;
            gx = A.seed + N;
            gy = A.seed + 2 * N;
            gz = A.seed + 3 * N;
        }
        // One tau partial per block of the adjoint grid (the launch shape may
        // have changed since the forward pass).
        const dim3 g = h->grid(), b = h->block();
        const std::size_t blocks = static_cast<std::size_t>(g.x) * g.y * g.z;
        if (A.tau_blocks < blocks) {
            device_free(A.tau_partials);
            A.tau_partials = nullptr;
            A.tau_blocks = 0;
            A.tau_partials = static_cast<double*>(device_alloc(blocks * sizeof(double), "tau gradient partials"));
            A.tau_blocks = blocks;
        }
        check_cuda(cudaMemsetAsync(A.grad_ns, 0, N * sizeof(double), h->stream), "cudaMemsetAsync");
        check_cuda(cudaMemsetAsync(A.tau_partials, 0, blocks * sizeof(double), h->stream), "cudaMemsetAsync");

        const int es = storage_bytes(h->key.storage);
        const int lam_es = h->key.storage == kStoreF64 ? 8 : 4;
        const double tau = h->cfg.tau;
        AdjointArgs X{};
        X.grad_ns = A.grad_ns;
        X.tau_partials = A.tau_partials;
        X.dwp = -1.0 / (tau * tau);
        if (h->key.collision == kBGK) {
            X.dwm = X.dwp;
        } else if (h->cfg.trt_tau_minus > 0.0F) {
            X.dwm = 0.0;
        } else {
            const double lam = h->cfg.trt_magic, q = lam + 0.5 * (tau - 0.5);
            X.dwm = lam / (q * q);
        }
        X.g_rho = gr;
        X.g_ux = gx;
        X.g_uy = gy;
        X.g_uz = gz;
        X.f = h->args();
        X.l = h->args_at(A.lam, lam_es, 1);
        check_cuda(launch_adjoint_seed(h->key, X, g, b, h->stream), "adjoint seed kernel");
        const std::uint64_t segments = (A.steps + A.interval - 1U) / A.interval;
        std::uint64_t parity = 0;
        for (std::uint64_t s = segments; s-- > 0U;) {
            const std::uint64_t ts = A.t0 + s * A.interval;
            const std::uint64_t len = std::min<std::uint64_t>(A.interval, A.t0 + A.steps - ts);
            const int P = static_cast<int>(A.t0 & 1U); // every checkpoint and frame keeps the layout of t0
            // Recompute step from state `src` (time step ts + k - 1 of the forward) into `dst`.
            const auto recompute = [&](void* src, void* dst, std::uint64_t k) -> cudaError_t {
                LbmArgs a = h->args_at(src, es, P);
                a.round_seed = h->round_seed(ts + k - 1U); // the forward's step at this time
                return launch_step_oop(h->key, a, h->args_at(dst, es, P ^ 1), g, b, h->stream);
            };
            // Adjoint step k of the segment (reading its incoming state, the state k - 1).
            const auto adjoint = [&](void* state) -> cudaError_t {
                X.f = h->args_at(state, es, P);
                X.l = h->args_at(A.lam, lam_es, static_cast<int>(parity & 1U));
                ++parity;
                return launch_adjoint_step(h->key, X, g, b, h->stream);
            };
            // the segment's recompute and adjoint steps as one graph
            enqueue_captured(h, "adjoint segment kernels", [&]() -> cudaError_t {
                cudaError_t e = cudaSuccess;
                if (!two_level(A.sub, len)) {
                    for (std::uint64_t k = 1; k < len && e == cudaSuccess; ++k)
                        e = recompute(adjoint_frame(h, s, k - 1U), adjoint_frame(h, s, k), k);
                    for (std::uint64_t k = len; k >= 1U && e == cudaSuccess; --k) e = adjoint(adjoint_frame(h, s, k - 1U));
                    return e;
                }
                // Two levels: first the sub-checkpoints (every m-th state, the
                // others in two scratch frames), then each sub-segment from the
                // last: its states from its sub-checkpoint, then its adjoint steps.
                const std::uint64_t m = A.sub, nsub = (len + m - 1U) / m;
                const std::uint64_t nsub_full = (std::min<std::uint64_t>(A.interval, A.steps) + m - 1U) / m;
                const auto start = [&](std::uint64_t j) {
                    return j == 0U ? adjoint_frame(h, s, 0) : adjoint_subcheckpoint(h, j);
                };
                void* cur = start(0);
                for (std::uint64_t k = 1; k <= (nsub - 1U) * m && e == cudaSuccess; ++k) {
                    void* dst = k % m == 0U ? adjoint_subcheckpoint(h, k / m) : adjoint_subframe(h, nsub_full, 1U + (k & 1U));
                    e = recompute(cur, dst, k);
                    cur = dst;
                }
                for (std::uint64_t j = nsub; j-- > 0U && e == cudaSuccess;) {
                    const std::uint64_t k0 = j * m, kend = std::min<std::uint64_t>(k0 + m, len);
                    const auto state = [&](std::uint64_t k) {
                        return k == k0 ? start(j) : adjoint_subframe(h, nsub_full, k - k0);
                    };
                    for (std::uint64_t k = k0 + 1U; k < kend && e == cudaSuccess; ++k) e = recompute(state(k - 1U), state(k), k);
                    for (std::uint64_t k = kend; k > k0 && e == cudaSuccess; --k) e = adjoint(state(k - 1U));
                }
                return e;
            });
        }
        check_cuda(launch_sum_partials(A.tau_partials, blocks, A.tau_out, h->stream), "adjoint tau reduction");
        if (grad_ns) {
            const cudaMemcpyKind kind = grad_where == CFDX_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
            check_cuda(cudaMemcpyAsync(grad_ns, A.grad_ns, N * sizeof(double), kind, h->stream),
                       "cudaMemcpyAsync (n_s gradient)");
            if (grad_where == CFDX_HOST) h->d2h += N * sizeof(double);
        }
        double tau_host = 0.0;
        check_cuda(cudaMemcpyAsync(&tau_host, A.tau_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                   "cudaMemcpyAsync (tau gradient)");
        h->d2h += sizeof(double);
        h->sync();
        if (grad_tau) *grad_tau = tau_host;
    });
}

CFDX_API int cfdx_lbm_adjoint_memory(cfdx_lbm* h, std::size_t* bytes) {
    return guarded([&] {
        checked(h);
        require(bytes != nullptr, "null output pointer");
        const auto& A = h->adj;
        *bytes = A.checkpoint_bytes + A.frame_bytes + A.lam_bytes + (A.grad_ns ? h->N * sizeof(double) : 0U) +
                 A.tau_blocks * sizeof(double) + (A.tau_out ? sizeof(double) : 0U) +
                 (A.seed ? 4U * h->N * sizeof(float) : 0U);
    });
}

CFDX_API int cfdx_lbm_adjoint_release(cfdx_lbm* h) {
    return guarded([&] {
        checked(h);
        if (h->stream) h->sync();
        release_adjoint(h);
    });
}

// ---------------------------------------------------------------- voxelizer
namespace {

void check_voxel_inputs(const double* tris, std::size_t count, std::size_t nx, std::size_t ny, std::size_t nz,
                        const double* lo, const double* hi, std::uint32_t z_count) {
    require(tris != nullptr && lo != nullptr && hi != nullptr, "null voxelization argument");
    // reference voxelize.cpp:5 ("invalid voxelization inputs")
    require(count > 0 && nx > 0 && ny > 0 && nz > 0 && hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2],
            "invalid voxelization inputs");
    for (int k = 0; k < 3; ++k) require(std::isfinite(lo[k]) && std::isfinite(hi[k]), "voxel grid bounds must be finite");
    for (std::size_t i = 0; i < 9 * count; ++i) require(std::isfinite(tris[i]), "triangle coordinates must be finite");
    require(nx <= (1ULL << 30) && ny <= 65535U && nz <= 0xffffffffULL && z_count >= 1U && z_count <= 65535U,
            "voxel grid exceeds launch limits");
    require(static_cast<unsigned long long>(ny) * z_count < (1ULL << 31), "voxel grid has too many rows");
    require(count <= (1ULL << 26), "too many triangles (at most 2^26 per call)");
}

void run_voxelizer(const double* tris, std::size_t count, const VoxelRequest& q, std::uint8_t* out, cudaStream_t s) {
    const char* what = "voxelizer";
    const cudaError_t e = voxelize_device(tris, count, q, out, s, &what);
    check_cuda(e, what);
}

} // namespace

CFDX_API int cfdx_voxelize(const double* triangles, std::size_t count, const cfdx_voxel_grid* grid,
                           std::uint32_t z_first, std::uint32_t z_count, std::uint8_t solid_value, std::uint8_t* out,
                           int where, int device) {
    return guarded([&] {
        require(grid != nullptr && out != nullptr, "null grid or output");
        const cfdx_voxel_grid& g = *grid;
        check_voxel_inputs(triangles, count, g.nx, g.ny, g.nz, g.minimum, g.maximum, z_count);
        require(z_first < g.nz, "z_first outside the grid");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        int devices = 0;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
            fail(CFDX_ERR_CUDA, "no CUDA device is available (the B200 engine has no CPU fallback)");
        require(device >= 0 && device < devices, "device ordinal out of range");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        VoxelRequest q{g.nx, g.ny, g.nz, {g.minimum[0], g.minimum[1], g.minimum[2]},
                       {g.maximum[0], g.maximum[1], g.maximum[2]}, z_first, z_count, solid_value, nullptr};
        const std::size_t bytes = g.nx * g.ny * static_cast<std::size_t>(z_count);
        cudaStream_t s = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        std::uint8_t* dev = where == CFDX_DEVICE ? out : nullptr;
        try {
            if (!dev) dev = static_cast<std::uint8_t*>(device_alloc(bytes, "voxel mask"));
            run_voxelizer(triangles, count, q, dev, s);
            if (where == CFDX_HOST) {
                check_cuda(cudaMemcpyAsync(out, dev, bytes, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync (mask)");
                check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            }
        } catch (...) {
            if (where == CFDX_HOST) device_free(dev);
            cudaStreamDestroy(s);
            throw;
        }
        if (where == CFDX_HOST) device_free(dev);
        cudaStreamDestroy(s);
    });
}

CFDX_API int cfdx_lbm_set_flags_surface(cfdx_lbm* h, const double* triangles, std::size_t count,
                                        const double* minimum, const double* maximum, std::uint8_t solid_value,
                                        const std::uint8_t* base_flags, int where) {
    return guarded([&] {
        checked(h);
        const std::size_t nz = h->slab.on ? h->slab.nz_global : h->cfg.nz;
        const auto planes = static_cast<std::uint32_t>(h->cfg.nz);
        check_voxel_inputs(triangles, count, h->cfg.nx, h->cfg.ny, nz, minimum, maximum, planes);
        require(solid_value >= 1U && solid_value < CFDX_MAX_WALL_IDS, "solid_value must be a wall id (1..15)");
        VoxelRequest q{h->cfg.nx, h->cfg.ny, nz, {minimum[0], minimum[1], minimum[2]},
                       {maximum[0], maximum[1], maximum[2]},
                       h->slab.on ? (h->slab.z_begin + h->slab.nz_global - 1U) % h->slab.nz_global : 0U, planes,
                       solid_value, nullptr};
        std::uint8_t* staging = static_cast<std::uint8_t*>(device_alloc(2 * h->N, "voxel staging"));
        try {
            if (base_flags) {
                upload(h, staging + h->N, base_flags, h->N, where);
                q.base = staging + h->N;
            }
            run_voxelizer(triangles, count, q, staging, h->stream);
            apply_flags(h, staging, CFDX_DEVICE);
        } catch (...) {
            device_free(staging);
            throw;
        }
        device_free(staging);
    });
}

// ------------------------------------------------------------ field export
extern "C++" {
namespace {

// Writer failures: size errors stay CFDX_ERR_INVALID, file errors become CFDX_ERR_IO.
template <class F> void as_io(F&& write) {
    try {
        write();
    } catch (const std::invalid_argument&) {
        throw;
    } catch (const std::runtime_error& e) {
        fail(CFDX_ERR_IO, e.what());
    }
}

void check_q_grid(std::size_t nx, std::size_t ny, std::size_t nz, double dx, double dy, double dz) {
    // reference visualization.cpp:124-125
    require(nx >= 3 && ny >= 3 && nz >= 3 && dx > 0.0 && dy > 0.0 && dz > 0.0, "invalid LBM Q-criterion grid");
    require(nx <= (1ULL << 30) && ny <= 65535U && nz <= 65535U, "Q-criterion grid exceeds launch limits");
}

} // namespace
} // extern "C++"

CFDX_API int cfdx_write_vtk_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, const double* scalar,
                               const double* velocity, const std::uint8_t* solid, const char* scalar_name,
                               int binary) {
    return guarded([&] {
        require(path != nullptr && scalar != nullptr, "null path or scalar field");
        as_io([&] { write_vtk_3d(path, nx, ny, nz, scalar, velocity, solid, scalar_name ? scalar_name : "field",
                                 binary != 0); });
    });
}

CFDX_API int cfdx_write_json_state_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz,
                                      std::uint64_t step, const double* scalar, const std::uint8_t* solid,
                                      const char* scalar_name) {
    return guarded([&] {
        require(path != nullptr && scalar != nullptr, "null path or scalar field");
        as_io([&] { write_json_state_3d(path, nx, ny, nz, step, scalar, solid, scalar_name ? scalar_name : "field"); });
    });
}

CFDX_API int cfdx_q_criterion(const double* velocity, std::size_t nx, std::size_t ny, std::size_t nz, double dx,
                              double dy, double dz, double* q, int where, int device) {
    return guarded([&] {
        require(velocity != nullptr && q != nullptr, "null velocity or output");
        check_q_grid(nx, ny, nz, dx, dy, dz);
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        int devices = 0;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
            fail(CFDX_ERR_CUDA, "no CUDA device is available (the B200 engine has no CPU fallback)");
        require(device >= 0 && device < devices, "device ordinal out of range");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        const std::size_t n = nx * ny * nz;
        cudaStream_t s = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        double* staging = nullptr;
        try {
            const double* u = velocity;
            double* out = q;
            if (where == CFDX_HOST) {
                void* p = nullptr;
                check_cuda(scratch_alloc(&p, 4 * n * sizeof(double), s), "Q-criterion staging");
                staging = static_cast<double*>(p);
                check_cuda(cudaMemcpyAsync(staging, velocity, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s),
                           "cudaMemcpyAsync (velocity)");
                u = staging;
                out = staging + 3 * n;
            }
            check_cuda(launch_q_criterion(u, u + 1, u + 2, true, 3, nx, ny, nz, dx, dy, dz, out, s),
                       "Q-criterion kernel");
            if (where == CFDX_HOST)
                check_cuda(cudaMemcpyAsync(q, out, n * sizeof(double), cudaMemcpyDeviceToHost, s),
                           "cudaMemcpyAsync (Q)");
            check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        } catch (...) {
            scratch_free(staging, s);
            cudaStreamDestroy(s);
            throw;
        }
        scratch_free(staging, s);
        cudaStreamDestroy(s);
    });
}

CFDX_API int cfdx_lbm_q_criterion(cfdx_lbm* h, double dx, double dy, double dz, double* q, int where) {
    return guarded([&] {
        checked(h);
        require(q != nullptr, "null output");
        require(!h->slab.on, "the Q-criterion of a slab needs its neighbours' velocities: gather the whole lattice");
        check_q_grid(h->cfg.nx, h->cfg.ny, h->cfg.nz, dx, dy, dz);
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t n = h->N;
        // rho | ux | uy | uz as cfdx_lbm_macroscopic_f64 reports them, then Q
        void* p = nullptr;
        check_cuda(scratch_alloc(&p, (where == CFDX_HOST ? 5 : 4) * n * sizeof(double), h->stream),
                   "Q-criterion staging");
        double* s = static_cast<double*>(p);
        try {
            check_cuda(launch_macro(h->key, h->args(), s, s + n, s + 2 * n, s + 3 * n, true, h->grid(), h->block(),
                                    h->stream),
                       "macroscopic kernel");
            double* out = where == CFDX_HOST ? s + 4 * n : q;
            check_cuda(launch_q_criterion(s + n, s + 2 * n, s + 3 * n, true, 1, h->cfg.nx, h->cfg.ny, h->cfg.nz, dx,
                                          dy, dz, out, h->stream),
                       "Q-criterion kernel");
            if (where == CFDX_HOST) {
                check_cuda(cudaMemcpyAsync(q, out, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                           "cudaMemcpyAsync (Q)");
                h->d2h += n * sizeof(double);
            }
            h->sync();
        } catch (...) {
            device_free(s);
            throw;
        }
        device_free(s);
    });
}

// ------------------------------------------------- resident thermal lattice
// The resident solvers index cells with 32-bit integers.
constexpr std::size_t kResidentMaxCells = 0xFFFF0000ULL;

struct cfdx_thermal {
    cfdx_lbm* flow = nullptr; // borrowed: its device and stream
    ThermalGrid grid{};
    float tau = 0.0F, omega = 0.0F;
    float* g = nullptr;
    float* next = nullptr;
    float* scalar = nullptr;     // temperature scratch, lazily allocated
    double* partials = nullptr;  // FP64 total: per-block sums, then the total
    double* host_total = nullptr; // pinned
    int blocks = 0;
    std::uint64_t h2d = 0, d2h = 0;
};

namespace {

cfdx_thermal* checked_thermal(cfdx_thermal* t) {
    if (!t || !t->flow) throw std::invalid_argument("null cfdx_thermal handle");
    t->flow->set_device();
    return t;
}

void release_thermal(cfdx_thermal* t) {
    if (!t) return;
    if (t->flow) {
        cudaSetDevice(t->flow->cfg.device);
        cudaStreamSynchronize(t->flow->stream);
    }
    device_free(t->g);
    device_free(t->next);
    device_free(t->scalar);
    device_free(t->partials);
    if (t->host_total) cudaFreeHost(t->host_total);
    delete t;
}

float* thermal_scalar(cfdx_thermal* t) {
    if (!t->scalar) t->scalar = static_cast<float*>(device_alloc(t->grid.cells * sizeof(float), "temperature scratch"));
    check_cuda(launch_thermal_scalar(t->g, t->grid, t->scalar, t->flow->stream), "temperature kernel");
    return t->scalar;
}

} // namespace

CFDX_API int cfdx_thermal_create(cfdx_lbm* flow, float diffusivity, cfdx_thermal** out, char* error,
                                 std::size_t cap) {
    cfdx_thermal* t = nullptr;
    const int rc = guarded([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        checked(flow);
        require(!flow->slab.on, "the resident thermal lattice covers whole lattices, not slabs");
        // reference resident_multiphysics_sycl.hpp:64-66
        require(diffusivity > 0.0F && std::isfinite(diffusivity), "invalid resident thermal lattice");
        require(flow->N <= kResidentMaxCells, "resident thermal lattices hold at most 2^32 - 2^16 cells");
        t = new cfdx_thermal();
        t->flow = flow;
        t->grid = ThermalGrid{static_cast<std::uint32_t>(flow->cfg.nx), static_cast<std::uint32_t>(flow->cfg.ny),
                              static_cast<std::uint32_t>(flow->cfg.nz), static_cast<std::uint32_t>(flow->N)};
        t->tau = 0.5F + 4.0F * diffusivity;
        t->omega = 1.0F / t->tau;
        const std::size_t bytes = 7U * flow->N * sizeof(float);
        t->g = static_cast<float*>(device_alloc(bytes, "thermal lattice"));
        t->next = static_cast<float*>(device_alloc(bytes, "thermal lattice"));
        t->blocks = static_cast<int>(std::min<std::size_t>(592U, (7U * flow->N + 255U) / 256U));
        t->partials = static_cast<double*>(device_alloc((static_cast<std::size_t>(t->blocks) + 1U) * sizeof(double),
                                                        "thermal reduction scratch"));
        check_cuda(cudaMallocHost(&t->host_total, sizeof(double)), "cudaMallocHost");
        check_cuda(launch_thermal_uniform(t->g, t->grid, 0.0F, flow->stream), "thermal init kernel");
        flow->sync();
        *out = t;
    });
    if (rc != CFDX_OK) {
        release_thermal(t);
        copy_error(error, cap, g_error);
    }
    return rc;
}

CFDX_API int cfdx_thermal_destroy(cfdx_thermal* t) {
    return guarded([&] { release_thermal(t); });
}

CFDX_API int cfdx_thermal_init_uniform(cfdx_thermal* t, float temperature) {
    return guarded([&] {
        checked_thermal(t);
        require(std::isfinite(temperature), "thermal state must be finite");
        check_cuda(launch_thermal_uniform(t->g, t->grid, temperature, t->flow->stream), "thermal init kernel");
    });
}

CFDX_API int cfdx_thermal_init_field(cfdx_thermal* t, const float* temperature, int where) {
    return guarded([&] {
        checked_thermal(t);
        require(temperature != nullptr, "null temperature field");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t bytes = t->grid.cells * sizeof(float);
        const float* src = temperature;
        if (where == CFDX_HOST) {
            float* s = thermal_scalar(t); // scratch, overwritten below
            check_cuda(cudaMemcpyAsync(s, temperature, bytes, cudaMemcpyHostToDevice, t->flow->stream),
                       "cudaMemcpyAsync (temperature)");
            t->h2d += bytes;
            src = s;
        }
        check_cuda(launch_thermal_field(t->g, t->grid, src, t->flow->stream), "thermal init kernel");
        if (where == CFDX_HOST) t->flow->sync();
    });
}

CFDX_API int cfdx_thermal_step(cfdx_thermal* t, const float* ux, const float* uy, const float* uz,
                               std::uint64_t count) {
    return guarded([&] {
        checked_thermal(t);
        require(ux != nullptr && uy != nullptr && uz != nullptr, "null velocity field");
        for (std::uint64_t k = 0; k < count; ++k) {
            check_cuda(launch_thermal_step(t->g, t->next, t->grid, ux, uy, uz, t->omega, t->flow->stream),
                       "thermal step kernel");
            std::swap(t->g, t->next);
        }
    });
}

CFDX_API int cfdx_thermal_refresh_device_scalar(cfdx_thermal* t, float** temperature) {
    return guarded([&] {
        checked_thermal(t);
        require(temperature != nullptr, "null output pointer");
        *temperature = thermal_scalar(t);
    });
}

CFDX_API int cfdx_thermal_temperature(cfdx_thermal* t, float* out, int where) {
    return guarded([&] {
        checked_thermal(t);
        require(out != nullptr, "null output buffer");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t bytes = t->grid.cells * sizeof(float);
        float* s = thermal_scalar(t);
        check_cuda(cudaMemcpyAsync(out, s, bytes, where == CFDX_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                   t->flow->stream),
                   "cudaMemcpyAsync (temperature)");
        if (where == CFDX_HOST) t->d2h += bytes;
        t->flow->sync();
    });
}

CFDX_API int cfdx_thermal_add_boussinesq(cfdx_thermal* t, float* ax, float* ay, float* az, float t_ref, float beta,
                                         float gx, float gy, float gz) {
    return guarded([&] {
        checked_thermal(t);
        require(ax != nullptr && ay != nullptr && az != nullptr, "null acceleration field");
        // reference resident_multiphysics_sycl.hpp:141-145
        require(std::isfinite(t_ref) && std::isfinite(beta) && std::isfinite(gx) && std::isfinite(gy) &&
                    std::isfinite(gz),
                "invalid resident Boussinesq coupling");
        if (!t->scalar)
            t->scalar = static_cast<float*>(device_alloc(t->grid.cells * sizeof(float), "temperature scratch"));
        check_cuda(launch_thermal_boussinesq(t->g, t->grid, t->scalar, ax, ay, az, t_ref, beta, gx, gy, gz,
                                             t->flow->stream),
                   "Boussinesq kernel");
    });
}

CFDX_API int cfdx_thermal_total(cfdx_thermal* t, double* total) {
    return guarded([&] {
        checked_thermal(t);
        require(total != nullptr, "null output");
        double* out = t->partials + t->blocks;
        check_cuda(launch_thermal_total(t->g, t->grid, t->partials, t->blocks, out, t->flow->stream),
                   "thermal total kernel");
        check_cuda(cudaMemcpyAsync(t->host_total, out, sizeof(double), cudaMemcpyDeviceToHost, t->flow->stream),
                   "cudaMemcpyAsync (thermal total)");
        t->flow->sync();
        *total = *t->host_total;
    });
}

CFDX_API int cfdx_thermal_info(cfdx_thermal* t, std::size_t* resident_bytes, std::uint64_t* host_to_device,
                               std::uint64_t* device_to_host) {
    return guarded([&] {
        require(t != nullptr && resident_bytes && host_to_device && device_to_host, "null handle or output");
        *resident_bytes = 14U * static_cast<std::size_t>(t->grid.cells) * sizeof(float) +
                          (t->scalar ? t->grid.cells * sizeof(float) : 0U) +
                          (static_cast<std::size_t>(t->blocks) + 1U) * sizeof(double);
        *host_to_device = t->h2d;
        *device_to_host = t->d2h;
    });
}

// ------------------------------------------------- resident free surface
struct cfdx_surface {
    cfdx_lbm* flow = nullptr; // borrowed: its device and stream
    ThermalGrid grid{};
    float* fill = nullptr;
    float* next = nullptr;
    float* geometry = nullptr;   // normals x | y | z | curvature
    double* partials = nullptr;  // FP64 volume: per-block sums, then the total
    double* host_total = nullptr; // pinned
    int blocks = 0;
    std::uint64_t h2d = 0, d2h = 0;
};

// ------------------------------------------------- resident particles
struct cfdx_particles {
    cfdx_lbm* flow = nullptr;
    ThermalGrid grid{};
    std::uint32_t count = 0;
    float* state = nullptr; // x | y | z | vx | vy | vz | mass | response, count floats each
    std::uint64_t h2d = 0, d2h = 0;
};

// ------------------------------------------------- resident diagnostics
struct cfdx_diagnostics {
    cfdx_lbm* flow = nullptr;
    ThermalGrid grid{};
    float* q = nullptr;
};

extern "C++" {
namespace {

// the resident solvers cover whole lattices of at least `minimum` cells per axis
ThermalGrid resident_grid(cfdx_lbm* flow, std::size_t minimum, const char* what) {
    checked(flow);
    require(!flow->slab.on, (std::string(what) + " covers whole lattices, not slabs").c_str());
    require(flow->cfg.nx >= minimum && flow->cfg.ny >= minimum && flow->cfg.nz >= minimum,
            (std::string("invalid ") + what + " lattice").c_str());
    require(flow->N <= kResidentMaxCells, (std::string(what) + " lattices hold at most 2^32 - 2^16 cells").c_str());
    return ThermalGrid{static_cast<std::uint32_t>(flow->cfg.nx), static_cast<std::uint32_t>(flow->cfg.ny),
                       static_cast<std::uint32_t>(flow->cfg.nz), static_cast<std::uint32_t>(flow->N)};
}

template <class H> H* checked_resident(H* h, const char* what) {
    if (!h || !h->flow) throw std::invalid_argument(std::string("null ") + what + " handle");
    h->flow->set_device();
    return h;
}

template <class H> void sync_flow(H* h) {
    if (h && h->flow) {
        cudaSetDevice(h->flow->cfg.device);
        cudaStreamSynchronize(h->flow->stream);
    }
}

void release_surface(cfdx_surface* s) {
    if (!s) return;
    sync_flow(s);
    device_free(s->fill);
    device_free(s->next);
    device_free(s->geometry);
    device_free(s->partials);
    if (s->host_total) cudaFreeHost(s->host_total);
    delete s;
}

void release_particles(cfdx_particles* p) {
    if (!p) return;
    sync_flow(p);
    device_free(p->state);
    delete p;
}

void release_diagnostics(cfdx_diagnostics* d) {
    if (!d) return;
    sync_flow(d);
    device_free(d->q);
    delete d;
}

void require_velocity(const float* ux, const float* uy, const float* uz) {
    require(ux != nullptr && uy != nullptr && uz != nullptr, "null velocity field");
}

void require_acceleration(const float* ax, const float* ay, const float* az) {
    require(ax != nullptr && ay != nullptr && az != nullptr, "null acceleration field");
}

// normals and curvature of the current fill (reference resident_multiphysics_sycl.hpp:269-298)
void surface_geometry(cfdx_surface* s) {
    check_cuda(launch_fill_geometry(s->fill, s->geometry, s->grid, s->flow->stream), "free-surface geometry kernel");
}

} // namespace
} // extern "C++"

CFDX_API int cfdx_surface_create(cfdx_lbm* flow, cfdx_surface** out, char* error, std::size_t cap) {
    cfdx_surface* s = nullptr;
    const int rc = guarded([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        // reference resident_multiphysics_sycl.hpp:204-206
        const ThermalGrid grid = resident_grid(flow, 2U, "resident free-surface");
        s = new cfdx_surface();
        s->flow = flow;
        s->grid = grid;
        const std::size_t bytes = flow->N * sizeof(float);
        s->fill = static_cast<float*>(device_alloc(bytes, "free-surface fill"));
        s->next = static_cast<float*>(device_alloc(bytes, "free-surface fill"));
        s->geometry = static_cast<float*>(device_alloc(4U * bytes, "free-surface geometry"));
        s->blocks = static_cast<int>(std::min<std::size_t>(592U, (flow->N + 255U) / 256U));
        s->partials = static_cast<double*>(device_alloc((static_cast<std::size_t>(s->blocks) + 1U) * sizeof(double),
                                                        "free-surface reduction scratch"));
        check_cuda(cudaMallocHost(&s->host_total, sizeof(double)), "cudaMallocHost");
        check_cuda(launch_fill_uniform(s->fill, s->grid, 0.0F, flow->stream), "free-surface init kernel");
        flow->sync();
        *out = s;
    });
    if (rc != CFDX_OK) {
        release_surface(s);
        copy_error(error, cap, g_error);
    }
    return rc;
}

CFDX_API int cfdx_surface_destroy(cfdx_surface* s) {
    return guarded([&] { release_surface(s); });
}

CFDX_API int cfdx_surface_init_uniform(cfdx_surface* s, float fill) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        // reference resident_multiphysics_sycl.hpp:223-224
        require(fill >= 0.0F && fill <= 1.0F, "free-surface fill must be in [0,1]");
        check_cuda(launch_fill_uniform(s->fill, s->grid, fill, s->flow->stream), "free-surface init kernel");
    });
}

CFDX_API int cfdx_surface_init_half_space_x(cfdx_surface* s, float interface_x) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require(std::isfinite(interface_x), "invalid free-surface interface position");
        check_cuda(launch_fill_half_space_x(s->fill, s->grid, interface_x, s->flow->stream),
                   "free-surface init kernel");
    });
}

CFDX_API int cfdx_surface_init_field(cfdx_surface* s, const float* fill, int where) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require(fill != nullptr, "null fill field");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        const std::size_t bytes = s->grid.cells * sizeof(float);
        if (where == CFDX_HOST) {
            for (std::size_t n = 0; n < s->grid.cells; ++n)
                require(fill[n] >= 0.0F && fill[n] <= 1.0F, "free-surface fill must be in [0,1]");
            s->h2d += bytes;
        }
        check_cuda(cudaMemcpyAsync(s->fill, fill, bytes,
                                   where == CFDX_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                   s->flow->stream),
                   "cudaMemcpyAsync (fill)");
        if (where == CFDX_HOST) s->flow->sync();
    });
}

CFDX_API int cfdx_surface_advect(cfdx_surface* s, const float* ux, const float* uy, const float* uz, float dt) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require_velocity(ux, uy, uz);
        // reference resident_multiphysics_sycl.hpp:238-239
        require(dt > 0.0F, "invalid resident free-surface advection");
        check_cuda(launch_fill_advect(s->fill, s->next, s->grid, ux, uy, uz, dt, s->flow->stream),
                   "free-surface advection kernel");
        std::swap(s->fill, s->next);
    });
}

CFDX_API int cfdx_surface_device_fill(cfdx_surface* s, float** fill) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require(fill != nullptr, "null output pointer");
        *fill = s->fill;
    });
}

CFDX_API int cfdx_surface_refresh_geometry(cfdx_surface* s, float** geometry) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        surface_geometry(s);
        if (geometry) *geometry = s->geometry;
    });
}

CFDX_API int cfdx_surface_add_tension(cfdx_surface* s, float* ax, float* ay, float* az, float surface_tension,
                                      float density) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require_acceleration(ax, ay, az);
        // reference resident_multiphysics_sycl.hpp:302-304
        require(surface_tension >= 0.0F && density > 0.0F && std::isfinite(surface_tension) &&
                    std::isfinite(density),
                "invalid resident surface-tension coupling");
        surface_geometry(s);
        check_cuda(launch_surface_tension(s->fill, s->geometry + 3U * static_cast<std::size_t>(s->grid.cells),
                                          s->grid, ax, ay, az, surface_tension, density, s->flow->stream),
                   "surface-tension kernel");
    });
}

CFDX_API int cfdx_surface_volume(cfdx_surface* s, double* volume) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require(volume != nullptr, "null output");
        double* out = s->partials + s->blocks;
        check_cuda(launch_sum_floats(s->fill, s->grid.cells, s->partials, s->blocks, out, s->flow->stream),
                   "free-surface volume kernel");
        check_cuda(cudaMemcpyAsync(s->host_total, out, sizeof(double), cudaMemcpyDeviceToHost, s->flow->stream),
                   "cudaMemcpyAsync (volume)");
        s->flow->sync();
        *volume = *s->host_total;
    });
}

CFDX_API int cfdx_surface_fill(cfdx_surface* s, float* out, int which, int where) {
    return guarded([&] {
        checked_resident(s, "cfdx_surface");
        require(out != nullptr, "null output buffer");
        require(where == CFDX_HOST || where == CFDX_DEVICE, "where must be CFDX_HOST or CFDX_DEVICE");
        require(which >= 0 && which <= 4, "which must be 0 (fill) or 1-4 (normal x, y, z, curvature)");
        const std::size_t bytes = s->grid.cells * sizeof(float);
        const float* src = which == 0 ? s->fill : s->geometry + (static_cast<std::size_t>(which) - 1U) * s->grid.cells;
        check_cuda(cudaMemcpyAsync(out, src, bytes, where == CFDX_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                   s->flow->stream),
                   "cudaMemcpyAsync (fill)");
        if (where == CFDX_HOST) s->d2h += bytes;
        s->flow->sync();
    });
}

CFDX_API int cfdx_surface_info(cfdx_surface* s, std::size_t* resident_bytes, std::uint64_t* host_to_device,
                               std::uint64_t* device_to_host) {
    return guarded([&] {
        require(s != nullptr && resident_bytes && host_to_device && device_to_host, "null handle or output");
        *resident_bytes = 6U * static_cast<std::size_t>(s->grid.cells) * sizeof(float) +
                          (static_cast<std::size_t>(s->blocks) + 1U) * sizeof(double);
        *host_to_device = s->h2d;
        *device_to_host = s->d2h;
    });
}

CFDX_API int cfdx_particles_create(cfdx_lbm* flow, std::size_t count, cfdx_particles** out, char* error,
                                   std::size_t cap) {
    cfdx_particles* p = nullptr;
    const int rc = guarded([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        // reference resident_multiphysics_sycl.hpp:326-329
        const ThermalGrid grid = resident_grid(flow, 2U, "resident particle");
        require(count <= (std::size_t{1} << 28), "too many resident particles");
        p = new cfdx_particles();
        p->flow = flow;
        p->grid = grid;
        p->count = static_cast<std::uint32_t>(count);
        if (count) p->state = static_cast<float*>(device_alloc(8U * count * sizeof(float), "particle state"));
        *out = p;
    });
    if (rc != CFDX_OK) {
        release_particles(p);
        copy_error(error, cap, g_error);
    }
    return rc;
}

CFDX_API int cfdx_particles_destroy(cfdx_particles* p) {
    return guarded([&] { release_particles(p); });
}

CFDX_API int cfdx_particles_upload(cfdx_particles* p, const double* particles, std::size_t count) {
    return guarded([&] {
        checked_resident(p, "cfdx_particles");
        // reference resident_multiphysics_sycl.hpp:337-344
        require(count == p->count, "resident particle count mismatch");
        require(particles != nullptr || count == 0U, "null particle array");
        std::vector<float> host(8U * count);
        for (std::size_t i = 0; i < count; ++i) {
            const double* q = particles + 8U * i;
            require(q[6] > 0.0 && q[7] > 0.0, "particle mass and response time must be positive");
            for (std::size_t k = 0; k < 8U; ++k) host[k * count + i] = static_cast<float>(q[k]);
        }
        if (count) {
            check_cuda(cudaMemcpyAsync(p->state, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice,
                                       p->flow->stream),
                       "cudaMemcpyAsync (particles)");
            p->flow->sync();
            p->h2d += host.size() * sizeof(float);
        }
    });
}

CFDX_API int cfdx_particles_download(cfdx_particles* p, double* particles, std::size_t count) {
    return guarded([&] {
        checked_resident(p, "cfdx_particles");
        require(count == p->count, "resident particle count mismatch");
        require(particles != nullptr || count == 0U, "null particle array");
        std::vector<float> host(8U * count);
        if (count) {
            check_cuda(cudaMemcpyAsync(host.data(), p->state, host.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                       p->flow->stream),
                       "cudaMemcpyAsync (particles)");
            p->flow->sync();
            p->d2h += host.size() * sizeof(float);
        }
        for (std::size_t i = 0; i < count; ++i)
            for (std::size_t k = 0; k < 8U; ++k) particles[8U * i + k] = static_cast<double>(host[k * count + i]);
    });
}

CFDX_API int cfdx_particles_device_state(cfdx_particles* p, float** state) {
    return guarded([&] {
        checked_resident(p, "cfdx_particles");
        require(state != nullptr, "null output pointer");
        *state = p->state;
    });
}

CFDX_API int cfdx_particles_advance(cfdx_particles* p, const float* ux, const float* uy, const float* uz, float* ax,
                                    float* ay, float* az, float dt, int two_way, float gx, float gy, float gz) {
    return guarded([&] {
        checked_resident(p, "cfdx_particles");
        require_velocity(ux, uy, uz);
        if (two_way) require_acceleration(ax, ay, az);
        // reference resident_multiphysics_sycl.hpp:351-352
        require(dt > 0.0F && std::isfinite(dt), "invalid resident particle coupling");
        require(std::isfinite(gx) && std::isfinite(gy) && std::isfinite(gz), "invalid resident particle gravity");
        check_cuda(launch_particles_advance(p->state, p->count, p->grid, ux, uy, uz, ax, ay, az, dt, two_way != 0, gx,
                                            gy, gz, p->flow->stream),
                   "particle kernel");
    });
}

CFDX_API int cfdx_particles_info(cfdx_particles* p, std::size_t* resident_bytes, std::uint64_t* host_to_device,
                                 std::uint64_t* device_to_host) {
    return guarded([&] {
        require(p != nullptr && resident_bytes && host_to_device && device_to_host, "null handle or output");
        *resident_bytes = 8U * static_cast<std::size_t>(p->count) * sizeof(float);
        *host_to_device = p->h2d;
        *device_to_host = p->d2h;
    });
}

CFDX_API int cfdx_diagnostics_create(cfdx_lbm* flow, cfdx_diagnostics** out, char* error, std::size_t cap) {
    cfdx_diagnostics* d = nullptr;
    const int rc = guarded([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        // reference resident_multiphysics_sycl.hpp:389-392
        const ThermalGrid grid = resident_grid(flow, 3U, "Q-criterion (at least 3x3x3)");
        d = new cfdx_diagnostics();
        d->flow = flow;
        d->grid = grid;
        d->q = static_cast<float*>(device_alloc(flow->N * sizeof(float), "Q-criterion field"));
        *out = d;
    });
    if (rc != CFDX_OK) {
        release_diagnostics(d);
        copy_error(error, cap, g_error);
    }
    return rc;
}

CFDX_API int cfdx_diagnostics_destroy(cfdx_diagnostics* d) {
    return guarded([&] { release_diagnostics(d); });
}

CFDX_API int cfdx_diagnostics_q_criterion(cfdx_diagnostics* d, const float* ux, const float* uy, const float* uz,
                                          float** q) {
    return guarded([&] {
        checked_resident(d, "cfdx_diagnostics");
        require_velocity(ux, uy, uz);
        require(q != nullptr, "null output pointer");
        check_cuda(launch_resident_q(ux, uy, uz, d->grid, d->q, d->flow->stream), "Q-criterion kernel");
        *q = d->q;
    });
}

CFDX_API int cfdx_diagnostics_info(cfdx_diagnostics* d, std::size_t* resident_bytes) {
    return guarded([&] {
        require(d != nullptr && resident_bytes != nullptr, "null handle or output");
        *resident_bytes = static_cast<std::size_t>(d->grid.cells) * sizeof(float);
    });
}

CFDX_API int cfdx_lbm_debug_slot_audit(cfdx_lbm* h, int parity, cfdx_slot_audit* out) {
    std::uint32_t* counters = nullptr;
    AuditCounts* counts = nullptr;
    const int rc = guarded([&] {
        checked(h);
        require(out != nullptr, "null output");
        require(parity == 0 || parity == 1, "parity must be 0 or 1");
        const std::size_t slots = static_cast<std::size_t>(h->key.q) * h->N;
        require(slots <= (std::size_t{1} << 28), "the slot audit takes lattices of at most 2^28 slots");
        counters =
            static_cast<std::uint32_t*>(device_alloc((5U * slots + 1U) * sizeof(std::uint32_t), "slot audit counters"));
        counts = static_cast<AuditCounts*>(device_alloc(sizeof(AuditCounts), "slot audit counts"));
        const LbmArgs a = h->args_at(counters, static_cast<int>(sizeof(std::uint32_t)), parity);
        check_cuda(launch_slot_audit(h->key, a, counters, h->grid(), h->block(), counts, h->stream), "slot audit");
        AuditCounts host{};
        check_cuda(cudaMemcpyAsync(&host, counts, sizeof host, cudaMemcpyDeviceToHost, h->stream),
                   "cudaMemcpyAsync (slot audit)");
        h->sync();
        *out = cfdx_slot_audit{slots,          host.touched,    host.read_twice, host.written_twice,
                               host.read_only, host.write_only, host.foreign,    host.out_of_range};
    });
    device_free(counters);
    device_free(counts);
    return rc;
}

CFDX_API int cfdx_debug_audit_classify(uint32_t reads, uint32_t writes, uint32_t lowest_reader,
                                       uint32_t highest_reader, uint32_t writer, unsigned* classes) {
    return guarded([&] {
        require(classes != nullptr, "null output");
        *classes = audit_classify(reads, writes, lowest_reader, highest_reader, writer);
    });
}

CFDX_API int cfdx_release_scratch(int device) {
    return guarded([&] {
        int devices = 0;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
            fail(CFDX_ERR_CUDA, "no CUDA device is available (the B200 engine has no CPU fallback)");
        require(device >= 0 && device < devices, "device ordinal out of range");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        check_cuda(scratch_release(device), "cudaMemPoolTrimTo");
    });
}

CFDX_API int cfdx_debug_fail_allocations(int count) {
    g_fail_allocations.store(count > 0 ? count : 0);
    return CFDX_OK;
}

CFDX_API int cfdx_lbm_debug_force_wide_slots(cfdx_lbm* h, int wide) {
    return guarded([&] {
        checked(h);
        h->force_wide = wide != 0;
        if (h->force_wide) h->variant = h->variant == 1 ? 1 : 0; // the paired kernels need 32-bit offsets
        h->choose_variant();
        refresh_near_list(h, false);
    });
}

CFDX_API int cfdx_debug_retry_allocations(int count, unsigned long long* retries) {
    if (count >= 0) g_retry_allocations.store(count);
    if (retries) *retries = g_allocation_retries.load();
    return CFDX_OK;
}

} // extern "C"
