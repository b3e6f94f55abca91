// Launch arguments shared by the host dispatcher and the device kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cfdx {

constexpr int kMaxWallIds = 16;

// Internal per-cell flag byte, derived on the device from the caller's flags
// (0 fluid, 1 stationary wall, 2..15 moving wall id):
//   bits 0-3  wall id (0 = fluid)
//   bit 6     fluid cell with a moving-wall neighbour
//   bit 7     fluid cell with at least one wall neighbour
constexpr std::uint8_t kFlagTypeMask = 0x0f;
constexpr std::uint8_t kFlagNearMoving = 0x40;
constexpr std::uint8_t kFlagNearWall = 0x80;

enum Storage : int { kStoreF32 = 0, kStoreF64 = 1, kStoreF16S = 2 };
enum Collision : int { kBGK = 0, kTRT = 1 };

// Cell indices are 32-bit: n = (z*ny + y)*nx + x < 2^32 for every lattice
// that fits in HBM.  Population slots are addressed through per-parity base
// pointers held in the parameter bank, so the kernels carry no [q][N]
// offsets and no parity selects in registers:
//   rest     base of direction 0
//   pa[p]    base of the slot pair p reads at the neighbour nb = n + c_{2p+2}
//            (direction 2p+1 at even parity, 2p+2 at odd parity)
//   pb[p]    base of the slot pair p reads at the cell itself
//            (direction 2p+2 at even parity, 2p+1 at odd parity)
//   fd[d]    base of direction d (parity-free layouts: logical dumps, init)
//   base, rest_off, pa_off[p], pb_off[p]: the same slots as element offsets
//            from one base pointer (valid when q*N < 2^32; used by the
//            paired-cell step kernel)
struct LbmArgs {
    void* rest;
    void* pa[13];
    void* pb[13];
    void* fd[27];
    void* base;
    std::uint32_t rest_off;
    std::uint32_t pa_off[13];
    std::uint32_t pb_off[13];
    const std::uint8_t* flags; // internal flags or nullptr
    // Per fluid cell next to a wall: bit 2p set when direction 2p+1's source
    // n + c_{2p+2} is a wall, bit 2p+1 when direction 2p+2's source n + c_{2p+1}
    // is (computed once with the flags; nullptr without flags).
    const std::uint32_t* wall_mask;
    const float* ax_field;     // per-cell acceleration components or nullptr
    const float* ay_field;
    const float* az_field;
    const float* ns;           // N gray-LBM solid fractions or nullptr
    std::uint32_t nx, ny, nz;
    std::uint32_t N;
    int odd;                   // parity of the time step being executed / read
    int has_force;             // uniform or per-cell acceleration present
    double tau;                // base symmetric relaxation time
    double omega_minus;        // antisymmetric rate when fixed (> 0), else from magic / = omega+
    double trt_magic;
    double les_k;              // Smagorinsky K (0 = off)
    double ax, ay, az;         // uniform acceleration
    // FP32 copies of the parameters above for the FP32/FP16 kernels (no
    // double-to-float conversion per thread) and the omega- rule as an int:
    // 1 fixed (omega_minus), 0 TRT magic, -1 BGK.
    float tau_f, omega_minus_f, trt_magic_f, les_k_f, ax_f, ay_f, az_f;
    int minus_mode;
    float wall_u[kMaxWallIds][3];
    float scale[27];           // FP16S per-direction scale
    float inv_scale[27];
    // FP16S store rounding: the rounding bits of cell n's stores derive from
    // hash(n ^ round_seed) & round_mask, plus round_add (stochastic: mask ~0,
    // add 0, seed per step; nearest: mask 0, add = half a step in each field).
    std::uint32_t round_seed;
    std::uint32_t round_mask;
    std::uint32_t round_add;
    // Added to the local cell index before hashing: a z-slab hashes the
    // global index, so a decomposed lattice rounds like the whole one.
    std::uint32_t hash_base;
    // Fluid cells of the x-pairs the two-cell FP16 step leaves out (pairs
    // with a wall or a near-wall cell), in cell order; k_step_list steps them.
    const std::uint32_t* near_list;
    std::uint32_t near_count;
    // z-planes each thread of the z-marching pair kernel (k_step_w2) steps.
    std::uint32_t planes;
    // Planes [z_first, z_end) a step launch covers (0 and nz for a whole step;
    // a slab's two-phase step launches its edge planes and its interior
    // separately).  Honoured by every step kernel (k_step, k_step_w2, k_step_h2,
    // k_step_x2); the other kernels cover the whole lattice.
    std::uint32_t z_first, z_end;
};

// Parameters of the adjoint kernels (lbm_adjoint.cuh).
struct AdjointArgs {
    LbmArgs f;            // forward state read by the step (a recompute frame or the live lattice)
    LbmArgs l;            // adjoint lattice at the adjoint parity (updated in place)
    double* grad_ns;      // N, dJ/dn_s accumulated over steps
    double* tau_partials; // one per block, dJ/dtau accumulated over steps
    double dwp, dwm;      // d omega+ / d tau, d omega- / d tau
    const float* g_rho;   // seed: dJ/drho of the final state (N, may be null)
    const float* g_ux;    // seed: dJ/du of the final state (N each)
    const float* g_uy;
    const float* g_uz;
};

// Initial state for k_init.
struct InitSpec {
    int kind; // 0 uniform, 1 Taylor-Green, 2 per-cell fields
    float rho, ux, uy, uz, amplitude;
    const float* fields; // 4*N (rho|ux|uy|uz), device
    // Global z of local plane z: (z + z_origin) mod nz_total (a z-slab's
    // Taylor-Green field is the whole lattice's); 0 and nz for a whole lattice.
    std::uint32_t z_origin, nz_total;
};

// Output of the fluid-cell reduction, accumulated in FP64.
constexpr int kReduceFields = 7; // mass, mx, my, mz, 2*KE, max|u|, non-finite cells

} // namespace cfdx
