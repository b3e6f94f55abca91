// Host-side launch interface of the lattice kernels (one implementation per
// storage type, compiled in separate translation units).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_args.h"

namespace cfdx {

struct LaunchShape {
    int block_x = 0; // 0 = choose from nx
    int block_y = 0;
};

// Kernel selection that is fixed per handle.
struct KernelKey {
    int storage;   // Storage
    int q;         // 19 / 27
    int collision; // Collision
    bool les;
    bool flags;
    bool gray;
    int cells_per_thread; // reserved (one cell per thread)
    bool paired;          // use the paired-cell step kernel (two adjacent x cells per thread)
    bool w2;              // FP16: the wall-aware z-marching pair kernel (k_step_w2)
    bool w2_pipe;         // k_step_w2 with its cp.async shared-memory pipeline
    bool narrow;          // 32-bit slot offsets (q * cells < 2^32)
};

dim3 cell_block(long long nx, long long ny, const LaunchShape& s);
dim3 cell_grid(long long nx, long long ny, long long nz, dim3 block);

template <int STORAGE> struct Launcher {
    static cudaError_t step(const KernelKey& k, const LbmArgs& a, dim3 grid, dim3 block, cudaStream_t s);
    static cudaError_t init(const KernelKey& k, const LbmArgs& a, const InitSpec& spec, dim3 grid, dim3 block,
                            cudaStream_t s);
    static cudaError_t macro(const KernelKey& k, const LbmArgs& a, void* rho, void* ux, void* uy, void* uz,
                             bool out_f64, dim3 grid, dim3 block, cudaStream_t s);
    static cudaError_t logical(const KernelKey& k, const LbmArgs& a, float* out, dim3 grid, dim3 block,
                               cudaStream_t s);
    static cudaError_t reduce(const KernelKey& k, const LbmArgs& a, double* partials, int blocks, double* out,
                              cudaStream_t s);
    // Checkpoint I/O of direction d (k_slot_out / k_slot_in).
    static cudaError_t slot_io(const KernelKey& k, const LbmArgs& a, int d, float* buffer, bool in, dim3 grid,
                               dim3 block, cudaStream_t s);
    // Adjoint (lbm_adjoint.cuh); all three need 32-bit slot offsets.
    static cudaError_t step_oop(const KernelKey& k, const LbmArgs& src, const LbmArgs& dst, dim3 grid, dim3 block,
                                cudaStream_t s);
    static cudaError_t adjoint_seed(const KernelKey& k, const AdjointArgs& a, dim3 grid, dim3 block, cudaStream_t s);
    static cudaError_t adjoint_step(const KernelKey& k, const AdjointArgs& a, dim3 grid, dim3 block, cudaStream_t s);
};

cudaError_t launch_step(const KernelKey& k, const LbmArgs& a, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_init(const KernelKey& k, const LbmArgs& a, const InitSpec& spec, dim3 grid, dim3 block,
                        cudaStream_t s);
cudaError_t launch_macro(const KernelKey& k, const LbmArgs& a, void* rho, void* ux, void* uy, void* uz,
                         bool out_f64, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_logical(const KernelKey& k, const LbmArgs& a, float* out, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_reduce(const KernelKey& k, const LbmArgs& a, double* partials, int blocks, double* out,
                          cudaStream_t s);
cudaError_t launch_step_oop(const KernelKey& k, const LbmArgs& src, const LbmArgs& dst, dim3 grid, dim3 block,
                            cudaStream_t s);
cudaError_t launch_adjoint_seed(const KernelKey& k, const AdjointArgs& a, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_adjoint_step(const KernelKey& k, const AdjointArgs& a, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_slot_io(const KernelKey& k, const LbmArgs& a, int d, float* buffer, bool in, dim3 grid,
                           dim3 block, cudaStream_t s);
cudaError_t launch_sum_partials(const double* partials, std::size_t count, double* out, cudaStream_t s);
// Fluid cells of the pairs that are not interior (near_list.cu), in cell order:
// the CUB select of `cells` indices into `out`, the count to *count (device).
// With temp == nullptr it only sets *temp_bytes.
cudaError_t select_near_cells(const std::uint8_t* flags, std::uint32_t cells, std::uint32_t* out,
                              std::uint32_t* count, void* temp, std::size_t* temp_bytes, cudaStream_t s);

// ghost: planes 0 and nz-1 are a z-slab's ghost planes (k_prepare_flags).
cudaError_t launch_prepare_flags(int q, const LbmArgs& a, const std::uint8_t* user, std::uint8_t* out,
                                 std::uint32_t* mask, bool ghost, dim3 grid, dim3 block, cudaStream_t s);

} // namespace cfdx
