/*
 * cfdx_lbm.h -- C ABI of the B200 in-place Esoteric-Pull lattice-Boltzmann engine.
 *
 * Plain C types only (pointers, sizes, ints, floats); no CUDA or torch types
 * appear in any signature.  Every entry point returns an int status
 * (CFDX_OK = 0) and never throws or aborts; the message of the last failure on
 * the calling thread is available through cfdx_last_error().  The status and
 * error-copy convention follows the reference C ABI
 * (include/cfd/python/c_api.h:3-12, src/python/c_api.cpp:8-16: 0 ok,
 * 1 std::exception, 2 unknown), extended with CUDA-specific codes.
 *
 * Each entry point replaces one member of the reference solver classes
 *   cfd::lbm::EsotericPullSolver<D>      include/cfd/solvers/lbm/esoteric_pull.hpp:104-515
 *   cfd::lbm::EsotericPullSyclSolver<D>  include/cfd/solvers/lbm/esoteric_pull_sycl.hpp:18-475
 * as cited beside it.  The reference has no C ABI for this path; the C++
 * class cfd::lbm::EsotericPullCudaSolver<D> (include/cfd/solvers/lbm/
 * esoteric_pull_cuda.hpp) and the Python package cfd_solvers_b200 are thin
 * layers over these functions.
 *
 * Threading: a handle is not thread-safe; use one handle per thread or
 * serialise calls.  Each handle owns one CUDA stream; cfdx_lbm_step() is
 * asynchronous on it, every call that returns data to the caller
 * synchronises it.
 */
#ifndef CFDX_LBM_H
#define CFDX_LBM_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define CFDX_API __declspec(dllexport)
#else
#define CFDX_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define CFDX_OK 0
#define CFDX_ERR_INVALID 1   /* invalid argument / configuration (std::invalid_argument in the reference) */
#define CFDX_ERR_UNKNOWN 2   /* unknown failure */
#define CFDX_ERR_CUDA 3      /* CUDA runtime error, including "no CUDA device" */
#define CFDX_ERR_OOM 4       /* device allocation failed (std::bad_alloc in the reference) */
#define CFDX_ERR_NONFINITE 5 /* a reduction met NaN/Inf populations */
#define CFDX_ERR_IO 6        /* checkpoint file could not be written or read / is corrupt */
#define CFDX_ERR_RANGE 7     /* index out of range (std::out_of_range in the reference) */

/* Lattices (value = q). */
#define CFDX_D3Q19 19
#define CFDX_D3Q27 27

/* Population storage. */
#define CFDX_STORE_F32 0  /* FP32 populations, FP32 arithmetic (the reference's layout) */
#define CFDX_STORE_F64 1  /* FP64 populations, FP64 arithmetic (at-scale FP64 oracle) */
#define CFDX_STORE_F16S 2 /* FP16 shifted populations h = half((f - w_d) * s_d), FP32 arithmetic */

/* Collision operators. */
#define CFDX_BGK 0 /* single relaxation time (esoteric_pull.hpp:408-432) */
#define CFDX_TRT 1 /* two relaxation times (one_step_pull.hpp:187-204) */

/* Where a caller buffer lives. */
#define CFDX_HOST 0
#define CFDX_DEVICE 1

/* Cell flags passed to cfdx_lbm_set_flags(). */
#define CFDX_FLUID 0
#define CFDX_WALL 1       /* stationary half-way bounce-back wall */
#define CFDX_MOVING_WALL_MIN 2
#define CFDX_MAX_WALL_IDS 16 /* ids 2..15 are moving walls with a velocity from cfdx_lbm_set_wall_velocity() */

/* Reduction slots of cfdx_lbm_reduce(). */
#define CFDX_REDUCE_MASS 0
#define CFDX_REDUCE_MOMENTUM_X 1
#define CFDX_REDUCE_MOMENTUM_Y 2
#define CFDX_REDUCE_MOMENTUM_Z 3
#define CFDX_REDUCE_KINETIC_ENERGY 4
#define CFDX_REDUCE_MAX_SPEED 5
#define CFDX_REDUCE_NONFINITE 6
#define CFDX_REDUCE_COUNT 7

typedef struct cfdx_lbm cfdx_lbm; /* opaque handle */

/* Solver configuration.  The first eight fields are the reference's
 * InPlaceLbmConfig (esoteric_pull.hpp:20-29); the rest extend it. */
/* Rounding of FP16-shifted population stores.  STOCHASTIC (sm_100a
 * cvt.rs with per-cell, per-step hashed random bits) keeps increments
 * smaller than half an FP16 step from being lost every step (small forces,
 * slow flows) -- an unbiased rounding, reproducible run to run for a given
 * seed.  NEAREST rounds half away from zero (the reference codec's rule,
 * compressed_pull.hpp:27,35). */
enum { CFDX_ROUND_NEAREST = 0, CFDX_ROUND_STOCHASTIC = 1 };

typedef struct cfdx_lbm_config {
    size_t nx, ny, nz;
    float tau;               /* > 0.5 */
    float acceleration_x;    /* uniform body acceleration (Guo forcing) */
    float acceleration_y;
    float acceleration_z;
    int smagorinsky_les;     /* 0/1 */
    int lattice;             /* CFDX_D3Q19 / CFDX_D3Q27 */
    int collision;           /* CFDX_BGK / CFDX_TRT */
    int storage;             /* CFDX_STORE_* */
    float smagorinsky_cs;    /* <= 0: the reference's fixed coefficient (Cs = sqrt(8/27)/pi) */
    float trt_magic;         /* TRT magic parameter Lambda (default 3/16) */
    float trt_tau_minus;     /* > 0: fixed antisymmetric relaxation time instead of Lambda */
    int device;              /* CUDA device ordinal */
    int fp16_rounding;       /* CFDX_STORE_F16S stores: CFDX_ROUND_STOCHASTIC (default) or CFDX_ROUND_NEAREST */
    uint32_t rounding_seed;  /* seed of the stochastic rounding bits */
} cfdx_lbm_config;

/* Handle information. */
typedef struct cfdx_lbm_info {
    size_t cells;
    int q;
    int storage;
    uint64_t time_step;          /* reference time_step(), esoteric_pull.hpp:271 */
    size_t population_bytes;     /* reference population_bytes(), esoteric_pull.hpp:272-274 */
    size_t resident_bytes;       /* reference SYCL resident_bytes(), esoteric_pull_sycl.hpp:387-391 */
    uint64_t host_to_device_bytes; /* reference DeviceTransferStats, core/device_residency.hpp:11-42 */
    uint64_t device_to_host_bytes;
    uint64_t synchronizations;
    int fluid_flags;             /* 1 when a flag field is active */
} cfdx_lbm_info;

/* Library version string. Replaces cfd_solvers_version (c_api.h:11). */
CFDX_API const char* cfdx_version(void);

/* Copies the calling thread's last error message (error-copy convention of
 * src/python/c_api.cpp:8).  Returns the status of that failure. */
CFDX_API int cfdx_last_error(char* buffer, size_t capacity);

/* Fills *config with defaults (128^3 D3Q19 BGK FP32, tau 0.6, Lambda 3/16).
 * Reference: InPlaceLbmConfig defaults, esoteric_pull.hpp:20-29. */
CFDX_API int cfdx_lbm_config_default(cfdx_lbm_config* config);

/* Allocates the single population lattice on the device and initialises it
 * to rest (rho = 1).  Reference: EsotericPullSolver(InPlaceLbmConfig),
 * esoteric_pull.hpp:109-115; EsotericPullSyclSolver ctor, esoteric_pull_sycl.hpp:23-33.
 * error/error_capacity may be NULL/0. */
CFDX_API int cfdx_lbm_create(const cfdx_lbm_config* config, cfdx_lbm** out, char* error, size_t error_capacity);

/* Frees every device buffer of the handle.  Reference: ~EsotericPullSyclSolver, esoteric_pull_sycl.hpp:35-45. */
CFDX_API int cfdx_lbm_destroy(cfdx_lbm* lbm);

/* Reference: initialize_uniform, esoteric_pull.hpp:117-119 / esoteric_pull_sycl.hpp:52-60. */
CFDX_API int cfdx_lbm_init_uniform(cfdx_lbm* lbm, float rho, float ux, float uy, float uz);

/* Reference: initialize_taylor_green, esoteric_pull.hpp:121-137 / esoteric_pull_sycl.hpp:62-85. */
CFDX_API int cfdx_lbm_init_taylor_green(cfdx_lbm* lbm, float amplitude);

/* Equilibrium from per-cell fields rho|ux|uy|uz (4*N floats, host or device).
 * Reference: the initializer callback of initialize, esoteric_pull.hpp:312-333. */
CFDX_API int cfdx_lbm_init_fields(cfdx_lbm* lbm, const float* fields, int where);

/* Cell flags (N bytes, host or device): 0 fluid, 1 wall, 2..15 moving wall.
 * NULL clears.  Half-way bounce-back is applied in place.  Set flags before
 * initialising.  Reference: set_solid_mask / clear_solid_mask,
 * esoteric_pull.hpp:161-177 (mask != 0 => wall). */
CFDX_API int cfdx_lbm_set_flags(cfdx_lbm* lbm, const uint8_t* flags, int where);

/* Velocity of moving-wall id (2..15).  Formula: reference src/lbm/d2q9.cpp:109-115,220-223. */
CFDX_API int cfdx_lbm_set_wall_velocity(cfdx_lbm* lbm, int wall_id, float ux, float uy, float uz);

/* Per-cell acceleration ax|ay|az (3*N floats, host or device); NULL clears.
 * Reference: set_local_body_acceleration / clear_local_body_acceleration,
 * esoteric_pull.hpp:144-157; esoteric_pull_sycl.hpp:355-372. */
CFDX_API int cfdx_lbm_set_local_acceleration(cfdx_lbm* lbm, const float* accel, int where);

/* Device pointer to the per-cell acceleration buffer (3*N floats), allocated
 * and zeroed on first use.  Reference: device_local_acceleration, esoteric_pull_sycl.hpp:349-353. */
CFDX_API int cfdx_lbm_device_local_acceleration(cfdx_lbm* lbm, float** accel);

/* Zeroes the per-cell acceleration buffer on the device, ordered on the
 * handle's stream (no host transfer; nothing when there is no buffer).
 * Reference: clear_local_body_acceleration, esoteric_pull_sycl.hpp:355-358 (a queue memset). */
CFDX_API int cfdx_lbm_clear_device_acceleration(cfdx_lbm* lbm);

/* Gray-LBM solid fraction n_s per cell (N floats in [0,1), host or device);
 * NULL clears.  Partial bounce-back f_i <- (1-n_s) f_i* + n_s f_opp(i).
 * No reference counterpart (Walsh, Burwinkle & Saar 2009). */
CFDX_API int cfdx_lbm_set_solid_fraction(cfdx_lbm* lbm, const float* ns, int where);

/* FP16S only: q per-direction scales s_d (directions of equal lattice weight
 * must share a scale); NULL restores the default power-of-two scales near 1/w_d.
 * Reference codec: ShiftedHalfCodec (s_d = 1), compressed_pull.hpp:71-79. */
CFDX_API int cfdx_lbm_set_storage_scale(cfdx_lbm* lbm, const float* scale);

/* Enqueues count fused stream+collide steps.  Reference: step(count),
 * esoteric_pull.hpp:139-142 / esoteric_pull_sycl.hpp:87-211. */
CFDX_API int cfdx_lbm_step(cfdx_lbm* lbm, uint64_t count);

/* Waits for all work of the handle.  Reference: wait(), esoteric_pull_sycl.hpp:213-216. */
CFDX_API int cfdx_lbm_synchronize(cfdx_lbm* lbm);

/* rho and u + a/2 per cell into caller buffers (N floats each; host or
 * device); wall cells report 0.  Reference: compute_macroscopic,
 * esoteric_pull.hpp:180-209; download_macroscopic, esoteric_pull_sycl.hpp:309-325. */
CFDX_API int cfdx_lbm_macroscopic(cfdx_lbm* lbm, float* rho, float* ux, float* uy, float* uz, int where);

/* Same in double precision (N doubles each); exact for CFDX_STORE_F64. */
CFDX_API int cfdx_lbm_macroscopic_f64(cfdx_lbm* lbm, double* rho, double* ux, double* uy, double* uz, int where);

/* Device pointers to a handle-owned rho|ux|uy|uz scratch (4*N floats)
 * refreshed from the current state.  Reference: refresh_device_macroscopic,
 * esoteric_pull_sycl.hpp:226-307. */
CFDX_API int cfdx_lbm_refresh_device_macroscopic(cfdx_lbm* lbm, float** rho, float** ux, float** uy, float** uz);

/* FP64-accumulated reductions over fluid cells into out[CFDX_REDUCE_COUNT]
 * (mass, momentum xyz, kinetic energy 0.5*sum rho|u|^2, max |u|, non-finite
 * cell count).  Returns CFDX_ERR_NONFINITE (with out filled) when any fluid
 * cell is NaN/Inf.  Reference: mass, kinetic_energy, max_speed,
 * esoteric_pull.hpp:211-255; total_mass, esoteric_pull_sycl.hpp:327-339. */
CFDX_API int cfdx_lbm_reduce(cfdx_lbm* lbm, double* out);

/* mass + kinetic energy (the checksum of examples/phase02_lbm_taylor_green.cpp:3). */
CFDX_API int cfdx_lbm_checksum(cfdx_lbm* lbm, double* checksum);

/* Parity-independent populations [d][n] (q*N floats, host or device).
 * Reference: logical_populations, esoteric_pull.hpp:257-267. */
CFDX_API int cfdx_lbm_logical_populations(cfdx_lbm* lbm, float* out, int where);

/* Reference: time_step, population_bytes, cells, resident_bytes, transfer_stats. */
CFDX_API int cfdx_lbm_get_info(cfdx_lbm* lbm, cfdx_lbm_info* info);

/* The handle's CUDA stream (a cudaStream_t) for callers that time or order
 * work around the step. */
CFDX_API int cfdx_lbm_stream(cfdx_lbm* lbm, void** stream);

/* Device pointer and size of the raw population storage (esoteric layout).
 * Reference: raw_storage, esoteric_pull.hpp:276-278. */
CFDX_API int cfdx_lbm_raw_populations(cfdx_lbm* lbm, void** device_ptr, size_t* bytes);

/* Launch shape of the cell kernels: threads per block (x, y) and the step
 * kernel variant: 0 automatic, 1 one cell per thread, 2 two adjacent x cells
 * per thread (FP32/FP16 storage, even nx), 3 / 4 the wall-aware FP16 pair
 * kernel that marches along z, with / without its shared-memory prefetch of
 * the next plane (FP16 storage, even nx).  All variants give bitwise equal
 * results.  Automatic: two cells for D3Q19 FP16 on lattices without flags,
 * the wall-aware pair kernel (3) for D3Q19 FP16 with flags and without gray
 * cells, one cell otherwise.  Zeros restore the defaults.
 * Reference: no counterpart (the OpenMP loop of step_once,
 * esoteric_pull.hpp:494-515, has no launch shape). */
CFDX_API int cfdx_lbm_set_launch_shape(cfdx_lbm* lbm, int block_x, int block_y, int variant);

/* z-planes each thread of the z-marching pair kernel (variants 3 and 4)
 * steps, in [1, 4096]; 0 restores the default.  Results do not depend on it.
 * Reference: no counterpart. */
CFDX_API int cfdx_lbm_set_step_planes(cfdx_lbm* lbm, int planes);

/* The reduction of cfdx_lbm_reduce() without any allocation: no
 * cudaMalloc, cudaFree or other allocating routine, for callers that cannot
 * allocate at this point -- a process whose device memory is held by another
 * allocator, a monitoring loop that must not take the device-wide
 * synchronisation of cudaMalloc/cudaFree, or an FFI caller with no CUDA
 * allocation API of its own.  No counterpart in the reference.
 * `out` is host memory for CFDX_REDUCE_COUNT doubles, same layout and status
 * codes as cfdx_lbm_reduce().  Scratch is a fixed static device array
 * (229,432 bytes on every GPU that loads the library, held until exit) with
 * the partial sums of min(ny*nz, 4096) reduction blocks, so every lattice
 * size is accepted.  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) and keeps it; make that first call
 * before any stream capture, and do not call this entry point again after
 * resetting the device.  All calls share the array: calls whose work overlaps
 * on the GPU (different handles' streams, or threads) race and must be
 * serialised by the caller. */
CFDX_API int cfdx_lbm_reduce_noalloc(cfdx_lbm* lbm, double* out);

/* Checkpoint files in the reference's CFDCHK3 version-1 layout
 * (include/cfd/solvers/lbm/distributed_pull.hpp:176-245, one brick covering
 * the lattice): header, time step, tau and acceleration, then q*N float
 * populations [d][z][y][x] -- what each fluid cell gathers at the stored
 * time step (before moving-wall corrections), 0 on walls.  Load restores the
 * time step and the lattice so that stepping continues bit for bit (FP32
 * storage); the header must match the handle (q, extents, tau, acceleration)
 * and the payload must be complete, else CFDX_ERR_IO and nothing changes.
 * Reference: DistributedPullSolver::save_checkpoint / load_checkpoint. */
CFDX_API int cfdx_lbm_checkpoint_save(cfdx_lbm* lbm, const char* path);
CFDX_API int cfdx_lbm_checkpoint_load(cfdx_lbm* lbm, const char* path);

/* Symmetric relaxation time (> 0.5) for the following steps; the adjoint's
 * dJ/dtau is taken with respect to it.  Reference: InPlaceLbmConfig::tau,
 * esoteric_pull.hpp:20-29 (fixed at construction there). */
CFDX_API int cfdx_lbm_set_tau(cfdx_lbm* lbm, float tau);

/* ---- Discrete adjoint of the gray-LBM step (no reference counterpart: the
 * reference has neither gray LBM nor an adjoint).  Scope: BGK/TRT, uniform
 * or per-cell force, gray n_s, stationary walls, periodic faces; Smagorinsky
 * LES and moving walls are rejected with CFDX_ERR_INVALID; q*cells < 2^32.
 *
 * cfdx_lbm_adjoint_forward: runs `steps` steps from the current state like
 * cfdx_lbm_step, keeping a device copy of the lattice every `interval` steps
 * (ceil(steps/interval) copies, in the storage precision) plus the reverse
 * sweep's recompute frames (max(interval-1, 2) lattices with one level of
 * recompute; see cfdx_lbm_adjoint_set_subinterval).  It runs the out-of-place form of the
 * step that the reverse sweep recomputes with, so the recomputed states equal
 * the forward's bit for bit; the final state equals cfdx_lbm_step(steps)'s to
 * within the last bit of the arithmetic type. */
CFDX_API int cfdx_lbm_adjoint_forward(cfdx_lbm* lbm, uint64_t steps, uint32_t interval);

/* Sub-checkpoint interval m of the reverse sweep for the following
 * cfdx_lbm_adjoint_forward calls: 0 (the default) recomputes each segment once
 * and holds its interval - 1 states; 2 <= m < interval recomputes it twice
 * (first every m-th state, then each sub-segment of m steps from its
 * sub-checkpoint) and holds ceil(interval/m) - 1 + max(m - 1, 2) frames
 * instead, e.g. 14 instead of 63 for interval 64 and m = 8.  The gradients are
 * bitwise the same.  1 is rejected (CFDX_ERR_INVALID). */
CFDX_API int cfdx_lbm_adjoint_set_subinterval(cfdx_lbm* lbm, uint32_t subinterval);

/* Reverse sweep for an objective J of the final state, given dJ/drho (N
 * floats, may be NULL) and dJ/du_x,y,z (N floats each) of the fields
 * cfdx_lbm_macroscopic reports (u includes +a/2), all on `where` (host or
 * device).  Writes dJ/dn_s per cell (N doubles, 0 on walls; `grad_where`;
 * NULL skips) and dJ/dtau (*grad_tau, host; NULL skips).  Recomputes each
 * segment from its checkpoint; the lattice and its parameters must not have
 * changed since cfdx_lbm_adjoint_forward (else CFDX_ERR_INVALID).  FP32
 * adjoint arithmetic for FP32/FP16 storage, FP64 for FP64 storage; the
 * gradients are accumulated in FP64.  May be called again with another seed. */
CFDX_API int cfdx_lbm_adjoint_backward(cfdx_lbm* lbm, const float* g_rho, const float* g_ux, const float* g_uy,
                                       const float* g_uz, int where, double* grad_ns, int grad_where,
                                       double* grad_tau);

/* Device bytes the adjoint's buffers hold. */
CFDX_API int cfdx_lbm_adjoint_memory(cfdx_lbm* lbm, size_t* bytes);

/* Frees the adjoint's buffers (checkpoints, frames, adjoint lattice). */
CFDX_API int cfdx_lbm_adjoint_release(cfdx_lbm* lbm);

/* ---- z-slab decomposition (multi-GPU).  The reference cuts its distributed
 * two-grid solver into bricks (DistributedPullBlock, distributed_pull.hpp:35-60;
 * make_brick / partition_axis, distributed/cartesian.hpp:132-159) and sends
 * only the populations that cross a face (selective_halo.hpp:24-62).  Here the
 * in-place lattice is cut along z only, one slab per rank, by the same
 * partition rule (the first nz % parts slabs get one extra plane); the slabs
 * form a periodic ring, as the lattice is periodic in z.
 *
 * A slab handle holds nx*ny*(z_extent + 2) cells: local plane k is global
 * plane (z_begin - 1 + k) mod nz, so planes 0 and z_extent + 1 ("ghost
 * planes") hold copies of the neighbours' edge planes.  Every per-cell array
 * the other entry points take or return (flags, fields, accelerations, n_s,
 * macroscopic fields, logical populations) covers the local planes.  Ghost
 * plane flags must be the neighbours' flags (they set the bounce-back links of
 * the edge planes); the other ghost-plane inputs are ignored and ghost-plane
 * outputs are 0.  Reductions, checksums and checkpoints cover the slab's own
 * planes; checkpoints record the slab as a CFDCHK3 brick
 * (begin = (0, 0, z_begin), extent = (nx, ny, z_extent)).
 *
 * After each step every cut carries one message each way (5 chunks for D3Q19,
 * 9 for D3Q27, of nx*ny populations in the storage type): the ghost slots this
 * slab's edge cells wrote, and the edge slots the neighbour's edge cells read
 * next.  A slab steps once, exchanges through both sides (pack -> transport ->
 * unpack, or cfdx_lbm_halo_exchange between two handles of one process), then
 * steps again; cfdx_lbm_step refuses to start a step while a side of the
 * previous one has not been received.  A slab that is the whole ring
 * (z_extent == nz) exchanges with itself inside cfdx_lbm_step.  The discrete
 * adjoint is not available on slab handles. */
typedef struct cfdx_halo_entry {
    uint32_t plane;     /* local plane, 0 .. z_extent + 1 */
    uint32_t direction; /* lattice direction (storage slot) */
} cfdx_halo_entry;

#define CFDX_SIDE_LOWER 0 /* towards global plane z_begin - 1 */
#define CFDX_SIDE_UPPER 1 /* towards global plane z_begin + z_extent */

/* Creates the slab [z_begin, z_begin + z_extent) of the lattice `global`
 * describes (global->nz is the whole lattice's extent); z_extent >= 1. */
CFDX_API int cfdx_lbm_create_slab(const cfdx_lbm_config* global, uint32_t z_begin, uint32_t z_extent,
                                  cfdx_lbm** out, char* error, size_t error_capacity);

/* Slab geometry of a handle (a plain handle reports 0, nz, nz). */
CFDX_API int cfdx_lbm_slab_info(cfdx_lbm* lbm, uint32_t* z_begin, uint32_t* z_extent, uint32_t* nz_global);

/* Message layout of one side, host-only (no device needed): after a step of
 * parity `odd` on a slab of z_extent planes, chunk k of the message sent
 * through `side` is local (send[k].plane, send[k].direction), and chunk k of
 * the message arriving through `side` is written to (recv[k].plane,
 * recv[k].direction).  *count = 5 (D3Q19) or 9 (D3Q27); capacity >= *count. */
CFDX_API int cfdx_halo_plan(int lattice, int odd, int side, uint32_t z_extent, cfdx_halo_entry* send,
                            cfdx_halo_entry* recv, int capacity, int* count);

/* Bytes of one message (chunks * nx * ny * storage bytes). */
CFDX_API int cfdx_lbm_halo_bytes(cfdx_lbm* lbm, size_t* bytes);

/* One time step of a slab in two launches, so that its halo exchange can
 * overlap the interior of the step.  CFDX_STEP_EDGES steps the slab's first
 * and last own planes -- the cells whose stores the messages carry -- and
 * counts the time step: from then on the messages of the step can be packed
 * (cfdx_lbm_halo_pack) and sent.  CFDX_STEP_INTERIOR steps the remaining
 * planes.  The arriving messages may be unpacked before or after the
 * interior phase (they fill slots no cell of the slab touches during the
 * step), but before the next step.  Between the phases only the halo calls,
 * cfdx_lbm_synchronize and cfdx_lbm_stream are accepted.  Results equal
 * cfdx_lbm_step's bit for bit.  Reference: the interior / boundary-shell
 * split of DistributedPullBlock (distributed_pull.hpp:97-116). */
#define CFDX_STEP_EDGES 1
#define CFDX_STEP_INTERIOR 2
CFDX_API int cfdx_lbm_step_phase(cfdx_lbm* lbm, int phase);

/* Copies the message for `side` of the step just taken into device memory
 * `buffer` (this device's or a peer's), stream-ordered after the step. */
CFDX_API int cfdx_lbm_halo_pack(cfdx_lbm* lbm, int side, void* device_buffer);

/* Writes the message that arrived through `side` (device memory) into the
 * slab, stream-ordered; the buffer must stay valid until the slab's stream
 * has passed this point. */
CFDX_API int cfdx_lbm_halo_unpack(cfdx_lbm* lbm, int side, const void* device_buffer);

/* Both messages of the cut between `lower` (its upper side) and `upper` (its
 * lower side), two slab handles of this process on one device or on devices
 * with peer access: one copy kernel, slot to slot, ordered after both
 * handles' steps and before their next ones.  lower == upper is the ring of
 * one slab. */
CFDX_API int cfdx_lbm_halo_exchange(cfdx_lbm* lower, cfdx_lbm* upper);

/* ---- Triangle-surface voxelizer (reference cfd::lbm::voxelize_surface,
 * src/lbm/voxelize.cpp:4-5; SYCL voxelize_surface_sycl, src/sycl/voxelize_sycl.cpp:13-68).
 * Cell (i, j, k) of the nx*ny*nz grid over [minimum, maximum] is solid when
 * the ray from (min.x + (i+0.5)dx, min.y + (j+0.5)dy + 1e-10 dx,
 * min.z + (k+0.5)dz + 2e-10 dx) in direction +x crosses the surface an odd
 * number of times (Moller-Trumbore hits with |det| >= 1e-12 and distance >
 * 1e-10), in FP64 with the reference's operation order: the mask equals the
 * reference CPU voxelizer's bit for bit.  Triangles are 9 doubles each
 * (a, b, c) in host memory; the surface need not be closed or oriented (a
 * ray's parity decides).  Non-finite coordinates are rejected. */
typedef struct cfdx_voxel_grid {
    size_t nx, ny, nz;
    double minimum[3];
    double maximum[3];
} cfdx_voxel_grid;

/* Voxelizes global planes z_first .. z_first + z_count - 1 (mod nz) into
 * `out` (nx*ny*z_count bytes, host or device memory of `device`): `solid_value`
 * inside, 0 outside. */
CFDX_API int cfdx_voxelize(const double* triangles, size_t count, const cfdx_voxel_grid* grid, uint32_t z_first,
                           uint32_t z_count, uint8_t solid_value, uint8_t* out, int where, int device);

/* Sets the handle's flags from a surface: the handle's lattice (a slab: its
 * local planes of the whole lattice) is the voxel grid over [minimum, maximum];
 * cells inside get `solid_value` (1 wall, 2..15 moving wall), the others
 * base_flags[n] (the handle's cells, `where` memory) or 0 when base_flags is
 * NULL.  The same as voxelizing and calling cfdx_lbm_set_flags, without the
 * host round trip.  Reference use: voxelize_surface + set_solid_mask
 * (examples/real_lbm3d_model.cpp:146-150). */
CFDX_API int cfdx_lbm_set_flags_surface(cfdx_lbm* lbm, const double* triangles, size_t count, const double* minimum,
                                        const double* maximum, uint8_t solid_value, const uint8_t* base_flags,
                                        int where);

/* ---- Field export (reference visualization.hpp:17-22, src/lbm/visualization.cpp:39-148).
 * Host-only writers: legacy-VTK structured points (one scalar, optional
 * velocity vectors as 3 doubles per cell x,y,z, optional solid bytes) and the
 * JSON live state (written to "<path>.tmp", then renamed over path).  ASCII
 * VTK and JSON text equal the reference writers' output byte for byte;
 * binary = 1 writes the big-endian binary legacy format instead (the
 * reference writes ASCII only).  I/O failures return CFDX_ERR_IO. */
CFDX_API int cfdx_write_vtk_3d(const char* path, size_t nx, size_t ny, size_t nz, const double* scalar,
                               const double* velocity, const uint8_t* solid, const char* scalar_name, int binary);
CFDX_API int cfdx_write_json_state_3d(const char* path, size_t nx, size_t ny, size_t nz, uint64_t step,
                                      const double* scalar, const uint8_t* solid, const char* scalar_name);

/* Q-criterion (|Omega|^2 - |S|^2)/2 of a velocity field (3 doubles per cell,
 * x,y,z; host or device memory of `device`) with central differences over
 * spacings dx, dy, dz, 0 on the outer layer of cells: reference q_criterion_3d
 * (visualization.cpp:122-148) on the device, equal to it bit for bit.  Grids
 * need nx, ny, nz >= 3. */
CFDX_API int cfdx_q_criterion(const double* velocity, size_t nx, size_t ny, size_t nz, double dx, double dy,
                              double dz, double* q, int where, int device);

/* The Q-criterion of the handle's current velocity (u + a/2 as
 * cfdx_lbm_macroscopic_f64 reports it; walls 0), without a host round trip.
 * Whole lattices only (a slab's edge planes need the neighbours' velocities). */
CFDX_API int cfdx_lbm_q_criterion(cfdx_lbm* lbm, double dx, double dy, double dz, double* q, int where);

/* ---- Resident D3Q7 temperature lattice coupled to a flow handle (reference
 * ResidentThermalD3Q7Sycl, resident_multiphysics_sycl.hpp:51-200): a two-grid
 * BGK advection-diffusion lattice (c_s^2 = 1/4, tau = 1/2 + 4 D) on the flow's
 * grid, device and stream, driven by the flow's device velocity
 * (cfdx_lbm_refresh_device_macroscopic) and adding Boussinesq buoyancy into
 * the flow's device acceleration field (cfdx_lbm_device_local_acceleration):
 * no field passes through the host while coupled.  Whole lattices only;
 * destroy it before its flow handle.  Every call is ordered on the flow's
 * stream. */
typedef struct cfdx_thermal cfdx_thermal;

/* Reference constructor (resident_multiphysics_sycl.hpp:62-71); starts at T = 0. */
CFDX_API int cfdx_thermal_create(cfdx_lbm* flow, float diffusivity, cfdx_thermal** out, char* error,
                                 size_t error_capacity);
CFDX_API int cfdx_thermal_destroy(cfdx_thermal* thermal);
/* Reference initialize_uniform (:84-92); init_field sets a per-cell temperature (N floats). */
CFDX_API int cfdx_thermal_init_uniform(cfdx_thermal* thermal, float temperature);
CFDX_API int cfdx_thermal_init_field(cfdx_thermal* thermal, const float* temperature, int where);
/* Reference step(flow view, count) (:94-130): `count` steps with the device velocity ux/uy/uz. */
CFDX_API int cfdx_thermal_step(cfdx_thermal* thermal, const float* ux, const float* uy, const float* uz,
                               uint64_t count);
/* Reference refresh_device_scalar (:132-139): device pointer to the temperature (owned by the lattice). */
CFDX_API int cfdx_thermal_refresh_device_scalar(cfdx_thermal* thermal, float** temperature);
CFDX_API int cfdx_thermal_temperature(cfdx_thermal* thermal, float* out, int where);
/* Reference add_boussinesq_acceleration (:141-159): a += -beta (T - t_ref) g per cell (device arrays). */
CFDX_API int cfdx_thermal_add_boussinesq(cfdx_thermal* thermal, float* ax, float* ay, float* az, float t_ref,
                                         float beta, float gx, float gy, float gz);
/* Reference total_scalar (:161-171), summed in FP64. */
CFDX_API int cfdx_thermal_total(cfdx_thermal* thermal, double* total);
/* Reference resident_bytes / transfer_stats (:173-176). */
CFDX_API int cfdx_thermal_info(cfdx_thermal* thermal, size_t* resident_bytes, uint64_t* host_to_device,
                               uint64_t* device_to_host);

/* ---- Resident free surface (reference ResidentFreeSurfaceSycl3D,
 * resident_multiphysics_sycl.hpp:202-318): a fill fraction in [0, 1] per
 * cell, advected by the flow's device velocity with first-order upwind face
 * fluxes (face velocity = mean of the two cells) and clamped, its normals and
 * curvature from central differences, and the surface-tension acceleration
 * sigma * kappa * grad(fill) / rho added into the flow's device acceleration.
 * Periodic in every axis; whole lattices with nx, ny, nz >= 2; ordered on the
 * flow's stream; destroy it before its flow handle. */
typedef struct cfdx_surface cfdx_surface;

/* Reference constructor (:204-212); starts empty (fill 0). */
CFDX_API int cfdx_surface_create(cfdx_lbm* flow, cfdx_surface** out, char* error, size_t error_capacity);
CFDX_API int cfdx_surface_destroy(cfdx_surface* surface);
/* Reference initialize_uniform (:222-226): fill in [0, 1] else CFDX_ERR_INVALID. */
CFDX_API int cfdx_surface_init_uniform(cfdx_surface* surface, float fill);
/* Reference initialize_half_space_x (:227-236): the fraction of each cell left of x = interface_x. */
CFDX_API int cfdx_surface_init_half_space_x(cfdx_surface* surface, float interface_x);
/* A per-cell fill (N floats, host values checked to lie in [0, 1]). */
CFDX_API int cfdx_surface_init_field(cfdx_surface* surface, const float* fill, int where);
/* Reference advect(flow view, dt) (:238-264): one upwind step with the device velocity; dt > 0. */
CFDX_API int cfdx_surface_advect(cfdx_surface* surface, const float* ux, const float* uy, const float* uz,
                                 float dt);
/* Reference fill_device (:266-267): device pointer to the current fill (valid until the next advect). */
CFDX_API int cfdx_surface_device_fill(cfdx_surface* surface, float** fill);
/* Reference refresh_geometry (:269-298): normals (0 where |grad| <= 1e-12) and
 * curvature -div(n)/2; *geometry (may be NULL) = device [normal x | y | z | curvature], 4 N floats. */
CFDX_API int cfdx_surface_refresh_geometry(cfdx_surface* surface, float** geometry);
/* Reference add_surface_tension_acceleration (:300-318): refreshes the geometry,
 * then a += sigma * kappa / rho * grad(fill); sigma >= 0, rho > 0. */
CFDX_API int cfdx_surface_add_tension(cfdx_surface* surface, float* ax, float* ay, float* az, float surface_tension,
                                      float density);
/* Reference volume (:322-327): the sum of the fill (in FP64 here; the reference sums in FP32). */
CFDX_API int cfdx_surface_volume(cfdx_surface* surface, double* volume);
/* Copy out the fill (which 0) or a geometry component (1-3 normal x/y/z, 4 curvature). */
CFDX_API int cfdx_surface_fill(cfdx_surface* surface, float* out, int which, int where);
CFDX_API int cfdx_surface_info(cfdx_surface* surface, size_t* resident_bytes, uint64_t* host_to_device,
                               uint64_t* device_to_host);

/* ---- Resident point particles (reference ResidentParticlesSycl3D,
 * resident_multiphysics_sycl.hpp:333-382): per particle x, y, z, vx, vy, vz,
 * mass, response time on the device.  advance() interpolates the flow's
 * device velocity trilinearly (periodic), applies the drag m (u - v) / tau_p
 * and gravity with an explicit Euler step, wraps the position, and with
 * two_way != 0 spreads -drag onto the eight surrounding cells of the flow's
 * device acceleration with atomic adds (whose order, and so the last bits of
 * the sum where particles share a cell, is not fixed). */
typedef struct cfdx_particles cfdx_particles;

/* Reference constructor (:326-330); count may be 0. */
CFDX_API int cfdx_particles_create(cfdx_lbm* flow, size_t count, cfdx_particles** out, char* error,
                                   size_t error_capacity);
CFDX_API int cfdx_particles_destroy(cfdx_particles* particles);
/* Reference upload (:337-346): `count` records of 8 doubles laid out as the
 * reference's ImmersedBoundaryParticle (position x y z, velocity x y z, mass,
 * response_time; particles.hpp:13-18); mass and response time > 0. */
CFDX_API int cfdx_particles_upload(cfdx_particles* particles, const double* records, size_t count);
/* Reference download (:371-380): the same 8-double records. */
CFDX_API int cfdx_particles_download(cfdx_particles* particles, double* records, size_t count);
/* Device state, 8 planes of `count` floats (x | y | z | vx | vy | vz | mass | response). */
CFDX_API int cfdx_particles_device_state(cfdx_particles* particles, float** state);
/* Reference advance(flow view, force view, dt, two_way, gravity) (:348-369). */
CFDX_API int cfdx_particles_advance(cfdx_particles* particles, const float* ux, const float* uy, const float* uz,
                                    float* ax, float* ay, float* az, float dt, int two_way, float gx, float gy,
                                    float gz);
CFDX_API int cfdx_particles_info(cfdx_particles* particles, size_t* resident_bytes, uint64_t* host_to_device,
                                 uint64_t* device_to_host);

/* ---- Resident FP32 Q-criterion of a device velocity (reference
 * ResidentFlowDiagnosticsSycl3D, resident_multiphysics_sycl.hpp:384-405):
 * periodic central differences, Q = (|Omega|^2 - |S|^2) / 2 in FP32, into a
 * device field owned by the handle.  Whole lattices with nx, ny, nz >= 3. */
typedef struct cfdx_diagnostics cfdx_diagnostics;

CFDX_API int cfdx_diagnostics_create(cfdx_lbm* flow, cfdx_diagnostics** out, char* error, size_t error_capacity);
CFDX_API int cfdx_diagnostics_destroy(cfdx_diagnostics* diagnostics);
/* *q = the device Q field (N floats, owned by the handle; overwritten by the next call). */
CFDX_API int cfdx_diagnostics_q_criterion(cfdx_diagnostics* diagnostics, const float* ux, const float* uy,
                                          const float* uz, float** q);
CFDX_API int cfdx_diagnostics_info(cfdx_diagnostics* diagnostics, size_t* resident_bytes);

/* Temporary buffers of single calls (cfdx_voxelize / cfdx_lbm_set_flags_surface
 * scratch, cfdx_q_criterion / cfdx_lbm_q_criterion staging) come from a
 * stream-ordered memory pool the library keeps per device, which keeps up to
 * 8 GiB mapped between calls so that repeated calls do not map memory anew or
 * synchronise the device in cudaFree.  This returns the pool's unused memory on
 * `device` to the driver (after synchronising the device). */
CFDX_API int cfdx_release_scratch(int device);

/* ---- Slot-ownership audit (a test hook standing in for a race detector).
 * In-place streaming is race-free because, within a step, every population
 * slot is loaded and then stored by exactly one cell.  The audit runs the
 * one-cell step kernel's own addressing (gather, wall links, moving walls,
 * slab ghost planes) for the step of the given parity with a storage type that
 * records, per slot, its loads, its stores and the threads that made them,
 * and counts the slots in each class below.  The lattice is not modified; the
 * audit uses 20 bytes per slot of scratch (at most 2^28 slots).  A race-free
 * step has written_twice = foreign = 0 (and read_twice = out_of_range = 0).  A fluid cell
 * touches q slots plus one per link into a wall cell: such a link loads one of
 * the wall cell's two slots of the pair and stores the other (half-way
 * bounce-back in place), so read_only = write_only = the number of wall links,
 * and touched = q * fluid cells + wall links. */
typedef struct cfdx_slot_audit {
    uint64_t slots;         /* q * cells */
    uint64_t touched;       /* read or written */
    uint64_t read_twice;    /* loaded more than once */
    uint64_t written_twice; /* stored more than once: a write-write race */
    uint64_t read_only;     /* loaded, never stored */
    uint64_t write_only;    /* stored, never loaded */
    uint64_t foreign;       /* stored by a thread other than the one that loaded it */
    uint64_t out_of_range;  /* loads and stores outside the lattice's slots (counted, not performed) */
} cfdx_slot_audit;

CFDX_API int cfdx_lbm_debug_slot_audit(cfdx_lbm* lbm, int parity, cfdx_slot_audit* out);

/* The audit's classification of one slot from its counters (loads, stores,
 * lowest and highest loading thread, storing thread; threads numbered from
 * 1): a bit set of 1 touched, 2 read twice, 4 written twice, 8 read only,
 * 16 write only, 32 foreign.  Host-only; lets the classification be tested
 * without a GPU. */
CFDX_API int cfdx_debug_audit_classify(uint32_t reads, uint32_t writes, uint32_t lowest_reader,
                                       uint32_t highest_reader, uint32_t writer, unsigned* classes);

/* Test hook: the next `count` device allocations of this process fail with
 * cudaErrorMemoryAllocation (0 disables).  Used to test CFDX_ERR_OOM paths
 * without exhausting the device. */
CFDX_API int cfdx_debug_fail_allocations(int count);

/* Test hook: with wide != 0 the handle addresses slots through 64-bit
 * per-parity pointers, the form every kernel uses when q * cells >= 2^32
 * (e.g. D3Q27 above about 542^3), instead of 32-bit element offsets, so that
 * small lattices test that path; the paired-cell kernels, which need the
 * offsets, are not used then, and the adjoint refuses the handle as it
 * refuses such lattices.  Reference: no counterpart (esoteric_pull.hpp:304-310
 * indexes with size_t throughout). */
CFDX_API int cfdx_lbm_debug_force_wide_slots(cfdx_lbm* lbm, int wide);

/* Test hook of the out-of-memory retry: the next `count` device allocations
 * (count >= 0; < 0 leaves it unchanged) see out-of-memory from their first
 * attempt, return the idle scratch-pool memory to the driver and try again.
 * *retries (may be NULL) receives the number of retries taken so far in
 * this process. */
CFDX_API int cfdx_debug_retry_allocations(int count, unsigned long long* retries);

#ifdef __cplusplus
}
#endif
#endif /* CFDX_LBM_H */
