/*
 * CPU oracle for the in-place Esoteric-Pull lattice-Boltzmann step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path is
 * compared against; it is never linked into, loaded by or called from the
 * product library (cfd_solvers_b200/libcfdx_lbm.so).  Only tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline leg of bench.py use it.
 *
 * It restates, in plain C, the algorithm of the reference solver
 *   cfd::lbm::EsotericPullSolver<D>   include/cfd/solvers/lbm/esoteric_pull.hpp:104-515
 * and extends it with the features the reference keeps elsewhere or lacks:
 *   - TRT collision          include/cfd/solvers/lbm/one_step_pull.hpp:187-204
 *   - Smagorinsky with a parametrised coefficient (reference: fixed K,
 *                            include/cfd/solvers/lbm/esoteric_pull.hpp:72-97)
 *   - half-way bounce-back, done in place (reference: 3-pass push path,
 *                            include/cfd/solvers/lbm/esoteric_pull.hpp:434-492)
 *   - moving-wall bounce-back (reference formula, D2Q9 only: src/lbm/d2q9.cpp:206-226)
 *   - gray-LBM partial bounce-back (absent from the reference; Walsh,
 *     Burwinkle & Saar, Geophys. Res. Lett. 36 (2009) L15405)
 *   - FP16 shifted storage with per-direction scale (reference codec, two-grid
 *     only: include/cfd/solvers/lbm/compressed_pull.hpp:72-79)
 *   - FP64 storage and arithmetic.
 *
 * Parity pin: the FP32 variant evaluates every expression of the reference
 * in the reference's order, so with floating-point contraction disabled in
 * both builds it reproduces the reference's populations bit for bit on the
 * features the reference has (BGK + Guo + fixed-K Smagorinsky, periodic;
 * static-mask bounce-back).  tests/test_oracle_vs_reference.py checks this
 * against the reference compiled from its own sources (oracle/_ref).
 */
#ifndef CFDX_LBM_ORACLE_H
#define CFDX_LBM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_STORE_F32 = 0, ORA_STORE_F64 = 1, ORA_STORE_F16S = 2 };
enum { ORA_BGK = 0, ORA_TRT = 1 };
/* Cell flags: 0 fluid, 1 stationary wall, 2..15 moving wall with wall_u[id]. */
enum { ORA_FLUID = 0, ORA_WALL = 1 };
#define ORA_MAX_WALL_IDS 16

typedef struct ora_cfg {
    int q;                    /* 19 or 27 */
    size_t nx, ny, nz;
    int storage;              /* ORA_STORE_* */
    int collision;            /* ORA_BGK / ORA_TRT */
    double tau;               /* symmetric (shear) relaxation time, > 0.5 */
    double tau_minus;         /* TRT antisymmetric relaxation time; 0 => from magic */
    double trt_magic;         /* Lambda = (tau+ - 1/2)(tau- - 1/2) */
    double les_k;             /* Smagorinsky coefficient K (0 = off); K = 18*sqrt(2)*Cs^2 */
    double ax, ay, az;        /* uniform body acceleration */
    const float* local_a;     /* NULL or 3*N floats (ax | ay | az) added per cell */
    const uint8_t* flags;     /* NULL or N cell flags */
    const float* wall_u;      /* 3*ORA_MAX_WALL_IDS wall velocities (may be NULL) */
    const float* solid_fraction; /* NULL or N gray-LBM n_s in [0,1) */
    const float* scale;       /* F16S only: q per-direction scales (NULL => 1) */
} ora_cfg;

/* Number of bytes a population array of this configuration occupies. */
size_t ora_population_bytes(const ora_cfg* c);

/* Equilibrium initialisation into the esoteric slots (time step 0).
 * kind 0: uniform (p[0..3] = rho, ux, uy, uz)
 * kind 1: Taylor-Green (p[0] = amplitude)
 * kind 2: per-cell fields (fields = rho|ux|uy|uz, 4*N floats)
 * Reference: esoteric_pull.hpp:117-137,312-333. */
int ora_init(const ora_cfg* c, void* f, int kind, const float* p, const float* fields);

/* One fused stream+collide step at parity (t & 1).  Reference: esoteric_pull.hpp:494-515. */
int ora_step(const ora_cfg* c, void* f, uint64_t t);

/* The same step for the cells of planes [z_begin, z_end) only: the other
 * planes are read and written by those cells' streaming but not updated
 * themselves (a z-slab with ghost planes in the decomposition tests). */
int ora_step_planes(const ora_cfg* c, void* f, uint64_t t, size_t z_begin, size_t z_end);

/* Macroscopic fields of the state at time t (rho, u + a/2); non-fluid cells
 * report rho = 0, u = 0.  Outputs are float for F32/F16S and double for F64.
 * Reference: esoteric_pull.hpp:180-209. */
int ora_macroscopic(const ora_cfg* c, const void* f, uint64_t t, void* rho, void* ux, void* uy, void* uz);

/* Reductions over fluid cells: out[0] mass, out[1..3] momentum (rho*u),
 * out[4] kinetic energy 0.5*sum rho|u|^2, out[5] max |u|, out[6] non-finite
 * cell count.  Per-cell sums in the arithmetic type, accumulation in double.
 * Reference: esoteric_pull.hpp:211-255, core/parallel.hpp:108-168. */
int ora_reduce(const ora_cfg* c, const void* f, uint64_t t, double out[7]);

/* Parity-independent populations [d][n] (pre-collision, after streaming and
 * boundary handling).  Reference: esoteric_pull.hpp:257-267. */
int ora_logical(const ora_cfg* c, const void* f, uint64_t t, void* out);

/* FP64 discrete adjoint (lbm_adjoint_oracle.c), on logical populations x
 * ([d][n], what ora_logical returns) with the forward's cfg (BGK/TRT, Guo
 * forcing, gray n_s, stationary walls; no LES, no moving walls).
 * ora_adjoint_forward: x_end = x after `steps` logical steps.
 * ora_adjoint: for J with dJ/drho = g_rho (N, may be NULL) and dJ/du = g_u
 * (3*N, ux | uy | uz) at the final state, grad_ns[n] = dJ/dn_s(n) and
 * *grad_tau = dJ/dtau. */
int ora_adjoint_forward(const ora_cfg* c, const double* x0, uint64_t steps, double* x_end);
int ora_adjoint(const ora_cfg* c, const double* x0, uint64_t steps, const double* g_rho, const double* g_u,
                double* grad_ns, double* grad_tau);

/* Triangle-surface voxelizer and rigid transform (voxel_oracle.c; reference
 * src/lbm/voxelize.cpp:4-6).  Triangles are 9 doubles (a, b, c); mask
 * [(k*ny + j)*nx + i] is 1 inside.  ora_voxelize returns 1 on the inputs the
 * reference rejects (no triangles, an empty grid or box). */
int ora_voxelize(const double* tris, size_t count, size_t nx, size_t ny, size_t nz, const double* lo,
                 const double* hi, uint8_t* mask);
int ora_transform_surface(const double* tris, size_t count, const double* translation, const double* axis,
                          double angle, double* out);

/* IEEE binary16 round-to-nearest-even conversion used by the F16S storage. */
uint16_t ora_f32_to_f16(float v);
float ora_f16_to_f32(uint16_t h);

/* Reference Smagorinsky coefficient 16*sqrt(2)/(3*pi^2) evaluated in float
 * exactly as esoteric_pull.hpp:94-95 does. */
float ora_reference_les_k(void);

#ifdef __cplusplus
}
#endif
#endif
