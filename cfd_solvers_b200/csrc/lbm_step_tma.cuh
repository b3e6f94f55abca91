// Row-staged variant of the step kernel: whole x-rows move between HBM and
// shared memory with 1-D bulk copies (the TMA engine, cp.async.bulk), so the
// bytes in flight no longer depend on registers.
//
// A persistent CTA walks rows r = blockIdx.x + t * gridDim.x.  For row r the
// slots its cells own at this parity are q full rows of the population array:
// the rest row and the pb rows of r itself, and for every pair p the pa row of
// the neighbouring row r + off(c_j) -- every slot of that row belongs to a cell
// of row r (the x shift wraps within the row).  Each stage holds those q rows
// (plus the flag row); one thread issues the copies onto the stage's mbarrier,
// S - 1 rows ahead of the row being computed.  Threads update the stage in
// place (each slot is read and written by exactly one thread) and the same
// thread writes the q rows back with bulk stores.  Rows of different r never
// share a slot, so the staging keeps the in-place update race-free; wall
// cells leave their slots untouched and the write-back rewrites the same
// bytes.  Bounce-back links read the partner slot from global memory (it is
// not owned by any cell at this parity, so no tile writes it).
//
// Every mbarrier wait is bounded: on timeout the kernel sets *a.status, waits
// (bounded) for its own copies and returns.  No multicast is used.
#pragma once

#include "lbm_device.cuh"

namespace cfdx {

constexpr unsigned kTmaSpinLimit = 1U << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(std::uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(std::uint64_t* bar, unsigned bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(std::uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0U;
}

// Bounded wait on one phase of an mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(std::uint64_t* bar, unsigned parity) {
    for (unsigned k = 0; k < kTmaSpinLimit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, std::uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Waits until at most N bulk store groups still read shared memory.
template <int N> __device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory layout of the row pipeline (host computes, kernel reads).
struct RowStages {
    unsigned stages;      // S >= 2
    unsigned row_bytes;   // nx * element size (multiple of 16)
    unsigned stage_bytes; // q rows + flag row, rounded up to 128
};

// Row index of the neighbour row r + (c_y, c_z) with periodic wrap, as the
// element index of its x = 0 cell.
template <class L, int D> __device__ __forceinline__ u32 nbr_row(const LbmArgs& a, u32 y, u32 z) {
    u32 yy = y, zz = z;
    if constexpr (L::cy(D) > 0) yy = y + 1U == a.ny ? 0U : y + 1U;
    if constexpr (L::cy(D) < 0) yy = y == 0U ? a.ny - 1U : y - 1U;
    if constexpr (L::cz(D) > 0) zz = z + 1U == a.nz ? 0U : z + 1U;
    if constexpr (L::cz(D) < 0) zz = z == 0U ? a.nz - 1U : z - 1U;
    return (zz * a.ny + yy) * a.nx;
}

// Stage row order: 0 rest, 1 + p pb rows, 1 + PAIRS + p pa rows, then flags.
template <class L, class S, bool FLAGS, int P = 0>
__device__ __forceinline__ void issue_pairs(const LbmArgs& a, const RowStages& g, unsigned char* st, u32 row, u32 y,
                                            u32 z, std::uint64_t* bar) {
    using T = typename S::T;
    if constexpr (P < L::PAIRS) {
        constexpr int j = 2 * P + 2;
        const T* base = static_cast<const T*>(a.base);
        bulk_load(st + (1U + P) * g.row_bytes, base + (a.pb_off[P] + row), g.row_bytes, bar);
        bulk_load(st + (1U + L::PAIRS + P) * g.row_bytes, base + (a.pa_off[P] + nbr_row<L, j>(a, y, z)), g.row_bytes,
                  bar);
        issue_pairs<L, S, FLAGS, P + 1>(a, g, st, row, y, z, bar);
    }
}

template <class L, class S, bool FLAGS>
__device__ __forceinline__ void issue_row(const LbmArgs& a, const RowStages& g, unsigned char* st, u32 r,
                                          std::uint64_t* bar) {
    using T = typename S::T;
    const u32 y = r % a.ny, z = r / a.ny;
    const u32 row = r * a.nx;
    mbar_arrive_expect_tx(bar, static_cast<unsigned>(L::Q) * g.row_bytes + (FLAGS ? a.nx : 0U));
    bulk_load(st, static_cast<const T*>(a.base) + (a.rest_off + row), g.row_bytes, bar);
    issue_pairs<L, S, FLAGS>(a, g, st, row, y, z, bar);
    if constexpr (FLAGS) bulk_load(st + L::Q * g.row_bytes, a.flags + row, a.nx, bar);
}

template <class L, class S, int P = 0>
__device__ __forceinline__ void store_pairs(const LbmArgs& a, const RowStages& g, const unsigned char* st, u32 row,
                                            u32 y, u32 z) {
    using T = typename S::T;
    if constexpr (P < L::PAIRS) {
        constexpr int j = 2 * P + 2;
        T* base = static_cast<T*>(a.base);
        bulk_store(base + (a.pb_off[P] + row), st + (1U + P) * g.row_bytes, g.row_bytes);
        bulk_store(base + (a.pa_off[P] + nbr_row<L, j>(a, y, z)), st + (1U + L::PAIRS + P) * g.row_bytes, g.row_bytes);
        store_pairs<L, S, P + 1>(a, g, st, row, y, z);
    }
}

template <class L, class S>
__device__ __forceinline__ void store_row(const LbmArgs& a, const RowStages& g, const unsigned char* st, u32 r) {
    using T = typename S::T;
    const u32 y = r % a.ny, z = r / a.ny;
    const u32 row = r * a.nx;
    bulk_store(static_cast<T*>(a.base) + (a.rest_off + row), st, g.row_bytes);
    store_pairs<L, S>(a, g, st, row, y, z);
    bulk_commit();
}

// x index of the pa slot of a cell at x for a pair whose neighbour direction has x-shift s.
__device__ __forceinline__ u32 shifted_x(int s, u32 x, u32 nx) {
    return s > 0 ? (x + 1U == nx ? 0U : x + 1U) : (s < 0 ? (x == 0U ? nx - 1U : x - 1U) : x);
}

template <class L, class S, bool RAW, int P = 0>
__device__ __forceinline__ void stage_gather(const LbmArgs& a, const typename S::T* stage, u32 nx, u32 x,
                                             typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        fin[j] = ld<S, L, j, RAW>(stage + (1U + P) * nx + x, a);
        fin[i] = ld<S, L, i, RAW>(stage + (1U + L::PAIRS + P) * nx + shifted_x(L::cx(j), x, nx), a);
        stage_gather<L, S, RAW, P + 1>(a, stage, nx, x, fin);
    }
}

template <class L, class S, bool RAW, int P = 0>
__device__ __forceinline__ void stage_scatter(const LbmArgs& a, typename S::T* stage, u32 nx, u32 x,
                                              const typename S::R* fout) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        st<S, L, i, RAW>(stage + (1U + P) * nx + x, fout[i], a);
        st<S, L, j, RAW>(stage + (1U + L::PAIRS + P) * nx + shifted_x(L::cx(j), x, nx), fout[j], a);
        stage_scatter<L, S, RAW, P + 1>(a, stage, nx, x, fout);
    }
}

// Bounce-back fix-up from global memory (wall links only).
template <class L, class S, bool RAW, int P = 0>
__device__ __forceinline__ void stage_bounce(const LbmArgs& a, u32 n, const Nbr& o, unsigned walls,
                                             typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const typename S::T* base = static_cast<const typename S::T*>(a.base);
        if ((walls >> (2 * P)) & 1U) fin[i] = ld<S, L, i, RAW>(base + (a.pb_off[P] + (n + nbr_off<L, j>(o))), a);
        if ((walls >> (2 * P + 1)) & 1U) fin[j] = ld<S, L, j, RAW>(base + (a.pa_off[P] + n), a);
        stage_bounce<L, S, RAW, P + 1>(a, n, o, walls, fin);
    }
}

template <class L, class S, bool LES, bool FLAGS, bool GRAY>
__global__ void __launch_bounds__(512, 2) k_step_rows(const __grid_constant__ LbmArgs a, const RowStages g) {
    using R = typename S::R;
    using T = typename S::T;
    constexpr bool RAW = S::scaled;
    extern __shared__ __align__(128) unsigned char smem[];
    std::uint64_t* full = reinterpret_cast<std::uint64_t*>(smem);
    unsigned char* stages = smem + 128;
    const u32 rows = a.ny * a.nz;
    const u32 tiles = blockIdx.x < rows ? (rows - blockIdx.x + gridDim.x - 1U) / gridDim.x : 0U;
    const bool leader = threadIdx.x == 0;
    if (leader) {
        for (unsigned s = 0; s < g.stages; ++s) mbar_init(&full[s], 1U);
        mbar_fence_init();
    }
    __syncthreads();
    if (leader)
        for (u32 t = 0; t < tiles && t < g.stages; ++t)
            issue_row<L, S, FLAGS>(a, g, stages + t * g.stage_bytes, blockIdx.x + t * gridDim.x, &full[t]);
    const bool force = a.has_force != 0;
    for (u32 t = 0; t < tiles; ++t) {
        const u32 s = t % g.stages;
        const unsigned parity = (t / g.stages) & 1U;
        const bool late = !mbar_wait_bounded(&full[s], parity);
        if (__syncthreads_or(late)) {
            // A stage never completed: record it, let this CTA's own copies
            // finish (bounded) and leave without touching HBM again.
            if (leader) {
                atomicExch(a.status, 1);
                for (u32 u = t; u < tiles && u < t + g.stages; ++u)
                    mbar_wait_bounded(&full[u % g.stages], (u / g.stages) & 1U);
                bulk_wait_all();
            }
            return;
        }
        const u32 r = blockIdx.x + t * gridDim.x;
        const u32 y = r % a.ny, z = r / a.ny;
        unsigned char* st_bytes = stages + s * g.stage_bytes;
        T* stage = reinterpret_cast<T*>(st_bytes);
        for (u32 x = threadIdx.x; x < a.nx; x += blockDim.x) {
            const u32 n = r * a.nx + x;
            std::uint8_t flag = 0;
            if constexpr (FLAGS) {
                flag = st_bytes[L::Q * g.row_bytes + x];
                if (flag & kFlagTypeMask) continue; // walls keep their slots
            }
            R fin[L::Q];
            fin[0] = ld<S, L, 0, RAW>(stage + x, a);
            stage_gather<L, S, RAW>(a, stage, a.nx, x, fin);
            if constexpr (FLAGS) {
                if (flag & (kFlagNearWall | kFlagNearMoving)) {
                    const Nbr o = make_nbr(a, x, y, z);
                    if (flag & kFlagNearWall) stage_bounce<L, S, RAW>(a, n, o, wall_links<L>(a, n, o), fin);
                    if constexpr (RAW)
                        gather_fixup_scaled<L>(a, n, o, flag, fin);
                    else
                        gather_fixup<L, S, true>(a, n, o, flag, fin);
                }
            }
            if constexpr (RAW) {
                if (force)
                    collide_scaled<L, LES, GRAY, true>(a, n, fin);
                else
                    collide_scaled<L, LES, GRAY, false>(a, n, fin);
            } else {
                if (force)
                    collide<L, R, LES, GRAY, true, S::delta>(a, n, fin);
                else
                    collide<L, R, LES, GRAY, false, S::delta>(a, n, fin);
            }
            st<S, L, 0, RAW>(stage + x, fin[0], a);
            stage_scatter<L, S, RAW>(a, stage, a.nx, x, fin);
        }
        fence_proxy_async(); // this thread's shared-memory writes before the bulk stores read them
        __syncthreads();
        if (leader) {
            store_row<L, S>(a, g, st_bytes, r);
            // Refill the stage freed one row ago, once its bulk stores have read it.
            if (t >= 1U && t - 1U + g.stages < tiles) {
                const u32 prev = (t - 1U) % g.stages;
                bulk_wait_read<1>();
                issue_row<L, S, FLAGS>(a, g, stages + prev * g.stage_bytes, blockIdx.x + (t - 1U + g.stages) * gridDim.x,
                                       &full[prev]);
            }
        }
    }
    if (leader) bulk_wait_all();
}

} // namespace cfdx
