// Two-cell step kernel for FP16-shifted storage (sm_100a), and the list
// kernel that steps the cells it leaves out.
//
// A thread owns the cells x0 = 2t and x0 + 1 of one x-row (nx even, so n0 is
// even and every FP16 pair (x0, x0+1) is one aligned 32-bit word).  Per
// direction it moves one word instead of two 16-bit values, and it relaxes
// both cells at once in packed f32x2 arithmetic (collide_scaled with
// V = float2), which halves the arithmetic issue slots of the collision.
//
// Walls.  The two-cell kernel steps only interior pairs: both cells fluid and
// neither next to a wall or a moving wall.  Every other pair's fluid cells
// are on a list built when the flags are set (near_list / near_count) and are
// stepped one cell per thread by k_step_list, with the one-cell kernel's
// arithmetic.  In the in-place step each slot is touched by exactly one cell,
// so the two launches never touch the same slot, and since both kernels
// compute a cell bit for bit alike the split changes no result.  The pair
// kernel thereby carries no bounce-back fix-ups, no moving-wall corrections
// and no per-cell store predicates.
//
// Loads.  The rest slot, the pb slots (at the cell itself) and the pa slots
// of pairs whose neighbour direction j has c_x(j) = 0 are aligned words.
// A pa slot with s = c_x(j) = +-1 is shifted by one element: its two values
// straddle two aligned words, both loaded (the neighbouring threads load the
// same words, so the second load hits L1) and spliced with one byte permute.
// No warp shuffles: threads are independent, a block may end mid-row.
// Stores mirror the loads: aligned words where the slot pair is aligned, two
// 16-bit stores where it is shifted.
//
// Rounding: the stochastic rounding bits of a (cell, direction) are the same
// as in the one-cell kernel (round_bits of the cell's hash, low field for a
// pair's first direction, high field for its second), so both kernels write
// identical bits.
#pragma once

#include "lbm_device.cuh"

namespace cfdx {

__device__ __forceinline__ u32 ld_word(const __half* p) { return *reinterpret_cast<const u32*>(p); }
__device__ __forceinline__ void st_word(__half* p, u32 w) { *reinterpret_cast<u32*>(p) = w; }
__device__ __forceinline__ void st_half(__half* p, u32 bits) {
    *reinterpret_cast<unsigned short*>(p) = static_cast<unsigned short>(bits);
}
// (hi half of a, lo half of b): the two elements that straddle two aligned words.
__device__ __forceinline__ u32 splice(u32 a, u32 b) { return __byte_perm(a, b, 0x5432); }
__device__ __forceinline__ float2 unpack(u32 w) {
    return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
// Low (sel 0x5410) / high (0x7632) 16-bit halves of two rounding words.
__device__ __forceinline__ u32 lo_halves(u32 x, u32 y) { return __byte_perm(x, y, 0x5410); }
__device__ __forceinline__ u32 hi_halves(u32 x, u32 y) { return __byte_perm(x, y, 0x7632); }

struct H2Ctx {
    u32 x0, xl, xr, row, n0; // xl / xr: x of the aligned words left / right of x0 (periodic)
    u32 oy[3], oz[3];
};

template <class L, int D> __device__ __forceinline__ u32 h2_row(const H2Ctx& c) {
    return c.row + c.oy[L::cy(D) + 1] + c.oz[L::cz(D) + 1];
}

// All words of the thread, loaded before any is decoded.
template <class L> struct H2Raw {
    u32 rest;
    u32 pb[L::PAIRS];
    u32 pa[L::PAIRS];
    u32 pa2[L::PAIRS]; // second word of shifted pa slots
};

template <class L, int P = 0>
__device__ __forceinline__ void h2_issue(const LbmArgs& a, const __half* base, const H2Ctx& c, H2Raw<L>& r) {
    if constexpr (P < L::PAIRS) {
        constexpr int j = 2 * P + 2;
        constexpr int s = L::cx(j);
        const u32 rj = a.pa_off[P] + h2_row<L, j>(c);
        r.pb[P] = ld_word(base + (a.pb_off[P] + c.n0));
        if constexpr (s == 0) {
            r.pa[P] = ld_word(base + (rj + c.x0));
        } else if constexpr (s > 0) { // elements x0+1, x0+2
            r.pa[P] = ld_word(base + (rj + c.x0));
            r.pa2[P] = ld_word(base + (rj + c.xr));
        } else { // elements x0-1, x0
            r.pa[P] = ld_word(base + (rj + c.xl));
            r.pa2[P] = ld_word(base + (rj + c.x0));
        }
        h2_issue<L, P + 1>(a, base, c, r);
    }
}

template <class L, int P = 0> __device__ __forceinline__ void h2_decode(const H2Raw<L>& r, float2* f) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        f[j] = unpack(r.pb[P]);
        if constexpr (L::cx(j) == 0)
            f[i] = unpack(r.pa[P]);
        else
            f[i] = unpack(splice(r.pa[P], r.pa2[P]));
        h2_decode<L, P + 1>(r, f);
    }
}

template <class L, int P = 0>
__device__ __forceinline__ void h2_stores(const LbmArgs& a, __half* base, const H2Ctx& c, const float2* f, u32 h0,
                                          u32 h1) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        constexpr int s = L::cx(j);
        const u32 k0 = round_bits(a, h0, P + 1), k1 = round_bits(a, h1, P + 1);
        // fout_i -> pb at the cells themselves
        st_word(base + (a.pb_off[P] + c.n0), f16x2_rs(f[i].y, f[i].x, lo_halves(k0, k1)));
        // fout_j -> pa at the neighbours n + c_j
        const u32 wj = f16x2_rs(f[j].y, f[j].x, hi_halves(k0, k1));
        const u32 rj = a.pa_off[P] + h2_row<L, j>(c);
        if constexpr (s == 0) {
            st_word(base + (rj + c.x0), wj);
        } else if constexpr (s > 0) { // x0 -> x0+1, x0+1 -> xr
            st_half(base + (rj + c.x0 + 1U), wj);
            st_half(base + (rj + c.xr), wj >> 16);
        } else { // x0 -> xl+1, x0+1 -> x0
            st_half(base + (rj + c.xl + 1U), wj);
            st_half(base + (rj + c.x0), wj >> 16);
        }
        h2_stores<L, P + 1>(a, base, c, f, h0, h1);
    }
}

// Resident blocks per SM (register cap 65536 / (128 * blocks)), measured on
// B200 at 512^3 D3Q19: 4 (128 registers) without Smagorinsky, 6 (80
// registers) with it.  The macros exist for tuning builds.
#ifndef CFDX_H2_MIN_BLOCKS
#define CFDX_H2_MIN_BLOCKS 4
#endif
#ifndef CFDX_H2_MIN_BLOCKS_LES
#define CFDX_H2_MIN_BLOCKS_LES 6
#endif
template <class L, bool LES, bool FLAGS, bool GRAY>
__global__ void __launch_bounds__(128, LES ? CFDX_H2_MIN_BLOCKS_LES : CFDX_H2_MIN_BLOCKS)
    k_step_h2(const __grid_constant__ LbmArgs a) {
    H2Ctx c;
    c.x0 = 2U * (blockIdx.x * blockDim.x + threadIdx.x);
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = a.z_first + blockIdx.z;
    if (c.x0 >= a.nx || y >= a.ny) return;
    c.row = (z * a.ny + y) * a.nx;
    c.n0 = c.row + c.x0;
    if constexpr (FLAGS) {
        // walls, and fluid cells next to walls, belong to k_step_list
        const unsigned both = *reinterpret_cast<const unsigned short*>(a.flags + c.n0);
        constexpr unsigned not_interior = (kFlagTypeMask | kFlagNearWall | kFlagNearMoving) * 0x0101U;
        if (both & not_interior) return;
    }
    c.xl = c.x0 == 0U ? a.nx - 2U : c.x0 - 2U;
    c.xr = c.x0 + 2U == a.nx ? 0U : c.x0 + 2U;
    const u32 plane = a.nx * a.ny;
    c.oy[0] = y == 0 ? (a.ny - 1U) * a.nx : 0U - a.nx;
    c.oy[1] = 0U;
    c.oy[2] = y == a.ny - 1U ? 0U - (a.ny - 1U) * a.nx : a.nx;
    c.oz[0] = z == 0 ? (a.nz - 1U) * plane : 0U - plane;
    c.oz[1] = 0U;
    c.oz[2] = z == a.nz - 1U ? 0U - (a.nz - 1U) * plane : plane;

    __half* base = static_cast<__half*>(a.base);
    H2Raw<L> raw;
    raw.rest = ld_word(base + (a.rest_off + c.n0));
    h2_issue<L>(a, base, c, raw);
    float2 f[L::Q];
    f[0] = unpack(raw.rest);
    h2_decode<L>(raw, f);
    if (a.has_force)
        collide_scaled<L, LES, GRAY, true>(a, c.n0, f);
    else
        collide_scaled<L, LES, GRAY, false>(a, c.n0, f);
    const u32 h0 = round_hash(a, c.n0), h1 = round_hash(a, c.n0 + 1U);
    st_word(base + (a.rest_off + c.n0),
            f16x2_rs(f[0].y, f[0].x, lo_halves(round_bits(a, h0, 0), round_bits(a, h1, 0))));
    h2_stores<L>(a, base, c, f, h0, h1);
}

// The fluid cells of the pairs k_step_h2 leaves out (a.near_list, sorted by
// cell index), one per thread, with the one-cell kernel's arithmetic: the
// wall-link gather, the moving-wall correction, the collision and the store.
template <class L, class S, bool LES, bool GRAY>
__global__ void __launch_bounds__(128, step_min_blocks<L, S>()) k_step_list(const __grid_constant__ LbmArgs a) {
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.near_count) return;
    const u32 n = a.near_list[k];
    const u32 plane = a.nx * a.ny;
    const u32 z = n / plane;
    if (z < a.z_first || z >= a.z_end) return; // outside this launch's planes
    const u32 r = n - z * plane;
    const u32 y = r / a.nx;
    const u32 x = r - y * a.nx;
    const std::uint8_t flag = a.flags[n];
    const Nbr o = make_nbr(a, x, y, z);
    typename S::R fin[L::Q];
    gather_loads<L, S, true, true, S::scaled>(a, n, o, flag, fin);
    if constexpr (S::scaled) {
        gather_fixup_scaled<L>(a, n, o, flag, fin);
        if (a.has_force)
            collide_scaled<L, LES, GRAY, true>(a, n, fin);
        else
            collide_scaled<L, LES, GRAY, false>(a, n, fin);
    } else {
        gather_fixup<L, S, true>(a, n, o, flag, fin);
        if (a.has_force)
            collide<L, typename S::R, LES, GRAY, true, S::delta>(a, n, fin);
        else
            collide<L, typename S::R, LES, GRAY, false, S::delta>(a, n, fin);
    }
    scatter<L, S, true, S::scaled>(a, n, o, fin, sizeof(typename S::T) == 2 ? round_hash(a, n) : 0U);
}

} // namespace cfdx
