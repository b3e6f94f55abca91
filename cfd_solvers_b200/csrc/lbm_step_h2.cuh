// Two-cell step kernel for FP16-shifted storage (sm_100a).
//
// A thread owns the cells x0 = 2t and x0 + 1 of one x-row (nx even, so n0 is
// even and every FP16 pair (x0, x0+1) is one aligned 32-bit word).  Per
// direction it moves one word instead of two 16-bit values, and it relaxes
// both cells at once in packed f32x2 arithmetic (collide_scaled with
// V = float2), which halves the arithmetic issue slots of the collision.
//
// Loads.  The rest slot, the pb slots (at the cell itself) and the pa slots
// of pairs whose neighbour direction j has c_x(j) = 0 are aligned words.
// A pa slot with s = c_x(j) = +-1 is shifted by one element: its two values
// straddle two aligned words, both loaded (the neighbouring threads load the
// same words, so the second load hits L1) and spliced with one byte permute.
// No warp shuffles: threads are independent, a block may end mid-row.
//
// Stores mirror the loads: aligned words where the slot pair is aligned and
// both cells are fluid, single 16-bit stores otherwise (a wall cell's slots
// can hold bounced populations of its fluid neighbours and are not touched).
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
    bool live0, live1;
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

// Stores one converted word w (low half: cell x0, high half: cell x0+1) to an
// aligned slot pair.  BOTH: both cells are fluid (no per-cell predicates).
template <bool BOTH> __device__ __forceinline__ void h2_store_aligned(__half* p, u32 w, bool live0, bool live1) {
    if (BOTH || (live0 && live1)) {
        st_word(p, w);
    } else {
        if (live0) st_half(p, w);
        if (live1) st_half(p + 1, w >> 16);
    }
}

template <class L, bool BOTH, int P = 0>
__device__ __forceinline__ void h2_stores(const LbmArgs& a, __half* base, const H2Ctx& c, const float2* f, u32 h0,
                                          u32 h1) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        constexpr int s = L::cx(j);
        const u32 k0 = round_bits(a, h0, P + 1), k1 = round_bits(a, h1, P + 1);
        // fout_i -> pb at the cells themselves
        h2_store_aligned<BOTH>(base + (a.pb_off[P] + c.n0), f16x2_rs(f[i].y, f[i].x, lo_halves(k0, k1)), c.live0,
                               c.live1);
        // fout_j -> pa at the neighbours n + c_j
        const u32 wj = f16x2_rs(f[j].y, f[j].x, hi_halves(k0, k1));
        const u32 rj = a.pa_off[P] + h2_row<L, j>(c);
        if constexpr (s == 0) {
            h2_store_aligned<BOTH>(base + (rj + c.x0), wj, c.live0, c.live1);
        } else if constexpr (s > 0) { // x0 -> x0+1, x0+1 -> xr
            if (BOTH || c.live0) st_half(base + (rj + c.x0 + 1U), wj);
            if (BOTH || c.live1) st_half(base + (rj + c.xr), wj >> 16);
        } else { // x0 -> xl+1, x0+1 -> x0
            if (BOTH || c.live0) st_half(base + (rj + c.xl + 1U), wj);
            if (BOTH || c.live1) st_half(base + (rj + c.x0), wj >> 16);
        }
        h2_stores<L, BOTH, P + 1>(a, base, c, f, h0, h1);
    }
}

// Half-way bounce-back of one cell (lane LANE of the packed values): wall
// links reload the partner slot -- direction i from pb at its source n + c_j,
// direction j from pa at the cell itself -- straight into the lane.
template <int LANE> __device__ __forceinline__ float& lane_of(float2& v) {
    if constexpr (LANE == 0) return v.x; else return v.y;
}

template <class L, int LANE, int P = 0>
__device__ __forceinline__ void h2_bounce(const LbmArgs& a, const __half* base, const H2Ctx& c, u32 walls,
                                          float2* f) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        constexpr int s = L::cx(j);
        const u32 n = c.n0 + LANE;
        if ((walls >> (2 * P)) & 1U) {
            // x of n + c_j: lane 0 -> x0 + s, lane 1 -> x0 + 1 + s (periodic)
            const u32 xs = s == 0 ? c.x0 + LANE
                                  : (s > 0 ? (LANE == 0 ? c.x0 + 1U : c.xr) : (LANE == 0 ? c.xl + 1U : c.x0));
            lane_of<LANE>(f[i]) = __half2float(base[a.pb_off[P] + h2_row<L, j>(c) + xs]);
        }
        if ((walls >> (2 * P + 1)) & 1U) lane_of<LANE>(f[j]) = __half2float(base[a.pa_off[P] + n]);
        h2_bounce<L, LANE, P + 1>(a, base, c, walls, f);
    }
}

// Near-wall fix-ups of one cell: bounce-back reloads, then (next to a moving
// wall, rare) the moving-wall correction on a copy of the lane.
template <class L, int LANE>
__device__ __forceinline__ void h2_fixup(const LbmArgs& a, const __half* base, const H2Ctx& c, u32 y, u32 z,
                                         std::uint8_t flag, float2* f) {
    const u32 n = c.n0 + LANE;
    if (flag & kFlagNearWall) h2_bounce<L, LANE>(a, base, c, a.wall_mask[n], f);
    if (flag & kFlagNearMoving) {
        float v[L::Q];
#pragma unroll
        for (int d = 0; d < L::Q; ++d) v[d] = lane_of<LANE>(f[d]);
        gather_fixup_scaled<L>(a, n, make_nbr(a, c.x0 + LANE, y, z), flag, v);
#pragma unroll
        for (int d = 0; d < L::Q; ++d) lane_of<LANE>(f[d]) = v[d];
    }
}

// Resident blocks per SM (register cap 65536 / (128 * blocks)), measured on
// B200 at 512^3 D3Q19: 4 (128 registers, no spills) for the plain periodic
// step (64.0 GLUPS BGK vs 57.1 uncapped), 6 (80 registers) with Smagorinsky
// or walls (LES cavity 45.9 GLUPS vs 34.3 uncapped and 40.2 at 4): the
// near-wall paths need the occupancy.  The predicate-free store path for
// fully fluid pairs pays off without LES only (LES cavity 45.2 without it,
// 42.6 with: it costs spills at 80 registers).
#ifndef CFDX_H2_MIN_BLOCKS
#define CFDX_H2_MIN_BLOCKS 4
#endif
#ifndef CFDX_H2_MIN_BLOCKS_LES
#define CFDX_H2_MIN_BLOCKS_LES 6
#endif
#ifndef CFDX_H2_MIN_BLOCKS_WALLS
#define CFDX_H2_MIN_BLOCKS_WALLS 6
#endif
#ifndef CFDX_H2_FAST_STORES
#define CFDX_H2_FAST_STORES 1
#endif
template <class L, bool LES, bool FLAGS, bool GRAY>
__global__ void __launch_bounds__(128, LES ? CFDX_H2_MIN_BLOCKS_LES
                                          : (FLAGS ? CFDX_H2_MIN_BLOCKS_WALLS : CFDX_H2_MIN_BLOCKS))
    k_step_h2(const __grid_constant__ LbmArgs a) {
    H2Ctx c;
    c.x0 = 2U * (blockIdx.x * blockDim.x + threadIdx.x);
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (c.x0 >= a.nx || y >= a.ny) return;
    c.row = (z * a.ny + y) * a.nx;
    c.n0 = c.row + c.x0;
    std::uint8_t fl0 = 0, fl1 = 0;
    if constexpr (FLAGS) {
        const unsigned short both = *reinterpret_cast<const unsigned short*>(a.flags + c.n0);
        fl0 = static_cast<std::uint8_t>(both & 0xffU);
        fl1 = static_cast<std::uint8_t>(both >> 8);
    }
    c.live0 = (fl0 & kFlagTypeMask) == 0;
    c.live1 = (fl1 & kFlagTypeMask) == 0;
    if (!c.live0 && !c.live1) return;
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
    if constexpr (FLAGS) {
        if (c.live0 && (fl0 & (kFlagNearWall | kFlagNearMoving))) h2_fixup<L, 0>(a, base, c, y, z, fl0, f);
        if (c.live1 && (fl1 & (kFlagNearWall | kFlagNearMoving))) h2_fixup<L, 1>(a, base, c, y, z, fl1, f);
    }
    if (a.has_force)
        collide_scaled<L, LES, GRAY, true>(a, c.n0, f);
    else
        collide_scaled<L, LES, GRAY, false>(a, c.n0, f);
    const u32 h0 = round_hash(a, c.n0), h1 = round_hash(a, c.n0 + 1U);
    const u32 w0 = f16x2_rs(f[0].y, f[0].x, lo_halves(round_bits(a, h0, 0), round_bits(a, h1, 0)));
    if (CFDX_H2_FAST_STORES && !LES && c.live0 && c.live1) { // the common case: no per-cell predicates
        h2_store_aligned<true>(base + (a.rest_off + c.n0), w0, true, true);
        h2_stores<L, true>(a, base, c, f, h0, h1);
    } else {
        h2_store_aligned<false>(base + (a.rest_off + c.n0), w0, c.live0, c.live1);
        h2_stores<L, false>(a, base, c, f, h0, h1);
    }
}


} // namespace cfdx
