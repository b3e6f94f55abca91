// Paired-cell variant of the step kernel: each thread owns the two adjacent
// cells x0 = 2t and x0 + 1 of one x-row, so every population moves as one
// 64-bit (FP32) or 32-bit (FP16) word per thread instead of two scalars.
//
// Word alignment per direction (nx even, so the cell index n0 of x0 is even):
//   * the rest slot and the pb slots sit at n0, n0+1: one aligned word;
//   * pa slots of pairs whose neighbour direction j has c_x(j) = 0 sit at the
//     same x in a neighbouring row: one aligned word;
//   * pa slots with s = c_x(j) = +-1 are shifted by one element: the thread
//     loads the aligned word W whose low half is its second cell's value; its
//     first cell's value is the high half of lane-1's word (one warp
//     shuffle).  Lane 0 loads that element directly.  Stores mirror this: a
//     thread writes W = (its second cell's value, lane+1's first cell's
//     value) when both cells are fluid, and single elements otherwise, so no
//     slot owned by a wall (which may carry a bounced population) is touched.
// All words of a thread are loaded before the first is decoded or shuffled,
// so the loads overlap.  Bounce-back is a fix-up: near-wall cells reload only
// their wall links from the partner slot.  Addresses are element offsets from
// one base pointer (32-bit, q*N < 2^32), so each access is one add and one
// wide multiply-add.
// Blocks are whole warps along x (blockDim.x a multiple of 32), so a warp
// never spans two rows.
#pragma once

#include "lbm_device.cuh"

namespace cfdx {

template <class S> struct Pair;

template <> struct Pair<StF32> {
    using W = float2;
    template <class L, int D> __device__ __forceinline__ static void decode(W w, float& lo, float& hi, const LbmArgs&) {
        lo = w.x;
        hi = w.y;
    }
    template <class L, int D> __device__ __forceinline__ static W encode(float lo, float hi, const LbmArgs&) {
        return make_float2(lo, hi);
    }
};

// FP16 words stay in storage units (see collide_scaled).
template <> struct Pair<StF16> {
    using W = __half2;
    template <class L, int D> __device__ __forceinline__ static void decode(W w, float& lo, float& hi, const LbmArgs&) {
        const float2 f = __half22float2(w);
        lo = f.x;
        hi = f.y;
    }
    template <class L, int D> __device__ __forceinline__ static W encode(float lo, float hi, const LbmArgs&) {
        return __floats2half2_rn(lo, hi);
    }
};

// Per-thread context of one cell pair.
struct PairCtx {
    u32 lane, x0, row, n0;
    u32 h0, h1, h2; // FP16 rounding hashes of cells n0, n0+1 and n0+2 (lane+1's first cell)
    u32 oy[3], oz[3];
    unsigned live0_mask, live1_mask; // ballots over the warp
    bool live0, live1, valid;
};

template <class L, int D> __device__ __forceinline__ u32 row_of(const PairCtx& c) {
    return c.row + c.oy[L::cy(D) + 1] + c.oz[L::cz(D) + 1];
}

// x of the aligned word W holding the second cell's pa value (shift s), and
// x of the first cell's pa value, both with periodic wrap.
__device__ __forceinline__ u32 word_x(int s, u32 x0, u32 nx) { return s > 0 ? (x0 + 2U == nx ? 0U : x0 + 2U) : x0; }
__device__ __forceinline__ u32 first_x(int s, u32 x0, u32 nx) { return s > 0 ? x0 + 1U : (x0 == 0U ? nx - 1U : x0 - 1U); }

// Raw words of one cell pair, loaded before any of them is used so that all
// loads of the thread are in flight together.
template <class L, class S> struct PairRaw {
    typename Pair<S>::W rest;
    typename Pair<S>::W pb[L::PAIRS];
    typename Pair<S>::W pa[L::PAIRS];
    typename S::T first[L::PAIRS]; // lane 0: the first cell's shifted pa element
};

// Address of the aligned pa word of pair P (x-shift s = c_x(j)).
template <class L, int P> __device__ __forceinline__ u32 pa_word(const LbmArgs& a, const PairCtx& c) {
    constexpr int j = 2 * P + 2;
    constexpr int s = L::cx(j);
    return a.pa_off[P] + row_of<L, j>(c) + (s == 0 ? c.x0 : word_x(s, c.x0, a.nx));
}

template <class L, class S, int P = 0>
__device__ __forceinline__ void pair_issue(const LbmArgs& a, const typename S::T* base, const PairCtx& c,
                                           PairRaw<L, S>& r) {
    using V = typename Pair<S>::W;
    if constexpr (P < L::PAIRS) {
        constexpr int j = 2 * P + 2;
        constexpr int s = L::cx(j);
        // Lanes past the row end read the row start instead (values unused).
        r.pb[P] = *reinterpret_cast<const V*>(base + (a.pb_off[P] + (c.valid ? c.n0 : c.row)));
        r.pa[P] = *reinterpret_cast<const V*>(base + (c.valid ? pa_word<L, P>(a, c) : a.pa_off[P] + row_of<L, j>(c)));
        if constexpr (s != 0) {
            if (c.lane == 0U && c.valid)
                r.first[P] = base[a.pa_off[P] + row_of<L, j>(c) + first_x(s, c.x0, a.nx)];
        }
        pair_issue<L, S, P + 1>(a, base, c, r);
    }
}

template <class L, class S, int P = 0>
__device__ __forceinline__ void pair_decode(const LbmArgs& a, const PairCtx& c, const PairRaw<L, S>& r,
                                            typename S::R* f0, typename S::R* f1) {
    using R = typename S::R;
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        constexpr int s = L::cx(j);
        Pair<S>::template decode<L, j>(r.pb[P], f0[j], f1[j], a);
        if constexpr (s == 0) {
            Pair<S>::template decode<L, i>(r.pa[P], f0[i], f1[i], a);
        } else {
            R lo, hi;
            Pair<S>::template decode<L, i>(r.pa[P], lo, hi, a);
            f1[i] = lo;
            const R up = __shfl_up_sync(0xffffffffU, hi, 1);
            f0[i] = c.lane == 0U ? ld<S, L, i, S::scaled>(&r.first[P], a) : up;
        }
        pair_decode<L, S, P + 1>(a, c, r, f0, f1);
    }
}

// Writes the two values of one aligned word, or only the live one.  FP16:
// rb holds the rounding bits of v0 in [12:0] and of v1 in [28:16] (the same
// bits the one-cell kernel uses for these cells and this direction).
template <class L, class S, int D>
__device__ __forceinline__ void store_word(const LbmArgs& a, typename S::T* p, bool live0, bool live1,
                                           typename S::R v0, typename S::R v1, u32 rb) {
    using V = typename Pair<S>::W;
    if constexpr (sizeof(typename S::T) == 2) {
        if (live0 && live1) {
            *reinterpret_cast<u32*>(p) = f16x2_rs(v1, v0, rb);
        } else {
            if (live0) st_h16(p, v0, rb);
            if (live1) st_h16(p + 1, v1, rb >> 16);
        }
    } else {
        if (live0 && live1) {
            *reinterpret_cast<V*>(p) = Pair<S>::template encode<L, D>(v0, v1, a);
        } else {
            if (live0) st<S, L, D, S::scaled>(p, v0, a);
            if (live1) st<S, L, D, S::scaled>(p + 1, v1, a);
        }
    }
}

// Low (sel 0x5410) or high (0x7632) 16-bit halves of two rounding words.
__device__ __forceinline__ u32 low_halves(u32 x, u32 y) { return __byte_perm(x, y, 0x5410); }
__device__ __forceinline__ u32 high_halves(u32 x, u32 y) { return __byte_perm(x, y, 0x7632); }

template <class L, class S, int P = 0>
__device__ __forceinline__ void pair_stores(const LbmArgs& a, typename S::T* base, const PairCtx& c,
                                            const typename S::R* f0, const typename S::R* f1) {
    using R = typename S::R;
    using V = typename Pair<S>::W;
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        constexpr int s = L::cx(j);
        constexpr bool h16 = sizeof(typename S::T) == 2;
        // rounding words of this pair for cells n0, n0+1, n0+2 (FP16 only)
        const u32 k0 = h16 ? round_bits(a, c.h0, P + 1) : 0U;
        const u32 k1 = h16 ? round_bits(a, c.h1, P + 1) : 0U;
        // fout_i -> pb at the pair itself
        store_word<L, S, i>(a, base + (a.pb_off[P] + c.n0), c.live0, c.live1, f0[i], f1[i], low_halves(k0, k1));
        // fout_j -> pa at the neighbour nb = n + c_j
        const u32 rj = row_of<L, j>(c);
        if constexpr (s == 0) {
            store_word<L, S, j>(a, base + (a.pa_off[P] + rj + c.x0), c.live0, c.live1, f0[j], f1[j],
                                high_halves(k0, k1));
        } else {
            const bool next_live0 = c.lane < 31U && ((c.live0_mask >> (c.lane + 1U)) & 1U);
            const bool prev_live1 = c.lane > 0U && ((c.live1_mask >> (c.lane - 1U)) & 1U);
            const R next = __shfl_down_sync(0xffffffffU, f0[j], 1);
            typename S::T* pw = base + (a.pa_off[P] + rj + word_x(s, c.x0, a.nx));
            if (c.live1) {
                if constexpr (h16) {
                    // cells n0+1 (this thread) and n0+2 (lane+1's first cell)
                    const u32 rb = high_halves(k1, round_bits(a, c.h2, P + 1));
                    if (next_live0)
                        *reinterpret_cast<u32*>(pw) = f16x2_rs(next, f1[j], rb);
                    else
                        st_h16(pw, f1[j], rb);
                } else {
                    if (next_live0)
                        *reinterpret_cast<V*>(pw) = Pair<S>::template encode<L, j>(f1[j], next, a);
                    else
                        st<S, L, j, S::scaled>(pw, f1[j], a);
                }
            }
            if (c.live0 && !prev_live1) {
                typename S::T* pf = base + (a.pa_off[P] + rj + first_x(s, c.x0, a.nx));
                if constexpr (h16)
                    st_h16(pf, f0[j], k0 >> 16);
                else
                    st<S, L, j, S::scaled>(pf, f0[j], a);
            }
        }
        pair_stores<L, S, P + 1>(a, base, c, f0, f1);
    }
}

template <class L, class S, bool LES, bool FLAGS, bool GRAY>
__global__ void __launch_bounds__(128, pair_min_blocks<S>()) k_step_x2(const __grid_constant__ LbmArgs a) {
    using R = typename S::R;
    using T = typename S::T;
    PairCtx c;
    c.lane = threadIdx.x & 31U;
    c.x0 = 2U * (blockIdx.x * blockDim.x + threadIdx.x);
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = a.z_first + blockIdx.z;
    if (y >= a.ny) return; // warp-uniform: a warp never spans rows
    c.valid = c.x0 < a.nx;
    c.row = (z * a.ny + y) * a.nx;
    c.n0 = c.row + c.x0;
    std::uint8_t fl0 = 0, fl1 = 0;
    if constexpr (FLAGS) {
        if (c.valid) {
            const unsigned short both = *reinterpret_cast<const unsigned short*>(a.flags + c.n0);
            fl0 = static_cast<std::uint8_t>(both & 0xffU);
            fl1 = static_cast<std::uint8_t>(both >> 8);
        }
    }
    c.live0 = c.valid && (fl0 & kFlagTypeMask) == 0;
    c.live1 = c.valid && (fl1 & kFlagTypeMask) == 0;
    c.live0_mask = __ballot_sync(0xffffffffU, c.live0);
    c.live1_mask = __ballot_sync(0xffffffffU, c.live1);
    if ((c.live0_mask | c.live1_mask) == 0U) return; // warp-uniform
    const u32 plane = a.nx * a.ny;
    c.oy[0] = y == 0 ? (a.ny - 1U) * a.nx : 0U - a.nx;
    c.oy[1] = 0U;
    c.oy[2] = y == a.ny - 1U ? 0U - (a.ny - 1U) * a.nx : a.nx;
    c.oz[0] = z == 0 ? (a.nz - 1U) * plane : 0U - plane;
    c.oz[1] = 0U;
    c.oz[2] = z == a.nz - 1U ? 0U - (a.nz - 1U) * plane : plane;

    T* base = static_cast<T*>(a.base);
    PairRaw<L, S> raw;
    raw.rest = *reinterpret_cast<const typename Pair<S>::W*>(base + (a.rest_off + (c.valid ? c.n0 : c.row)));
    pair_issue<L, S>(a, base, c, raw);
    R f0[L::Q], f1[L::Q];
    Pair<S>::template decode<L, 0>(raw.rest, f0[0], f1[0], a);
    pair_decode<L, S>(a, c, raw, f0, f1);

    if constexpr (FLAGS) {
        if (c.live0 && (fl0 & (kFlagNearWall | kFlagNearMoving))) {
            const Nbr o = make_nbr(a, c.x0, y, z);
            if (fl0 & kFlagNearWall) bounce_fixup<L, S>(a, base, c.n0, o, a.wall_mask[c.n0], f0);
            if constexpr (S::scaled)
                gather_fixup_scaled<L>(a, c.n0, o, fl0, f0);
            else
                gather_fixup<L, S, true>(a, c.n0, o, fl0, f0);
        }
        if (c.live1 && (fl1 & (kFlagNearWall | kFlagNearMoving))) {
            const Nbr o = make_nbr(a, c.x0 + 1U, y, z);
            if (fl1 & kFlagNearWall) bounce_fixup<L, S>(a, base, c.n0 + 1U, o, a.wall_mask[c.n0 + 1U], f1);
            if constexpr (S::scaled)
                gather_fixup_scaled<L>(a, c.n0 + 1U, o, fl1, f1);
            else
                gather_fixup<L, S, true>(a, c.n0 + 1U, o, fl1, f1);
        }
    }

    const bool force = a.has_force != 0;
    auto relax = [&](u32 n, R* f) {
        if constexpr (S::scaled) {
            if (force)
                collide_scaled<L, LES, GRAY, true>(a, n, f);
            else
                collide_scaled<L, LES, GRAY, false>(a, n, f);
        } else {
            if (force)
                collide<L, R, LES, GRAY, true, S::delta>(a, n, f);
            else
                collide<L, R, LES, GRAY, false, S::delta>(a, n, f);
        }
    };
    if (c.live0) relax(c.n0, f0);
    if (c.live1) relax(c.n0 + 1U, f1);

    if constexpr (sizeof(T) == 2) {
        c.h0 = round_hash(a, c.n0);
        c.h1 = round_hash(a, c.n0 + 1U);
        c.h2 = __shfl_down_sync(0xffffffffU, c.h0, 1); // lane 31's value is never used
    } else {
        c.h0 = c.h1 = c.h2 = 0U;
    }
    store_word<L, S, 0>(a, base + (a.rest_off + c.n0), c.live0, c.live1, f0[0], f1[0],
                        low_halves(round_bits(a, c.h0, 0), round_bits(a, c.h1, 0)));
    pair_stores<L, S>(a, base, c, f0, f1);
}

} // namespace cfdx
