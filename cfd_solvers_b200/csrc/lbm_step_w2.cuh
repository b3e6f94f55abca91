// Wall-aware two-cell step kernel for FP16-shifted storage (sm_100a).
//
// A thread owns the cells x0 = 2t and x0 + 1 of an x-row (nx even) and
// marches through `planes` consecutive z-planes.  Every FP16 slot pair
// (x0, x0+1) is one aligned 32-bit word, so a pair of cells costs one word
// access per direction where the one-cell kernel spends two 16-bit ones, and
// both cells relax together in packed f32x2 arithmetic (collide_scaled with
// V = float2).
//
// Loads.  Per plane a thread reads the rest word, the pb words at its own
// cells and the pa words at the neighbours n + c_j: aligned rows where
// c_x(j) = 0, and two aligned words spliced by one byte permute where the row
// is shifted by one element (the neighbouring thread reads the same words,
// so the second access hits L1).  In the pipelined form (PIPE) the words of
// plane z + 1 are copied into the thread's own shared-memory slots with
// 4-byte cp.async while plane z is relaxed, so loads stay in flight through
// the collision without holding registers; each thread reads back only what
// it copied itself, so no block barrier is involved (cp.async.wait_group
// makes a thread's own copies visible to it).
//
// Walls (half-way bounce-back in place, as the one-cell kernel's gather).  A
// wall link only changes which slot a load takes: the source's other slot at
// the same address (same element, the other table).  Stores are the same
// slots with or without walls.  A pair holding a wall cell stores its fluid
// cell's halves alone: the wall cell is not stepped, and its slots hold what
// fluid neighbours wrote in the previous step and read back in this one.  A
// cell next to a moving wall gets the one-cell kernel's correction lane by
// lane.  Warps without near-wall cells skip all of this on uniform branches,
// so there is no near-wall cell list and no second launch.
//   Pipelined form: the flags of a plane are read three planes ahead (a ring
// in shared memory) and the wall-link masks of its near-wall pairs two
// planes ahead of the issue (two spare words of the stage), so when the words
// of plane z + 1 are issued their tables are known.  A warp holding a
// near-wall pair copies every word from the table a wall link selects: a
// shifted word (one cell's element) by its cell's link, an aligned word (both
// cells' elements) by the link of the pair's fluid cell, or of cell x0 when
// both are fluid.  Where two fluid cells disagree on an aligned link, the
// second cell's half is fixed with one 16-bit load once the words arrive (the
// fix bits are written beside the words).  The relaxation waits on no mask.
//   Unpipelined form: plain words for every pair; the cells with wall links
// replace their bounced halves with 16-bit loads of the partner slots.
//
// Results equal the one-cell kernel's bit for bit: the same loads, the same
// explicitly rounded collision (collide_scaled), the moving-wall correction
// by the same function, and the same stochastic rounding bits per (cell,
// direction).
//
// In-place safety of the prefetch: within a step every slot is read and
// written by exactly one cell, so the words of plane z + 1 that a thread
// copies early are slots no other cell writes in this step.  The only other
// data in those words are the unused halves of shifted words (another cell's
// slot), which are discarded.
#pragma once

#include "lbm_step_h2.cuh"

namespace cfdx {

// Word slots of one thread's pair of cells, in issue order: 0 the rest word,
// 1 + p the pb word of pair p, then the pa words of each pair (two for a pair
// whose neighbour direction j has c_x(j) != 0).
template <class L> struct W2Words {
    __host__ __device__ static constexpr bool shifted(int p) { return L::cx(2 * p + 2) != 0; }
    __host__ __device__ static constexpr int pa_slot(int p) {
        int k = 1 + L::PAIRS;
        for (int q = 0; q < p; ++q) k += shifted(q) ? 2 : 1;
        return k;
    }
    static constexpr int count = pa_slot(L::PAIRS);
    // pair of pa word slot k (k > PAIRS)
    __host__ __device__ static constexpr int pa_pair(int k) {
        int p = 0;
        while (p + 1 < L::PAIRS && pa_slot(p + 1) <= k) ++p;
        return p;
    }
    // Word slot k (k >= 1) holds both cells' elements (an aligned pb or pa word);
    // otherwise it is one of the two words of a shifted pa slot.
    __host__ __device__ static constexpr bool aligned(int k) { return k <= L::PAIRS || !shifted(pa_pair(k)); }
    // Cell whose source element a shifted word holds: the first word holds cell
    // x0's (x0 + 1 or x0 - 1), the second cell x0 + 1's (x0 + 2 or x0).
    __host__ __device__ static constexpr int cell_of(int k) { return k - pa_slot(pa_pair(k)); }
    // Wall-link bit of slot k (k >= 1): a pb word carries direction j = 2p + 2
    // (bit 2p + 1), a pa word direction i = 2p + 1 (bit 2p).
    __host__ __device__ static constexpr u32 link_bit(int k) {
        return k <= L::PAIRS ? (2U << (2 * (k - 1))) : (1U << (2 * pa_pair(k)));
    }
    // Wall-link bits of the aligned slots.
    __host__ __device__ static constexpr u32 aligned_bits() {
        u32 m = 0U;
        for (int k = 1; k < count; ++k) m |= aligned(k) ? link_bit(k) : 0U;
        return m;
    }
};

// Per-thread indices; n0 / nl / nr (the plane's row index plus x0 / xl / xr)
// change with the plane, the rest does not.
struct W2Ctx {
    u32 x0, xl, xr, y, z; // xl / xr: x of the aligned words left / right of x0 (periodic)
    u32 n0, nl, nr;
    u32 oy[3], oz[3];     // row offsets of the y / z neighbours (periodic), [c + 1]
};

__device__ __forceinline__ void w2_thread(const LbmArgs& a, u32 x0, u32 y, W2Ctx& c) {
    c.x0 = x0;
    c.y = y;
    c.xl = x0 == 0U ? a.nx - 2U : x0 - 2U;
    c.xr = x0 + 2U == a.nx ? 0U : x0 + 2U;
    c.oy[0] = y == 0 ? (a.ny - 1U) * a.nx : 0U - a.nx;
    c.oy[1] = 0U;
    c.oy[2] = y == a.ny - 1U ? 0U - (a.ny - 1U) * a.nx : a.nx;
}

__device__ __forceinline__ void w2_plane(const LbmArgs& a, u32 z, W2Ctx& c) {
    c.z = z;
    const u32 row = (z * a.ny + c.y) * a.nx;
    c.n0 = row + c.x0;
    c.nl = row + c.xl;
    c.nr = row + c.xr;
    const u32 plane = a.nx * a.ny;
    c.oz[0] = z == 0 ? (a.nz - 1U) * plane : 0U - plane;
    c.oz[1] = 0U;
    c.oz[2] = z == a.nz - 1U ? 0U - (a.nz - 1U) * plane : plane;
}

// Offset from a cell's row to the row of its neighbour n + c_D (periodic in y and z).
template <class L, int D> __device__ __forceinline__ u32 w2_dyz(const W2Ctx& c) {
    return c.oy[L::cy(D) + 1] + c.oz[L::cz(D) + 1];
}

// Slot tables as pointers: a slot address is a table pointer (uniform across
// the launch, built from the kernel parameters) plus one 32-bit per-thread
// index.  Measured on B200 against widening a 32-bit sum of table offset and
// index per access: +10 % on the 512^3 FP16 cavity.
__device__ __forceinline__ __half* w2_tab(const LbmArgs& a, u32 off) { return static_cast<__half*>(a.base) + off; }

// Element index (within its table) of the first element of word slot K >= 1,
// and the slot's table offset: plain, or (ALT) the table a wall link reads.
template <class L, int K> __device__ __forceinline__ u32 w2_word_idx(const W2Ctx& c) {
    if constexpr (K <= L::PAIRS) {
        return c.n0;
    } else {
        constexpr int p = W2Words<L>::pa_pair(K);
        constexpr int second = K - W2Words<L>::pa_slot(p);
        constexpr int j = 2 * p + 2, s = L::cx(j);
        const u32 dyz = w2_dyz<L, j>(c);
        if constexpr (s == 0) return c.n0 + dyz;
        else if constexpr (s > 0) return (second ? c.nr : c.n0) + dyz;
        else return (second ? c.n0 : c.nl) + dyz;
    }
}
template <class L, int K, bool ALT> __device__ __forceinline__ u32 w2_table(const LbmArgs& a) {
    if constexpr (K <= L::PAIRS) return ALT ? a.pa_off[K - 1] : a.pb_off[K - 1];
    else return ALT ? a.pb_off[W2Words<L>::pa_pair(K)] : a.pa_off[W2Words<L>::pa_pair(K)];
}

// Address of word slot K.
template <class L, int K> __device__ __forceinline__ const __half* w2_word_ptr(const LbmArgs& a, const W2Ctx& c) {
    if constexpr (K == 0) {
        return w2_tab(a, a.rest_off) + c.n0;
    } else if constexpr (K <= L::PAIRS) {
        return w2_tab(a, a.pb_off[K - 1]) + c.n0;
    } else {
        constexpr int p = W2Words<L>::pa_pair(K);
        constexpr int second = K - W2Words<L>::pa_slot(p);
        constexpr int j = 2 * p + 2, s = L::cx(j);
        const u32 dyz = w2_dyz<L, j>(c);
        const __half* t = w2_tab(a, a.pa_off[p]);
        if constexpr (s == 0) return t + (c.n0 + dyz);
        else if constexpr (s > 0) return t + ((second ? c.nr : c.n0) + dyz); // elements x0+1, x0+2
        else return t + ((second ? c.n0 : c.nl) + dyz);                      // elements x0-1, x0
    }
}

// Calls f(std::integral_constant<int, k>, address) for every word slot k.
template <class L, int K = 0, class F> __device__ __forceinline__ void w2_words(const LbmArgs& a, const W2Ctx& c, F&& f) {
    if constexpr (K < W2Words<L>::count) {
        f(std::integral_constant<int, K>{}, w2_word_ptr<L, K>(a, c));
        w2_words<L, K + 1>(a, c, f);
    }
}

__device__ __forceinline__ u32 ld_u16(const __half* p) { return *reinterpret_cast<const unsigned short*>(p); }
__device__ __forceinline__ u32 with_lo(u32 w, u32 h) { return (w & 0xffff0000U) | h; }
__device__ __forceinline__ u32 with_hi(u32 w, u32 h) { return (w & 0x0000ffffU) | (h << 16); }

// Near-wall form: calls f(std::integral_constant<int, k>, address) for every
// word slot k with the table a wall link selects: for a shifted word the
// link of the cell whose source it holds (masks m0, m1 of cells x0, x0 + 1),
// for an aligned word (both cells' elements) the links in ma.
template <class L, int K = 0, class F>
__device__ __forceinline__ void w2_near_words(const LbmArgs& a, const W2Ctx& c, u32 m0, u32 m1, u32 ma, F&& f) {
    using W = W2Words<L>;
    if constexpr (K < W::count) {
        if constexpr (K == 0) {
            f(std::integral_constant<int, 0>{}, w2_word_ptr<L, 0>(a, c));
        } else {
            constexpr u32 bit = W::link_bit(K);
            const u32 m = W::aligned(K) ? ma : (W::cell_of(K) ? m1 : m0);
            const u32 t = (m & bit) ? w2_table<L, K, true>(a) : w2_table<L, K, false>(a);
            f(std::integral_constant<int, K>{}, w2_tab(a, t) + w2_word_idx<L, K>(c));
        }
        w2_near_words<L, K + 1>(a, c, m0, m1, ma, f);
    }
}

// Direction whose half-pair an aligned word slot K >= 1 holds: j of a pb word, i of a pa word.
template <class L, int K> constexpr int w2_dir() {
    return K <= L::PAIRS ? 2 * K : 2 * W2Words<L>::pa_pair(K) + 1;
}

// Cell x0 + 1's half of the aligned words whose table differs from cell x0's
// (a pair whose two fluid cells disagree on such a link): reloaded from the
// other table (bits in to_alt: the alternative table, in to_plain: the plain one).
template <class L, int K = 1>
__device__ __forceinline__ void w2_fix_second(const LbmArgs& a, const W2Ctx& c, u32 to_alt, u32 to_plain, u32* pw) {
    using W = W2Words<L>;
    if constexpr (K < W::count) {
        if constexpr (W::aligned(K)) {
            constexpr u32 bit = W::link_bit(K);
            constexpr int d = w2_dir<L, K>();
            if ((to_alt | to_plain) & bit) {
                const u32 t = (to_alt & bit) ? w2_table<L, K, true>(a) : w2_table<L, K, false>(a);
                pw[d] = with_hi(pw[d], ld_u16(w2_tab(a, t) + (w2_word_idx<L, K>(c) + 1U)));
            }
        }
        w2_fix_second<L, K + 1>(a, c, to_alt, to_plain, pw);
    }
}

// Pair words (low half: cell x0, high half: cell x0 + 1) of every direction
// from the raw words, as if the pair had no walls.
template <class L> __device__ __forceinline__ void w2_assemble(const u32* raw, u32* pw) {
    pw[0] = raw[0];
    static_for_pairs<L>([&](auto PP) {
        constexpr int p = decltype(PP)::value;
        constexpr int i = 2 * p + 1, j = i + 1;
        constexpr int k = W2Words<L>::pa_slot(p);
        pw[j] = raw[1 + p];
        if constexpr (W2Words<L>::shifted(p))
            pw[i] = splice(raw[k], raw[k + 1]);
        else
            pw[i] = raw[k];
    });
}


// Index, within the cell's own row plane, of the source element of cell
// x0 + C for a direction with c_x = S (the halves of the shifted words of
// w2_words; periodic in x).  Add w2_dyz for the neighbour's row.
template <int S, int C> __device__ __forceinline__ u32 w2_src(const W2Ctx& c) {
    if constexpr (S == 0) return c.n0 + C;
    else if constexpr (S > 0) return C == 0 ? c.n0 + 1U : c.nr;
    else return C == 0 ? c.nl + 1U : c.n0;
}

// Half-way bounce-back of the cells with wall links (masks m0, m1; the
// one-cell gather_walls rule): direction i = 2p+1 whose source n + c_j is a
// wall reads the pb slot at that source; direction j whose source n + c_i is a
// wall reads the pa slot at the cell.

template <class L>
__device__ __forceinline__ void w2_bounce(const LbmArgs& a, const W2Ctx& c, u32 m0, u32 m1, u32* pw) {
    const u32 m = m0 | m1;
    static_for_pairs<L>([&](auto PP) {
        constexpr int p = decltype(PP)::value;
        constexpr int i = 2 * p + 1, j = i + 1, s = L::cx(j);
        constexpr u32 bi = 1U << (2 * p), bj = 2U << (2 * p);
        if (m & bi) {
            const u32 dyz = w2_dyz<L, j>(c);
            if (m0 & bi) pw[i] = with_lo(pw[i], ld_u16(w2_tab(a, a.pb_off[p]) + (w2_src<s, 0>(c) + dyz)));
            if (m1 & bi) pw[i] = with_hi(pw[i], ld_u16(w2_tab(a, a.pb_off[p]) + (w2_src<s, 1>(c) + dyz)));
        }
        if (m & bj) {
            if (m0 & bj) pw[j] = with_lo(pw[j], ld_u16(w2_tab(a, a.pa_off[p]) + c.n0));
            if (m1 & bj) pw[j] = with_hi(pw[j], ld_u16(w2_tab(a, a.pa_off[p]) + (c.n0 + 1U)));
        }
    });
}

// Moving-wall correction of one lane (cell x0 + C) with the one-cell kernel's function.
template <class L, int C>
__device__ __noinline__ void w2_moving_lane(const LbmArgs& a, const W2Ctx c, std::uint8_t flag, float2* f) {
    float h[L::Q];
#pragma unroll
    for (int d = 0; d < L::Q; ++d) h[d] = C ? f[d].y : f[d].x;
    gather_fixup_scaled<L>(a, c.n0 + C, make_nbr(a, c.x0 + C, c.y, c.z), flag, h);
#pragma unroll
    for (int d = 0; d < L::Q; ++d) {
        if (C)
            f[d].y = h[d];
        else
            f[d].x = h[d];
    }
}

// Stores: aligned words where the slot pair is aligned, two 16-bit stores
// where the pa row is shifted (h2_stores' rule).
// MERGE (a warp holding a pair with a wall cell): a wall cell is not stepped,
// and its slots must keep their bits, so a pair with one live cell (live0 /
// live1) stores that cell's halves alone, as 16-bit stores.  No cell writes a
// wall cell's slots within a step, so its slots keep their bits.  An aligned
// word is one predicated word store or one predicated half store at a
// per-lane offset: measured on B200, 53.3 instead of 52.6 GLUPS on the 512^3
// cavity and 47.3 instead of 46.5 on the sphere pack against a three-way
// choice per word (word, low half, high half).
template <class L, bool MERGE>
__device__ __forceinline__ void w2_stores(const LbmArgs& a, const W2Ctx& c, const float2* f, u32 h0, u32 h1,
                                          bool live0, bool live1) {
    // a pair with one live cell: that cell's half (element offset hoff, bit shift hsh)
    const bool both = live0 && live1;
    const u32 hoff = live0 ? 0U : 1U, hsh = live0 ? 0U : 16U;
    const auto store_aligned = [&](__half* ptr, u32 w) {
        if constexpr (MERGE) {
            if (both)
                st_word(ptr, w);
            else
                st_half(ptr + hoff, w >> hsh);
        } else {
            st_word(ptr, w);
        }
    };
    store_aligned(w2_tab(a, a.rest_off) + c.n0,
                  f16x2_rs(f[0].y, f[0].x, lo_halves(round_bits(a, h0, 0), round_bits(a, h1, 0))));
    static_for_pairs<L>([&](auto PP) {
        constexpr int p = decltype(PP)::value;
        constexpr int i = 2 * p + 1, j = i + 1, s = L::cx(j);
        const u32 k0 = round_bits(a, h0, p + 1), k1 = round_bits(a, h1, p + 1);
        store_aligned(w2_tab(a, a.pb_off[p]) + c.n0, f16x2_rs(f[i].y, f[i].x, lo_halves(k0, k1)));
        const u32 wj = f16x2_rs(f[j].y, f[j].x, hi_halves(k0, k1));
        __half* t = w2_tab(a, a.pa_off[p]);
        const u32 dyz = w2_dyz<L, j>(c);
        if constexpr (s == 0) {
            store_aligned(t + (c.n0 + dyz), wj);
        } else if constexpr (MERGE) {
            if (live0) st_half(t + (w2_src<s, 0>(c) + dyz), wj);
            if (live1) st_half(t + (w2_src<s, 1>(c) + dyz), wj >> 16);
        } else {
            st_half(t + (w2_src<s, 0>(c) + dyz), wj);
            st_half(t + (w2_src<s, 1>(c) + dyz), wj >> 16);
        }
    });
}

// One pair of cells from its pair words pw (low half cell x0).  fl2: the two
// internal flag bytes (cell x0 in the low byte).  BOUNCE: pw holds the plain
// words and the cells with wall links reload their bounced halves here (the
// unpipelined form; the pipelined one assembles them from the near-wall form).
// The moving-wall correction is a call, not inlined code: inlined, its
// per-lane arrays raised the register demand of the whole kernel and the
// interior path spilled.  It gets a copy of the populations (tmp), since an
// array whose address reaches a call lives in local memory on every path.
// The bounce-back loads stay inline: they run in every warp that holds a
// near-wall pair (on a cavity, the first and last warp of each row), and a
// call there saved and restored the live registers through local memory.
template <class L, bool LES, bool FLAGS, bool GRAY, bool BOUNCE>
__device__ __forceinline__ void w2_cell_pair(const LbmArgs& a, const W2Ctx& c, u32* pw, unsigned fl2) {
    constexpr unsigned kNearWall2 = kFlagNearWall * 0x0101U;
    constexpr unsigned kNearMoving2 = kFlagNearMoving * 0x0101U;
    constexpr unsigned kType2 = kFlagTypeMask * 0x0101U;
    if constexpr (FLAGS && BOUNCE) {
        if (fl2 & kNearWall2) {
            // wall cells have empty masks; a fluid cell's mask is loaded only when it has links
            const u32 m0 = (fl2 & kFlagNearWall) ? a.wall_mask[c.n0] : 0U;
            const u32 m1 = (fl2 & (kFlagNearWall << 8)) ? a.wall_mask[c.n0 + 1U] : 0U;
            w2_bounce<L>(a, c, m0, m1, pw);
        }
    }
    float2 f[L::Q];
#pragma unroll
    for (int d = 0; d < L::Q; ++d) f[d] = unpack(pw[d]);
    if constexpr (FLAGS) {
        if (fl2 & kNearMoving2) {
            float2 tmp[L::Q];
#pragma unroll
            for (int d = 0; d < L::Q; ++d) tmp[d] = f[d];
            w2_moving_lane<L, 0>(a, c, static_cast<std::uint8_t>(fl2), tmp);
            w2_moving_lane<L, 1>(a, c, static_cast<std::uint8_t>(fl2 >> 8), tmp);
#pragma unroll
            for (int d = 0; d < L::Q; ++d) f[d] = tmp[d];
        }
    }
    if (a.has_force)
        collide_scaled<L, LES, GRAY, true>(a, c.n0, f);
    else
        collide_scaled<L, LES, GRAY, false>(a, c.n0, f);
    const u32 h0 = round_hash(a, c.n0), h1 = round_hash(a, c.n0 + 1U);
    if constexpr (FLAGS) {
        const bool wall0 = (fl2 & kFlagTypeMask) != 0U, wall1 = (fl2 & (kFlagTypeMask << 8)) != 0U;
        // warp-uniform choice: the merging stores cost every thread of the warp the same
        if (__any_sync(__activemask(), (fl2 & kType2) != 0U)) {
            w2_stores<L, true>(a, c, f, h0, h1, !wall0, !wall1);
            return;
        }
    }
    w2_stores<L, false>(a, c, f, h0, h1, true, true);
}

// ---------------------------------------------------------------- cp.async
template <int OFF> __device__ __forceinline__ void cp_async4(u32 smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0+%2], [%1], 4;\n" ::"r"(smem), "l"(gmem), "n"(OFF) : "memory");
}
__device__ __forceinline__ void cp_async8(u32 smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Resident 128-thread blocks per SM (register cap 65536 / (128 * blocks)).
// The macros exist for tuning builds.
#ifndef CFDX_W2_MIN_BLOCKS
#define CFDX_W2_MIN_BLOCKS 5
#endif
#ifndef CFDX_W2_MIN_BLOCKS_Q27
#define CFDX_W2_MIN_BLOCKS_Q27 5
#endif
template <class L> constexpr int w2_min_blocks() { return L::Q == 27 ? CFDX_W2_MIN_BLOCKS_Q27 : CFDX_W2_MIN_BLOCKS; }

// Threads per block of k_step_w2 (the shared-memory slots of the pipelined
// form are laid out for it, so their offsets are immediates).
constexpr unsigned kW2Threads = 128;

// Shared memory of the pipelined form, per thread, in groups of four words
// (one 16-byte load reads four): two stages, each with the count word slots,
// two words of second-cell fixes (w2_fix_second's bits, written when the
// plane's words are issued) and two words holding the wall-link masks of the
// plane three ahead of the one the stage holds (same parity); then a ring of
// four planes' pair flags.  D3Q19: 7 groups per stage, 30 KB per block.
// Measured and replaced (512^3 cavity, FP16): a near-wall form with a word
// per cell for every aligned slot (42 KB per block: the L1 left beside five
// blocks' shared memory cost the interior 5 %); one stage read into
// registers before the next plane's copies (24 KB; the pair words live
// through the issue spilled); staging the second cell's fix words too (up to
// eight per pair, 38 KB per block): 49.1 instead of 52.2 GLUPS on the cavity
// and 38.8 instead of 46.2 on the 512x256x256 sphere pack, whose mixed pairs
// paid more for the issue than the fix loads cost.  A stage stride of a
// power of two groups (8) made ptxas spill.
template <class L> constexpr unsigned w2_groups() { return (static_cast<unsigned>(W2Words<L>::count) + 4U + 3U) / 4U; }
template <class L> constexpr unsigned w2_fix_slot() { return static_cast<unsigned>(W2Words<L>::count); }
template <class L> constexpr unsigned w2_mask_slot() { return 4U * w2_groups<L>() - 2U; } // 8-byte aligned
constexpr unsigned kW2FlagRing = 4;
template <class L> constexpr unsigned w2_smem_bytes() {
    return 2U * w2_groups<L>() * kW2Threads * 16U + kW2FlagRing * kW2Threads * 4U;
}

// Grid: x over pairs (blockDim.x threads, nx/2 pairs), y over rows
// (blockDim.x * blockDim.y == kW2Threads), z over chunks of a.planes planes
// of [a.z_first, a.z_end).
template <class L, bool LES, bool FLAGS, bool GRAY, bool PIPE>
__global__ void __launch_bounds__(kW2Threads, w2_min_blocks<L>()) k_step_w2(const __grid_constant__ LbmArgs a) {
    using Wd = W2Words<L>;
    constexpr int W = Wd::count;
    const u32 x0 = 2U * (blockIdx.x * blockDim.x + threadIdx.x);
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x0 >= a.nx || y >= a.ny) return;
    const u32 zb = a.z_first + blockIdx.z * a.planes;
    const u32 ze = min(a.z_end, zb + a.planes);
    W2Ctx c;
    w2_thread(a, x0, y, c);
    constexpr unsigned kNear2 = kFlagNearWall * 0x0101U;
    // pair flags (cell x0 in the low byte) of plane z
    const auto flags_at = [&](u32 z) -> unsigned {
        if constexpr (FLAGS)
            return *reinterpret_cast<const unsigned short*>(a.flags + ((z * a.ny + y) * a.nx + x0));
        else
            return 0U;
    };
    // both cells walls: nothing to step
    const auto both_walls = [](unsigned fl2) {
        return FLAGS && (fl2 & kFlagTypeMask) != 0U && (fl2 & (kFlagTypeMask << 8)) != 0U;
    };
    if constexpr (!PIPE) {
        for (u32 z = zb; z < ze; ++z) {
            w2_plane(a, z, c);
            const unsigned fl2 = flags_at(z);
            if (both_walls(fl2)) continue;
            u32 raw[W];
            w2_words<L>(a, c, [&](auto K, const __half* p) { raw[decltype(K)::value] = ld_word(p); });
            u32 pw[L::Q];
            w2_assemble<L>(raw, pw);
            w2_cell_pair<L, LES, FLAGS, GRAY, true>(a, c, pw, fl2);
        }
    } else {
        // Word k of stage st: component k % 4 of w2_stage[(st * G + k / 4) * kW2Threads + tid]; the
        // masks of a plane at word w2_mask_slot of the stage of its parity.  After the stages, ring
        // slot r of the flags: the pair flags of a plane, bit 16 set when its words were issued in
        // the near-wall form.  Plane z uses stage (z - zb) % 2 and flag slot (z - zb) % 4.
        // Iteration z issues the words of z + 1 and the masks of z + 3, then waits for everything
        // but that (so the masks of z + 1, fetched two iterations earlier, have arrived).
        constexpr u32 G = w2_groups<L>();
        constexpr u32 GW = (static_cast<u32>(W) + 3U) / 4U; // groups holding words
        constexpr u32 kStageBytes = G * kW2Threads * 16U;
        constexpr u32 kMask = w2_mask_slot<L>(), kFix = w2_fix_slot<L>();
        static_assert(kFix + 2U <= kMask, "second-cell fixes between the words and the masks");
        extern __shared__ uint4 w2_stage[];
        const u32 tid = threadIdx.y * blockDim.x + threadIdx.x;
        const uint4* mine = w2_stage + tid;
        const u32 sbase = static_cast<u32>(__cvta_generic_to_shared(mine));
        u32* const fring = reinterpret_cast<u32*>(w2_stage + 2U * G * kW2Threads) + tid;
        const auto slot_at = [&](u32 st, u32 k) { // byte offset of word slot k of stage st from sbase
            return st * kStageBytes + (k / 4U) * kW2Threads * 16U + (k % 4U) * 4U;
        };
        const auto slot_ptr = [&](u32 st, u32 k) {
            return reinterpret_cast<u32*>(reinterpret_cast<char*>(w2_stage + tid) + slot_at(st, k));
        };
        // wall-link masks of plane z into the stage of its parity (n0 even: 8-byte aligned)
        const auto fetch_masks = [&](u32 z) {
            cp_async8(sbase + slot_at((z - zb) & 1U, kMask), a.wall_mask + ((z * a.ny + y) * a.nx + x0));
        };
        // Copies the words of plane z into stage st, with the tables its wall links select when a
        // lane of the warp has links (the warp's vote: the form costs every lane the same); returns
        // the ring word.  A wall cell's halves are never stored, so an aligned word takes the
        // table of its pair's fluid cell; when both cells are fluid and disagree on a link, cell
        // x0's choice is taken and the second cell's half is fixed after the words arrive.
        const auto issue = [&](u32 z, u32 st, unsigned fl2, uint2 m) -> unsigned {
            W2Ctx cn = c;
            w2_plane(a, z, cn);
            const u32 s0 = sbase + st * kStageBytes;
            bool near = false;
            if constexpr (FLAGS) near = __any_sync(__activemask(), (fl2 & kNear2) != 0U);
            const auto copy = [&](auto K, const __half* p) {
                constexpr int k = decltype(K)::value;
                cp_async4<(k / 4) * kW2Threads * 16 + (k % 4) * 4>(s0, p);
            };
            if (!both_walls(fl2)) {
                if (near) {
                    // wall cells have empty masks; a fluid cell's mask was fetched only when it has links
                    const u32 m0 = (fl2 & kFlagNearWall) ? m.x : 0U;
                    const u32 m1 = (fl2 & (kFlagNearWall << 8)) ? m.y : 0U;
                    const u32 m0e = (fl2 & kFlagTypeMask) != 0U ? m1 : m0;
                    const u32 m1e = (fl2 & (kFlagTypeMask << 8)) != 0U ? m0 : m1;
                    const u32 mixed = (m0e ^ m1e) & Wd::aligned_bits();
                    w2_near_words<L>(a, cn, m0, m1, m0e, copy);
                    u32* fix = slot_ptr(st, kFix);
                    fix[0] = mixed & m1e;  // the second cell reads the alternative table
                    fix[1] = mixed & ~m1e; // the second cell reads the plain table
                } else {
                    w2_words<L>(a, cn, copy);
                }
            }
            return fl2 | (near ? 0x10000U : 0U);
        };
        // prologue: flags of the first four planes, masks of the first three, words of the first
        const unsigned f0 = flags_at(zb);
        const unsigned f1 = zb + 1U < ze ? flags_at(zb + 1U) : 0U;
        const unsigned f2 = zb + 2U < ze ? flags_at(zb + 2U) : 0U;
        unsigned ahead = zb + 3U < ze ? flags_at(zb + 3U) : 0U; // flags of plane z + 3 in iteration z
        fring[kW2Threads] = f1;
        fring[2U * kW2Threads] = f2;
        uint2 m0v = make_uint2(0U, 0U);
        if constexpr (FLAGS) {
            if (zb + 1U < ze && (f1 & kNear2)) fetch_masks(zb + 1U);
            if (zb + 2U < ze && (f2 & kNear2)) fetch_masks(zb + 2U);
        }
        cp_async_commit();
        if constexpr (FLAGS) {
            if (f0 & kNear2) m0v = *reinterpret_cast<const uint2*>(a.wall_mask + ((zb * a.ny + y) * a.nx + x0));
        }
        fring[0] = issue(zb, 0U, f0, m0v);
        cp_async_commit();
        cp_async_wait<1>(); // the masks of planes zb + 1, zb + 2
        for (u32 z = zb; z < ze; ++z) {
            const u32 r = z - zb;
            const unsigned f3 = ahead;
            if (z + 3U < ze) fring[((r + 3U) & 3U) * kW2Threads] = f3;
            ahead = z + 4U < ze ? flags_at(z + 4U) : 0U;
            if (z + 1U < ze) {
                u32* const slot = fring + ((r + 1U) & 3U) * kW2Threads;
                const unsigned fn = *slot;
                uint2 mn = make_uint2(0U, 0U);
                if (FLAGS && (fn & kNear2)) mn = *reinterpret_cast<const uint2*>(slot_ptr((r + 1U) & 1U, kMask));
                *slot = issue(z + 1U, (r + 1U) & 1U, fn, mn);
            }
            if constexpr (FLAGS) {
                // after the read above: the masks of z + 3 go where those of z + 1 were
                if (z + 3U < ze && (f3 & kNear2)) fetch_masks(z + 3U);
            }
            cp_async_commit();
            cp_async_wait<1>(); // all but this iteration's copies: the words of z
            const unsigned ring = fring[(r & 3U) * kW2Threads];
            const unsigned fl2 = ring & 0xffffU;
            if (both_walls(fl2)) continue;
            const uint4* groups = mine + (r & 1U) * (G * kW2Threads);
            u32 raw[4 * GW];
#pragma unroll
            for (u32 g = 0; g < GW; ++g) {
                const uint4 v = groups[g * kW2Threads];
                raw[4 * g] = v.x;
                raw[4 * g + 1] = v.y;
                raw[4 * g + 2] = v.z;
                raw[4 * g + 3] = v.w;
            }
            u32 pw[L::Q];
            w2_assemble<L>(raw, pw);
            w2_plane(a, z, c);
            if (FLAGS && (ring & 0x10000U) != 0U) {
                const u32* fix = slot_ptr(r & 1U, kFix);
                const u32 to_alt = fix[0], to_plain = fix[1];
                if ((to_alt | to_plain) != 0U) w2_fix_second<L>(a, c, to_alt, to_plain, pw);
            }
            w2_cell_pair<L, LES, FLAGS, GRAY, false>(a, c, pw, fl2);
        }
        cp_async_wait_all();
    }
}

} // namespace cfdx
