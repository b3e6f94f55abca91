// Device side of the in-place Esoteric-Pull lattice-Boltzmann step (sm_100a).
//
// One thread owns CPT cells stacked in z.  Every launch reads and writes each
// population slot exactly once: a cell reads the q slots its pairs own at this
// parity and writes the post-collision values back into the same q slots, so
// the update is race-free with a single lattice in HBM (access pattern:
// Lehmann, Computation 10(6) 92, 2022; reference esoteric_pull.hpp:349-382).
//
// Layout in HBM: populations are a structure of arrays f[d][n] with
// n = (z*ny + y)*nx + x (reference esoteric_pull.hpp:304-310), so a warp
// reads 32 consecutive x cells of one direction: c_x = 0 directions are
// aligned rows, c_x = +-1 directions are shifted by one element and share
// their edge sector with the neighbouring warp, which L1/L2 absorb.
//
// The step is HBM-bound (no tensor-core work: it is a stencil, not a
// contraction).  What limits it is bytes in flight per SM and instruction
// issue: all loads of a thread's CPT cells are issued before the first
// collision; addressing is 32-bit off per-parity slot tables held in the
// parameter bank (no parity selects, no 64-bit offsets in registers); the
// collision works on opposite-pair sums and differences.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

#include "lattice.cuh"
#include "lbm_args.h"

namespace cfdx {

using u32 = std::uint32_t;

// ------------------------------------------------------------- storage traits
// `delta` storage types hand the kernels the deviation f - w_d from the rest
// weight instead of f itself; the collision then works in deviation space
// (see collide), so decoding and encoding are one multiply each.
struct StF32 {
    using T = float;
    using R = float;
    static constexpr bool delta = false;
    static constexpr bool scaled = false;
};
struct StF64 {
    using T = double;
    using R = double;
    static constexpr bool delta = false;
    static constexpr bool scaled = false;
};
// FP16 shifted storage: h = half((f - w_d) * s_d); kernels see f - w_d = h / s_d.
// Scales are equal within an opposite pair, so a bounced load that reads the
// partner direction's slot decodes with the same constant.
// The step kernel keeps FP16 populations in storage units h (`scaled`) and
// applies the scales per weight class (collide_scaled).
struct StF16 {
    using T = __half;
    using R = float;
    static constexpr bool delta = true;
    static constexpr bool scaled = true;
};

// Slot-ownership audit (a test hook; see slot_audit.cu): a storage type whose
// loads and stores record who touched each slot instead of moving data.  The
// step kernels instantiated with it run their real addressing code.  Per slot
// there are five 32-bit counters, `stride` = q * cells apart: reads, writes,
// lowest and highest reading thread, writing thread (threads numbered from 1);
// one more word counts accesses outside the slots.
template <bool SCALED> struct StAudit {
    using T = std::uint32_t;
    using R = float;
    static constexpr bool delta = SCALED;
    static constexpr bool scaled = SCALED;
};
template <class S> struct IsAudit {
    static constexpr bool value = false;
};
template <bool SCALED> struct IsAudit<StAudit<SCALED>> {
    static constexpr bool value = true;
};
__device__ __forceinline__ std::uint32_t audit_thread() {
    const std::uint32_t block = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    return block * (blockDim.x * blockDim.y) + threadIdx.y * blockDim.x + threadIdx.x + 1U;
}
// An address outside the lattice's q * cells slots is not accessed: it is
// counted in the word after the five arrays.
__device__ __forceinline__ bool audit_in_range(const std::uint32_t* p, const void* base, std::uint32_t stride) {
    const auto* b = static_cast<const std::uint32_t*>(base);
    if (p >= b && p < b + stride) return true;
    atomicAdd(const_cast<std::uint32_t*>(b) + 5U * stride, 1U);
    return false;
}
__device__ __forceinline__ void audit_read(std::uint32_t* p, const void* base, std::uint32_t stride) {
    if (!audit_in_range(p, base, stride)) return;
    const std::uint32_t id = audit_thread();
    atomicAdd(p, 1U);
    atomicMin(p + 2U * stride, id);
    atomicMax(p + 3U * stride, id);
}
__device__ __forceinline__ void audit_write(std::uint32_t* p, const void* base, std::uint32_t stride) {
    if (!audit_in_range(p, base, stride)) return;
    atomicAdd(p + stride, 1U);
    atomicExch(p + 4U * stride, audit_thread());
}

// RAW: FP16 values stay in storage units h (no scale applied).
template <class S, class L, int D, bool RAW = false>
__device__ __forceinline__ typename S::R ld(const typename S::T* p, const LbmArgs& a) {
    if constexpr (IsAudit<S>::value) {
        audit_read(const_cast<std::uint32_t*>(p), a.base, static_cast<std::uint32_t>(L::Q) * a.N);
        return 0.0F;
    } else if constexpr (sizeof(typename S::T) == 2) {
        if constexpr (RAW)
            return __half2float(*p);
        else
            return __half2float(*p) * a.inv_scale[D];
    } else {
        return *p;
    }
}

template <class S, class L, int D, bool RAW = false>
__device__ __forceinline__ void st(typename S::T* p, typename S::R v, const LbmArgs& a) {
    if constexpr (IsAudit<S>::value) {
        (void)v;
        audit_write(p, a.base, static_cast<std::uint32_t>(L::Q) * a.N);
    } else if constexpr (sizeof(typename S::T) == 2) {
        if constexpr (RAW)
            *p = __float2half_rn(v);
        else
            *p = __float2half_rn(v * a.scale[D]);
    } else {
        *p = v;
    }
}

// ------------------------------------------------------- FP16 store rounding
// FP16 stores go through sm_100a's cvt.rs (stochastic rounding): it converts
// two FP32 values to an FP16 pair, adding rbits[12:0] (low half) and
// rbits[28:16] (high half) below the FP16 mantissa and truncating.  Uniform
// random bits make the rounding unbiased, so increments smaller than half an
// FP16 step -- a small body force, a slow flow -- survive on average instead
// of being rounded away every step.  Constant bits 0x1000 in both fields give
// round-half-away-from-zero (the "nearest" mode).  The bits come from a hash
// of the cell index and a per-step seed (LbmArgs::round_*), with one 32-bit
// word per opposite pair: the same bits for a (cell, direction) in every
// kernel, so the one-cell, paired and out-of-place steps stay bitwise equal.

// lowbias32 integer hash (C. Wellons, "hash-prospector", public domain).
__device__ __forceinline__ u32 round_hash(const LbmArgs& a, u32 n) {
    u32 x = (n + a.hash_base) ^ a.round_seed;
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x & a.round_mask;
}

// Rounding word of pair slot k (0: rest, p + 1: pair p) of a cell with hash h:
// bits [12:0] round the pair's first direction 2p+1 (or the rest population),
// bits [28:16] its second direction 2p+2.
__device__ __forceinline__ u32 round_bits(const LbmArgs& a, u32 h, int k) {
    return h * (0x9E3779B9U * (2U * static_cast<u32>(k) + 1U)) + a.round_add;
}

// (hi, lo) -> FP16 pair, rounded with rbits (see above).
__device__ __forceinline__ u32 f16x2_rs(float hi, float lo, u32 rbits) {
    u32 d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// One FP16 store rounded with rbits[12:0].
__device__ __forceinline__ void st_h16(__half* p, float v, u32 rbits) {
    *reinterpret_cast<unsigned short*>(p) = static_cast<unsigned short>(f16x2_rs(0.0F, v, rbits));
}

// Value the kernels hold for an absolute population f of direction D.
template <class S, class L, int D> __device__ __forceinline__ typename S::R held(typename S::R f) {
    if constexpr (S::delta) {
        return f - typename S::R(L::w(D));
    } else {
        return f;
    }
}

// Absolute population from a held value.
template <class S, class L> __device__ __forceinline__ typename S::R absolute(typename S::R v, int d) {
    if constexpr (S::delta) {
        return v + typename S::R(L::w(d));
    } else {
        return v;
    }
}

// ------------------------------------------------ lattice-vector products
// c_D . (x, y, z) for a direction with components in {-1, 0, 1}, written as
// the signed sum of its nonzero terms (positive terms first).  The generic
// form c_x * x + c_y * y + c_z * z costs a multiply-add per zero component:
// IEEE semantics (NaN, signed zero) forbid folding x * 0 away.
template <int A, int B, int C, class R> __device__ __forceinline__ R signed_sum(R x, R y, R z) {
    if constexpr (A > 0) {
        R r = x;
        if constexpr (B > 0) r = r + y;
        if constexpr (C > 0) r = r + z;
        if constexpr (B < 0) r = r - y;
        if constexpr (C < 0) r = r - z;
        return r;
    } else if constexpr (B > 0) {
        R r = y;
        if constexpr (C > 0) r = r + z;
        if constexpr (A < 0) r = r - x;
        if constexpr (C < 0) r = r - z;
        return r;
    } else if constexpr (C > 0) {
        R r = z;
        if constexpr (A < 0) r = r - x;
        if constexpr (B < 0) r = r - y;
        return r;
    } else if constexpr (A < 0) {
        R r = -x;
        if constexpr (B < 0) r = r - y;
        if constexpr (C < 0) r = r - z;
        return r;
    } else if constexpr (B < 0) {
        R r = -y;
        if constexpr (C < 0) r = r - z;
        return r;
    } else if constexpr (C < 0) {
        return -z;
    } else {
        return R(0);
    }
}

template <class L, int D, class R> __device__ __forceinline__ R cdot(R x, R y, R z) {
    return signed_sum<L::cx(D), L::cy(D), L::cz(D), R>(x, y, z);
}

// Compile-time loop over the opposite pairs: f(std::integral_constant<int, p>).
template <class L, int P = 0, class F> __device__ __forceinline__ void static_for_pairs(F&& f) {
    if constexpr (P < L::PAIRS) {
        f(std::integral_constant<int, P>{});
        static_for_pairs<L, P + 1>(f);
    }
}

// ------------------------------------------------------- periodic neighbours
// Offsets of the x-1/x/x+1, y-1/y/y+1, z-1/z/z+1 neighbours with periodic wrap
// (reference esoteric_pull.hpp:40-46), indexed by c + 1.  Unsigned wrap-around
// arithmetic keeps n + offset exact because the true neighbour index is in [0, N).
struct Nbr {
    u32 ox[3], oy[3], oz[3];
};

__device__ __forceinline__ Nbr make_nbr(const LbmArgs& a, u32 x, u32 y, u32 z) {
    Nbr o;
    const u32 plane = a.nx * a.ny;
    o.ox[0] = x == 0 ? a.nx - 1U : 0xffffffffU;
    o.ox[1] = 0U;
    o.ox[2] = x == a.nx - 1U ? 1U - a.nx : 1U;
    o.oy[0] = y == 0 ? (a.ny - 1U) * a.nx : 0U - a.nx;
    o.oy[1] = 0U;
    o.oy[2] = y == a.ny - 1U ? 0U - (a.ny - 1U) * a.nx : a.nx;
    o.oz[0] = z == 0 ? (a.nz - 1U) * plane : 0U - plane;
    o.oz[1] = 0U;
    o.oz[2] = z == a.nz - 1U ? 0U - (a.nz - 1U) * plane : plane;
    return o;
}

template <class L, int D> __device__ __forceinline__ u32 nbr_off(const Nbr& o) {
    return o.ox[L::cx(D) + 1] + o.oy[L::cy(D) + 1] + o.oz[L::cz(D) + 1];
}

// ------------------------------------------------------------------- gather
// Incoming (post-streaming, pre-collision) populations of fluid cell n.
// Pair p = (i, j = i+1), nb = n + c_j is the source of direction i,
// nf = n + c_i the source of direction j.
//   even step: fin_i = f[i][nb], fin_j = f[j][n]
//   odd step:  fin_i = f[j][nb], fin_j = f[i][n]
// i.e. fin_i = pa[p][nb], fin_j = pb[p][n] with the per-parity tables.
// Half-way bounce-back in place: when the source is a wall, the incoming
// value is this cell's own outgoing opposite population of the previous
// step, which sits in the other slot of the same address -- the load takes
// the other table.  Moving walls add 6 w_k rho (c_k . u_wall) (reference
// src/lbm/d2q9.cpp:220-223) with rho this cell's pre-correction density.
// Slot addressing: NARROW kernels use 32-bit element offsets from one base
// pointer (q*N < 2^32: one add and one wide multiply-add per access, no
// per-access pointer loads); the wide form reads the 64-bit per-parity
// pointer tables.
template <class S, bool NARROW> struct Slots {
    using T = typename S::T;
    __device__ __forceinline__ static T* at(const LbmArgs& a, bool use_pa, int p, u32 idx) {
        if constexpr (NARROW) {
            return static_cast<T*>(a.base) + ((use_pa ? a.pa_off[p] : a.pb_off[p]) + idx);
        } else {
            return static_cast<T*>(use_pa ? a.pa[p] : a.pb[p]) + idx;
        }
    }
    __device__ __forceinline__ static T* rest(const LbmArgs& a, u32 idx) {
        if constexpr (NARROW) {
            return static_cast<T*>(a.base) + (a.rest_off + idx);
        } else {
            return static_cast<T*>(a.rest) + idx;
        }
    }
};

template <class L, class S, bool NARROW, bool RAW = false, int P = 0>
__device__ __forceinline__ void gather_plain(const LbmArgs& a, u32 n, const Nbr& o, typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        fin[i] = ld<S, L, i, RAW>(Slots<S, NARROW>::at(a, true, P, n + nbr_off<L, j>(o)), a);
        fin[j] = ld<S, L, j, RAW>(Slots<S, NARROW>::at(a, false, P, n), a);
        gather_plain<L, S, NARROW, RAW, P + 1>(a, n, o, fin);
    }
}

template <class L, class S, bool NARROW, bool RAW = false, int P = 0>
__device__ __forceinline__ void gather_walls(const LbmArgs& a, u32 n, const Nbr& o, unsigned walls,
                                             typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const bool sb = ((walls >> (2 * P)) & 1U) != 0U;
        const bool sf = ((walls >> (2 * P + 1)) & 1U) != 0U;
        fin[i] = ld<S, L, i, RAW>(Slots<S, NARROW>::at(a, !sb, P, n + nbr_off<L, j>(o)), a);
        fin[j] = ld<S, L, j, RAW>(Slots<S, NARROW>::at(a, sf, P, n), a);
        gather_walls<L, S, NARROW, RAW, P + 1>(a, n, o, walls, fin);
    }
}


template <class L, class R, int P = 0>
__device__ __forceinline__ void moving_wall_pairs(const LbmArgs& a, u32 n, const Nbr& o, R rw, R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const int idb = a.flags[n + nbr_off<L, j>(o)] & kFlagTypeMask;
        if (idb >= 2) {
            const R cu = cdot<L, i, R>(R(a.wall_u[idb][0]), R(a.wall_u[idb][1]), R(a.wall_u[idb][2]));
            fin[i] += R(6.0) * R(L::w(i)) * rw * cu;
        }
        const int idf = a.flags[n + nbr_off<L, i>(o)] & kFlagTypeMask;
        if (idf >= 2) {
            const R cu = cdot<L, j, R>(R(a.wall_u[idf][0]), R(a.wall_u[idf][1]), R(a.wall_u[idf][2]));
            fin[j] += R(6.0) * R(L::w(j)) * rw * cu;
        }
        moving_wall_pairs<L, R, P + 1>(a, n, o, rw, fin);
    }
}

// With flags every fluid cell takes the wall-link path; cells without a wall
// neighbour have an empty mask, so the links pick the plain slots.  A warp of
// mixed near-wall and interior cells then runs one gather instead of both
// (measured on B200, 512^3 LES cavity / 512x256x256 sphere pack: +14 % / +13 %
// FP16, +2 % / +7 % FP32 over branching on the near-wall bit).
template <class L, class S, bool FLAGS, bool NARROW = false, bool RAW = false>
__device__ __forceinline__ void gather_loads(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                             typename S::R* fin) {
    fin[0] = ld<S, L, 0, RAW>(Slots<S, NARROW>::rest(a, n), a);
    if constexpr (FLAGS) {
        gather_walls<L, S, NARROW, RAW>(a, n, o, (flag & kFlagNearWall) ? a.wall_mask[n] : 0U, fin);
        return;
    }
    gather_plain<L, S, NARROW, RAW>(a, n, o, fin);
}

// Bounce-back fix-up of one near-wall cell whose values were gathered as if
// it had no walls (the paired kernels): wall links reload the partner slot.
template <class L, class S, int P = 0>
__device__ __forceinline__ void bounce_fixup(const LbmArgs& a, const typename S::T* base, u32 n, const Nbr& o,
                                             unsigned walls, typename S::R* f) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        if ((walls >> (2 * P)) & 1U) f[i] = ld<S, L, i, S::scaled>(base + (a.pb_off[P] + (n + nbr_off<L, j>(o))), a);
        if ((walls >> (2 * P + 1)) & 1U) f[j] = ld<S, L, j, S::scaled>(base + (a.pa_off[P] + n), a);
        bounce_fixup<L, S, P + 1>(a, base, n, o, walls, f);
    }
}

// Moving-wall correction for values held in FP16 storage units: the
// correction 6 w_k rho (c_k . u_wall) is scaled by s_k.  Explicitly rounded
// operations: the paired kernels call this out of line, the one-cell kernel
// inline, and both must round alike.
template <class L, int P = 0>
__device__ __forceinline__ void moving_wall_pairs_scaled(const LbmArgs& a, u32 n, const Nbr& o, float rw, float* h) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const int idb = a.flags[n + nbr_off<L, j>(o)] & kFlagTypeMask;
        if (idb >= 2) {
            const float cu = cdot<L, i, float>(a.wall_u[idb][0], a.wall_u[idb][1], a.wall_u[idb][2]);
            h[i] = __fmaf_rn(a.scale[i], __fmul_rn(__fmul_rn(6.0F * float(L::w(i)), rw), cu), h[i]);
        }
        const int idf = a.flags[n + nbr_off<L, i>(o)] & kFlagTypeMask;
        if (idf >= 2) {
            const float cu = cdot<L, j, float>(a.wall_u[idf][0], a.wall_u[idf][1], a.wall_u[idf][2]);
            h[j] = __fmaf_rn(a.scale[j], __fmul_rn(__fmul_rn(6.0F * float(L::w(j)), rw), cu), h[j]);
        }
        moving_wall_pairs_scaled<L, P + 1>(a, n, o, rw, h);
    }
}

template <class L>
__device__ __forceinline__ void gather_fixup_scaled(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                                    float* h) {
    if (flag & kFlagNearMoving) {
        float rho0 = 1.0F;
#pragma unroll
        for (int d = 0; d < L::Q; ++d) rho0 = __fmaf_rn(h[d], a.inv_scale[d], rho0);
        const float rw = rho0 > 1.0e-8F ? rho0 : 1.0e-8F;
        moving_wall_pairs_scaled<L>(a, n, o, rw, h);
    }
}

template <class L, class S, bool FLAGS>
__device__ __forceinline__ void gather_fixup(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                             typename S::R* fin) {
    using R = typename S::R;
    if constexpr (FLAGS) {
        if (flag & kFlagNearMoving) {
            R rho0 = S::delta ? R(1) : R(0);
#pragma unroll
            for (int d = 0; d < L::Q; ++d) rho0 += fin[d];
            const R rw = rho0 > R(1.0e-8) ? rho0 : R(1.0e-8);
            moving_wall_pairs<L, R>(a, n, o, rw, fin);
        }
    }
}

template <class L, class S, bool FLAGS>
__device__ __forceinline__ void gather(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                       typename S::R* fin) {
    gather_loads<L, S, FLAGS>(a, n, o, flag, fin);
    gather_fixup<L, S, FLAGS>(a, n, o, flag, fin);
}

// ------------------------------------------------------------------ scatter
// Post-collision values go back to the slots the pair was read from
// (reference esoteric_pull.hpp:367-382):
//   even step: f[j][n] = fout_i, f[i][nb] = fout_j
//   odd step:  f[i][n] = fout_i, f[j][nb] = fout_j
// i.e. fout_i -> pb[p][n], fout_j -> pa[p][nb].
template <class L, class S, bool NARROW, bool RAW = false, int P = 0>
__device__ __forceinline__ void scatter_pairs(const LbmArgs& a, u32 n, const Nbr& o, const typename S::R* fout,
                                              u32 h) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        auto* pi = Slots<S, NARROW>::at(a, false, P, n);
        auto* pj = Slots<S, NARROW>::at(a, true, P, n + nbr_off<L, j>(o));
        if constexpr (sizeof(typename S::T) == 2) {
            const float vi = RAW ? fout[i] : fout[i] * a.scale[i];
            const float vj = RAW ? fout[j] : fout[j] * a.scale[j];
            const u32 w = f16x2_rs(vj, vi, round_bits(a, h, P + 1));
            *reinterpret_cast<unsigned short*>(pi) = static_cast<unsigned short>(w);
            *reinterpret_cast<unsigned short*>(pj) = static_cast<unsigned short>(w >> 16);
        } else {
            st<S, L, i, RAW>(pi, fout[i], a);
            st<S, L, j, RAW>(pj, fout[j], a);
        }
        scatter_pairs<L, S, NARROW, RAW, P + 1>(a, n, o, fout, h);
    }
}

// h: the cell's rounding hash (round_hash; FP16 storage only).
template <class L, class S, bool NARROW, bool RAW = false>
__device__ __forceinline__ void scatter(const LbmArgs& a, u32 n, const Nbr& o, const typename S::R* fout, u32 h) {
    if constexpr (sizeof(typename S::T) == 2) {
        const float v0 = RAW ? fout[0] : fout[0] * a.scale[0];
        st_h16(Slots<S, NARROW>::rest(a, n), v0, round_bits(a, h, 0));
    } else {
        st<S, L, 0, RAW>(Slots<S, NARROW>::rest(a, n), fout[0], a);
    }
    scatter_pairs<L, S, NARROW, RAW>(a, n, o, fout, h);
}

// ------------------------------------------------------------------ helpers
// Reciprocals.  rcp: the hardware approximation (__fdividef, within 2 ulp),
// for relaxation rates, which enter a cell's mass and momentum alike.
// rcp_unbiased, for 1/rho in u = j / rho: the collision returns the momentum
// rho u, so an error in 1/rho that leans one way (an approximation's does)
// moves every cell's momentum the same way each step.  One Newton-Raphson step
// r + r (1 - x r) on the approximation leaves a symmetric error of about half
// an ulp at the cost of two fused multiply-adds.
__device__ __forceinline__ float rcp(float x) { return __fdividef(1.0F, x); }
__device__ __forceinline__ float rcp_unbiased(float x) {
    const float r = __fdividef(1.0F, x);
    return fmaf(r, fmaf(-x, r, 1.0F), r);
}
__device__ __forceinline__ double rcp_unbiased(double x) { return 1.0 / x; }
__device__ __forceinline__ double rcp(double x) { return 1.0 / x; }

// ---------------------------------------------------------------- moments
// rho and u of a cell (reference esoteric_pull.hpp:384-406), summed per
// opposite pair: s_p = f_i + f_j, d_p = f_i - f_j (c_j = -c_i).
template <class L, class R, int P = 0>
__device__ __forceinline__ void pair_sums(const R* f, R* s, R* d) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        s[P] = f[i] + f[j];
        d[P] = f[i] - f[j];
        pair_sums<L, R, P + 1>(f, s, d);
    }
}

// DELTA: the values are deviations f - w, whose rest weights sum to 1.
template <class L, class R, bool DELTA = false>
__device__ __forceinline__ void pair_moments(R f0, const R* s, const R* d, R& rho, R& jx, R& jy, R& jz) {
    R r = f0, x = R(0), y = R(0), z = R(0);
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        const int i = 2 * p + 1;
        r += s[p];
        if (L::cx(i) > 0) x += d[p];
        if (L::cx(i) < 0) x -= d[p];
        if (L::cy(i) > 0) y += d[p];
        if (L::cy(i) < 0) y -= d[p];
        if (L::cz(i) > 0) z += d[p];
        if (L::cz(i) < 0) z -= d[p];
    }
    rho = DELTA ? R(1) + r : r;
    jx = x;
    jy = y;
    jz = z;
}

template <class L, class R, bool DELTA = false>
__device__ __forceinline__ void moments(const R* fin, R& rho, R& ux, R& uy, R& uz) {
    R s[L::PAIRS], d[L::PAIRS], jx, jy, jz;
    pair_sums<L, R>(fin, s, d);
    pair_moments<L, R, DELTA>(fin[0], s, d, rho, jx, jy, jz);
    // reference esoteric_pull.hpp:397-405: u = 0 when rho <= 0
    const R inv = rho > R(0) ? rcp_unbiased(rho) : R(0);
    ux = jx * inv;
    uy = jy * inv;
    uz = jz * inv;
}

// Scalar parameters in the arithmetic type (FP32 kernels read the float copies).
template <class R> __device__ __forceinline__ R p_tau(const LbmArgs& a) {
    if constexpr (sizeof(R) == 8) return a.tau; else return a.tau_f;
}
template <class R> __device__ __forceinline__ R p_les_k(const LbmArgs& a) {
    if constexpr (sizeof(R) == 8) return a.les_k; else return a.les_k_f;
}

template <class R> __device__ __forceinline__ void cell_acceleration(const LbmArgs& a, u32 n, R& ax, R& ay, R& az) {
    if constexpr (sizeof(R) == 8) {
        ax = a.ax;
        ay = a.ay;
        az = a.az;
    } else {
        ax = a.ax_f;
        ay = a.ay_f;
        az = a.az_f;
    }
    if (a.ax_field) {
        ax += R(a.ax_field[n]);
        ay += R(a.ay_field[n]);
        az += R(a.az_field[n]);
    }
}

// Smagorinsky relaxation time (reference esoteric_pull.hpp:72-97 with the
// coefficient K = 18 sqrt(2) Cs^2 as a parameter).  The non-equilibrium
// momentum flux is formed as sum c_a c_b f - rho (delta_ab / 3 + u_a u_b),
// which equals sum c_a c_b (f - feq) on D3Q19/D3Q27 (both lattices are
// fourth-order isotropic) and needs no per-direction equilibria; c_a c_b is
// even in c, so the sums run over pair sums s_p.
template <class L, class R, bool DELTA = false>
__device__ __forceinline__ R les_tau(const R* s, R rho, R irho, R ux, R uy, R uz, R tau, R k) {
    if (!(rho > R(0))) return tau;
    R sxx = R(0), syy = R(0), szz = R(0), sxy = R(0), sxz = R(0), syz = R(0);
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        const int i = 2 * p + 1;
        if (L::cx(i) != 0) sxx += s[p];
        if (L::cy(i) != 0) syy += s[p];
        if (L::cz(i) != 0) szz += s[p];
        if (L::cx(i) * L::cy(i) > 0) sxy += s[p];
        if (L::cx(i) * L::cy(i) < 0) sxy -= s[p];
        if (L::cx(i) * L::cz(i) > 0) sxz += s[p];
        if (L::cx(i) * L::cz(i) < 0) sxz -= s[p];
        if (L::cy(i) * L::cz(i) > 0) syz += s[p];
        if (L::cy(i) * L::cz(i) < 0) syz -= s[p];
    }
    const R third = R(1.0 / 3.0);
    if constexpr (DELTA) { // sum_d c_a c_b w_d = delta_ab / 3
        sxx += third;
        syy += third;
        szz += third;
    }
    const R pxx = sxx - rho * (third + ux * ux);
    const R pyy = syy - rho * (third + uy * uy);
    const R pzz = szz - rho * (third + uz * uz);
    const R pxy = sxy - rho * ux * uy;
    const R pxz = sxz - rho * ux * uz;
    const R pyz = syz - rho * uy * uz;
    const R q = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz);
    return R(0.5) * (tau + sqrt(tau * tau + k * sqrt(q) * irho));
}

// ---------------------------------------------------------------- collision
// Two-relaxation-time collision with Guo forcing (reference
// one_step_pull.hpp:187-204; BGK, esoteric_pull.hpp:408-432, is the case
// omega- = omega+), evaluated per opposite pair on s = f_i + f_j and
// d = f_i - f_j:
//   equilibrium  s_eq = 2 w rho t,  t = 1 - 1.5 u^2 + 4.5 (c.u)^2,   d_eq = 2 w rho (3 c.u)
//   Guo source   s_F  = 2 w (9 (c.u)(c.F) - 3 u.F),                d_F  = 6 w (c.F)
//   s' = s - omega+ (s - s_eq) + (1 - omega+/2) s_F
//   d' = d - omega- (d - d_eq) + (1 - omega-/2) d_F
//   f_i' = (s' + d') / 2,  f_j' = (s' - d') / 2
// The halves s'/2 and d'/2 are formed directly with per-weight-class
// coefficients computed once per cell, so a pair costs a handful of fused
// multiply-adds.  With DELTA the values are deviations f - w: s_eq becomes
// 2 w (rho t - 1) (w_i = w_j within a pair, so d is unchanged).  Gray-LBM
// partial bounce-back then mixes in the incoming opposite population:
// f_i <- (1 - n_s) f_i' + n_s fin_j (Walsh, Burwinkle & Saar 2009).
//
// Rounding: the mass and momentum coefficients both derive from the per-cell
// product w rho (rounded differently in every cell), then times omega+ or
// omega-.  A coefficient formed from constants alone (3 omega- w) carries one
// rounding error shared by every cell and every step, which the collision
// turns into a steady gain or loss of momentum against mass: with
// 3 omega- w rho, a 64^3 Taylor-Green vortex in FP32 gained kinetic energy at
// 2.3e-7 relative per step against FP64.  What remains is the representation
// error of the FP32 weights themselves, as in the reference.
template <class R> struct ClassCoef {
    R a;  // omega+ w rho          (s'/2 equilibrium term: a * t)
    R a0; // omega+ w              (DELTA: subtracted)
    R c;  // omega- w rho          (d'/2 equilibrium term: c * (3 c.u))
    R g1; // 3 (1 - omega+/2) w    (s'/2 force term: g1 * ((3 c.u)(c.F) - u.F))
    R g2; // 3 (1 - omega-/2) w    (d'/2 force term)
};

template <class L, class R, bool FORCE, bool GRAY, bool DELTA, int P = 0>
__device__ __forceinline__ void collide_pairs(R* f, const R* s, const R* d, const ClassCoef<R>* cc, R ux3, R uy3,
                                              R uz3, R ux15, R uy15, R uz15, R fx, R fy, R fz, R base, R uf, R a1,
                                              R b1, R ns) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const ClassCoef<R>& k = cc[weight_class<L>(i)];
        const R cu3 = cdot<L, i>(ux3, uy3, uz3);     // 3 c.u
        const R cu15 = cdot<L, i>(ux15, uy15, uz15); // 1.5 c.u
        const R t = cu3 * cu15 + base;
        R sp = DELTA ? k.a * t + (a1 * s[P] - k.a0) : k.a * t + a1 * s[P];
        R dp = k.c * cu3 + b1 * d[P];
        if constexpr (FORCE) {
            const R cf = cdot<L, i>(fx, fy, fz);
            sp += k.g1 * (cu3 * cf - uf);
            dp += k.g2 * cf;
        }
        R oi = sp + dp;
        R oj = sp - dp;
        if constexpr (GRAY) {
            const R fi = R(0.5) * (s[P] + d[P]);
            const R fj = R(0.5) * (s[P] - d[P]);
            oi = (R(1) - ns) * oi + ns * fj;
            oj = (R(1) - ns) * oj + ns * fi;
        }
        f[i] = oi;
        f[j] = oj;
        collide_pairs<L, R, FORCE, GRAY, DELTA, P + 1>(f, s, d, cc, ux3, uy3, uz3, ux15, uy15, uz15, fx, fy, fz, base,
                                                       uf, a1, b1, ns);
    }
}

// Relaxation rates of a cell: omega+ from tau (LES-adjusted) and omega- by
// the configured rule.
template <class R> __device__ __forceinline__ R omega_minus_of(const LbmArgs& a, R tau, R omega) {
    if (a.minus_mode > 0) return sizeof(R) == 8 ? R(a.omega_minus) : R(a.omega_minus_f); // fixed TRT rate
    if (a.minus_mode < 0) return omega;                                                  // BGK
    // TRT magic: tau- = 1/2 + Lambda / (tau+ - 1/2)
    const R sp = tau - R(0.5);
    const R lam = sizeof(R) == 8 ? R(a.trt_magic) : R(a.trt_magic_f);
    return sp * rcp(lam + R(0.5) * sp);
}

// Per weight class coefficients; `scale` multiplies every term (FP16 storage
// units), 1 otherwise.
template <class L, class R>
__device__ __forceinline__ void class_coefficients(ClassCoef<R>* cc, R rho, R omega, R omega_m, R gp, R gm,
                                                   const R* scale) {
    constexpr int K = L::Q == 27 ? 3 : 2;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        const R w = R(L::w(class_rep(k))) * scale[k];
        const R wr = w * rho;
        cc[k].a0 = omega * w;
        cc[k].a = omega * wr;
        cc[k].c = omega_m * wr;
        cc[k].g1 = R(3) * gp * w;
        cc[k].g2 = R(3) * gm * w;
    }
}

template <class L, class R, bool LES, bool GRAY, bool FORCE, bool DELTA = false>
__device__ __forceinline__ void collide(const LbmArgs& a, u32 n, R* f) {
    R s[L::PAIRS], d[L::PAIRS];
    pair_sums<L, R>(f, s, d);
    R rho, jx, jy, jz;
    pair_moments<L, R, DELTA>(f[0], s, d, rho, jx, jy, jz);
    const R inv = rho > R(0) ? rcp_unbiased(rho) : R(0);
    R ux = jx * inv, uy = jy * inv, uz = jz * inv;
    R ax = R(0), ay = R(0), az = R(0);
    if constexpr (FORCE) {
        cell_acceleration<R>(a, n, ax, ay, az);
        ux += R(0.5) * ax;
        uy += R(0.5) * ay;
        uz += R(0.5) * az;
    }
    R tau = p_tau<R>(a);
    if constexpr (LES) tau = les_tau<L, R, DELTA>(s, rho, inv, ux, uy, uz, tau, p_les_k<R>(a));
    const R omega = rcp(tau);
    const R omega_m = omega_minus_of<R>(a, tau, omega);
    const R base = R(1) - R(1.5) * (ux * ux + uy * uy + uz * uz);
    R fx = R(0), fy = R(0), fz = R(0), uf = R(0);
    if constexpr (FORCE) {
        fx = rho * ax;
        fy = rho * ay;
        fz = rho * az;
        uf = ux * fx + uy * fy + uz * fz;
    }
    const R gp = R(1) - R(0.5) * omega;
    const R gm = R(1) - R(0.5) * omega_m;
    R ns = R(0);
    if constexpr (GRAY) ns = R(a.ns[n]);
    {
        constexpr R w0 = R(L::w(0));
        const R f0 = f[0];
        R o0 = (R(1) - omega) * f0 + omega * (DELTA ? w0 * (rho * base - R(1)) : (w0 * rho) * base);
        if constexpr (FORCE) o0 -= gp * w0 * (R(3) * uf);
        if constexpr (GRAY) o0 = (R(1) - ns) * o0 + ns * f0;
        f[0] = o0;
    }
    ClassCoef<R> cc[4];
    const R unit[4] = {R(1), R(1), R(1), R(1)};
    class_coefficients<L, R>(cc, rho, omega, omega_m, gp, gm, unit);
    collide_pairs<L, R, FORCE, GRAY, DELTA>(f, s, d, cc, R(3) * ux, R(3) * uy, R(3) * uz, R(1.5) * ux, R(1.5) * uy,
                                            R(1.5) * uz, fx, fy, fz, base, uf, R(0.5) * (R(1) - omega),
                                            R(0.5) * (R(1) - omega_m), ns);
}

// --------------------------------------------------- FP16 scaled collision
// The same TRT/Guo/gray update as collide, for values held in FP16 storage
// units h = (f - w) s_k, with s_k constant within each weight class k.
// Pair sums stay in storage units: the moments scale each class's partial
// sums once, and the scales are folded into the per-class coefficients, so
// decoding and encoding cost only the half <-> float conversions.
//
// Written once for V = float (one cell) and V = float2 (two cells, sm_100a
// packed f32x2 instructions: one issue slot for both cells).  Every operation
// is an explicitly rounded intrinsic, so the compiler cannot contract the two
// forms differently and the one-cell and two-cell kernels stay bitwise equal.

__device__ __forceinline__ float v_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float v_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float v_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float v_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float2 v_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 v_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b = RN(b * (-1) + a), the same rounding as the scalar subtraction
__device__ __forceinline__ float2 v_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0F, -1.0F), a); }
__device__ __forceinline__ float2 v_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }

template <class V> __device__ __forceinline__ V v_splat(float c) {
    if constexpr (sizeof(V) == 8) return make_float2(c, c); else return c;
}
template <class V> constexpr int v_lanes() { return sizeof(V) / sizeof(float); }
__device__ __forceinline__ float v_lane(float v, int) { return v; }
__device__ __forceinline__ float v_lane(float2 v, int k) { return k ? v.y : v.x; }
__device__ __forceinline__ void v_set(float& v, int, float x) { v = x; }
__device__ __forceinline__ void v_set(float2& v, int k, float x) { if (k) v.y = x; else v.x = x; }
// Applies a scalar function lane by lane.
template <class V, class F> __device__ __forceinline__ V v_map(V v, F f) {
    V r = v;
#pragma unroll
    for (int k = 0; k < v_lanes<V>(); ++k) v_set(r, k, f(v_lane(v, k), k));
    return r;
}

// Signed sum of lattice-vector components, V form (see signed_sum).
template <int A, int B, int C, class V> __device__ __forceinline__ V v_signed_sum(V x, V y, V z) {
    static_assert(A > 0 || B > 0 || C > 0, "the pair's first direction has a positive component");
    if constexpr (A > 0) {
        V r = x;
        if constexpr (B > 0) r = v_add(r, y);
        if constexpr (C > 0) r = v_add(r, z);
        if constexpr (B < 0) r = v_sub(r, y);
        if constexpr (C < 0) r = v_sub(r, z);
        return r;
    } else if constexpr (B > 0) {
        V r = y;
        if constexpr (C > 0) r = v_add(r, z);
        if constexpr (A < 0) r = v_sub(r, x);
        if constexpr (C < 0) r = v_sub(r, z);
        return r;
    } else {
        V r = z;
        if constexpr (A < 0) r = v_sub(r, x);
        if constexpr (B < 0) r = v_sub(r, y);
        return r;
    }
}
template <class L, int D, class V> __device__ __forceinline__ V v_cdot(V x, V y, V z) {
    return v_signed_sum<L::cx(D), L::cy(D), L::cz(D), V>(x, y, z);
}

// Sum over pairs p in [P, PAIRS) of coef(p) * val[p], coef(p) in {-1, 0, 1}
// given by Coef::at(p); started from the first nonzero term, so no
// instruction is spent adding to zero.
template <class Coef, int P, int E, class V> __device__ __forceinline__ V v_csum_from(V acc, const V* val) {
    if constexpr (P < E) {
        constexpr int c = Coef::at(P);
        if constexpr (c > 0) acc = v_add(acc, val[P]);
        if constexpr (c < 0) acc = v_sub(acc, val[P]);
        return v_csum_from<Coef, P + 1, E>(acc, val);
    } else {
        return acc;
    }
}
template <class Coef, int P, int E, class V> __device__ __forceinline__ V v_csum(const V* val) {
    if constexpr (P >= E) {
        return v_splat<V>(0.0F);
    } else {
        constexpr int c = Coef::at(P);
        if constexpr (c > 0) return v_csum_from<Coef, P + 1, E>(val[P], val);
        else if constexpr (c < 0) return v_csum_from<Coef, P + 1, E>(v_sub(v_splat<V>(0.0F), val[P]), val);
        else return v_csum<Coef, P + 1, E>(val);
    }
}
// Coefficients of pair p (first direction i = 2p+1) in the class-k sums:
// component moments (c_a, 0 = all ones) and second moments (c_a c_b).
template <class L, int K, int A> struct CoefFirst {
    static constexpr int at(int p) {
        const int i = 2 * p + 1;
        if (weight_class<L>(i) != K) return 0;
        return A == 0 ? 1 : (A == 1 ? L::cx(i) : (A == 2 ? L::cy(i) : L::cz(i)));
    }
};
template <class L, int K, int A, int B> struct CoefSecond {
    static constexpr int comp(int i, int c) { return c == 1 ? L::cx(i) : (c == 2 ? L::cy(i) : L::cz(i)); }
    static constexpr int at(int p) {
        const int i = 2 * p + 1;
        return weight_class<L>(i) != K ? 0 : comp(i, A) * comp(i, B);
    }
};
template <class L, int K, int A, class V> __device__ __forceinline__ V class_sum(const V* v) {
    return v_csum<CoefFirst<L, K, A>, 0, L::PAIRS>(v);
}
template <class L, int K, int A, int B, class V> __device__ __forceinline__ V class_sum2(const V* v) {
    return v_csum<CoefSecond<L, K, A, B>, 0, L::PAIRS>(v);
}
// sum_k sum_k-class(v) / s_k over the weight classes 1..K, as a multiply-add chain.
template <class L, int A, class V> __device__ __forceinline__ V scaled_moment(const V* v, const float* inv, V init) {
    V r = v_fma(class_sum<L, 1, A>(v), v_splat<V>(inv[1]), init);
    r = v_fma(class_sum<L, 2, A>(v), v_splat<V>(inv[2]), r);
    if constexpr (L::Q == 27) r = v_fma(class_sum<L, 3, A>(v), v_splat<V>(inv[3]), r);
    return r;
}
template <class L, int A, int B, class V>
__device__ __forceinline__ V scaled_moment2(const V* v, const float* inv, V init) {
    V r = v_fma(class_sum2<L, 1, A, B>(v), v_splat<V>(inv[1]), init);
    r = v_fma(class_sum2<L, 2, A, B>(v), v_splat<V>(inv[2]), r);
    if constexpr (L::Q == 27) r = v_fma(class_sum2<L, 3, A, B>(v), v_splat<V>(inv[3]), r);
    return r;
}

// sqrt for the Smagorinsky rate: hardware reciprocal square root (2 ulp);
// the eddy viscosity needs no correctly rounded square root, and FP16
// storage rounding is far larger.  x >= 0; x = 0 gives 0.
__device__ __forceinline__ float les_sqrt(float x) { return __fmul_rn(x, rsqrtf(fmaxf(x, 1.0e-30F))); }

// n: the first cell of V's lanes (lane k is cell n + k).
template <class L, bool LES, bool GRAY, bool FORCE, class V>
__device__ __forceinline__ void collide_scaled(const LbmArgs& a, u32 n, V* h) {
    constexpr int K = L::Q == 27 ? 3 : 2;
    const V one = v_splat<V>(1.0F);
    V sh[L::PAIRS], dh[L::PAIRS];
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        sh[p] = v_add(h[2 * p + 1], h[2 * p + 2]);
        dh[p] = v_sub(h[2 * p + 1], h[2 * p + 2]);
    }
    float inv[4], scl[4];
#pragma unroll
    for (int k = 0; k <= K; ++k) {
        inv[k] = a.inv_scale[class_rep(k)];
        scl[k] = a.scale[class_rep(k)];
    }
    const V rho = v_add(scaled_moment<L, 0>(sh, inv, v_mul(h[0], v_splat<V>(inv[0]))), one);
    const V zero = v_splat<V>(-0.0F); // x + (-0) == x for every x
    const V jx = scaled_moment<L, 1>(dh, inv, zero);
    const V jy = scaled_moment<L, 2>(dh, inv, zero);
    const V jz = scaled_moment<L, 3>(dh, inv, zero);
    const V irho = v_map(rho, [](float r, int) { return r > 0.0F ? rcp_unbiased(r) : 0.0F; });
    V ux = v_mul(jx, irho), uy = v_mul(jy, irho), uz = v_mul(jz, irho);
    V ax = zero, ay = zero, az = zero;
    if constexpr (FORCE) {
        ax = v_map(ax, [&](float, int k) { float x, y, z; cell_acceleration<float>(a, n + k, x, y, z); return x; });
        ay = v_map(ay, [&](float, int k) { float x, y, z; cell_acceleration<float>(a, n + k, x, y, z); return y; });
        az = v_map(az, [&](float, int k) { float x, y, z; cell_acceleration<float>(a, n + k, x, y, z); return z; });
        const V half = v_splat<V>(0.5F);
        ux = v_fma(ax, half, ux);
        uy = v_fma(ay, half, uy);
        uz = v_fma(az, half, uz);
    }
    V omega, omega_m;
    if constexpr (LES) {
        const V third = v_splat<V>(1.0F / 3.0F);
        const V sxx = scaled_moment2<L, 1, 1>(sh, inv, third);
        const V syy = scaled_moment2<L, 2, 2>(sh, inv, third);
        const V szz = scaled_moment2<L, 3, 3>(sh, inv, third);
        const V sxy = scaled_moment2<L, 1, 2>(sh, inv, zero);
        const V sxz = scaled_moment2<L, 1, 3>(sh, inv, zero);
        const V syz = scaled_moment2<L, 2, 3>(sh, inv, zero);
        const V nrho = v_mul(rho, v_splat<V>(-1.0F));
        const V pxx = v_fma(nrho, v_fma(ux, ux, third), sxx);
        const V pyy = v_fma(nrho, v_fma(uy, uy, third), syy);
        const V pzz = v_fma(nrho, v_fma(uz, uz, third), szz);
        const V nrux = v_mul(nrho, ux), nruy = v_mul(nrho, uy);
        const V pxy = v_fma(nrux, uy, sxy);
        const V pxz = v_fma(nrux, uz, sxz);
        const V pyz = v_fma(nruy, uz, syz);
        V off = v_mul(pxy, pxy);
        off = v_fma(pxz, pxz, off);
        off = v_fma(pyz, pyz, off);
        V q = v_fma(pxx, pxx, v_add(off, off));
        q = v_fma(pyy, pyy, q);
        q = v_fma(pzz, pzz, q);
        const float tau0 = a.tau_f, kles = a.les_k_f;
        V tau = v_map(q, [&](float qq, int k) {
            const float r = v_lane(rho, k);
            // tau0/2 + sqrt(tau0^2 + K sqrt(Q) / rho) / 2, every operation explicitly rounded: the
            // same bits in every kernel, whatever the compiler hoists out of a loop around it
            const float t = __fmul_rn(__fmul_rn(kles, les_sqrt(qq)), v_lane(irho, k));
            return r > 0.0F ? __fmul_rn(0.5F, __fadd_rn(tau0, les_sqrt(__fmaf_rn(tau0, tau0, t)))) : tau0;
        });
        omega = v_map(tau, [](float t, int) { return rcp(t); });
        omega_m = v_map(tau, [&](float t, int k) { return omega_minus_of<float>(a, t, v_lane(omega, k)); });
    } else {
        const float w = rcp(a.tau_f);
        omega = v_splat<V>(w);
        omega_m = v_splat<V>(omega_minus_of<float>(a, a.tau_f, w));
    }
    V base = v_mul(ux, ux);
    base = v_fma(uy, uy, base);
    base = v_fma(uz, uz, base);
    base = v_fma(base, v_splat<V>(-1.5F), one);
    V fx = zero, fy = zero, fz = zero, nuf = zero;
    if constexpr (FORCE) {
        fx = v_mul(rho, ax);
        fy = v_mul(rho, ay);
        fz = v_mul(rho, az);
        V uf = v_mul(ux, fx);
        uf = v_fma(uy, fy, uf);
        uf = v_fma(uz, fz, uf);
        nuf = v_mul(uf, v_splat<V>(-1.0F));
    }
    const V nhalf = v_splat<V>(-0.5F);
    const V gp = v_fma(omega, nhalf, one), gm = v_fma(omega_m, nhalf, one);
    V ns = zero, keep = one;
    if constexpr (GRAY) {
        ns = v_map(ns, [&](float, int k) { return a.ns[n + k]; });
        keep = v_sub(one, ns);
    }
    {
        const float w0 = float(L::w(0)) * scl[0];
        const V h0 = h[0];
        // (1 - omega) h0 + s0 omega w0 (rho base - 1)  [- s0 (1 - omega/2) w0 3 u.F]
        V o0 = v_fma(v_sub(one, omega), h0, v_mul(v_mul(omega, v_splat<V>(w0)), v_fma(rho, base, v_splat<V>(-1.0F))));
        if constexpr (FORCE) o0 = v_fma(v_mul(gp, v_splat<V>(3.0F * w0)), nuf, o0);
        if constexpr (GRAY) o0 = v_fma(keep, o0, v_mul(ns, h0));
        h[0] = o0;
    }
    // per weight class: a = omega w rho, a0 = omega w, c = omega- w rho (w includes the storage scale)
    V ka[4], nka0[4], kc[4], g1[4], g2[4];
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        const float w = float(L::w(class_rep(k))) * scl[k];
        const V wr = v_mul(rho, v_splat<V>(w));
        ka[k] = v_mul(omega, wr);
        kc[k] = v_mul(omega_m, wr);
        nka0[k] = v_mul(omega, v_splat<V>(-w));
        if constexpr (FORCE) {
            g1[k] = v_mul(gp, v_splat<V>(3.0F * w));
            g2[k] = v_mul(gm, v_splat<V>(3.0F * w));
        }
    }
    const V a1 = v_mul(v_sub(one, omega), v_splat<V>(0.5F));
    const V b1 = v_mul(v_sub(one, omega_m), v_splat<V>(0.5F));
    const V ux3 = v_mul(ux, v_splat<V>(3.0F)), uy3 = v_mul(uy, v_splat<V>(3.0F)), uz3 = v_mul(uz, v_splat<V>(3.0F));
    const V ux15 = v_mul(ux, v_splat<V>(1.5F)), uy15 = v_mul(uy, v_splat<V>(1.5F)), uz15 = v_mul(uz, v_splat<V>(1.5F));
    static_for_pairs<L>([&](auto PP) {
        constexpr int p = decltype(PP)::value;
        constexpr int i = 2 * p + 1, j = i + 1;
        constexpr int k = weight_class<L>(i);
        const V cu3 = v_cdot<L, i>(ux3, uy3, uz3);
        const V cu15 = v_cdot<L, i>(ux15, uy15, uz15);
        const V t = v_fma(cu3, cu15, base);
        V sp = v_fma(ka[k], t, v_fma(a1, sh[p], nka0[k]));
        V dp = v_fma(kc[k], cu3, v_mul(b1, dh[p]));
        if constexpr (FORCE) {
            const V cf = v_cdot<L, i>(fx, fy, fz);
            sp = v_fma(g1[k], v_fma(cu3, cf, nuf), sp);
            dp = v_fma(g2[k], cf, dp);
        }
        V oi = v_add(sp, dp);
        V oj = v_sub(sp, dp);
        if constexpr (GRAY) {
            const V hi = h[i], hj = h[j];
            oi = v_fma(keep, oi, v_mul(ns, hj));
            oj = v_fma(keep, oj, v_mul(ns, hi));
        }
        h[i] = oi;
        h[j] = oj;
    });
}

// ---------------------------------------------------------------- the step
// CPT cells per thread (stacked in z): the loads of all of a thread's cells are
// issued before the first collision.  One cell per thread measured best on
// B200 (more cells cost occupancy through registers), and the launcher uses 1.
// Minimum resident 128-thread blocks per SM the step kernels are compiled for;
// it caps registers at 65536 / (128 * blocks).  The step is latency bound at
// the occupancy its natural register count allows: measured on B200 at 512^3,
// 10 blocks (48 registers, a few spilled words that stay in L1) beat the
// uncapped 64-96 registers by 10-55% for FP32 and FP16 storage, and for D3Q19
// 12 blocks (40 registers) beat 10 once the wall path stopped branching (LES
// cavity FP16 48.4 vs 46.9, FP32 40.6 vs 40.0; sphere pack within 0.5 %);
// FP64 storage keeps its full register set.  The macros exist for tuning builds.
#ifndef CFDX_STEP_MIN_BLOCKS_Q19
#define CFDX_STEP_MIN_BLOCKS_Q19 12
#endif
#ifndef CFDX_STEP_MIN_BLOCKS_Q27_F16
#define CFDX_STEP_MIN_BLOCKS_Q27_F16 10
#endif
#ifndef CFDX_STEP_MIN_BLOCKS_Q27_F32
#define CFDX_STEP_MIN_BLOCKS_Q27_F32 8
#endif
#ifndef CFDX_PAIR_MIN_BLOCKS
#define CFDX_PAIR_MIN_BLOCKS 8
#endif
// Gray-LBM forms (partial bounce-back) keep the solid fraction and the
// pre-collision populations alive through the collision and spilled up to
// 112 (D3Q19 FP32) and 368 (D3Q27 FP16) bytes per thread at the caps above.
// Measured on B200, gray TRT channel forward step: D3Q27 FP16 256^3 at 8
// blocks (64 registers) 548 us vs 744 us at 10; D3Q19 FP32 128^3 at 8 blocks
// 63.7 us vs 65.9 us at 12 (10 blocks, 48 registers, keeps 24 bytes of spill).
#ifndef CFDX_STEP_MIN_BLOCKS_Q19_GRAY
#define CFDX_STEP_MIN_BLOCKS_Q19_GRAY 10
#endif
#ifndef CFDX_STEP_MIN_BLOCKS_Q27_F16_GRAY
#define CFDX_STEP_MIN_BLOCKS_Q27_F16_GRAY 8
#endif

template <class L, class S, bool GRAY = false> constexpr int step_min_blocks() {
    if constexpr (sizeof(typename S::T) == 8) {
        return 1;
    } else if constexpr (L::Q == 19) {
        return GRAY ? CFDX_STEP_MIN_BLOCKS_Q19_GRAY : CFDX_STEP_MIN_BLOCKS_Q19;
    } else if constexpr (sizeof(typename S::T) == 2) {
        return GRAY ? CFDX_STEP_MIN_BLOCKS_Q27_F16_GRAY : CFDX_STEP_MIN_BLOCKS_Q27_F16;
    } else {
        return CFDX_STEP_MIN_BLOCKS_Q27_F32;
    }
}
template <class S> constexpr int pair_min_blocks() { return sizeof(typename S::T) == 8 ? 1 : CFDX_PAIR_MIN_BLOCKS; }

template <class L, class S, bool LES, bool FLAGS, bool GRAY, int CPT, bool NARROW>
__global__ void __launch_bounds__(128, step_min_blocks<L, S, GRAY>()) k_step(const __grid_constant__ LbmArgs a) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z0 = a.z_first + blockIdx.z * CPT;
    if (x >= a.nx || y >= a.ny) return;
    R fin[CPT][L::Q];
    std::uint8_t flag[CPT];
    bool live[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        const u32 z = z0 + c;
        const u32 n = (z * a.ny + y) * a.nx + x;
        live[c] = z < a.z_end;
        flag[c] = 0;
        if constexpr (FLAGS) {
            if (live[c]) {
                flag[c] = a.flags[n];
                live[c] = (flag[c] & kFlagTypeMask) == 0; // walls hold no populations of their own
            }
        }
        if (live[c]) gather_loads<L, S, FLAGS, NARROW, S::scaled>(a, n, make_nbr(a, x, y, z), flag[c], fin[c]);
    }
    const bool force = a.has_force != 0;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        if (!live[c]) continue;
        const u32 z = z0 + c;
        const u32 n = (z * a.ny + y) * a.nx + x;
        const Nbr o = make_nbr(a, x, y, z);
        if constexpr (S::scaled) {
            if constexpr (FLAGS) gather_fixup_scaled<L>(a, n, o, flag[c], fin[c]);
            if (force)
                collide_scaled<L, LES, GRAY, true>(a, n, fin[c]);
            else
                collide_scaled<L, LES, GRAY, false>(a, n, fin[c]);
        } else {
            gather_fixup<L, S, FLAGS>(a, n, o, flag[c], fin[c]);
            if (force)
                collide<L, R, LES, GRAY, true, S::delta>(a, n, fin[c]);
            else
                collide<L, R, LES, GRAY, false, S::delta>(a, n, fin[c]);
        }
        const u32 h = sizeof(typename S::T) == 2 ? round_hash(a, n) : 0U;
        scatter<L, S, NARROW, S::scaled>(a, n, o, fin[c], h);
    }
}

// Equilibrium initialisation into the esoteric slots of time step 0
// (reference esoteric_pull.hpp:312-333; Taylor-Green field :121-137).  Wall
// links additionally seed the partner slot, so that the first step's bounced
// loads see the cell's own equilibrium exactly as the reference's first
// solid step does.  Uses the parity-0 tables.
template <class L, class S, bool FLAGS, int P = 0>
__device__ __forceinline__ void init_pairs(const LbmArgs& a, u32 n, const Nbr& o, unsigned walls, typename S::R rho,
                                           typename S::R ux, typename S::R uy, typename S::R uz,
                                           typename S::R usq15) {
    using R = typename S::R;
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const R cu = cdot<L, i>(ux, uy, uz);
        const R wr = R(L::w(i)) * rho;
        const R fi = wr * (R(1) + R(3) * cu + R(4.5) * cu * cu - usq15);
        const R fj = wr * (R(1) - R(3) * cu + R(4.5) * cu * cu - usq15);
        const u32 nb = n + nbr_off<L, j>(o);
        const R hi = held<S, L, i>(fi), hj = held<S, L, j>(fj);
        st<S, L, i>(static_cast<typename S::T*>(a.fd[i]) + nb, hi, a);
        st<S, L, j>(static_cast<typename S::T*>(a.fd[j]) + n, hj, a);
        if constexpr (FLAGS) {
            if ((walls >> (2 * P)) & 1U) st<S, L, j>(static_cast<typename S::T*>(a.fd[j]) + nb, hi, a);
            if ((walls >> (2 * P + 1)) & 1U) st<S, L, i>(static_cast<typename S::T*>(a.fd[i]) + n, hj, a);
        }
        init_pairs<L, S, FLAGS, P + 1>(a, n, o, walls, rho, ux, uy, uz, usq15);
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(128) k_init(const __grid_constant__ LbmArgs a, const InitSpec s) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    unsigned walls = 0U;
    const Nbr o = make_nbr(a, x, y, z);
    if constexpr (FLAGS) {
        const std::uint8_t flag = a.flags[n];
        if (flag & kFlagTypeMask) return;
        if (flag & kFlagNearWall) walls = a.wall_mask[n];
    }
    R rho, ux, uy, uz;
    if (s.kind == 0) {
        rho = R(s.rho);
        ux = R(s.ux);
        uy = R(s.uy);
        uz = R(s.uz);
    } else if (s.kind == 1) {
        // Evaluated in the arithmetic type, as the reference's FP32
        // (esoteric_pull.hpp:121-137) and FP64 (precision_pull.hpp:75-95) solvers do.
        const R two_pi = R(2) * R(3.14159265358979323846);
        const R xf = (R(x) + R(0.5)) / R(a.nx);
        const R yf = (R(y) + R(0.5)) / R(a.ny);
        const R zf = (R((z + s.z_origin) % s.nz_total) + R(0.5)) / R(s.nz_total);
        const R sx = sin(two_pi * xf), cx = cos(two_pi * xf);
        const R sy = sin(two_pi * yf), cy = cos(two_pi * yf);
        const R cz = cos(two_pi * zf);
        const R amp = R(s.amplitude);
        rho = R(1);
        ux = amp * sx * cy * cz;
        uy = -amp * cx * sy * cz;
        uz = R(0);
    } else {
        rho = R(s.fields[n]);
        ux = R(s.fields[std::size_t(a.N) + n]);
        uy = R(s.fields[2 * std::size_t(a.N) + n]);
        uz = R(s.fields[3 * std::size_t(a.N) + n]);
    }
    const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
    st<S, L, 0>(static_cast<typename S::T*>(a.fd[0]) + n, held<S, L, 0>(R(L::w(0)) * rho * (R(1) - usq15)), a);
    init_pairs<L, S, FLAGS>(a, n, o, walls, rho, ux, uy, uz, usq15);
}

// Macroscopic fields rho and u + a/2 (reference esoteric_pull.hpp:180-209 and
// esoteric_pull_sycl.hpp:229-307); wall cells report rho = 0, u = 0.
template <class L, class S, bool FLAGS, class OutT, bool NARROW = false>
__global__ void __launch_bounds__(128) k_macro(const __grid_constant__ LbmArgs a, OutT* rho_out, OutT* ux_out,
                                               OutT* uy_out, OutT* uz_out) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    std::uint8_t flag = 0;
    if constexpr (FLAGS) {
        flag = a.flags[n];
        if (flag & kFlagTypeMask) {
            rho_out[n] = OutT(0);
            ux_out[n] = OutT(0);
            uy_out[n] = OutT(0);
            uz_out[n] = OutT(0);
            return;
        }
    }
    R fin[L::Q];
    const Nbr o = make_nbr(a, x, y, z);
    gather_loads<L, S, FLAGS, NARROW>(a, n, o, flag, fin);
    gather_fixup<L, S, FLAGS>(a, n, o, flag, fin);
    R rho, ux, uy, uz, ax, ay, az;
    moments<L, R, S::delta>(fin, rho, ux, uy, uz);
    cell_acceleration<R>(a, n, ax, ay, az);
    rho_out[n] = OutT(rho);
    ux_out[n] = OutT(ux + R(0.5) * ax);
    uy_out[n] = OutT(uy + R(0.5) * ay);
    uz_out[n] = OutT(uz + R(0.5) * az);
}

// Parity-independent populations [d][n] (reference esoteric_pull.hpp:257-267).
template <class L, class S, bool FLAGS, class OutT>
__global__ void __launch_bounds__(128) k_logical(const __grid_constant__ LbmArgs a, OutT* out) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    R fin[L::Q];
    std::uint8_t flag = 0;
    bool wall = false;
    if constexpr (FLAGS) {
        flag = a.flags[n];
        wall = (flag & kFlagTypeMask) != 0;
    }
    if (!wall) gather<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), flag, fin);
#pragma unroll
    for (int d = 0; d < L::Q; ++d)
        out[static_cast<std::size_t>(d) * a.N + n] = wall ? OutT(0) : OutT(absolute<S, L>(fin[d], d));
}

// Checkpoint I/O of one direction d: the value a fluid cell gathers for d at
// the current parity, before any moving-wall correction (so that writing it
// back with k_slot_in restores the lattice exactly).  Walls: 0 / untouched.
template <class L, class S, bool FLAGS, int P = 0>
__device__ __forceinline__ typename S::T* slot_of(const LbmArgs& a, u32 n, const Nbr& o, unsigned walls, int d) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        if (d == i) {
            const bool sb = ((walls >> (2 * P)) & 1U) != 0U;
            return Slots<S, false>::at(a, !sb, P, n + nbr_off<L, j>(o));
        }
        if (d == j) {
            const bool sf = ((walls >> (2 * P + 1)) & 1U) != 0U;
            return Slots<S, false>::at(a, sf, P, n);
        }
        return slot_of<L, S, FLAGS, P + 1>(a, n, o, walls, d);
    } else {
        return Slots<S, false>::rest(a, n);
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(128) k_slot_out(const __grid_constant__ LbmArgs a, int d, float* out) {
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    unsigned walls = 0U;
    if constexpr (FLAGS) {
        const std::uint8_t flag = a.flags[n];
        if (flag & kFlagTypeMask) {
            out[n] = 0.0F;
            return;
        }
        if (flag & kFlagNearWall) walls = a.wall_mask[n];
    }
    const typename S::T* p = slot_of<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), walls, d);
    if constexpr (sizeof(typename S::T) == 2) {
        // FP16: deviation h / s_d plus the weight of direction d
        float w = d == 0 ? float(L::w(0)) : 0.0F;
        static_for_pairs<L>([&](auto PP) {
            constexpr int i = 2 * decltype(PP)::value + 1;
            if (d == i || d == i + 1) w = float(L::w(i));
        });
        out[n] = __half2float(*p) * a.inv_scale[d] + w;
    } else {
        out[n] = float(*p);
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(128) k_slot_in(const __grid_constant__ LbmArgs a, int d, const float* in) {
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    unsigned walls = 0U;
    if constexpr (FLAGS) {
        const std::uint8_t flag = a.flags[n];
        if (flag & kFlagTypeMask) return;
        if (flag & kFlagNearWall) walls = a.wall_mask[n];
    }
    typename S::T* p = slot_of<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), walls, d);
    if constexpr (sizeof(typename S::T) == 2) {
        float w = d == 0 ? float(L::w(0)) : 0.0F;
        static_for_pairs<L>([&](auto PP) {
            constexpr int i = 2 * decltype(PP)::value + 1;
            if (d == i || d == i + 1) w = float(L::w(i));
        });
        *p = __float2half_rn((in[n] - w) * a.scale[d]);
    } else {
        *p = typename S::T(in[n]);
    }
}

// Fluid-cell reduction with FP64 accumulation (reference
// esoteric_pull.hpp:211-255 accumulates per-cell FP32 sums in FP64; the
// reference's SYCL total_mass, esoteric_pull_sycl.hpp:327-339, used FP32).
// Each block writes its partial sums to scratch; k_reduce_final combines
// them in a fixed order, so results are bitwise reproducible for a given grid.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(0xffffffffU, v, s);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffU, v, s));
    return v;
}

constexpr int kReduceThreads = 256;

// Combines kReduceFields values over the block; thread 0 gets the result.
__device__ __forceinline__ void block_combine(double (&acc)[kReduceFields]) {
    __shared__ double sm[kReduceThreads / 32][kReduceFields];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kReduceFields; ++k) acc[k] = k == 5 ? warp_max(acc[k]) : warp_sum(acc[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) sm[warp][k] = acc[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) {
            const double v = lane < kReduceThreads / 32 ? sm[lane][k] : 0.0;
            acc[k] = k == 5 ? warp_max(v) : warp_sum(v);
        }
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(kReduceThreads) k_reduce(const __grid_constant__ LbmArgs a, double* partials) {
    using R = typename S::R;
    double acc[kReduceFields] = {0, 0, 0, 0, 0, 0, 0};
    const u32 rows = a.ny * a.nz;
    for (u32 row = blockIdx.x; row < rows; row += gridDim.x) {
        const u32 y = row % a.ny, z = row / a.ny;
        for (u32 x = threadIdx.x; x < a.nx; x += blockDim.x) {
            const u32 n = row * a.nx + x;
            std::uint8_t flag = 0;
            if constexpr (FLAGS) {
                flag = a.flags[n];
                if (flag & kFlagTypeMask) continue;
            }
            R fin[L::Q];
            gather<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), flag, fin);
            R rho, ux, uy, uz, ax, ay, az;
            moments<L, R, S::delta>(fin, rho, ux, uy, uz);
            cell_acceleration<R>(a, n, ax, ay, az);
            ux += R(0.5) * ax;
            uy += R(0.5) * ay;
            uz += R(0.5) * az;
            const double dr = double(rho), dx = double(ux), dy = double(uy), dz = double(uz);
            acc[0] += dr;
            acc[1] += dr * dx;
            acc[2] += dr * dy;
            acc[3] += dr * dz;
            acc[4] += dr * (dx * dx + dy * dy + dz * dz);
            const double speed = double(sqrt(ux * ux + uy * uy + uz * uz));
            acc[5] = fmax(acc[5], speed);
            if (!isfinite(dr) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz)) acc[6] += 1.0;
        }
    }
    block_combine(acc);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) partials[static_cast<std::size_t>(blockIdx.x) * kReduceFields + k] = acc[k];
}

static __global__ void __launch_bounds__(kReduceThreads) k_reduce_final(const double* partials, int blocks,
                                                                        double* out) {
    double acc[kReduceFields] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) {
            const double v = partials[static_cast<std::size_t>(b) * kReduceFields + k];
            acc[k] = k == 5 ? fmax(acc[k], v) : acc[k] + v;
        }
    block_combine(acc);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) out[k] = acc[k];
}

// Derives the internal flag byte (wall id, near-wall bits) from the caller's
// flags.  Near-wall bits let interior cells skip all neighbour-flag loads.
// With `ghost`, planes 0 and nz-1 are a z-slab's copies of its neighbours'
// edge planes: their flags still set the links of the cells next to them,
// but the cells themselves are marked as walls (id 1 unless a moving wall),
// so that no kernel steps, initialises, reduces or reports them.
template <class L>
__global__ void __launch_bounds__(128) k_prepare_flags(const __grid_constant__ LbmArgs a, const std::uint8_t* user,
                                                       std::uint8_t* out, std::uint32_t* mask, int ghost) {
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    const std::uint8_t t = user[n] & kFlagTypeMask;
    if (t != 0 || (ghost && (z == 0 || z == a.nz - 1U))) {
        out[n] = t != 0 ? t : std::uint8_t(1);
        mask[n] = 0U;
        return;
    }
    const Nbr o = make_nbr(a, x, y, z);
    std::uint8_t b = 0;
    std::uint32_t links = 0U;
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        const int i = 2 * p + 1, j = i + 1;
        // source of direction i is n + c_j, source of direction j is n + c_i
        const u32 mb = n + o.ox[L::cx(j) + 1] + o.oy[L::cy(j) + 1] + o.oz[L::cz(j) + 1];
        const u32 mf = n + o.ox[L::cx(i) + 1] + o.oy[L::cy(i) + 1] + o.oz[L::cz(i) + 1];
        const std::uint8_t ub = user[mb] & kFlagTypeMask, uf = user[mf] & kFlagTypeMask;
        if (ub != 0) links |= 1U << (2 * p);
        if (uf != 0) links |= 1U << (2 * p + 1);
        if (ub >= 2 || uf >= 2) b |= kFlagNearMoving;
    }
    if (links != 0U) b |= kFlagNearWall;
    out[n] = b;
    mask[n] = links;
}

} // namespace cfdx
