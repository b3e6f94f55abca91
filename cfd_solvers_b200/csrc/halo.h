// Halo messages of the z-slab decomposition of the in-place lattice.
//
// A slab of ze own planes is held with one ghost plane on each side (local
// planes 0 and ze+1 copy the neighbours' edge planes).  In the Esoteric-Pull
// step a cell touches, for each opposite pair p = (i, j = i+1), slot pa[p] of
// its neighbour n + c_j and slot pb[p] of itself (pa = i, pb = j at even
// parity, the reverse at odd), and every slot is touched by exactly one cell
// per step.  So across a cut at the upper side (c_j.z = +1 pairs leave
// upwards, c_j.z = -1 pairs downwards), after a step of parity t:
//   (i)  the edge cells wrote pa_t[p] of the ghost plane for the pairs that
//        leave through the cut: the neighbour's cells own those slots and
//        read them at step t+1 as pb_{t+1} = pa_t;
//   (ii) the edge plane's own slots pb_t[p] of the pairs that enter through
//        the cut are read at step t+1 by the neighbour's edge cells as
//        pa_{t+1} = pb_t, in the neighbour's ghost copy of this edge plane.
// Both are whole planes of one direction: contiguous runs of nx*ny elements
// in the [direction][z][y][x] layout.  The message through one side is (i)
// then (ii), pairs in ascending order; the receiver writes (i) into its edge
// plane (slot pa_t) and (ii) into its ghost plane (slot pb_t).  The count is
// the reference's crossing-population count per face cell
// (distributed/selective_halo.hpp:24-62): 5 for D3Q19, 9 for D3Q27.
//
// Slots a step never reads (those of walls) travel too; they are plane runs,
// and copying them keeps the message a few contiguous chunks.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "lattice.cuh"

namespace cfdx {

struct HaloEntry {
    std::uint32_t plane;
    std::uint32_t direction;
};

constexpr int kMaxHaloChunks = 9; // D3Q27: 9 pairs with a z component

// send[k] / recv[k] of the message through `side` (0 lower, 1 upper) after a
// step of parity `odd` on a slab of ze own planes; returns the chunk count.
template <class L>
int halo_plan(int odd, int side, std::uint32_t ze, HaloEntry* send, HaloEntry* recv) {
    const int out = side == 0 ? -1 : 1; // z component of the directions that leave through this side
    const std::uint32_t ghost = side == 0 ? 0U : ze + 1U;
    const std::uint32_t edge = side == 0 ? 1U : ze;
    int ks = 0, kr = 0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int p = 0; p < L::PAIRS; ++p) {
            const int i = 2 * p + 1, j = i + 1;
            const int cz = L::cz(j);
            if (cz == 0) continue;
            const std::uint32_t pa = static_cast<std::uint32_t>(odd ? j : i);
            const std::uint32_t pb = static_cast<std::uint32_t>(odd ? i : j);
            if (pass == 0) {
                if (cz == out) send[ks++] = HaloEntry{ghost, pa}; // (i) written into the ghost plane
                if (cz == -out) recv[kr++] = HaloEntry{edge, pa}; // neighbour's (i) lands in the edge plane
            } else {
                if (cz == -out) send[ks++] = HaloEntry{edge, pb}; // (ii) edge slots the neighbour reads next
                if (cz == out) recv[kr++] = HaloEntry{ghost, pb}; // neighbour's (ii) lands in the ghost plane
            }
        }
    }
    return ks; // == kr
}

inline int halo_plan(int q, int odd, int side, std::uint32_t ze, HaloEntry* send, HaloEntry* recv) {
    return q == 19 ? halo_plan<D3Q19>(odd, side, ze, send, recv) : halo_plan<D3Q27>(odd, side, ze, send, recv);
}

// One launch copies up to 2 * kMaxHaloChunks equal-sized chunks (a whole cut:
// both directions).
struct HaloCopy {
    const void* src[2 * kMaxHaloChunks];
    void* dst[2 * kMaxHaloChunks];
    int chunks;
};

cudaError_t launch_halo_copy(const HaloCopy& c, std::size_t chunk_bytes, cudaStream_t s);

} // namespace cfdx
