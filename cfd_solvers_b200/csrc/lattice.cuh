// Velocity sets of the in-place Esoteric-Pull path.
//
// The direction order is the reference's (include/cfd/solvers/lbm/descriptors.hpp:59-146):
// direction 0 is rest, pairs (2p+1, 2p+2) are opposite.  The order is an
// interface, not an implementation detail: logical populations, checkpoints
// and the parity tests index directions the same way the reference does.
#pragma once

#include <cstdint>

namespace cfdx {

struct D3Q19 {
    static constexpr int Q = 19;
    static constexpr int PAIRS = 9;
    __host__ __device__ static constexpr int cx(int d) {
        constexpr int v[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        return v[d];
    }
    __host__ __device__ static constexpr int cy(int d) {
        constexpr int v[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
        return v[d];
    }
    __host__ __device__ static constexpr int cz(int d) {
        constexpr int v[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
        return v[d];
    }
    __host__ __device__ static constexpr double w(int d) {
        return d == 0 ? 1.0 / 3.0 : (d <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
};

struct D3Q27 {
    static constexpr int Q = 27;
    static constexpr int PAIRS = 13;
    __host__ __device__ static constexpr int cx(int d) {
        constexpr int v[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
        return v[d];
    }
    __host__ __device__ static constexpr int cy(int d) {
        constexpr int v[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
        return v[d];
    }
    __host__ __device__ static constexpr int cz(int d) {
        constexpr int v[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};
        return v[d];
    }
    __host__ __device__ static constexpr double w(int d) {
        return d == 0 ? 8.0 / 27.0 : (d <= 6 ? 2.0 / 27.0 : (d <= 18 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
};

// Weight class of direction d: 0 rest, 1 axis, 2 face diagonal, 3 corner
// (|c_x| + |c_y| + |c_z|); the weights, and the FP16 storage scales, are
// constant within a class.
template <class L> __host__ __device__ constexpr int weight_class(int d) {
    return (L::cx(d) != 0 ? 1 : 0) + (L::cy(d) != 0 ? 1 : 0) + (L::cz(d) != 0 ? 1 : 0);
}

// A representative direction of each weight class.
__host__ __device__ constexpr int class_rep(int k) { return k == 0 ? 0 : (k == 1 ? 1 : (k == 2 ? 7 : 19)); }

} // namespace cfdx
