// Slot-ownership audit of the in-place step.  The race-freedom of in-place
// (Esoteric-Pull) streaming rests on one invariant: in a step every slot is
// loaded and then stored by one cell, its owner.  This file runs the one-cell
// step kernel k_step -- its real gather / scatter addressing, wall links,
// moving-wall and slab ghost handling -- with a storage type that records,
// per slot, how many loads and stores it saw and which threads made them,
// then classifies every slot.  A race-free step stores every slot at most once
// and only from the thread that loads it.  A fluid cell touches q slots, plus
// one per link into a wall cell: that link loads one of the wall cell's two
// slots of the pair and stores the other (they swap roles the next step).
#include "slot_audit.h"

#include "lbm_device.cuh"

namespace cfdx {
namespace {

__global__ void k_audit_reset(std::uint32_t* c, std::uint32_t slots) {
    if (blockIdx.x == 0 && threadIdx.x == 0) c[5U * slots] = 0U;
    for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
        c[i] = 0U;
        c[slots + i] = 0U;
        c[2U * slots + i] = 0xFFFFFFFFU;
        c[3U * slots + i] = 0U;
        c[4U * slots + i] = 0U;
    }
}

__global__ void k_audit_classify(const std::uint32_t* c, std::uint32_t slots, AuditCounts* out) {
    unsigned long long n[6] = {0, 0, 0, 0, 0, 0};
    for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
        const unsigned k = audit_classify(c[i], c[slots + i], c[2U * slots + i], c[3U * slots + i], c[4U * slots + i]);
        for (int b = 0; b < 6; ++b) n[b] += (k >> b) & 1U;
    }
    unsigned long long* o = &out->touched;
    for (int b = 0; b < 6; ++b)
        if (n[b]) atomicAdd(o + b, n[b]);
    if (blockIdx.x == 0 && threadIdx.x == 0) out->out_of_range = c[5U * slots];
}

template <class L, bool SCALED>
cudaError_t audit_step(bool flags, const LbmArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    // The collision (LES, gray) does not change which slots a cell touches.
    if (flags)
        k_step<L, StAudit<SCALED>, false, true, false, 1, true><<<g, b, 0, s>>>(a);
    else
        k_step<L, StAudit<SCALED>, false, false, false, 1, true><<<g, b, 0, s>>>(a);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_slot_audit(const KernelKey& k, const LbmArgs& a, std::uint32_t* counters, dim3 grid, dim3 block,
                              AuditCounts* device_counts, cudaStream_t s) {
    const std::uint32_t slots = static_cast<std::uint32_t>(k.q) * a.N;
    k_audit_reset<<<592, 256, 0, s>>>(counters, slots);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(device_counts, 0, sizeof(AuditCounts), s);
    if (e != cudaSuccess) return e;
    const bool scaled = k.storage == kStoreF16S;
    if (k.q == 19)
        e = scaled ? audit_step<D3Q19, true>(k.flags, a, grid, block, s) : audit_step<D3Q19, false>(k.flags, a, grid, block, s);
    else if (k.q == 27)
        e = scaled ? audit_step<D3Q27, true>(k.flags, a, grid, block, s) : audit_step<D3Q27, false>(k.flags, a, grid, block, s);
    else
        e = cudaErrorInvalidValue;
    if (e != cudaSuccess) return e;
    k_audit_classify<<<592, 256, 0, s>>>(counters, slots, device_counts);
    return cudaGetLastError();
}

} // namespace cfdx
