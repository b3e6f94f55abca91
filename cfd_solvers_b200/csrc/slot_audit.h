// Slot-ownership audit of the in-place step (slot_audit.cu): a test hook that
// replaces a race detector.  The one-cell step kernel runs with a storage type
// whose loads and stores only record who touched each slot (StAudit in
// lbm_device.cuh); a second kernel classifies every slot.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "lbm_args.h"
#include "lbm_launch.h"

namespace cfdx {

// Per-slot classes, counted over the q * cells slots of one step.
struct AuditCounts {
    unsigned long long touched;       // read or written
    unsigned long long read_twice;    // read more than once
    unsigned long long written_twice; // written more than once (two writers race)
    unsigned long long read_only;     // read, never written
    unsigned long long write_only;    // written, never read
    unsigned long long foreign;       // written by a thread that did not read it
    unsigned long long out_of_range;  // accesses outside the q * cells slots (not performed)
};

// The class bits of one slot from its five counters (host and device).
enum : unsigned {
    kAuditTouched = 1U,
    kAuditReadTwice = 2U,
    kAuditWrittenTwice = 4U,
    kAuditReadOnly = 8U,
    kAuditWriteOnly = 16U,
    kAuditForeign = 32U,
};
__host__ __device__ inline unsigned audit_classify(std::uint32_t reads, std::uint32_t writes, std::uint32_t rmin,
                                                   std::uint32_t rmax, std::uint32_t writer) {
    unsigned c = 0U;
    if (reads == 0U && writes == 0U) return c;
    c |= kAuditTouched;
    if (reads > 1U) c |= kAuditReadTwice;
    if (writes > 1U) c |= kAuditWrittenTwice;
    if (writes == 0U) c |= kAuditReadOnly;
    if (reads == 0U) c |= kAuditWriteOnly;
    if (reads > 0U && writes > 0U && (rmin != rmax || writer != rmin)) c |= kAuditForeign;
    return c;
}

// counters: 5 * q * cells + 1 words (reads | writes | lowest reader | highest
// reader | writer | out-of-range count), initialised here; `a` is the step's argument block with
// base / rest_off / pa_off / pb_off addressing the reads array (NARROW form).
cudaError_t launch_slot_audit(const KernelKey& k, const LbmArgs& a, std::uint32_t* counters, dim3 grid, dim3 block,
                              AuditCounts* device_counts, cudaStream_t s);

} // namespace cfdx
