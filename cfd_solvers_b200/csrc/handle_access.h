// Internal access to a live handle for entry points implemented outside
// capi.cu.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cfdx_lbm.h"
#include "lbm_launch.h"

namespace cfdx {

// What a reduction over the handle's current state needs.
struct ReduceView {
    KernelKey key;
    LbmArgs args;
    cudaStream_t stream;
    int device;
};

// Makes the handle's device current and fills *view.  Returns a CFDX_* status
// and records the thread's last error on failure.
int handle_reduce_view(cfdx_lbm* h, ReduceView* view);

// Records the calling thread's last error (read by cfdx_last_error) and
// returns status.
int record_error(int status, const char* message);

// Counts device-to-host bytes and one synchronisation against the handle's
// transfer statistics.
void record_download(cfdx_lbm* h, std::uint64_t bytes);

} // namespace cfdx
