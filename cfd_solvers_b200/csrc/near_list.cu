// The cells the two-cell FP16 step leaves to k_step_list (lbm_step_h2.cuh):
// the fluid cells of every x-pair (2k, 2k+1) that holds a wall or a cell next
// to a wall or a moving wall.  Selected once per flag field, in cell order.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "lbm_args.h"
#include "lbm_launch.h"

namespace cfdx {
namespace {

struct NotInteriorPair {
    const std::uint8_t* flags;
    __device__ bool operator()(std::uint32_t n) const {
        const std::uint8_t f = flags[n];
        if (f & kFlagTypeMask) return false; // walls are not stepped
        const std::uint8_t g = flags[n ^ 1U]; // the other cell of the pair (nx even: pairs never straddle rows)
        return ((f | g) & (kFlagTypeMask | kFlagNearWall | kFlagNearMoving)) != 0;
    }
};

} // namespace

cudaError_t select_near_cells(const std::uint8_t* flags, std::uint32_t cells, std::uint32_t* out,
                              std::uint32_t* count, void* temp, std::size_t* temp_bytes, cudaStream_t s) {
    return cub::DeviceSelect::If(temp, *temp_bytes, thrust::counting_iterator<std::uint32_t>(0), out, count,
                                 static_cast<int>(cells), NotInteriorPair{flags}, s);
}

} // namespace cfdx
