// Tiled matcher instantiated for 4x4-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

#include <cstdint>

namespace vsfeel {

size_t tile_plan_bytes_4x4(const StackJob& job, TileMode mode) {
    // an unaligned layout never fits (launch_grid_mode refuses it too)
    const SmemPlan p = smem_plan<4, 4>(job, mode);
    return smem_plan_aligned<4, 4>(p) ? p.bytes : SIZE_MAX;
}

cudaError_t launch_tiles_4x4(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<4, 4>(job, mode, s);
}

cudaError_t launch_batch_4x4(const BatchWork& work, TileMode mode, int lanes, size_t smem,
                                 int grid, cudaStream_t s) {
    return launch_batch<4, 4>(work, mode, lanes, smem, grid, s);
}

int batch_ctas_per_sm_4x4(TileMode mode, int lanes, size_t smem) {
    return batch_ctas_per_sm<4, 4>(mode, lanes, smem);
}

}  // namespace vsfeel
