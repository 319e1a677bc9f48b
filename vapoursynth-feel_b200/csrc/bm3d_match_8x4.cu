// Tiled matcher instantiated for 8x4-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

#include <cstdint>

namespace vsfeel {

size_t tile_plan_bytes_8x4(const StackJob& job, TileMode mode) {
    // an unaligned layout never fits (launch_grid_mode refuses it too)
    const SmemPlan p = smem_plan<8, 4>(job, mode);
    return smem_plan_aligned<8, 4>(p) ? p.bytes : SIZE_MAX;
}

cudaError_t launch_tiles_8x4(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<8, 4>(job, mode, s);
}

cudaError_t launch_batch_8x4(const BatchWork& work, TileMode mode, int lanes, size_t smem,
                                 int grid, cudaStream_t s) {
    return launch_batch<8, 4>(work, mode, lanes, smem, grid, s);
}

int batch_ctas_per_sm_8x4(TileMode mode, int lanes, size_t smem) {
    return batch_ctas_per_sm<8, 4>(mode, lanes, smem);
}

}  // namespace vsfeel
