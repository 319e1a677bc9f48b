// Tiled matcher instantiated for 8x2-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

#include <cstdint>

namespace vsfeel {

size_t tile_plan_bytes_8x2(const StackJob& job, TileMode mode) {
    // an unaligned layout never fits (launch_grid_mode refuses it too)
    const SmemPlan p = smem_plan<8, 2>(job, mode);
    return smem_plan_aligned<8, 2>(p) ? p.bytes : SIZE_MAX;
}

cudaError_t launch_tiles_8x2(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<8, 2>(job, mode, s);
}

cudaError_t launch_batch_8x2(const BatchWork& work, TileMode mode, int lanes, size_t smem,
                                 int grid, cudaStream_t s) {
    return launch_batch<8, 2>(work, mode, lanes, smem, grid, s);
}

int batch_ctas_per_sm_8x2(TileMode mode, int lanes, size_t smem) {
    return batch_ctas_per_sm<8, 2>(mode, lanes, smem);
}

}  // namespace vsfeel
