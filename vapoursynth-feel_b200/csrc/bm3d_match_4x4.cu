// Tiled matcher instantiated for 4x4-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

namespace vsfeel {

size_t tile_plan_bytes_4x4(const StackJob& job, TileMode mode) {
    return smem_plan<4, 4>(job, mode).bytes;
}

cudaError_t launch_tiles_4x4(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<4, 4>(job, mode, s);
}

cudaError_t launch_batch_4x4(const BatchWork& work, TileMode mode, size_t smem, int grid,
                                 cudaStream_t s) {
    return launch_batch<4, 4>(work, mode, smem, grid, s);
}

}  // namespace vsfeel
