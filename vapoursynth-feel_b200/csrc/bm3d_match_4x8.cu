// Tiled matcher instantiated for 4x8-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

namespace vsfeel {

size_t tile_plan_bytes_4x8(const StackJob& job, TileMode mode) {
    return smem_plan<4, 8>(job, mode).bytes;
}

cudaError_t launch_tiles_4x8(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<4, 8>(job, mode, s);
}

cudaError_t launch_batch_4x8(const BatchWork& work, TileMode mode, size_t smem, int grid,
                                 cudaStream_t s) {
    return launch_batch<4, 8>(work, mode, smem, grid, s);
}

}  // namespace vsfeel
