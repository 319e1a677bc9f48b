// Tiled matcher instantiated for 8x2-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

namespace vsfeel {

size_t tile_plan_bytes_8x2(const StackJob& job, TileMode mode) {
    return smem_plan<8, 2>(job, mode).bytes;
}

cudaError_t launch_tiles_8x2(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<8, 2>(job, mode, s);
}

cudaError_t launch_batch_8x2(const BatchWork& work, TileMode mode, size_t smem, int grid,
                                 cudaStream_t s) {
    return launch_batch<8, 2>(work, mode, smem, grid, s);
}

}  // namespace vsfeel
