// Tiled matcher instantiated for 16x2-block tiles (kernels in bm3d_match.cuh).
#include "bm3d_match.cuh"

namespace vsfeel {

size_t tile_plan_bytes_16x2(const StackJob& job, TileMode mode) {
    return smem_plan<16, 2>(job, mode).bytes;
}

cudaError_t launch_tiles_16x2(const StackJob& job, TileMode mode, cudaStream_t s) {
    return launch_grid_mode<16, 2>(job, mode, s);
}

cudaError_t launch_batch_16x2(const BatchWork& work, TileMode mode, size_t smem, int grid,
                                 cudaStream_t s) {
    return launch_batch<16, 2>(work, mode, smem, grid, s);
}

}  // namespace vsfeel
