// Host side of the tiled matcher: tile shapes, shared-memory fitting and
// the dispatch to the per-shape instantiations (bm3d_match_<shape>.cu; the
// kernels themselves are in bm3d_match.cuh).
#include "bm3d_device.cuh"

#include <algorithm>

namespace vsfeel {

#define VSFEEL_TILE_DECL(TX, TY)                                                              \
    size_t tile_plan_bytes_##TX##x##TY(const StackJob& job, TileMode mode);                   \
    cudaError_t launch_tiles_##TX##x##TY(const StackJob& job, TileMode mode, cudaStream_t s); \
    cudaError_t launch_batch_##TX##x##TY(const BatchWork& work, TileMode mode, int lanes,     \
                                         size_t smem, int grid, cudaStream_t s);            \
    int batch_ctas_per_sm_##TX##x##TY(TileMode mode, int lanes, size_t smem);
VSFEEL_TILE_DECL(8, 4)
VSFEEL_TILE_DECL(16, 2)
VSFEEL_TILE_DECL(4, 8)
VSFEEL_TILE_DECL(8, 2)
VSFEEL_TILE_DECL(4, 4)
#undef VSFEEL_TILE_DECL

namespace {

struct ShapeInfo {
    int tx, ty;
};
constexpr ShapeInfo kShapes[kTileShapes] = {{8, 4}, {16, 2}, {4, 8}, {8, 2}, {4, 4}};
constexpr size_t kSmemBudget = 220 * 1024;

size_t plan_bytes(const StackJob& job, TileShape shape, TileMode mode) {
    switch (shape) {
        case kTile8x4: return tile_plan_bytes_8x4(job, mode);
        case kTile16x2: return tile_plan_bytes_16x2(job, mode);
        case kTile4x8: return tile_plan_bytes_4x8(job, mode);
        case kTile8x2: return tile_plan_bytes_8x2(job, mode);
        default: return tile_plan_bytes_4x4(job, mode);
    }
}

}  // namespace

const char* tile_shape_name(TileShape shape) {
    static const char* names[kTileShapes] = {"8x4", "16x2", "4x8", "8x2", "4x4"};
    return (shape >= 0 && shape < kTileShapes) ? names[shape] : "?";
}

size_t tile_smem_bytes(const StackJob& job, TileShape shape, TileMode mode) {
    return plan_bytes(job, shape, mode);
}

int tile_count(const StackJob& job, TileShape shape) {
    const ShapeInfo si = kShapes[shape];
    return ((job.nbx + si.tx - 1) / si.tx) * ((job.nby + si.ty - 1) / si.ty);
}

// True when the tiled kernel handles this configuration with this shape:
// the sliding scan (radius < 3) in any mode or the exact scan (radius >= 3)
// writing the match table, its shared memory fits, and every temporal
// window is centred on a real match. (A corner block's spatial window holds
// (min(R, W-8)+1) * (min(R, H-8)+1) candidates; with fewer than ps_num of
// them the reference seeds a temporal window at (0, 0), which can lie
// outside the tile's staged region.) Otherwise the caller uses the
// direct-read kernel.
bool tile_shape_fits(const StackJob& job, TileShape shape, TileMode mode) {
    if (job.radius >= 3 && mode != kTableOnly) return false;  // exact scan: table mode only
    if (plan_bytes(job, shape, mode) > kSmemBudget) return false;
    // scan indices must stay below 2^21 (the kernels' div_small); the
    // shared-memory plan already keeps them far below
    const int64_t ws = 2 * (int64_t)job.bm_range + 1, wt = 2 * (int64_t)job.ps_range + 1;
    if (ws * ws >= (int64_t(1) << 21) || job.ps_num * wt * wt >= (int64_t(1) << 21)) return false;
    if (job.radius > 0) {
        const int cw = std::min(job.bm_range, job.width - 8) + 1;
        const int ch = std::min(job.bm_range, job.height - 8) + 1;
        if (cw * ch < job.ps_num) return false;
    }
    return true;
}

// The default shape of the plain path: the first that fits, largest tiles
// first.
int default_tile_shape(const StackJob& job, TileMode mode) {
    const TileShape order[] = {kTile8x4, kTile16x2, kTile8x2, kTile4x4};
    for (TileShape s : order)
        if (tile_shape_fits(job, s, mode)) return s;
    return -1;
}

cudaError_t launch_match_tiles(const StackJob& job, TileShape shape, TileMode mode,
                               cudaStream_t stream) {
    switch (shape) {
        case kTile8x4: return launch_tiles_8x4(job, mode, stream);
        case kTile16x2: return launch_tiles_16x2(job, mode, stream);
        case kTile4x8: return launch_tiles_4x8(job, mode, stream);
        case kTile8x2: return launch_tiles_8x2(job, mode, stream);
        default: return launch_tiles_4x4(job, mode, stream);
    }
}

int batch_ctas_per_sm(TileShape shape, TileMode mode, int lanes, size_t smem) {
    switch (shape) {
        case kTile8x4: return batch_ctas_per_sm_8x4(mode, lanes, smem);
        case kTile16x2: return batch_ctas_per_sm_16x2(mode, lanes, smem);
        case kTile4x8: return batch_ctas_per_sm_4x8(mode, lanes, smem);
        case kTile8x2: return batch_ctas_per_sm_8x2(mode, lanes, smem);
        default: return batch_ctas_per_sm_4x4(mode, lanes, smem);
    }
}

cudaError_t launch_batch_tiles(const BatchWork& work, TileShape shape, TileMode mode, int lanes,
                               size_t smem, int grid, cudaStream_t stream) {
    if (lanes != 8 && (lanes != 16 || mode != kTableOnly)) return cudaErrorInvalidValue;
    switch (shape) {
        case kTile8x4: return launch_batch_8x4(work, mode, lanes, smem, grid, stream);
        case kTile16x2: return launch_batch_16x2(work, mode, lanes, smem, grid, stream);
        case kTile4x8: return launch_batch_4x8(work, mode, lanes, smem, grid, stream);
        case kTile8x2: return launch_batch_8x2(work, mode, lanes, smem, grid, stream);
        default: return launch_batch_4x4(work, mode, lanes, smem, grid, stream);
    }
}

}  // namespace vsfeel
