// Device-side building blocks of the BM3Dv2 basic estimate for sm_100a.
//
// Every floating-point operation whose bits decide a block match or a
// threshold is spelled with an explicit round-to-nearest intrinsic
// (__fadd_rn, __fmul_rn, __fmaf_rn, ...), so the results do not depend on
// nvcc's contraction flags and equal the reference's operation order:
//   8-point DCT pair ............ src/bm3d.comp:91-181
//   column SSD .................. src/bm3d.comp:266-275 (e += d*d fused)
//   8-column reduction tree ..... src/bm3d.comp:280-282
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vsfeel {

constexpr int kMaxRadius = 4;
constexpr int kMaxTW = 2 * kMaxRadius + 1;
constexpr float kFltMax = 3.402823466e+38f;
constexpr int kSeqSentinel = 0x7fffffff;

// One stack: the reference blocks of frame m, searched in the slices
// z = 0..2r (frame clamp(m - r + z)).
struct StackJob {
    const float* slice_frame[kMaxTW];  // frame of each slice in the search clip (the clip
                                       // denoised too, except in the final pass)
    const float* slice_input[kMaxTW];  // final pass: the same frames of the clip denoised
    float* slice_dst[kMaxTW];          // numerator plane of each slice's target; null = dropped
    int64_t dst_plane;                 // floats from a numerator plane to its weight-origin
                                       // plane (each patch's weight at its origin)
    int pitch;                         // floats per frame row (inputs)
    int dst_pitch;                     // floats per accumulator row
    int width, height;
    int radius, step, bm_range, ps_num, ps_range;
    int nbx, nby;                      // block grid
    float thr;                         // SIGMA_Y: sigma * 0x3f021bb6 (basic) or 0x3e40c0c1
    int wiener;                        // final pass: Wiener filter against slice_frame
    float extractor;                   // 2^exp or 0
    uint32_t* match_xy;                // [nblocks][8]: x | y << 16
    uint32_t* match_z;                 // [nblocks]: 8 x 4-bit slice index
    uint64_t* mask_out;                // [nblocks][8] keep bits of the filter, or null
    int* status;                       // device word, set nonzero on an internal error
    int lanes;                         // tiled sliding matcher: lanes per block, 8 (also 0)
                                       // or 16 (table mode only, 512-thread CTAs)
    int tile_shape_plus1;              // 1 + TileShape the table-mode matcher uses (when it
                                       // fits); 0: the default order
    int probe_tile;                    // test hook: 1 + index of a tile whose staged-region
                                       // check reports a window outside (the tile sets
                                       // *status and scans nothing); 0 = none
};

// Per-output normalisation: numerator plane read at aggregation step i.
// The planes' rows (src_pitch floats) are padded to a multiple of 32 floats
// and their bases 16-byte aligned: the kernel reads them four floats at a
// time. A pixel's weight is the sum of its 8x8 window of the weight-origin
// plane.
struct NormalizeJob {
    const float* num[kMaxTW];
    int64_t den_offset;  // floats from a numerator plane to its weight-origin plane
    int tw, width, height, src_pitch, out_pitch;
    float* out;
    float* den_out;  // summed weights (the frozen denominator), or null
    int den_pitch;
};

// Many normalisations in one launch: output j covers the items
// tile_first[j] .. tile_first[j+1]-1, one 120x8-pixel tile each.
struct NormalizeBatch {
    const NormalizeJob* jobs;
    const int* tile_first;
    int njobs;
};

// Adjoint of the frozen-match operator over a whole clip: one launch covers
// every block of every stack. The saved state is what the forward pass
// recorded per stack (match table and keep bits) plus the per-output
// denominators.
struct AdjointJob {
    const unsigned char* saved;  // stack m's record at saved + m * stack_bytes
    int64_t stack_bytes, off_xy, off_z, off_mask;
    const float* gs;             // scaled output gradient dL/d(output) / D of frame f
                                 // in slot f % gs_slots, slots gs_frame floats apart
    int64_t gs_frame;
    int gs_pitch, gs_slots;
    float* grad_in;              // dL/d(input), accumulated (zero-filled by the caller)
    int64_t gi_frame;
    int gi_pitch;
    int nframes, radius, nblocks;
    int first_stack, stack_count;  // this launch: stacks first_stack .. +stack_count-1
    int width, height;           // match positions are clamped to the frame
};

// One output frame's scaled gradient for the adjoint: gs = g / D per pixel
// (the frozen denominator D of the forward's normalisation).
struct GradScaleJob {
    const float* go;   // dL/d(output) of the frame, go_pitch floats per row
    const float* den;  // its frozen denominator, den_pitch floats per row
    float* gs;         // out, gs_pitch floats per row
    int go_pitch, den_pitch, gs_pitch, width, height;
};

// Tiled matcher (bm3d_match.cu): tile shapes in blocks, and what a tile
// does after matching.
enum TileShape { kTile8x4 = 0, kTile16x2, kTile4x8, kTile8x2, kTile4x4, kTileShapes };
enum TileMode { kTableOnly = 0, kFused = 1, kFusedSave = 2 };

// The persistent form's work queue: tiles of jobs[0..njobs), job j owning
// items tile_first[j] .. tile_first[j+1]-1; counter is zeroed before a launch.
struct BatchWork {
    const StackJob* jobs;
    const int* tile_first;
    int njobs;
    int* counter;
};

// Host-side launchers (defined beside the kernels). Each returns the launch
// status and enqueues on `stream`.
cudaError_t launch_match(const StackJob& job, cudaStream_t stream);
cudaError_t launch_filter(const StackJob& job, cudaStream_t stream);
// The filter in CTAs of 8 groups, small enough to share an SM with a
// matcher CTA: the engine runs it beside the next stack's matching.
cudaError_t launch_filter_beside_match(const StackJob& job, cudaStream_t stream);
const char* tile_shape_name(TileShape shape);
bool tile_shape_fits(const StackJob& job, TileShape shape, TileMode mode);
int default_tile_shape(const StackJob& job, TileMode mode);  // -1: none fits
size_t tile_smem_bytes(const StackJob& job, TileShape shape, TileMode mode);
int tile_count(const StackJob& job, TileShape shape);
cudaError_t launch_match_tiles(const StackJob& job, TileShape shape, TileMode mode,
                               cudaStream_t stream);
// CTAs of the persistent kernel one SM holds at once (its grid: this many per SM)
int batch_ctas_per_sm(TileShape shape, TileMode mode, int lanes, size_t smem);
// mode: kTableOnly or kFused; lanes: 8, or 16 with kTableOnly
cudaError_t launch_batch_tiles(const BatchWork& work, TileShape shape, TileMode mode, int lanes,
                               size_t smem, int grid, cudaStream_t stream);

// Many stacks' filters in one launch: job j covers the items
// group_first[j] .. group_first[j+1]-1, 16 groups (blocks) each, with its
// matches in its own match table.
struct FilterBatch {
    const StackJob* jobs;
    const int* group_first;
    int njobs;
};
// groups: blocks per item (and CTA): 16, or 8 for CTAs small enough to run
// beside a matcher CTA
cudaError_t launch_filter_batch(const FilterBatch& work, int total_items, int groups,
                                cudaStream_t stream);
inline int filter_items(int nblocks, int groups = 16) { return (nblocks + groups - 1) / groups; }
cudaError_t launch_normalize(const NormalizeJob& job, cudaStream_t stream);
cudaError_t launch_adjoint(const AdjointJob& job, cudaStream_t stream);
cudaError_t launch_grad_scale(const GradScaleJob& job, cudaStream_t stream);
cudaError_t launch_normalize_batch(const NormalizeBatch& work, int total_tiles, cudaStream_t stream);
// The normaliser's tile: 2 rows (one warp each) of 120 pixels (30 lanes of
// 4 pixels, the warp's other 2 lanes reading the 8-column halo on the left).
// Its 64-thread CTAs are small enough (80 registers a thread) to sit on an SM
// beside a matcher CTA and a filter CTA, so that normalisations overlap the
// next stack's matching instead of waiting for the matcher grid's tail.
constexpr int kNormTileW = 120, kNormTileH = 2;
inline int normalize_tiles(int width, int height) {
    return ((width + kNormTileW - 1) / kNormTileW) * ((height + kNormTileH - 1) / kNormTileH);
}

// The kernels' status word: bit 0, a search window left its staged region
// (the window was not scanned); bit 1, a block's selection did not settle
// within its pass limit (its error table was not valid).
inline const char* status_text(int word) {
    if ((word & 3) == 3)
        return "internal error: a search window left the staged region; a block selection did "
               "not converge";
    if (word & 1) return "internal error: a search window left the staged region";
    if (word & 2) return "internal error: a block selection did not converge";
    return "internal error: unknown kernel status";
}

// Float add into global memory without a returned value (red.global):
// the accumulator planes' pointers reach the batched and persistent kernels
// through job arrays in memory, where the compiler cannot tell them from
// shared or local addresses and would emit a generic atomic that waits for
// its result (41% slower filtering at 1080p radius 0 than the reduction).
__device__ __forceinline__ void red_add_global(float* p, float v) {
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "f"(v)
                 : "memory");
}

__host__ __device__ inline int block_count(int extent, int step) {
    return (extent - 9 + 2 * step) / step;  // positions x0 = b*step < extent - 8 + step
}

__host__ __device__ inline int clamp_frame(int f, int nframes) {
    return f < 0 ? 0 : (f > nframes - 1 ? nframes - 1 : f);
}

// Aggregation slice that output n reads from stack clamp(n - r + i)
// (src/bm3d.cpp:369-371).
__host__ __device__ inline int agg_slice(int i, int n, int nframes, int radius) {
    if (radius == 0) return 0;
    const int a = 2 * radius - i, b = n - nframes + 1 + radius;
    const int lo = a > b ? a : b;
    return lo < n + radius ? lo : n + radius;
}

// How many times output n = clamp(m - r + z) sums slice z of stack m: the
// number of steps i with (clamp(n - r + i), agg_slice(i, n)) == (m, z). It
// is 0 for slices no output reads and above 1 only near the clip ends.
__host__ __device__ inline int slice_reads(int m, int z, int nframes, int radius) {
    const int n = clamp_frame(m - radius + z, nframes);
    int count = 0;
    for (int i = 0; i <= 2 * radius; ++i)
        if (clamp_frame(n - radius + i, nframes) == m && agg_slice(i, n, nframes, radius) == z)
            ++count;
    return count;
}

// ---------------------------------------------------------------------------
// 8-point DCT-II scaled x4 per axis, and its transpose. The statement order
// and the fused operations are those of the reference codelet.
__device__ __forceinline__ void dct8_fwd(float v[8]) {
    const float c414 = 0.414213562373095048801688724209698078569671875;
    const float c1847 = 1.847759065022573512256366378793576573644833252;
    const float c198 = 0.198912367379658006911597622644676228597850501;
    const float c1961 = 1.961570560806460898252364472268478073947867462;
    const float c1414 = 1.414213562373095048801688724209698078569671875;
    const float c668 = 0.668178637919298919997757686523080761552472251;
    const float c1662 = 1.662939224605090474157576755235811513477121624;
    const float c707 = 0.707106781186547524400844362104849039284835938;

    const float d07 = __fsub_rn(v[0], v[7]), s07 = __fadd_rn(v[0], v[7]);
    const float d43 = __fsub_rn(v[4], v[3]), s43 = __fadd_rn(v[4], v[3]);
    const float d25 = __fsub_rn(v[2], v[5]);
    const float d16 = __fsub_rn(v[1], v[6]);
    const float a = __fadd_rn(d25, d16);
    const float s16 = __fadd_rn(v[1], v[6]);
    const float b = __fsub_rn(d25, d16);
    const float s25 = __fadd_rn(v[2], v[5]);
    const float p = __fmaf_rn(-c707, a, d07);
    const float q = __fmaf_rn(-c707, b, d43);
    v[3] = __fmul_rn(c1662, __fmaf_rn(c668, q, p));
    v[5] = -__fmul_rn(c1662, __fmaf_rn(-c668, p, q));
    const float e0 = __fadd_rn(s07, s43), e1 = __fadd_rn(s25, s16);
    v[4] = __fmul_rn(c1414, __fsub_rn(e0, e1));
    v[0] = __fmul_rn(c1414, __fadd_rn(e0, e1));
    const float h = __fmaf_rn(c707, a, d07);
    const float i = __fmaf_rn(c707, b, d43);
    v[1] = __fmul_rn(c1961, __fmaf_rn(-c198, i, h));
    v[7] = __fmul_rn(c1961, __fmaf_rn(c198, h, i));
    const float l = __fsub_rn(s07, s43), o = __fsub_rn(s25, s16);
    v[2] = __fmul_rn(c1847, __fmaf_rn(-c414, o, l));
    v[6] = __fmul_rn(c1847, __fmaf_rn(c414, l, o));
}

__device__ __forceinline__ void dct8_inv(float v[8]) {
    const float c1662 = 1.662939224605090474157576755235811513477121624;
    const float c668 = 0.668178637919298919997757686523080761552472251;
    const float c1961 = 1.961570560806460898252364472268478073947867462;
    const float c198 = 0.198912367379658006911597622644676228597850501;
    const float c1847 = 1.847759065022573512256366378793576573644833252;
    const float c707 = 0.707106781186547524400844362104849039284835938;
    const float c414 = 0.414213562373095048801688724209698078569671875;
    const float c1414 = 1.414213562373095048801688724209698078569671875;

    const float dc = __fmul_rn(v[0], c1414);
    const float a = __fmaf_rn(c1414, v[4], dc);
    const float b = __fmaf_rn(-c1414, v[4], dc);
    const float c = __fmaf_rn(c414, v[6], v[2]);
    const float d = __fmaf_rn(c414, v[2], -v[6]);
    const float s53 = __fadd_rn(v[5], v[3]);
    const float d35 = __fsub_rn(v[3], v[5]);
    const float e = __fmaf_rn(c707, s53, v[1]);
    const float f = __fmaf_rn(-c707, d35, v[7]);
    const float g = __fmaf_rn(c707, d35, v[7]);
    const float h = __fmaf_rn(-c707, s53, v[1]);
    const float t0 = __fmaf_rn(c1847, c, a);
    const float t1 = __fmaf_rn(c198, g, e);
    const float t2 = __fmaf_rn(-c1847, d, b);
    const float t3 = __fmaf_rn(c668, h, f);
    const float t4 = __fmaf_rn(-c1847, c, a);
    const float t5 = __fmaf_rn(-c198, e, g);
    const float t6 = __fmaf_rn(c1847, d, b);
    const float t7 = __fmaf_rn(-c668, f, h);
    v[0] = __fmaf_rn(c1961, t1, t0);
    v[7] = __fmaf_rn(-c1961, t1, t0);
    v[2] = __fmaf_rn(c1662, t3, t2);
    v[5] = __fmaf_rn(-c1662, t3, t2);
    v[3] = __fmaf_rn(-c1961, t5, t4);
    v[4] = __fmaf_rn(c1961, t5, t4);
    v[6] = __fmaf_rn(-c1662, t7, t6);
    v[1] = __fmaf_rn(c1662, t7, t6);
}

// ---------------------------------------------------------------------------
// SSD of one 8-row column: block column `c` (8 values) against the source
// column at (cy .. cy+7, X). Even and odd rows accumulate separately.
__device__ __forceinline__ float column_ssd(const float cc[8], const float* __restrict__ col,
                                            int pitch) {
    float ev = 0.0f, od = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        const float d0 = __fsub_rn(cc[i], __ldg(col + (size_t)i * pitch));
        ev = __fmaf_rn(d0, d0, ev);
        const float d1 = __fsub_rn(cc[i + 1], __ldg(col + (size_t)(i + 1) * pitch));
        od = __fmaf_rn(d1, d1, od);
    }
    return __fadd_rn(ev, od);
}

__device__ __forceinline__ float tree8(const float col[8]) {
    return __fadd_rn(__fadd_rn(__fadd_rn(col[0], col[1]), __fadd_rn(col[2], col[3])),
                     __fadd_rn(__fadd_rn(col[4], col[5]), __fadd_rn(col[6], col[7])));
}

}  // namespace vsfeel
