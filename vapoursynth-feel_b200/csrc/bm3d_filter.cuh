// Collaborative filtering of one group (src/bm3d.comp:358-399, 666-716),
// shared by the standalone filter kernel and the fused match-and-filter tile
// kernel.
//
// Lane `sub` of a group's 8 lanes holds column sub of the 8 matched patches:
// d[k*8 + j] = patch k, row j. The 3D transform runs in the reference's axis
// order (rows of each column, columns of each row, then along the group; the
// inverse in the same order), with 8x8 transposes through shared memory. All
// 32 lanes of the warp must take part (4 groups per warp).
#pragma once

#include "bm3d_device.cuh"

namespace vsfeel {

constexpr int kRowStride = 9;                      // floats per transposed row
constexpr int kTileStride = 8 * kRowStride;        // one 8x8 tile
constexpr int kGroupStride = 8 * kTileStride + 8;  // one group's 8 tiles (+8: bank skew)
constexpr int kFilterGroupsPerCta = 16;

// new d_l[k*8 + i] = old d_i[k*8 + l] within each group
__device__ __forceinline__ void transpose_group(float d[64], float* buf, int sub) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int i = 0; i < 8; ++i) buf[k * kTileStride + i * kRowStride + sub] = d[k * 8 + i];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int i = 0; i < 8; ++i) d[k * 8 + i] = buf[k * kTileStride + sub * kRowStride + i];
    __syncwarp();
}

__device__ __forceinline__ void transform_rows(float d[64], bool inverse) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (inverse)
            dct8_inv(&d[k * 8]);
        else
            dct8_fwd(&d[k * 8]);
    }
}

__device__ __forceinline__ void transform_group_axis(float d[64], bool inverse) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = d[k * 8 + i];
        if (inverse)
            dct8_inv(v);
        else
            dct8_fwd(v);
#pragma unroll
        for (int k = 0; k < 8; ++k) d[k * 8 + i] = v[k];
    }
}

// Filters block b's group (matches mxy = x | y << 16, zp = 8 x 4-bit slice)
// and scatters it into the stack's slices. kSaveMask also records the keep
// bits, lane `sub` writing word mask_out[b * 8 + sub] (bit 8 * group
// frequency + vertical frequency, of horizontal frequency sub). An invalid
// group (valid == false) computes but writes nothing. buf: kGroupStride
// floats of shared memory owned by the group.
template <bool kSaveMask>
__device__ __forceinline__ void filter_group(const StackJob& job, int b, bool valid,
                                             const uint32_t mxy[8], uint32_t zp, int sub,
                                             float* buf) {
    const int pitch = job.pitch;
    float d[64];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int z = (int)((zp >> (4 * k)) & 15u);
        const float* __restrict__ f = job.slice_frame[z];
        const int mx = (int)(mxy[k] & 0xffffu), my = (int)(mxy[k] >> 16);
        const float* p = f + (size_t)my * pitch + mx + sub;
#pragma unroll
        for (int j = 0; j < 8; ++j) d[k * 8 + j] = __ldg(p + (size_t)j * pitch);
    }

    transform_rows(d, false);
    transpose_group(d, buf, sub);
    transform_rows(d, false);
    transpose_group(d, buf, sub);
    transform_group_axis(d, false);

    const float thr = job.thr;
    int kept = 0;
    uint64_t bits = 0;
#pragma unroll
    for (int i = 0; i < 64; ++i) {
        const float t = (i == 0 && sub == 0) ? 0.0f : thr;
        const bool keep = fabsf(d[i]) >= t;
        kept += keep ? 1 : 0;
        if (kSaveMask) bits |= keep ? (uint64_t(1) << i) : uint64_t(0);
        d[i] = keep ? __fmul_rn(d[i], 1.0f / 4096.0f) : 0.0f;
    }
    if (kSaveMask && valid) job.mask_out[(size_t)b * 8 + sub] = bits;
    kept += __shfl_xor_sync(0xffffffffu, kept, 1);
    kept += __shfl_xor_sync(0xffffffffu, kept, 2);
    kept += __shfl_xor_sync(0xffffffffu, kept, 4);
    const float w = __fdiv_rn(1.0f, (float)kept);

    transform_rows(d, true);
    transpose_group(d, buf, sub);
    transform_rows(d, true);
    transpose_group(d, buf, sub);
    transform_group_axis(d, true);

    if (!valid) return;
    const float E = job.extractor;
    const float wv = __fsub_rn(__fadd_rn(w, E), E);
    const int dpitch = job.dst_pitch;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int z = (int)((zp >> (4 * k)) & 15u);
        float* num = job.slice_dst[z];
        if (num == nullptr) continue;
        const int mx = (int)(mxy[k] & 0xffffu), my = (int)(mxy[k] >> 16);
        float* pn = num + (size_t)my * dpitch + mx + sub;
        float* pd = pn + job.dst_plane;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            atomicAdd(pn + (size_t)j * dpitch, __fsub_rn(__fmaf_rn(w, d[k * 8 + j], E), E));
            atomicAdd(pd + (size_t)j * dpitch, wv);
        }
    }
}

}  // namespace vsfeel
