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

// The 3D transform of a group held as d[k*8 + j] (patch k, row j; lane = column).
__device__ __forceinline__ void forward3(float d[64], float* buf, int sub) {
    transform_rows(d, false);
    transpose_group(d, buf, sub);
    transform_rows(d, false);
    transpose_group(d, buf, sub);
    transform_group_axis(d, false);
}

__device__ __forceinline__ void inverse3(float d[64], float* buf, int sub) {
    transform_rows(d, true);
    transpose_group(d, buf, sub);
    transform_rows(d, true);
    transpose_group(d, buf, sub);
    transform_group_axis(d, true);
}

__device__ __forceinline__ void gather_group(float d[64], const float* const frames[kMaxTW],
                                             int pitch, const uint32_t mxy[8], uint32_t zp,
                                             int sub) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int z = (int)((zp >> (4 * k)) & 15u);
        const int mx = (int)(mxy[k] & 0xffffu), my = (int)(mxy[k] >> 16);
        const float* p = frames[z] + (size_t)my * pitch + mx + sub;
#pragma unroll
        for (int j = 0; j < 8; ++j) d[k * 8 + j] = __ldg(p + (size_t)j * pitch);
    }
}

// Collaborative Wiener filtering of the final pass (src/bm3d.comp:401-443):
// d holds the transformed group of the clip denoised, r the transformed group
// of the basic estimate at the same positions. Per coefficient
// c = rr / (rr + SS) with rr = r*r and SS = SIGMA_Y*SIGMA_Y rounded products
// and an unfused sum (a shader compiler folds the specialisation constant's
// square), c = 1 at DC; d becomes d*c/4096. The squared coefficients are
// summed as the reference does: per lane four partial sums by index mod 4
// (ks += c*c fused), (ks0 + ks1) + (ks2 + ks3), then the pairwise tree over
// the group's lanes in lane order. Returns the weight 1 / sum.
__device__ __forceinline__ float wiener_coefficients(float d[64], const float r[64], float sy,
                                                     int sub) {
    const float ss = __fmul_rn(sy, sy);
    float ks[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 64; ++i) {
        const float rr = __fmul_rn(r[i], r[i]);
        float c = __fdiv_rn(rr, __fadd_rn(rr, ss));
        if (i == 0 && sub == 0) c = 1.0f;
        const float val = __fmul_rn(d[i], c);
        ks[i % 4] = __fmaf_rn(c, c, ks[i % 4]);
        d[i] = __fmul_rn(val, 1.0f / 4096.0f);
    }
    const float mine = __fadd_rn(__fadd_rn(ks[0], ks[1]), __fadd_rn(ks[2], ks[3]));
    const int base = (threadIdx.x & 31) & ~7;
    float k[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) k[l] = __shfl_sync(0xffffffffu, mine, base + l);
    const float sum = __fadd_rn(__fadd_rn(__fadd_rn(k[0], k[1]), __fadd_rn(k[2], k[3])),
                                __fadd_rn(__fadd_rn(k[4], k[5]), __fadd_rn(k[6], k[7])));
    return __fdiv_rn(1.0f, sum);
}

// Aggregation (src/bm3d.comp:697-715). The reference adds (w*p + E) - E to
// the numerator and (w + E) - E to the weight of every pixel of every
// matched patch. The weight is one value per group, so a pixel's weight sum
// is the sum of that value over the patches covering it: the filter adds it
// once per patch, at the patch's origin, into the slice's weight-origin
// plane, and the normaliser sums each pixel's 8x8 window of origins
// (bm3d_kernels.cu). With the extractor (E = 2^e) every addend is a multiple
// of ulp(E) and the sums are exact in any order, so the weights equal the
// reference's bit for bit; without it they differ only in float rounding
// order, as the reference's own atomics do from run to run.
//
// Numerators go to the slice's numerator plane with float atomics; `acc`,
// when given, is a tile-owned shared-memory accumulator that takes the
// patches of slice acc->z whose 8x8 footprint lies inside it (the caller
// flushes it into the plane once, see TileAccumulator).
struct TileAccumulator {
    float* num;  // shared: pixel (fx0 + c, fy0 + r) at num[r*w + c], w x h pixels
    float* org;  // shared: weight of origin (fx0 + c, fy0 + r) at org[r*(w-7) + c]
    int z;       // slice held (-1: none)
    int fx0, fy0, w, h;
};

__device__ __forceinline__ void scatter_group(const StackJob& job, const uint32_t mxy[8],
                                              uint32_t zp, int sub, const float d[64], float w,
                                              const TileAccumulator* acc = nullptr) {
    const float E = job.extractor;
    const float wv = __fsub_rn(__fadd_rn(w, E), E);
    const int dpitch = job.dst_pitch;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int z = (int)((zp >> (4 * k)) & 15u);
        float* num = job.slice_dst[z];
        if (num == nullptr) continue;
        const int mx = (int)(mxy[k] & 0xffffu), my = (int)(mxy[k] >> 16);
        if (acc && z == acc->z) {
            const int c = mx - acc->fx0, r = my - acc->fy0;
            if (c >= 0 && r >= 0 && c + 8 <= acc->w && r + 8 <= acc->h) {
                float* pn = acc->num + r * acc->w + c + sub;
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    atomicAdd(pn + j * acc->w, __fsub_rn(__fmaf_rn(w, d[k * 8 + j], E), E));
                if (sub == k) atomicAdd(acc->org + r * (acc->w - 7) + c, wv);
                continue;
            }
        }
        float* pn = num + (size_t)my * dpitch + mx + sub;
#pragma unroll
        for (int j = 0; j < 8; ++j)
            red_add_global(pn + (size_t)j * dpitch, __fsub_rn(__fmaf_rn(w, d[k * 8 + j], E), E));
        if (sub == k) red_add_global(num + job.dst_plane + (size_t)my * dpitch + mx, wv);
    }
}

// Filters block b's group (matches mxy = x | y << 16, zp = 8 x 4-bit slice)
// and scatters it into the stack's slices. kSaveMask also records the keep
// bits, lane `sub` writing word mask_out[b * 8 + sub] (bit 8 * group
// frequency + vertical frequency, of horizontal frequency sub). An invalid
// group (valid == false) computes but writes nothing. buf: kGroupStride
// floats of shared memory owned by the group.
template <bool kSaveMask, bool kWiener = false>
__device__ __forceinline__ void filter_group(const StackJob& job, int b, bool valid,
                                             const uint32_t mxy[8], uint32_t zp, int sub,
                                             float* buf, const TileAccumulator* acc = nullptr) {
    float d[64];
    float w;
    if (kWiener) {
        float r[64];
        gather_group(r, job.slice_frame, job.pitch, mxy, zp, sub);
        forward3(r, buf, sub);
        gather_group(d, job.slice_input, job.pitch, mxy, zp, sub);
        forward3(d, buf, sub);
        w = wiener_coefficients(d, r, job.thr, sub);
    } else {
        gather_group(d, job.slice_frame, job.pitch, mxy, zp, sub);
        forward3(d, buf, sub);
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
        w = __fdiv_rn(1.0f, (float)kept);
    }
    inverse3(d, buf, sub);

    if (!valid) return;
    scatter_group(job, mxy, zp, sub, d, w, acc);
}

}  // namespace vsfeel
