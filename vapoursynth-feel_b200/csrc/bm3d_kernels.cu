// sm_100a kernels of the BM3Dv2 basic estimate (hard-thresholding pass).
//
//   bm3d_match_kernel ..... block matching: spatial window, temporal
//                           predictive search, forced self-match
//                           (src/bm3d.comp:460-663); writes the match table
//   bm3d_filter_kernel .... gather, 3D DCT, hard threshold, inverse and the
//                           extractor-biased scatter into the output slices
//                           (src/bm3d.comp:358-399, 666-716)
//   bm3d_normalize_kernel . per-pixel FP64 sum over the TW slices and the
//                           division (src/bm3d_agg.comp:36-52)
//
// Lane layout of the matching and filtering kernels: 8 lanes per reference
// block, 4 blocks per warp. In matching, lane s scans the candidate rows
// top+s, top+s+8, ... (stride-8 linear order at radius >= 3) into its own
// sorted top-8; the 8 lists are merged with warp shuffles. Candidates are
// ordered by (SSD, scan index), so the merged list is the 8 smallest keys,
// exactly as in the reference.
#include "bm3d_device.cuh"
#include "bm3d_filter.cuh"

namespace vsfeel {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t pack_xy(int x, int y) {
    return (uint32_t)x | ((uint32_t)y << 16);
}

struct LaneTop8 {
    float e[8];
    uint32_t xy[8];
    int s[8];

    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            e[k] = kFltMax;
            xy[k] = 0;
            s[k] = kSeqSentinel;
        }
    }

    // strict `<`: an equal later candidate stays behind (src/bm3d.comp:284-302)
    __device__ __forceinline__ void insert(float err, uint32_t cxy, int seq) {
        if (err < e[7]) {
#pragma unroll
            for (int k = 7; k > 0; --k) {
                const bool sh = err < e[k - 1];
                const bool pl = err < e[k];
                e[k] = sh ? e[k - 1] : (pl ? err : e[k]);
                xy[k] = sh ? xy[k - 1] : (pl ? cxy : xy[k]);
                s[k] = sh ? s[k - 1] : (pl ? seq : s[k]);
            }
            const bool p0 = err < e[0];
            e[0] = p0 ? err : e[0];
            xy[0] = p0 ? cxy : xy[0];
            s[0] = p0 ? seq : s[0];
        }
    }
};

// Merge the 8 lane lists of this lane's group (lanes 8g..8g+7) into the 8
// smallest (error, seq) keys; every lane of the group receives the result.
// Ties between sentinels resolve to the lower lane, as in
// src/bm3d.comp:324-356.
__device__ __forceinline__ void merge_group(LaneTop8 L, float me[8], uint32_t mxy[8]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float e = L.e[0];
        int s = L.s[0];
        int src = lane;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
            const float oe = __shfl_xor_sync(kFull, e, off);
            const int os = __shfl_xor_sync(kFull, s, off);
            const int osrc = __shfl_xor_sync(kFull, src, off);
            const bool take = oe < e || (oe == e && (os < s || (os == s && osrc < src)));
            e = take ? oe : e;
            s = take ? os : s;
            src = take ? osrc : src;
        }
        me[k] = e;
        mxy[k] = __shfl_sync(kFull, L.xy[0], src);
        if (lane == src) {
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                L.e[q] = L.e[q + 1];
                L.xy[q] = L.xy[q + 1];
                L.s[q] = L.s[q + 1];
            }
            L.e[7] = kFltMax;
            L.xy[7] = 0;
            L.s[7] = kSeqSentinel;
        }
    }
}

// Scan one search window into this lane's list (src/bm3d.comp:493-526).
// kSliding (radius < 3): the reference's sliding column scan, whose slot c
// holds source column cx+c against block column min(c + cx-left, 7).
template <bool kSliding>
__device__ __forceinline__ void scan_window(const float cur[64], const float* __restrict__ f,
                                            int pitch, int left, int right, int top, int bottom,
                                            int seq_base, int sub, LaneTop8& L) {
    const int rw = right - left + 1;
    if (kSliding) {
        for (int cy = top + sub; cy <= bottom; cy += 8) {
            const float* row = f + (size_t)cy * pitch;
            float col[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) col[c] = column_ssd(&cur[c * 8], row + left + c, pitch);
            int seq = seq_base + (cy - top) * rw;
            L.insert(tree8(col), pack_xy(left, cy), seq);
            for (int cx = left + 1; cx <= right; ++cx) {
#pragma unroll
                for (int c = 0; c < 7; ++c) col[c] = col[c + 1];
                col[7] = column_ssd(&cur[56], row + cx + 7, pitch);
                ++seq;
                L.insert(tree8(col), pack_xy(cx, cy), seq);
            }
        }
    } else {
        const int total = (bottom - top + 1) * rw;
        int cy = top + sub / rw;
        int cx = left + sub % rw;
        for (int idx = sub; idx < total; idx += 8) {
            const float* p = f + (size_t)cy * pitch + cx;
            float col[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) col[c] = column_ssd(&cur[c * 8], p + c, pitch);
            L.insert(tree8(col), pack_xy(cx, cy), seq_base + idx);
            cx += 8;
            while (cx > right) {
                cx -= rw;
                cy += 1;
            }
        }
    }
}

// global list insertion of a temporal match (src/bm3d.comp:304-322)
__device__ __forceinline__ void ginsert(float ge[8], uint32_t gxy[8], int gz[8], float err,
                                        uint32_t cxy, int cz) {
    if (err < ge[7]) {
#pragma unroll
        for (int k = 7; k > 0; --k) {
            const bool sh = err < ge[k - 1];
            const bool pl = err < ge[k];
            ge[k] = sh ? ge[k - 1] : (pl ? err : ge[k]);
            gxy[k] = sh ? gxy[k - 1] : (pl ? cxy : gxy[k]);
            gz[k] = sh ? gz[k - 1] : (pl ? cz : gz[k]);
        }
        const bool p0 = err < ge[0];
        ge[0] = p0 ? err : ge[0];
        gxy[0] = p0 ? cxy : gxy[0];
        gz[0] = p0 ? cz : gz[0];
    }
}

}  // namespace

template <bool kSliding>
__global__ void __launch_bounds__(128) bm3d_match_kernel(const StackJob job) {
    const int lane = threadIdx.x & 31;
    const int sub = lane & 7;
    const int nblocks = job.nbx * job.nby;
    const int gblock = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
    const bool valid = gblock < nblocks;
    const int b = valid ? gblock : nblocks - 1;
    const int by = b / job.nbx;
    const int bx = b - by * job.nbx;
    const int x = min(bx * job.step, job.width - 8);
    const int y = min(by * job.step, job.height - 8);
    const int r = job.radius;
    const int pitch = job.pitch;
    const float* __restrict__ fc = job.slice_frame[r];

    float cur[64];
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int i = 0; i < 8; ++i) cur[c * 8 + i] = __ldg(fc + (size_t)(y + i) * pitch + x + c);

    float ge[8];
    uint32_t gxy[8];
    int gz[8];
    {
        LaneTop8 L;
        L.reset();
        const int R = job.bm_range;
        const int left = max(x - R, 0), right = min(x + R, job.width - 8);
        const int top = max(y - R, 0), bottom = min(y + R, job.height - 8);
        scan_window<kSliding>(cur, fc, pitch, left, right, top, bottom, 0, sub, L);
        merge_group(L, ge, gxy);
#pragma unroll
        for (int k = 0; k < 8; ++k) gz[k] = r;
    }

    // temporal predictive search (src/bm3d.comp:540-637): the spatial top-8
    // seeds both directions; each frame's merged top-8 seeds the next frame
    const int Q = job.ps_range;
    const int area = (2 * Q + 1) * (2 * Q + 1);
    uint32_t sxy[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) sxy[k] = gxy[k];
    for (int dir = -1; dir <= 1; dir += 2) {
        uint32_t pxy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) pxy[k] = sxy[k];
        for (int t = 1; t <= r; ++t) {
            const int z = r + dir * t;
            const float* __restrict__ ft = job.slice_frame[z];
            LaneTop8 L;
            L.reset();
            for (int i = 0; i < job.ps_num; ++i) {
                uint32_t p = pxy[0];
#pragma unroll
                for (int k = 1; k < 8; ++k) p = (i == k) ? pxy[k] : p;
                const int pxi = (int)(p & 0xffffu), pyi = (int)(p >> 16);
                const int left = max(pxi - Q, 0), right = min(pxi + Q, job.width - 8);
                const int top = max(pyi - Q, 0), bottom = min(pyi + Q, job.height - 8);
                scan_window<kSliding>(cur, ft, pitch, left, right, top, bottom, i * area, sub, L);
            }
            float fe[8];
            uint32_t fxy[8];
            merge_group(L, fe, fxy);
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i < job.ps_num) ginsert(ge, gxy, gz, fe[i], fxy[i], z);
#pragma unroll
            for (int k = 0; k < 8; ++k) pxy[k] = fxy[k];
        }
    }

    // forced self-match (src/bm3d.comp:639-663)
    const uint32_t self_xy = pack_xy(x, y);
    bool has_self = false;
#pragma unroll
    for (int k = 0; k < 8; ++k) has_self = has_self || (gxy[k] == self_xy && gz[k] == r);
    if (!has_self) {
#pragma unroll
        for (int k = 7; k > 0; --k) {
            gxy[k] = gxy[k - 1];
            gz[k] = gz[k - 1];
        }
        gxy[0] = self_xy;
        gz[0] = r;
    }

    if (valid && sub == 0) {
        uint4* dst = reinterpret_cast<uint4*>(job.match_xy + (size_t)b * 8);
        dst[0] = make_uint4(gxy[0], gxy[1], gxy[2], gxy[3]);
        dst[1] = make_uint4(gxy[4], gxy[5], gxy[6], gxy[7]);
        uint32_t zp = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) zp |= (uint32_t)gz[k] << (4 * k);
        job.match_z[b] = zp;
    }
}

// The standalone filter: kGroups groups of 8 lanes per CTA, matches read
// from the stack's match table. 16 groups when it runs alone; 8 when it
// runs beside the next stack's matching, so that one CTA fits on an SM next
// to a matcher CTA (18.7 KB of shared memory, 64 threads).
template <bool kSaveMask, bool kWiener, int kGroups = kFilterGroupsPerCta>
__global__ void __launch_bounds__(kGroups * 8) bm3d_filter_kernel(const StackJob job) {
    __shared__ float smem[kGroups * kGroupStride];
    const int sub = threadIdx.x & 7;
    float* buf = smem + (threadIdx.x >> 3) * kGroupStride;
    const int nblocks = job.nbx * job.nby;
    const int gblock = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
    const bool valid = gblock < nblocks;
    const int b = valid ? gblock : nblocks - 1;
    const uint4 m0 = reinterpret_cast<const uint4*>(job.match_xy + (size_t)b * 8)[0];
    const uint4 m1 = reinterpret_cast<const uint4*>(job.match_xy + (size_t)b * 8)[1];
    const uint32_t mxy[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
    filter_group<kSaveMask, kWiener>(job, b, valid, mxy, job.match_z[b], sub, buf);
}

// ---------------------------------------------------------------------------
// Normalisation (src/bm3d_agg.comp:36-52): out = float(sum_i double(num_i) /
// sum_i double(den_i)) over the tw slices, in the reference's order i = 0..tw-1.
// A slice's weight plane holds per-patch weights at the patches' origins
// (scatter_group): den_i of a pixel (x, y) is the sum of origins
// x-7..x by y-7..y, taken in float as the 8 vertical sums of its columns,
// then their sum from left to right.
//
// One warp covers 120 pixels of one row: lane l reads columns
// x0 - 8 + 4l .. +3 of the 8 origin rows (one float4 each) and forms their
// vertical sums; lanes 2..31 own the pixels x0 + 4(l-2) .. +3 and take the 7
// vertical sums left of their own from lanes l-2 and l-1 by shuffles (lanes
// 0 and 1 hold the tile's left halo). No shared memory, so the kernel's
// CTAs fit beside the matcher's. Origin planes exist for 0..W-8 x 0..H-8
// and are zero elsewhere within the padded plane; rows above the frame read
// as zero. The numerator planes are read four floats at a time (rows
// padded to 32 floats, bases 16-byte aligned).
__device__ __forceinline__ void normalize_tile(const NormalizeJob& job, int tx0, int ty0) {
    const int lane = threadIdx.x & 31;
    const int y = ty0 + (threadIdx.x >> 5);
    if (y >= job.height) return;  // whole warps leave: the shuffles below stay full
    const int col = tx0 - 8 + 4 * lane;          // first origin column of this lane
    const int x0 = tx0 + 4 * (lane - 2);         // first pixel of this lane (lanes >= 2)
    const bool has_px = lane >= 2 && x0 < job.width;
    const bool col_ok = col >= 0 && col + 3 < job.src_pitch;
    double acc[4] = {0.0, 0.0, 0.0, 0.0}, acw[4] = {0.0, 0.0, 0.0, 0.0};
    // slices indexed statically (the slice pointers stay in the parameter
    // space), in the reference's order
#pragma unroll
    for (int i = 0; i < kMaxTW; ++i) {
        if (i >= job.tw) break;
        const float* org = job.num[i] + job.den_offset;
        float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int dy = 7; dy >= 0; --dy) {
            const int oy = y - dy;
            float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (oy >= 0 && col_ok) a = *reinterpret_cast<const float4*>(org + (size_t)oy * job.src_pitch + col);
            v[0] = __fadd_rn(v[0], a.x);
            v[1] = __fadd_rn(v[1], a.y);
            v[2] = __fadd_rn(v[2], a.z);
            v[3] = __fadd_rn(v[3], a.w);
        }
        // vertical sums of columns c-8 .. c+3 (c = this lane's first column + 8)
        float h[12];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            h[k] = __shfl_up_sync(0xffffffffu, v[k], 2);
            h[4 + k] = __shfl_up_sync(0xffffffffu, v[k], 1);
            h[8 + k] = v[k];
        }
        float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (has_px) a = *reinterpret_cast<const float4*>(job.num[i] + (size_t)y * job.src_pitch + x0);
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            // pixel x0 + k: origins x0+k-7 .. x0+k, h[k+1] .. h[k+8]
            float w = h[k + 1];
#pragma unroll
            for (int dx = 2; dx <= 8; ++dx) w = __fadd_rn(w, h[k + dx]);
            acc[k] += (double)av[k];
            acw[k] += (double)w;
        }
    }
    if (!has_px) return;
    float* out = job.out + (size_t)y * job.out_pitch;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (x0 + k < job.width) {
            out[x0 + k] = (float)(acc[k] / acw[k]);
            if (job.den_out) job.den_out[(size_t)y * job.den_pitch + x0 + k] = (float)acw[k];
        }
    }
}

__global__ void __launch_bounds__(32 * kNormTileH) bm3d_normalize_kernel(const NormalizeJob job) {
    normalize_tile(job, blockIdx.x * kNormTileW, blockIdx.y * kNormTileH);
}

// Batched form: the filter of kGroups blocks of one stack per CTA.
template <int kGroups>
__global__ void __launch_bounds__(kGroups * 8) bm3d_filter_batch_kernel(const FilterBatch work) {
    __shared__ float smem[kGroups * kGroupStride];
    const int item = blockIdx.x;
    int lo = 0, hi = work.njobs - 1;
    while (lo < hi) {  // last job whose first item is <= item
        const int mid = (lo + hi + 1) >> 1;
        if (work.group_first[mid] <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    const StackJob& job = work.jobs[lo];
    const int sub = threadIdx.x & 7;
    float* buf = smem + (threadIdx.x >> 3) * kGroupStride;
    const int nblocks = job.nbx * job.nby;
    const int gblock = (item - work.group_first[lo]) * kGroups + (threadIdx.x >> 3);
    const bool valid = gblock < nblocks;
    const int b = valid ? gblock : nblocks - 1;
    const uint4 m0 = reinterpret_cast<const uint4*>(job.match_xy + (size_t)b * 8)[0];
    const uint4 m1 = reinterpret_cast<const uint4*>(job.match_xy + (size_t)b * 8)[1];
    const uint32_t mxy[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
    filter_group<false>(job, b, valid, mxy, job.match_z[b], sub, buf);
}

// Batched form: one CTA per normaliser tile of one output frame.
__global__ void __launch_bounds__(32 * kNormTileH) bm3d_normalize_batch_kernel(const NormalizeBatch work) {
    const int item = blockIdx.x;
    int lo = 0, hi = work.njobs - 1;
    while (lo < hi) {  // last job whose first tile is <= item
        const int mid = (lo + hi + 1) >> 1;
        if (work.tile_first[mid] <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    const NormalizeJob& job = work.jobs[lo];
    const int t = item - work.tile_first[lo];
    const int tiles_x = (job.width + kNormTileW - 1) / kNormTileW;
    normalize_tile(job, (t % tiles_x) * kNormTileW, (t / tiles_x) * kNormTileH);
}

// ---------------------------------------------------------------------------
// Adjoint of the frozen-match operator (no counterpart in the reference).
//
// With the match table, the keep bits and so the weights w = 1/kept frozen,
// the forward pass is linear in the input: every group adds
// w * S^T (F^-1 M F / 4096) S x to its slices, S gathering the 8 matched
// patches, F the scaled 3D DCT and M the keep mask, and output n divides the
// sum of the slices it reads by the frozen denominator D_n. F^-1 is F^T up
// to the same scale, so F^-1 M F / 4096 is symmetric and the adjoint of a
// group is the same transform, mask and inverse applied to the gathered
// output gradient. Per group: gather reads(m, z) * (g / D) from the scaled
// output gradient of each patch's frame (bm3d_grad_scale_kernel, once per
// frame), transform, mask, inverse, times w, then scatter-add into the input
// gradient of the same patches. One launch covers a range of stacks in
// order, so that its frames' scaled gradients and input gradients stay in
// L2. The extractor's rounding of the forward scatter is taken as the
// identity.
// Three CTAs per SM (at most 168 registers): without the bound the gathers
// all in flight take 211 registers and two CTAs per SM, 9.87 against 8.21 ms
// per 32-frame 1080p radius-2 backward.
__global__ void __launch_bounds__(128, 3) bm3d_adjoint_kernel(const AdjointJob job) {
    __shared__ float smem[kFilterGroupsPerCta * kGroupStride];
    const int lane = threadIdx.x & 31;
    const int sub = lane & 7;
    const int group_in_cta = threadIdx.x >> 3;
    float* buf = smem + group_in_cta * kGroupStride;
    const int64_t total = (int64_t)job.stack_count * job.nblocks;
    const int64_t gid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const bool valid = gid < total;
    const int64_t g = valid ? gid : total - 1;
    const int ml = (int)(g / job.nblocks);
    const int b = (int)(g - (int64_t)ml * job.nblocks);
    const int m = job.first_stack + ml;
    const unsigned char* rec = job.saved + (size_t)m * job.stack_bytes;

    const uint4* xy4 = reinterpret_cast<const uint4*>(rec + job.off_xy) + (size_t)b * 2;
    const uint4 m0 = xy4[0], m1 = xy4[1];
    uint32_t mxy[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
    // a damaged state must not send the gathers outside the frames
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t x = min(mxy[k] & 0xffffu, (uint32_t)(job.width - 8));
        const uint32_t y = min(mxy[k] >> 16, (uint32_t)(job.height - 8));
        mxy[k] = x | (y << 16);
    }
    const uint32_t zp = reinterpret_cast<const uint32_t*>(rec + job.off_z)[b];
    const uint64_t bits = reinterpret_cast<const uint64_t*>(rec + job.off_mask)[(size_t)b * 8 + sub];
    const int r = job.radius;

    float d[64];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int z = (int)((zp >> (4 * k)) & 15u);
        const int f = clamp_frame(m - r + z, job.nframes);
        const float reads = (float)slice_reads(m, z, job.nframes, r);
        const int mx = (int)(mxy[k] & 0xffffu), my = (int)(mxy[k] >> 16);
        const float* gs = job.gs + (size_t)(f % job.gs_slots) * job.gs_frame +
                          (size_t)my * job.gs_pitch + mx + sub;
#pragma unroll
        for (int j = 0; j < 8; ++j)
            d[k * 8 + j] = __fmul_rn(reads, __ldg(gs + (size_t)j * job.gs_pitch));
    }

    transform_rows(d, false);
    transpose_group(d, buf, sub);
    transform_rows(d, false);
    transpose_group(d, buf, sub);
    transform_group_axis(d, false);

    int kept = __popcll(bits);
    kept += __shfl_xor_sync(kFull, kept, 1);
    kept += __shfl_xor_sync(kFull, kept, 2);
    kept += __shfl_xor_sync(kFull, kept, 4);
    const float w = __fdiv_rn(1.0f, (float)max(kept, 1));
#pragma unroll
    for (int i = 0; i < 64; ++i)
        d[i] = ((bits >> i) & 1u) ? __fmul_rn(d[i], 1.0f / 4096.0f) : 0.0f;

    transform_rows(d, true);
    transpose_group(d, buf, sub);
    transform_rows(d, true);
    transpose_group(d, buf, sub);
    transform_group_axis(d, true);

    if (!valid) return;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int z = (int)((zp >> (4 * k)) & 15u);
        const int f = clamp_frame(m - r + z, job.nframes);
        const int mx = (int)(mxy[k] & 0xffffu), my = (int)(mxy[k] >> 16);
        float* gi = job.grad_in + (size_t)f * job.gi_frame + (size_t)my * job.gi_pitch + mx + sub;
#pragma unroll
        for (int j = 0; j < 8; ++j) red_add_global(gi + (size_t)j * job.gi_pitch, __fmul_rn(w, d[k * 8 + j]));
    }
}

// ---------------------------------------------------------------------------
namespace {
constexpr int kThreads = 128;  // 16 blocks (8 lanes each) per CTA
int block_grid(const StackJob& job) { return (job.nbx * job.nby * 8 + kThreads - 1) / kThreads; }
}  // namespace

cudaError_t launch_match(const StackJob& job, cudaStream_t stream) {
    int shape = default_tile_shape(job, kTableOnly);
    if (shape >= 0 && job.tile_shape_plus1 > 0 &&
        tile_shape_fits(job, TileShape(job.tile_shape_plus1 - 1), kTableOnly))
        shape = job.tile_shape_plus1 - 1;
    if (shape >= 0) return launch_match_tiles(job, TileShape(shape), kTableOnly, stream);
    if (job.radius < 3)
        bm3d_match_kernel<true><<<block_grid(job), kThreads, 0, stream>>>(job);
    else
        bm3d_match_kernel<false><<<block_grid(job), kThreads, 0, stream>>>(job);
    return cudaGetLastError();
}

cudaError_t launch_filter(const StackJob& job, cudaStream_t stream) {
    if (job.wiener)
        bm3d_filter_kernel<false, true><<<block_grid(job), kThreads, 0, stream>>>(job);
    else if (job.mask_out)
        bm3d_filter_kernel<true, false><<<block_grid(job), kThreads, 0, stream>>>(job);
    else
        bm3d_filter_kernel<false, false><<<block_grid(job), kThreads, 0, stream>>>(job);
    return cudaGetLastError();
}

cudaError_t launch_filter_beside_match(const StackJob& job, cudaStream_t stream) {
    constexpr int kSmall = 8, kSmallThreads = kSmall * 8;
    const int grid = (job.nbx * job.nby * 8 + kSmallThreads - 1) / kSmallThreads;
    if (job.wiener)
        bm3d_filter_kernel<false, true, kSmall><<<grid, kSmallThreads, 0, stream>>>(job);
    else if (job.mask_out)
        bm3d_filter_kernel<true, false, kSmall><<<grid, kSmallThreads, 0, stream>>>(job);
    else
        bm3d_filter_kernel<false, false, kSmall><<<grid, kSmallThreads, 0, stream>>>(job);
    return cudaGetLastError();
}

cudaError_t launch_filter_batch(const FilterBatch& work, int total_items, int groups,
                                cudaStream_t stream) {
    if (total_items <= 0) return cudaSuccess;
    if (groups == 8)
        bm3d_filter_batch_kernel<8><<<total_items, 64, 0, stream>>>(work);
    else
        bm3d_filter_batch_kernel<16><<<total_items, 128, 0, stream>>>(work);
    return cudaGetLastError();
}

cudaError_t launch_normalize_batch(const NormalizeBatch& work, int total_tiles,
                                   cudaStream_t stream) {
    if (total_tiles <= 0) return cudaSuccess;
    bm3d_normalize_batch_kernel<<<total_tiles, 32 * kNormTileH, 0, stream>>>(work);
    return cudaGetLastError();
}

cudaError_t launch_adjoint(const AdjointJob& job, cudaStream_t stream) {
    const int64_t threads = (int64_t)job.stack_count * job.nblocks * 8;
    const int64_t grid = (threads + kThreads - 1) / kThreads;
    if (grid <= 0) return cudaSuccess;
    if (grid > INT32_MAX) return cudaErrorInvalidValue;
    bm3d_adjoint_kernel<<<(unsigned)grid, kThreads, 0, stream>>>(job);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) bm3d_grad_scale_kernel(const GradScaleJob job) {
    const int x = blockIdx.x * 64 + (threadIdx.x & 63);
    const int y = blockIdx.y * 4 + (threadIdx.x >> 6);
    if (x >= job.width || y >= job.height) return;
    job.gs[(size_t)y * job.gs_pitch + x] = __fdiv_rn(__ldg(job.go + (size_t)y * job.go_pitch + x),
                                                     __ldg(job.den + (size_t)y * job.den_pitch + x));
}

cudaError_t launch_grad_scale(const GradScaleJob& job, cudaStream_t stream) {
    const dim3 grid((job.width + 63) / 64, (job.height + 3) / 4);
    bm3d_grad_scale_kernel<<<grid, 256, 0, stream>>>(job);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const NormalizeJob& job, cudaStream_t stream) {
    dim3 grid((job.width + kNormTileW - 1) / kNormTileW, (job.height + kNormTileH - 1) / kNormTileH);
    bm3d_normalize_kernel<<<grid, 32 * kNormTileH, 0, stream>>>(job);
    return cudaGetLastError();
}

}  // namespace vsfeel
