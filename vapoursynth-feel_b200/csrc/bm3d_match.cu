// Block matching for radius < 3: the reference's sliding column scan
// (src/bm3d.comp:479-538 spatial, 540-637 temporal), restructured for sm_100a.
//
// A CTA owns a tile of 8x4 reference blocks, 8 lanes per block. For each
// search phase (the spatial window in frame m, then one temporal step per
// frame) the CTA stages the frame region that every window of the tile can
// reach (tile +- bm_range + t*ps_range) in shared memory once, and all 32
// blocks search it from there.
//
// Within a block, lane s takes a chunk of K consecutive candidate rows of a
// window and sweeps the window's columns left to right. One step loads the
// K+7 source values of column X, updates the K column sums
//     V(X) = SSD(source column X, block column min(X - left, 7))
// and advances, per row, the reduction tree of the reference in incremental
// form: P(j) = V(j) + V(j+1), Q(j) = P(j) + P(j+2), E(j) = Q(j) + Q(j+4) --
// the same additions on the same operands as
// ((c0+c1)+(c2+c3))+((c4+c5)+(c6+c7)), so every candidate error carries the
// reference's bits.
//
// Ranking: candidates are 64-bit keys (error bits, scan index). The error is
// a non-negative float, so integer order is (error, index) order, and the 8
// smallest keys are exactly the reference's merged top-8 (per-lane strict
// insertion in index order + merge by (error, index)). Each lane keeps its 8
// smallest keys; a candidate is offered only if it beats the smallest 8th key
// among the block's 8 lanes, refreshed every 4 steps, so insertions are rare.
#include "bm3d_device.cuh"

#include <algorithm>

namespace vsfeel {

namespace {

constexpr int kTileBX = 8, kTileBY = 4;
constexpr int kMatchThreads = kTileBX * kTileBY * 8;  // 256
constexpr int kMaxK = 5;
constexpr uint64_t kKeyMax = (uint64_t(0x7f7fffffu) << 32) | 0x7fffffffu;  // (FLT_MAX, INT_MAX)

__device__ __forceinline__ uint64_t cand_key(float err, int seq) {
    return err < kFltMax ? ((uint64_t(__float_as_uint(err)) << 32) | uint32_t(seq)) : kKeyMax;
}

__device__ __forceinline__ float key_err(uint64_t k) { return __uint_as_float(uint32_t(k >> 32)); }

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

struct KeyList {
    uint64_t k[8];  // ascending

    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int i = 0; i < 8; ++i) k[i] = kKeyMax;
    }
    // keys are distinct, so `<` places c exactly
    __device__ __forceinline__ void insert(uint64_t c) {
#pragma unroll
        for (int i = 7; i > 0; --i) {
            const bool sh = c < k[i - 1];
            const bool pl = c < k[i];
            k[i] = sh ? k[i - 1] : (pl ? c : k[i]);
        }
        k[0] = c < k[0] ? c : k[0];
    }
};

__device__ __forceinline__ uint64_t group_min(uint64_t v, unsigned gmask) {
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) v = umin64(v, __shfl_xor_sync(gmask, v, off));
    return v;
}

__device__ __forceinline__ int group_max(int v, unsigned gmask) {
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) v = max(v, __shfl_xor_sync(gmask, v, off));
    return v;
}

// The `count` smallest keys of the group's 8 lane lists, in order; every
// lane of the group receives them. Equal keys (sentinels) resolve to the
// lower lane.
template <int kCount>
__device__ __forceinline__ void merge_keys(KeyList L, uint64_t out[8], int count, unsigned gmask) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < kCount; ++q) {
        if (q >= count) {
            out[q] = kKeyMax;
            continue;
        }
        uint64_t best = L.k[0];
        int src = lane;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
            const uint64_t o = __shfl_xor_sync(gmask, best, off);
            const int os = __shfl_xor_sync(gmask, src, off);
            const bool take = o < best || (o == best && os < src);
            best = take ? o : best;
            src = take ? os : src;
        }
        out[q] = best;
        if (lane == src) {
#pragma unroll
            for (int i = 0; i < 7; ++i) L.k[i] = L.k[i + 1];
            L.k[7] = kKeyMax;
        }
    }
}

// A search window: candidate columns left..left+rw-1, rows top..top+h-1,
// scan indices seq_base + (cy-top)*rw + (cx-left).
struct Window {
    int left, top, rw, h, seq_base;
};

__device__ __forceinline__ Window make_window(int cx, int cy, int range, int width, int height,
                                              int seq_base) {
    Window w;
    w.left = max(cx - range, 0);
    const int right = min(cx + range, width - 8);
    w.top = max(cy - range, 0);
    const int bottom = min(cy + range, height - 8);
    w.rw = right - w.left + 1;
    w.h = bottom - w.top + 1;
    w.seq_base = seq_base;
    return w;
}

// Source of a phase: the staged region in shared memory (kSmem) or the frame
// in global memory.
struct Source {
    const float* smem;  // region origin (rx0, ry0), row stride ss
    int rx0, ry0, ss;
    const float* __restrict__ frame;
    int pitch;
};

template <bool kSmem>
__device__ __forceinline__ float src_at(const Source& s, int row, int col) {
    if (kSmem) return s.smem[(row - s.ry0) * s.ss + (col - s.rx0)];
    return __ldg(s.frame + (size_t)row * s.pitch + col);
}

// SSD of one column of the block (bc, 8 values) against w[q..q+7].
template <int K>
__device__ __forceinline__ float column_ssd_at(const float bc[8], const float w[K + 7], int q) {
    float ev = 0.0f, od = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        const float d0 = __fsub_rn(bc[i], w[q + i]);
        ev = __fmaf_rn(d0, d0, ev);
        const float d1 = __fsub_rn(bc[i + 1], w[q + i + 1]);
        od = __fmaf_rn(d1, d1, od);
    }
    return __fadd_rn(ev, od);
}

// One lane's chunk: rows r0..r0+nrows-1 of window `win` (nrows may be 0),
// columns swept for `jcount` steps (uniform across the group; steps past the
// window's own width are padding). cur_s: the block's 64 values in shared
// memory, column-major; c7: block column 7 in registers.
template <int K, bool kSmem>
__device__ __forceinline__ void scan_chunk(const Source& src, const float* cur_s, const float c7[8],
                                           const Window& win, int r0, int nrows, int jcount,
                                           int row_max, unsigned gmask, KeyList& L,
                                           uint64_t& thr) {
    float vp[K], pr[K][2], qr[K][4];
    const int xmax = win.left + win.rw + 6;
    const int seq_row0 = win.seq_base + (r0 - win.top) * win.rw;
    // shared memory: rows past row_max exist (the region is padded) and only
    // feed masked rows; global memory: clamp them into the frame
    const float* sbase = kSmem ? src.smem + (r0 - src.ry0) * src.ss - src.rx0 : nullptr;
    const int ss = src.ss;

    auto load_col = [&](int X, float w[K + 7]) {
#pragma unroll
        for (int k = 0; k < K + 7; ++k) {
            if (kSmem)
                w[k] = sbase[k * ss + X];
            else
                w[k] = __ldg(src.frame + (size_t)min(r0 + k, row_max) * src.pitch + X);
        }
    };
    auto offer = [&](float e, int q, int d) {
        if (q < nrows && d < win.rw) {
            const uint64_t key = cand_key(e, seq_row0 + q * win.rw + d);
            if (key < thr) {
                L.insert(key);
                thr = umin64(thr, L.k[7]);
            }
        }
    };

    // warm-up: columns 0..7 of the block, steps j = 0..7 (candidate 0 at j = 7)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float bc[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) bc[i] = (j == 7) ? c7[i] : cur_s[j * 8 + i];
        float w[K + 7];
        load_col(min(win.left + j, xmax), w);
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const float v = column_ssd_at<K>(bc, w, q);
            if (j >= 1) {
                const float np = __fadd_rn(vp[q], v);          // P(j-1)
                if (j >= 3) {
                    const float nq = __fadd_rn(pr[q][(j + 1) & 1], np);  // Q(j-3)
                    if (j == 7) offer(__fadd_rn(qr[q][0], nq), q, 0);    // E(0)
                    qr[q][(j + 1) & 3] = nq;
                }
                pr[q][(j + 1) & 1] = np;
            }
            vp[q] = v;
        }
    }
    // steady state: block column 7, steps j = 8 .. jcount-1 (4 per iteration,
    // so the ring positions are static)
    for (int j0 = 8; j0 < jcount; j0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + u;
            float w[K + 7];
            load_col(min(win.left + j, xmax), w);
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const float v = column_ssd_at<K>(c7, w, q);
                const float np = __fadd_rn(vp[q], v);
                const float nq = __fadd_rn(pr[q][(u + 1) & 1], np);
                const float e = __fadd_rn(qr[q][(u + 1) & 3], nq);
                pr[q][(u + 1) & 1] = np;
                qr[q][(u + 1) & 3] = nq;
                vp[q] = v;
                if (j < jcount) offer(e, q, j - 7);
            }
        }
        thr = umin64(thr, group_min(L.k[7], gmask));
    }
}

template <int K>
__device__ __forceinline__ void scan_task(bool smem_ok, const Source& src, const float* cur_s,
                                          const float c7[8], const Window& win, int r0, int nrows,
                                          int jcount, int row_max, unsigned gmask, KeyList& L,
                                          uint64_t& thr) {
    if (smem_ok)
        scan_chunk<K, true>(src, cur_s, c7, win, r0, nrows, jcount, row_max, gmask, L, thr);
    else
        scan_chunk<K, false>(src, cur_s, c7, win, r0, nrows, jcount, row_max, gmask, L, thr);
}

// Scans windows[0..nwin) (rows split into chunks of K) into L. The windows
// live in the group's shared memory; every lane of the group makes the same
// choices (K, task count, source), so the group shuffles inside stay aligned.
__device__ void scan_windows(int K, const Source& src, int rx1, int ry1, const float* cur_s,
                             const float c7[8], const Window* wins, int nwin, int height,
                             int sub, unsigned gmask, KeyList& L) {
    int ntasks = 0;
    for (int i = 0; i < nwin; ++i) ntasks += (wins[i].h + K - 1) / K;
    uint64_t thr = kKeyMax;
    for (int t0 = 0; t0 < ntasks; t0 += 8) {
        const int task = t0 + sub;
        const bool has = task < ntasks;
        int wi = 0, c = has ? task : 0;
        while (wi < nwin - 1 && c >= (wins[wi].h + K - 1) / K) {
            c -= (wins[wi].h + K - 1) / K;
            ++wi;
        }
        const Window win = wins[wi];
        const int r0 = win.top + c * K;
        const int nrows = has ? min(K, win.h - c * K) : 0;
        const int jcount = group_max(has ? win.rw + 7 : 8, gmask);
        const int row_max = min(win.top + win.h - 1 + 7, height - 1);
        const bool inside = src.smem != nullptr && win.left >= src.rx0 &&
                            win.left + win.rw + 6 <= rx1 && win.top >= src.ry0 && row_max <= ry1;
        const bool smem_ok = __all_sync(gmask, inside);
        thr = umin64(thr, group_min(L.k[7], gmask));
        switch (K) {
            case 2: scan_task<2>(smem_ok, src, cur_s, c7, win, r0, nrows, jcount, row_max, gmask, L, thr); break;
            case 3: scan_task<3>(smem_ok, src, cur_s, c7, win, r0, nrows, jcount, row_max, gmask, L, thr); break;
            case 4: scan_task<4>(smem_ok, src, cur_s, c7, win, r0, nrows, jcount, row_max, gmask, L, thr); break;
            default: scan_task<5>(smem_ok, src, cur_s, c7, win, r0, nrows, jcount, row_max, gmask, L, thr); break;
        }
    }
}

__device__ __forceinline__ int rows_per_lane(int total_rows) {
    return min(kMaxK, max(2, (total_rows + 7) / 8));
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

// Position of a merged key. Sentinels decode to (0, 0) as in the reference.
__device__ __forceinline__ uint32_t key_xy(uint64_t key, const Window* wins, int area) {
    const uint32_t seq = uint32_t(key);
    if (key == kKeyMax) return 0u;
    const int wi = area > 0 ? int(seq) / area : 0;
    const Window w = wins[wi];
    const int rem = int(seq) - w.seq_base;
    const int dy = rem / w.rw;
    const int dx = rem - dy * w.rw;
    return uint32_t(w.left + dx) | (uint32_t(w.top + dy) << 16);
}

// A block's global match list and predictors (src/bm3d.comp:469-470,541-545).
struct GroupState {
    float ge[8];
    uint32_t gxy[8];
    int gz[8];
    uint32_t sxy[8];
    uint32_t pxy[8];
};

// Stages frame rows [ry0, ry1] x columns [rx0, rx1] into smem (row stride ss).
__device__ void stage_region(float* smem, const float* __restrict__ frame, int pitch, int rx0,
                             int ry0, int rx1, int ry1, int ss) {
    const int w = rx1 - rx0 + 1;
    const int h = ry1 - ry0 + 1;
    const int lane = threadIdx.x & 31;
    for (int yy = threadIdx.x >> 5; yy < h; yy += blockDim.x >> 5) {
        const float* __restrict__ row = frame + (size_t)(ry0 + yy) * pitch + rx0;
        for (int xx = lane; xx < w; xx += 32) smem[yy * ss + xx] = __ldg(row + xx);
    }
}

}  // namespace

// Shared memory: the block tiles' reference blocks (32 x 64 floats) followed
// by the staged region.
__global__ void __launch_bounds__(kMatchThreads, 1) bm3d_match_sliding_kernel(const StackJob job,
                                                                          int region_floats) {
    extern __shared__ float smem[];
    constexpr int kGroups = kTileBX * kTileBY;
    float* cur_all = smem;                                             // kGroups x 64
    Window* win_all = reinterpret_cast<Window*>(smem + kGroups * 64);   // kGroups x 8
    GroupState* gs_all = reinterpret_cast<GroupState*>(win_all + kGroups * 8);
    float* region = reinterpret_cast<float*>(gs_all + kGroups);

    const int lane = threadIdx.x & 31;
    const int sub = lane & 7;
    const int g = threadIdx.x >> 3;
    const unsigned gmask = 0xffu << (lane & ~7);
    const int tiles_x = (job.nbx + kTileBX - 1) / kTileBX;
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const int bx0 = tx * kTileBX, by0 = ty * kTileBY;
    const int bx_last = min(bx0 + kTileBX - 1, job.nbx - 1);
    const int by_last = min(by0 + kTileBY - 1, job.nby - 1);
    const int bxr = bx0 + (g % kTileBX), byr = by0 + (g / kTileBX);
    const bool valid = bxr < job.nbx && byr < job.nby;
    const int bx = min(bxr, job.nbx - 1), by = min(byr, job.nby - 1);
    const int W = job.width, H = job.height;
    const int x = min(bx * job.step, W - 8);
    const int y = min(by * job.step, H - 8);
    const int tile_x0 = min(bx0 * job.step, W - 8), tile_x1 = min(bx_last * job.step, W - 8);
    const int tile_y0 = min(by0 * job.step, H - 8), tile_y1 = min(by_last * job.step, H - 8);
    const int r = job.radius;
    const int R = job.bm_range, Q = job.ps_range, P = job.ps_num;
    const int pitch = job.pitch;

    // the reference block (column-major) and its column 7
    float* cur_s = cur_all + g * 64;
    Window* win = win_all + g * 8;
    const float* fc = job.slice_frame[r];
    {
        const int c = sub;
#pragma unroll
        for (int i = 0; i < 8; ++i) cur_s[c * 8 + i] = __ldg(fc + (size_t)(y + i) * pitch + x + c);
    }
    __syncwarp();
    float c7[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) c7[i] = cur_s[56 + i];

    auto stage = [&](const float* frame, int reach, Source& s, int& rx1, int& ry1) {
        const int rx0 = max(tile_x0 - reach, 0);
        rx1 = min(tile_x1 + reach, W - 8) + 7;
        const int ry0 = max(tile_y0 - reach, 0);
        ry1 = min(tile_y1 + reach, H - 8) + 7;
        const int ss = ((rx1 - rx0 + 1 + 31) & ~31) + 1;  // odd stride: rows hit distinct banks
        s.frame = frame;
        s.pitch = pitch;
        s.rx0 = rx0;
        s.ry0 = ry0;
        s.ss = ss;
        __syncthreads();  // previous phase finished reading the region
        if ((ry1 - ry0 + 1 + kMaxK + 7) * ss <= region_floats) {
            stage_region(region, frame, pitch, rx0, ry0, rx1, ry1, ss);
            s.smem = region;
        } else {
            s.smem = nullptr;  // too large for shared memory: read the frame directly
        }
        __syncthreads();
    };

    // the block's global match list, kept by lane 0 in shared memory
    GroupState* gs = gs_all + g;
    {
        Source s;
        int rx1, ry1;
        stage(fc, R, s, rx1, ry1);
        if (sub == 0) win[0] = make_window(x, y, R, W, H, 0);
        __syncwarp(gmask);
        KeyList L;
        L.reset();
        scan_windows(rows_per_lane(win[0].h), s, rx1, ry1, cur_s, c7, win, 1, H, sub, gmask, L);
        uint64_t mk[8];
        merge_keys<8>(L, mk, 8, gmask);
        if (sub == 0) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                gs->ge[k] = key_err(mk[k]);
                gs->gxy[k] = key_xy(mk[k], win, 0);
                gs->gz[k] = r;
                gs->sxy[k] = gs->gxy[k];
            }
        }
        __syncwarp(gmask);
    }

    const int area = (2 * Q + 1) * (2 * Q + 1);
    for (int dir = -1; dir <= 1; dir += 2) {
        if (sub == 0)
            for (int k = 0; k < 8; ++k) gs->pxy[k] = gs->sxy[k];
        for (int t = 1; t <= r; ++t) {
            const int z = r + dir * t;
            Source s;
            int rx1, ry1;
            stage(job.slice_frame[z], R + t * Q, s, rx1, ry1);
            if (sub == 0)
                for (int i = 0; i < P; ++i) {
                    const uint32_t p = gs->pxy[i];
                    win[i] = make_window(int(p & 0xffffu), int(p >> 16), Q, W, H, i * area);
                }
            __syncwarp(gmask);
            int total_rows = 0;
            for (int i = 0; i < P; ++i) total_rows += win[i].h;
            KeyList L;
            L.reset();
            scan_windows(rows_per_lane(total_rows), s, rx1, ry1, cur_s, c7, win, P, H, sub, gmask, L);
            uint64_t mk[8];
            merge_keys<8>(L, mk, P, gmask);
            if (sub == 0) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (i < P) {
                        const uint32_t fxy = key_xy(mk[i], win, area);
                        ginsert(gs->ge, gs->gxy, gs->gz, key_err(mk[i]), fxy, z);
                        gs->pxy[i] = fxy;
                    }
                }
            }
            __syncwarp(gmask);
        }
    }

    if (valid && sub == 0) {
        // forced self-match (src/bm3d.comp:639-663)
        uint32_t gxy[8];
        int gz[8];
        for (int k = 0; k < 8; ++k) {
            gxy[k] = gs->gxy[k];
            gz[k] = gs->gz[k];
        }
        const uint32_t self_xy = uint32_t(x) | (uint32_t(y) << 16);
        bool has_self = false;
        for (int k = 0; k < 8; ++k) has_self = has_self || (gxy[k] == self_xy && gz[k] == r);
        if (!has_self) {
            for (int k = 7; k > 0; --k) {
                gxy[k] = gxy[k - 1];
                gz[k] = gz[k - 1];
            }
            gxy[0] = self_xy;
            gz[0] = r;
        }
        const size_t b = (size_t)by * job.nbx + bx;
        uint4* dst = reinterpret_cast<uint4*>(job.match_xy + b * 8);
        dst[0] = make_uint4(gxy[0], gxy[1], gxy[2], gxy[3]);
        dst[1] = make_uint4(gxy[4], gxy[5], gxy[6], gxy[7]);
        uint32_t zp = 0;
        for (int k = 0; k < 8; ++k) zp |= uint32_t(gz[k]) << (4 * k);
        job.match_z[b] = zp;
    }
}

namespace {
constexpr int kRegionMaxFloats = 48 * 1024;  // 192 KB: larger regions read the frame directly
}

// Shared memory for one tile: blocks, windows and the largest staged region
// any phase needs (a full tile, reach bm_range + radius * ps_range).
size_t match_sliding_smem(const StackJob& job, int* region_floats) {
    const int reach = job.bm_range + job.radius * job.ps_range;
    const int tile_w = (kTileBX - 1) * job.step + 8, tile_h = (kTileBY - 1) * job.step + 8;
    const int w = std::min(tile_w + 2 * reach, job.width), h = std::min(tile_h + 2 * reach, job.height);
    const int ss = ((w + 31) & ~31) + 1;
    int floats = ss * (h + kMaxK + 7);  // + rows that masked chunk rows may read
    if (floats > kRegionMaxFloats) floats = 0;
    *region_floats = floats;
    constexpr int kGroups = kTileBX * kTileBY;
    return sizeof(float) * (kGroups * 64 + floats) + sizeof(Window) * kGroups * 8 +
           sizeof(GroupState) * kGroups;
}

cudaError_t launch_match_sliding(const StackJob& job, cudaStream_t stream) {
    int region_floats = 0;
    const size_t smem = match_sliding_smem(job, &region_floats);
    cudaError_t e = cudaFuncSetAttribute(bm3d_match_sliding_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int tiles = ((job.nbx + kTileBX - 1) / kTileBX) * ((job.nby + kTileBY - 1) / kTileBY);
    bm3d_match_sliding_kernel<<<tiles, kMatchThreads, smem, stream>>>(job, region_floats);
    return cudaGetLastError();
}

}  // namespace vsfeel
