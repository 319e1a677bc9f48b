// Block matching for radius < 3: the reference's sliding column scan
// (src/bm3d.comp:479-538 spatial, 540-637 temporal), restructured for sm_100a.
//
// A CTA owns a tile of 8x4 reference blocks, 8 lanes per block; a warp holds
// four blocks of one block row, two block columns apart. For each search
// phase (the spatial window in frame m, then one temporal step per frame) the
// CTA stages the frame region that every window of the tile can reach
// (tile +- bm_range + t*ps_range) in shared memory once (cp.async),
// row-major (the exact scan for radius >= 3 stages it column-major).
//
// Scan. Within a block, lane s takes a chunk of K consecutive candidate rows
// of a window and sweeps the window's columns left to right, two columns
// per iteration: the K+7 source rows of columns X, X+1 are K+7 8-byte pairs,
// and the column sums
//     V(X) = SSD(source column X, block column min(X - left, 7))
// of X and X+1 run in the two halves of f32x2 registers. Per row the
// reduction tree of the reference advances in incremental form:
// P(j) = V(j) + V(j+1), Q(j) = P(j) + P(j+2), E(j) = Q(j) + Q(j+4) --
// the same additions on the same operands as
// ((c0+c1)+(c2+c3))+((c4+c5)+(c6+c7)), so every candidate error carries the
// reference's bits. Every error is stored to the block's error table in
// shared memory; the lane also keeps each row's three smallest errors.
//
// Selection. The reference keeps per-lane sorted top-8 lists and merges them
// by (error, scan index); the result is the 8 smallest (error, index) keys.
// Here the block's 8 lanes bound the 8th smallest error by the 8th smallest
// of the window rows' three smallest errors, collect the few candidates at or
// below the bound from the table, and place each by counting the collected
// keys below it. The scan itself carries no branches or votes.
//
// Tile shapes. The tile is TX x TY blocks (32 or 16 groups, 256 or 128
// threads); warp w holds four blocks of one block row, TX/4 columns apart.
// Smaller tiles stage smaller regions, so configurations whose 8x4 region
// and error tables exceed shared memory (block_step 8 with a temporal
// search) still take this kernel. The batched form's autotuner picks the
// shape per shape class.
//
// Modes. kTableOnly writes the block's match table; kFused filters the
// tile's groups right after matching (bm3d_filter.cuh) and scatters them,
// so no match table goes through global memory and the filter's atomics
// overlap other tiles' matching; kFusedSave does both and records the
// filter's keep bits (the differentiable form's saved state).
//
// The persistent form (bm3d_batch_tile_kernel) runs the same tile body over
// a device work queue of (stack, tile) items spanning many stacks of many
// clips: each CTA pulls the next item with one atomic add until the queue
// is exhausted.
#pragma once

#include "bm3d_device.cuh"
#include "bm3d_filter.cuh"

#include <algorithm>

namespace vsfeel {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMinK = 2, kMaxK = 5;
constexpr int kCollect = 64;                // candidates a block collects per pass
constexpr int kLaneChunks = 4;              // chunks with hits a lane notes (first pass)
constexpr int kMaxSelectPasses = 64;        // bound tightenings before a table is deemed corrupt
constexpr uint64_t kKeyMax = (uint64_t(0x7f7fffffu) << 32) | 0x7fffffffu;  // (FLT_MAX, INT_MAX)

__device__ __forceinline__ uint64_t make_key(float err, int seq) {
    return (uint64_t(__float_as_uint(err)) << 32) | uint32_t(seq);
}

__device__ __forceinline__ float key_err(uint64_t k) { return __uint_as_float(uint32_t(k >> 32)); }

// floor(f / d) for 0 <= f < 2^21 and 1 <= d < 2^24, exactly: (f + 0.5)
// times the correctly rounded reciprocal of d, truncated. The relative
// error stays below 2^-23, less than the distance 0.5 / (f + 0.5) from
// (f + 0.5) / d to an integer, so the truncation is the integer quotient.
// The tiled kernels divide table indices and scan indices, which stay below
// 2^21 (tile_shape_fits sends larger windows to the direct-read kernel).
__device__ __forceinline__ int div_small(int f, int d) {
    return (int)__fmul_rn(__fadd_rn((float)f, 0.5f), __frcp_rn((float)d));
}

// the sliding kernel divides with div_small; the exact kernel (whose few
// divisions sit off its critical path) keeps the integer division
template <bool kExact>
__device__ __forceinline__ int qdiv(int f, int d) {
    return kExact ? f / d : div_small(f, d);
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) v = max(v, __shfl_xor_sync(kFull, v, off));
    return v;
}

// A search window: candidate columns left..left+rw-1, rows top..top+h-1,
// scan indices seq_base + (cy-top)*rw + (cx-left); its errors sit in the
// block's table at eoff + (cx-left)*h + (cy-top).
struct Window {
    int left, top, rw, h, seq_base, eoff;
};

__device__ __forceinline__ Window make_window(int cx, int cy, int range, int width, int height,
                                              int seq_base, int eoff) {
    Window w;
    w.left = max(cx - range, 0);
    const int right = min(cx + range, width - 8);
    w.top = max(cy - range, 0);
    const int bottom = min(cy + range, height - 8);
    w.rw = right - w.left + 1;
    w.h = bottom - w.top + 1;
    w.seq_base = seq_base;
    w.eoff = eoff;
    return w;
}

// The staged region. The exact scan stages it column-major with column
// stride cs (odd), so the K+7 source rows a lane needs at one column are
// consecutive words. The sliding scan stages it row-major with row stride
// rs (even, 2 mod 4, one column of padding), so the columns X and X+1 of a
// row (X even) form one 8-byte pair.
struct Region {
    const float* smem;
    int rx0, ry0, cs;
    int rx1, ry1;  // last staged column and row
    int rs;
};

__host__ __device__ inline int row_stride(int w) {
    int rs = (w + 2) & ~1;
    if ((rs & 3) == 0) rs += 2;
    return rs;
}

__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

// Two independent round-to-nearest float additions, one per half.
__device__ __forceinline__ unsigned long long add_f32x2(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// One lane's chunk: rows r0..r0+nrows-1 of window `win` (nrows may be 0),
// `jcount` column steps (warp-uniform; steps past the window's width are
// padding). cur_s: the block's 64 values in shared memory, column-major; c7:
// block column 7 in registers. Errors go to table E; each row's three smallest
// errors are merged into lb, this lane's 8 smallest such values (ascending).
//
// The sweep takes two steps at a time: source columns X and X+1 (X even in
// the row-major region; a window starting at an odd column starts one
// column early, on a step whose sums no candidate uses) are one 8-byte pair
// per row, and V(j), V(j+1) are the two halves of one f32x2 register, each
// half running the scalar even-row and odd-row chains against block columns
// min(j, 7) and min(j+1, 7). Per row the tree then advances two candidates
// on the reference's operands: P(j-1) = V(j-1) + V(j), P(j) = V(j) + V(j+1),
// Q(j-3) = P(j-3) + P(j-1), Q(j-2) = P(j-2) + P(j), E(j-7) = Q(j-7) + Q(j-3),
// E(j-6) = Q(j-6) + Q(j-2).
template <int K>
__device__ __forceinline__ void scan_chunk(const Region& reg, const float* cur_s, const float c7[8],
                                           const Window& win, int r0, int nrows, int jcount,
                                           float* E, float lb[8]) {
    using u64 = unsigned long long;
    float m1[K], m2[K], m3[K];
    float vprev[K], pa[K], pb[K], qa[K][2], qb[K][2];
#pragma unroll
    for (int q = 0; q < K; ++q) {
        m1[q] = m2[q] = m3[q] = kFltMax;
        vprev[q] = pa[q] = pb[q] = 0.0f;
        qa[q][0] = qa[q][1] = qb[q][0] = qb[q][1] = 0.0f;
    }
    const int xs = win.left - reg.rx0;    // the window's first source column
    const int jst = -(xs & 1);            // first step: an even column
    const int xlast = (xs + win.rw + 6) & ~1;  // last pair holding a needed column
    // rows past the window exist in the region (padding) and only feed masked rows
    const float* rbase = reg.smem + (r0 - reg.ry0) * reg.rs;
    const int rs = reg.rs;
    float* ecol = E + win.eoff + (r0 - win.top);
    const int npairs = (jcount + 2) >> 1;

    auto emit = [&](float e, int q, int d) {
        if (q < nrows && d >= 0 && d < win.rw) {
            ecol[d * win.h + q] = e;
            m3[q] = fminf(m3[q], fmaxf(m2[q], e));
            m2[q] = fminf(m2[q], fmaxf(m1[q], e));
            m1[q] = fminf(m1[q], e);
        }
    };
    // iteration t: steps j = jst + 2t and j + 1 against the block pairs b
    auto step = [&](int t, const u64 b[8], int ring) {
        const int j = jst + 2 * t;
        const int X = min(xs + j, xlast);
        u64 w[K + 7];
#pragma unroll
        for (int k = 0; k < K + 7; ++k) w[k] = *reinterpret_cast<const u64*>(rbase + k * rs + X);
#pragma unroll
        for (int q = 0; q < K; ++q) {
            u64 ev = 0ull, od = 0ull;  // {+0.0f, +0.0f}
#pragma unroll
            for (int i = 0; i < 8; i += 2) {
                u64 d;
                asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(b[i]), "l"(w[q + i]));
                asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(ev) : "l"(d), "l"(ev));
                asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(b[i + 1]), "l"(w[q + i + 1]));
                asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(od) : "l"(d), "l"(od));
            }
            u64 v;
            asm("add.rn.f32x2 %0, %1, %2;" : "=l"(v) : "l"(ev), "l"(od));
            float va, vb;
            asm("mov.b64 {%0, %1}, %2;" : "=f"(va), "=f"(vb) : "l"(v));
            // (the tree in scalar form: as f32x2 pairs it measured 2% slower,
            // the pairs {V(j-1), V(j)} need packing moves)
            const float p_a = __fadd_rn(vprev[q], va);  // P(j-1)
            const float p_b = __fadd_rn(va, vb);        // P(j)
            const float q_a = __fadd_rn(pa[q], p_a);    // Q(j-3)
            const float q_b = __fadd_rn(pb[q], p_b);    // Q(j-2)
            const float e_a = __fadd_rn(qa[q][ring], q_a);  // E(j-7)
            const float e_b = __fadd_rn(qb[q][ring], q_b);  // E(j-6)
            vprev[q] = vb;
            pa[q] = p_a;
            pb[q] = p_b;
            qa[q][ring] = q_a;
            qb[q][ring] = q_b;
            emit(e_a, q, j - 7);
            emit(e_b, q, j - 6);
        }
    };

    // warm-up: iterations 0..3 cover steps up to 7 (block columns j, j+1,
    // clamped to 0..7, per lane as its first step is 0 or -1)
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int ca = max(jst + 2 * t, 0), cb = jst + 2 * t + 1;
        u64 b[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) b[i] = pack_f32x2(cur_s[ca * 8 + i], cur_s[cb * 8 + i]);
        step(t, b, t & 1);
    }
    // steady state: block column 7 in both halves
    u64 b7[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) b7[i] = pack_f32x2(c7[i], c7[i]);
    for (int t0 = 4; t0 < npairs; t0 += 2) {
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (t0 + u < npairs) step(t0 + u, b7, u);
    }
    // merge the rows' three smallest into the lane's 8 smallest (three per
    // row bound the 8th smallest tighter than two, so fewer candidates pass
    // the selection's bound; a fourth costs more than it saves): a bitonic
    // sorting network over the 3K values, then one bitonic merge with lb --
    // a few parallel stages instead of a dependent chain of insertions
    constexpr int N = 3 * K > 8 ? 16 : 8;
    float v[N];
#pragma unroll
    for (int i = 0; i < N; ++i)
        v[i] = i < K ? m1[i] : (i < 2 * K ? m2[i - K] : (i < 3 * K ? m3[i - 2 * K] : kFltMax));
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int jj = k >> 1; jj > 0; jj >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int l = i ^ jj;
                if (l > i) {
                    const float a = v[i], b = v[l];
                    const bool up = (i & k) == 0;
                    v[i] = up ? fminf(a, b) : fmaxf(a, b);
                    v[l] = up ? fmaxf(a, b) : fminf(a, b);
                }
            }
    // the 8 smallest of both ascending lists form a bitonic sequence ...
#pragma unroll
    for (int i = 0; i < 8; ++i) lb[i] = fminf(lb[i], v[7 - i]);
    // ... which three compare-exchange levels sort
#pragma unroll
    for (int dd = 4; dd > 0; dd >>= 1)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if ((i & dd) == 0) {
                const float a = lb[i], b = lb[i + dd];
                lb[i] = fminf(a, b);
                lb[i + dd] = fmaxf(a, b);
            }
}

// Exact scan (radius >= 3, src/bm3d.comp:512-526): candidate cx (relative
// to the window's left column) has the true 8x8 SSD
//     E = ((S0 + S1) + (S2 + S3)) + ((S4 + S5) + (S6 + S7)),
//     S_c = SSD(source column left + cx + c, block column c),
// each column SSD in the reference's even/odd order. Step j loads source
// column left + j and computes S_c for the 8 block columns; S_c belongs to
// candidate j - c. Per row the tree advances incrementally on the
// reference's operands: P01(j-1) = S0(j-1) + S1(j), P23(j-3) = S2(j-1) +
// S3(j), P45(j-5) = S4(j-1) + S5(j), P67(j-7) = S6(j-1) + S7(j),
// Q0123(j-3) = P01(j-3) + P23(j-3), Q4567(j-7) = P45(j-7) + P67(j-7),
// E(j-7) = Q0123(j-7) + Q4567(j-7). The block is read from shared memory
// once per step and used for all K rows. With 136 flops per candidate
// the selection is cheap next to the scan, so there is no error table: each
// candidate's (error, scan index) key goes straight into the lane's sorted
// top-8 (top, ascending), and the 8 lane lists are merged afterwards.
__device__ __forceinline__ void insert_key(uint64_t top[8], uint64_t key) {
    if (key < top[7]) {
#pragma unroll
        for (int k = 7; k > 0; --k) {
            const bool shift = key < top[k - 1];
            top[k] = shift ? top[k - 1] : (key < top[k] ? key : top[k]);
        }
        top[0] = key < top[0] ? key : top[0];
    }
}

// The column sums run two block columns at a time, c and c + 4, as the two
// halves of one f32x2 register: each half subtracts the same source value
// (duplicated into both halves) from its own block column and accumulates
// its own even-row and odd-row chain, so every sum carries exactly the
// scalar bits; cur_p holds the block's values interleaved that way,
// cur_p[2 * (8 * cp + i) + h] = block column cp + 4h, row i. The tree runs on
// the same pairs: {P01, P45} = {S0, S4}(j-1) + {S1, S5}(j), {P23, P67} =
// {S2, S6}(j-1) + {S3, S7}(j), {Q0123, Q4567} = {P01, P45} + {P23, P67}.

template <int K>
__device__ __forceinline__ void scan_chunk_exact(const Region& reg, const float* cur_p,
                                                 const Window& win, int r0, int nrows, int jcount,
                                                 uint64_t top[8]) {
    using u64 = unsigned long long;
    u64 s04p[K], s26p[K];  // {S0, S4} and {S2, S6} of the previous step
    u64 p0145[K][2];       // {P01, P45}, made two steps ago and one step ago
    float q0123[K][4];     // Q0123, made up to four steps ago
#pragma unroll
    for (int q = 0; q < K; ++q) {
        s04p[q] = s26p[q] = 0ull;
        p0145[q][0] = p0145[q][1] = 0ull;
#pragma unroll
        for (int i = 0; i < 4; ++i) q0123[q][i] = 0.0f;
    }
    const int xmax = win.left + win.rw + 6;
    const float* sbase = reg.smem + (r0 - reg.ry0) - reg.rx0 * reg.cs;
    const int cs = reg.cs;
    const int seq0 = win.seq_base + (r0 - win.top) * win.rw;
    const u64* bpair = reinterpret_cast<const u64*>(cur_p);

    // step j (ring positions u = j mod 4); in the first four steps (head)
    // the pairs with cp > j feed no candidate (S_c belongs to candidate
    // j - c < 0) and are skipped -- statically, as those steps are peeled
    auto step = [&](const int j, const int u, const bool head) {
        {
            u64 wd[K + 7];  // source values, each in both halves
            {
                const float* col = sbase + min(win.left + j, xmax) * cs;
#pragma unroll
                for (int k = 0; k < K + 7; ++k) wd[k] = pack_f32x2(col[k], col[k]);
            }
            u64 S[K][4];  // {S_cp, S_cp+4}
#pragma unroll
            for (int cp = 0; cp < 4; ++cp) {
                if (head && cp > u) {
#pragma unroll
                    for (int q = 0; q < K; ++q) S[q][cp] = 0ull;
                    continue;
                }
                u64 b[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) b[i] = bpair[8 * cp + i];
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    u64 ev = 0ull, od = 0ull;  // {+0.0f, +0.0f}
#pragma unroll
                    for (int i = 0; i < 8; i += 2) {
                        u64 d;
                        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(b[i]), "l"(wd[q + i]));
                        asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(ev) : "l"(d), "l"(ev));
                        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(b[i + 1]), "l"(wd[q + i + 1]));
                        asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(od) : "l"(d), "l"(od));
                    }
                    S[q][cp] = add_f32x2(ev, od);
                }
            }
            float e[K];
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const u64 np0145 = add_f32x2(s04p[q], S[q][1]);  // {P01, P45}(j-1), (j-5)
                const u64 np2367 = add_f32x2(s26p[q], S[q][3]);  // {P23, P67}(j-3), (j-7)
                // P01(j-3) and P45(j-7) were made two steps ago, Q0123(j-7) four
                const u64 nq = add_f32x2(p0145[q][u & 1], np2367);  // {Q0123(j-3), Q4567(j-7)}
                float nq0123, nq4567;
                asm("mov.b64 {%0, %1}, %2;" : "=f"(nq0123), "=f"(nq4567) : "l"(nq));
                e[q] = __fadd_rn(q0123[q][u & 3], nq4567);
                p0145[q][u & 1] = np0145;
                q0123[q][u & 3] = nq0123;
                s04p[q] = S[q][0];
                s26p[q] = S[q][2];
            }
            const int d = j - 7;
            if (d >= 0 && d < win.rw && j < jcount) {
#pragma unroll
                for (int q = 0; q < K; ++q)
                    // errors at or above FLT_MAX never count (src/bm3d.comp:284-302)
                    if (q < nrows && e[q] < kFltMax)
                        insert_key(top, make_key(e[q], seq0 + q * win.rw + d));
            }
        }
    };
#pragma unroll
    for (int u = 0; u < 4; ++u) step(u, u, true);
    // steps past jcount (the rest of the last group of four) would only feed
    // candidates right of every window of the warp: skipped (warp-uniform)
    for (int j0 = 4; j0 < jcount; j0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (j0 + u < jcount) step(j0 + u, u, false);
    }
}

// Rows per lane of the sliding scan: the lanes of a block share its window
// rows; 16 lanes per block carry at most 3 rows each (the 512-thread form
// runs at 128 registers per thread).
template <int kLanes>
__device__ __forceinline__ int rows_per_lane(int total_rows) {
    constexpr int kMax = kLanes == 8 ? kMaxK : 3;
    return min(kMax, max(kMinK, (total_rows + kLanes - 1) / kLanes));
}

// A block's global match list, spatial predictors, the phase's top-8 and the
// collection buffer (src/bm3d.comp:469-470, 541-545, 622-633).
struct GroupState {
    float ge[8];
    uint32_t gxy[8];
    int gz[8];
    uint32_t sxy[8];
    uint32_t pxy[8];
    uint64_t top[8];
    uint64_t buf[kCollect];
    int count;
};

// The 8 smallest keys of the group's 8 sorted lane lists, into gs->top.
__device__ __forceinline__ void merge_top8(uint64_t top[8], GroupState* gs, unsigned gmask) {
    const int sub = threadIdx.x & 7;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        uint64_t best = top[0];
        int src = sub;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
            const uint64_t o = __shfl_xor_sync(gmask, best, off);
            const int os = __shfl_xor_sync(gmask, src, off);
            const bool take = o < best || (o == best && os < src);
            best = take ? o : best;
            src = take ? os : src;
        }
        if (sub == 0) gs->top[r] = best;
        if (sub == src) {
#pragma unroll
            for (int i = 0; i < 7; ++i) top[i] = top[i + 1];
            top[7] = kKeyMax;
        }
    }
    __syncwarp(gmask);
}


// The 8 smallest (error, scan index) keys of the windows' error table into
// gs->top (padded with (FLT_MAX, INT_MAX) when fewer exist; errors >= FLT_MAX
// never count, as in the reference). lb: this lane's 8 smallest per-row
// minima (ascending). All 8 lanes of the group take part.
template <int kLanes>
__device__ void select_top8(const float* E, const Window* wins, int nwin, float lb[8],
                            GroupState* gs, unsigned gmask, int* status) {
    const int sub = threadIdx.x & (kLanes - 1);
    // bound: the 8th smallest of the rows' three smallest errors -- at least 8
    // candidates lie at or below it. Each lane's list is sorted; three
    // bitonic merge stages with the lanes 1, 2 and 4 apart leave every lane
    // with the group's 8 smallest, sorted.
#pragma unroll
    for (int off = 1; off < kLanes; off <<= 1) {
        float o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = __shfl_xor_sync(gmask, lb[i], off);
        // the 8 smallest of both lists form a bitonic sequence ...
#pragma unroll
        for (int i = 0; i < 8; ++i) lb[i] = fminf(lb[i], o[7 - i]);
        // ... which three compare-exchange levels sort
#pragma unroll
        for (int d = 4; d > 0; d >>= 1)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if ((i & d) == 0) {
                    const float a = lb[i], b = lb[i + d];
                    lb[i] = fminf(a, b);
                    lb[i + d] = fmaxf(a, b);
                }
    }
    const float bound = lb[7];
    uint64_t tkey = (uint64_t(__float_as_uint(bound)) << 32) | 0xffffffffu;
    int n = 0;
    // First pass: the sweep only notes, per lane, which chunks of 16 entries
    // hold hits (errors at or below the bound) and a hit bitmask for each --
    // no branch per entry; afterwards every lane expands its noted chunks in
    // one loop, so the hits of different lanes are handled together, and the
    // keys are placed by a prefix sum over the group. A group with a lane of
    // more than kLaneChunks such chunks, or more than kCollect hits in all,
    // takes the general loop below (rare).
    bool fast = false;
    {
        const float terr = bound;
        uint32_t ch[kLaneChunks], cm[kLaneChunks];
#pragma unroll
        for (int i = 0; i < kLaneChunks; ++i) ch[i] = cm[i] = 0u;
        int nc = 0;
        for (int wi = 0; wi < nwin; ++wi) {
            const Window w = wins[wi];
            const int n_w = w.rw * w.h;
            const int nq = (n_w + 3) >> 2;
            const float4* tab = reinterpret_cast<const float4*>(E + w.eoff);
            for (int v0 = 0; v0 < nq; v0 += 4 * kLanes) {
                float4 q[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int v = v0 + sub + kLanes * k;
                    q[k] = v < nq ? tab[v] : make_float4(kFltMax, kFltMax, kFltMax, kFltMax);
                }
                float mn = kFltMax;
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    mn = fminf(mn, fminf(fminf(q[k].x, q[k].y), fminf(q[k].z, q[k].w)));
                if (!(mn <= terr)) continue;
                uint32_t mask = 0u;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float ev[4] = {q[k].x, q[k].y, q[k].z, q[k].w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int f = 4 * (v0 + sub + kLanes * k) + u;
                        const bool hit = f < n_w && ev[u] <= terr && ev[u] < kFltMax;
                        mask |= hit ? (1u << (4 * k + u)) : 0u;
                    }
                }
                if (mask) {
#pragma unroll
                    for (int i = 0; i < kLaneChunks; ++i) {
                        ch[i] = i == nc ? (uint32_t(wi) << 24) | uint32_t(v0) : ch[i];
                        cm[i] = i == nc ? mask : cm[i];
                    }
                    ++nc;
                }
            }
        }
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kLaneChunks; ++i) cnt += __popc(cm[i]);
        int incl = cnt;
#pragma unroll
        for (int off = 1; off < kLanes; off <<= 1) {
            const int t = __shfl_up_sync(gmask, incl, off, kLanes);
            if (sub >= off) incl += t;
        }
        const int total = __shfl_sync(gmask, incl, kLanes - 1, kLanes);
        const bool overflow = __any_sync(gmask, nc > kLaneChunks) || total > kCollect;
        if (!overflow) {
            int pos = incl - cnt;
#pragma unroll
            for (int i = 0; i < kLaneChunks; ++i) {
                uint32_t m = cm[i];
                const Window w = wins[ch[i] >> 24];
                const int v0 = int(ch[i] & 0xffffffu);
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    const int f = 4 * (v0 + sub + kLanes * (b >> 2)) + (b & 3);
                    const int d = div_small(f, w.h);
                    const int row = f - d * w.h;
                    gs->buf[pos++] = make_key(E[w.eoff + f], w.seq_base + row * w.rw + d);
                }
            }
            n = total;
            fast = true;
        }
        __syncwarp(gmask);
    }
    // every pass at least shrinks the set of keys at or below the bound
    // (errors are sums of squares, never negative); the cap only guards
    // against a corrupted table, and reports it
    for (int pass = 0; !fast; ++pass) {
        if (pass == kMaxSelectPasses) {
            if (sub == 0) atomicOr(status, 2);
            n = kCollect;
            break;
        }
        if (sub == 0) gs->count = 0;
        __syncwarp(gmask);
        const float terr = key_err(tkey);
        const uint32_t tseq = uint32_t(tkey);
        // a window's table is rw*h contiguous words from a 4-aligned offset.
        // A group step covers 32 float4 (128 entries), four loads in flight
        // per lane; nearly every chunk of 16 entries lies above the bound and
        // costs one comparison of its minimum (entries past the window in its
        // last float4 only send a chunk down the exact path, which skips them)
        for (int wi = 0; wi < nwin; ++wi) {
            const Window w = wins[wi];
            const int n_w = w.rw * w.h;
            const int nq = (n_w + 3) >> 2;
            const float4* tab = reinterpret_cast<const float4*>(E + w.eoff);
            for (int v0 = 0; v0 < nq; v0 += 4 * kLanes) {
                float4 q[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int v = v0 + sub + kLanes * k;
                    q[k] = v < nq ? tab[v] : make_float4(kFltMax, kFltMax, kFltMax, kFltMax);
                }
                float mn = kFltMax;
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    mn = fminf(mn, fminf(fminf(q[k].x, q[k].y), fminf(q[k].z, q[k].w)));
                if (!(mn <= terr)) continue;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float ev[4] = {q[k].x, q[k].y, q[k].z, q[k].w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int f = 4 * (v0 + sub + kLanes * k) + u;
                        if (f < n_w && ev[u] <= terr && ev[u] < kFltMax) {
                            const int d = div_small(f, w.h);
                            const int row = f - d * w.h;
                            const uint32_t seq = uint32_t(w.seq_base + row * w.rw + d);
                            if (ev[u] < terr || seq <= tseq) {
                                const int pos = atomicAdd(&gs->count, 1);
                                if (pos < kCollect) gs->buf[pos] = make_key(ev[u], int(seq));
                            }
                        }
                    }
                }
            }
        }
        __syncwarp(gmask);
        n = gs->count;
        if (n <= kCollect) break;
        // more than kCollect at or below the bound: tighten it to the 8th
        // smallest key among the collected ones and collect again
        uint64_t t8 = kKeyMax;
        for (int j = sub; j < kCollect; j += kLanes) {
            const uint64_t kj = gs->buf[j];
            int rank = 0;
            for (int i = 0; i < kCollect; ++i) rank += gs->buf[i] < kj ? 1 : 0;
            if (rank == 7) t8 = kj;
        }
#pragma unroll
        for (int off = 1; off < kLanes; off <<= 1) {
            const uint64_t o = __shfl_xor_sync(gmask, t8, off);
            t8 = o < t8 ? o : t8;
        }
        tkey = t8;
        __syncwarp(gmask);
    }
    if (n <= 2 * kLanes) {
        // up to two keys per lane, ranked by shuffles (the keys are distinct:
        // every candidate of a phase has its own scan index)
        const uint64_t k0 = sub < n ? gs->buf[sub] : kKeyMax;
        const uint64_t k1 = sub + kLanes < n ? gs->buf[sub + kLanes] : kKeyMax;
        int r0 = 0, r1 = 0;
#pragma unroll
        for (int j = 0; j < kLanes; ++j) {
            const uint64_t o0 = __shfl_sync(gmask, k0, j, kLanes);
            const uint64_t o1 = __shfl_sync(gmask, k1, j, kLanes);
            r0 += (o0 < k0 ? 1 : 0) + (o1 < k0 ? 1 : 0);
            r1 += (o0 < k1 ? 1 : 0) + (o1 < k1 ? 1 : 0);
        }
        if (sub < 8) gs->top[sub] = kKeyMax;
        __syncwarp(gmask);
        if (sub < n && r0 < 8) gs->top[r0] = k0;
        if (sub + kLanes < n && r1 < 8) gs->top[r1] = k1;
        __syncwarp(gmask);
    } else {
        if (sub < 8) gs->top[sub] = kKeyMax;
        __syncwarp(gmask);
        for (int j = sub; j < n; j += kLanes) {
            const uint64_t kj = gs->buf[j];
            int rank = 0;
            for (int i = 0; i < n; ++i) rank += gs->buf[i] < kj ? 1 : 0;
            if (rank < 8) gs->top[rank] = kj;
        }
        __syncwarp(gmask);
    }
}

// Scans windows[0..nwin) of this lane's block into its error table, then
// selects the top-8 into gs->top. Rows are split into chunks of K
// (warp-uniform); chunk c of the block goes to lane c % 8 in round c / 8.
// after_scan() runs on every thread of the CTA once its warp has scanned,
// before the selection, which reads the tables but not the staged region
// (the caller stages the next phase's region there).
template <bool kExact, int kLanes, class AfterScan>
__device__ void search_windows(const Region& reg, const float* cur_s, const float c7[8],
                               const Window* wins, int nwin, float* E, GroupState* gs,
                               unsigned gmask, int* status, bool probe,
                               const AfterScan& after_scan) {
    static_assert(kLanes == 8 || (kLanes == 16 && !kExact), "16 lanes: sliding scan only");
    const int sub = threadIdx.x & (kLanes - 1);
    int total_rows = 0;
    for (int i = 0; i < nwin; ++i) total_rows += wins[i].h;
    // the exact scan keeps 8 column sums per row: 2 rows per lane, so that
    // its kernel fits 128 registers and two CTAs (16 warps) share an SM
    // (11.7% faster per 1080p r4 stack than 2 or 3 rows at one CTA per SM)
    int K;
    if (kExact)
        K = 2;
    else
        K = warp_max(rows_per_lane<kLanes>(total_rows));
    int ntasks = 0;
    for (int i = 0; i < nwin; ++i) ntasks += qdiv<kExact>(wins[i].h + K - 1, K);
    const int rounds = warp_max((ntasks + kLanes - 1) / kLanes);
    float lb[8];
    uint64_t top[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        lb[i] = kFltMax;
        top[i] = kKeyMax;
    }
    for (int round = 0; round < rounds; ++round) {
        const int task = round * kLanes + sub;
        const bool has = task < ntasks;
        int wi = 0, c = has ? task : 0;
        while (wi < nwin - 1 && c >= qdiv<kExact>(wins[wi].h + K - 1, K)) {
            c -= qdiv<kExact>(wins[wi].h + K - 1, K);
            ++wi;
        }
        Window win = wins[wi];
        int r0 = win.top + c * K;
        int nrows = has ? min(K, win.h - c * K) : 0;
        // every window lies inside the staged region by construction (the
        // host routes configurations that could place one outside to the
        // direct-read kernel); should one not, scan nothing here and report
        // (`probe`: the host's test hook makes this tile report)
        if (probe || win.left < reg.rx0 || win.left + win.rw + 6 > reg.rx1 || win.top < reg.ry0 ||
            win.top + win.h + 6 > reg.ry1) {
            if (has) atomicOr(status, 1);
            win = Window{reg.rx0, reg.ry0, 1, 1, 0, 0};
            r0 = reg.ry0;
            nrows = 0;
        }
        const int jcount = warp_max(has ? win.rw + 7 : 8);
        if (kExact) {
            // E: the block interleaved by column pairs (see scan_chunk_exact)
            scan_chunk_exact<2>(reg, E, win, r0, nrows, jcount, top);
        } else if (kLanes == 16) {
            if (K == 2)
                scan_chunk<2>(reg, cur_s, c7, win, r0, nrows, jcount, E, lb);
            else
                scan_chunk<3>(reg, cur_s, c7, win, r0, nrows, jcount, E, lb);
        } else {
            switch (K) {
                case 2: scan_chunk<2>(reg, cur_s, c7, win, r0, nrows, jcount, E, lb); break;
                case 3: scan_chunk<3>(reg, cur_s, c7, win, r0, nrows, jcount, E, lb); break;
                case 4: scan_chunk<4>(reg, cur_s, c7, win, r0, nrows, jcount, E, lb); break;
                default: scan_chunk<5>(reg, cur_s, c7, win, r0, nrows, jcount, E, lb); break;
            }
        }
    }
    __syncwarp(gmask);
    after_scan();
    // a window that was not scanned leaves stale values in the table; the
    // selection still ends (its pass limit) on in-range positions, and the
    // host reports the status word
    if constexpr (kExact)
        merge_top8(top, gs, gmask);
    else
        select_top8<kLanes>(E, wins, nwin, lb, gs, gmask, status);
}

// Position of a key. Sentinels decode to (0, 0) as in the reference.
template <bool kExact>
__device__ __forceinline__ uint32_t key_xy(uint64_t key, const Window* wins, int area) {
    if (key == kKeyMax) return 0u;
    const int seq = int(uint32_t(key));
    const int wi = area > 0 ? qdiv<kExact>(seq, area) : 0;
    const Window w = wins[wi];
    const int rem = seq - w.seq_base;
    const int dy = qdiv<kExact>(rem, w.rw);
    const int dx = rem - dy * w.rw;
    return uint32_t(w.left + dx) | (uint32_t(w.top + dy) << 16);
}

// Stages frame rows [ry0, ry1] x columns [rx0, rx1] into smem, column-major
// with column stride cs (odd, so the transposing stores of a warp hit
// distinct banks). Global reads are coalesced along rows. The copies are
// asynchronous (cp.async, 4 bytes each) and only issued here: a thread
// issues all of its copies, and the caller waits once (cp.async.wait_all)
// and synchronises the CTA before the region is read, so the L2 latency of
// the region is paid about once, and can overlap other work meanwhile.
__device__ void stage_region(float* smem, const float* __restrict__ frame, int pitch, int rx0,
                             int ry0, int rx1, int ry1, int cs) {
    const int w = rx1 - rx0 + 1;
    const int h = ry1 - ry0 + 1;
    const int lane = threadIdx.x & 31;
    for (int yy = threadIdx.x >> 5; yy < h; yy += blockDim.x >> 5) {
        const float* __restrict__ row = frame + (size_t)(ry0 + yy) * pitch + rx0;
        for (int xx = lane; xx < w; xx += 32) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(smem + xx * cs + yy);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(row + xx)
                         : "memory");
        }
    }
}

// The same region row-major with row stride rs (the sliding scan). The
// copies are issued right after the barrier that frees the region, on every
// warp's path to its selection (about 9% of a 1080p radius-2 launch with
// 4-byte copies), so when the source rows allow it (frame 8-byte aligned,
// even pitch, even first column -- region_of starts the sliding scan's
// region on an even column) each copy moves a column pair: 8-byte copies
// over the flattened (row, pair) index, and an odd last column as a 4-byte
// copy, so nothing past column rx1 is read. Otherwise 4-byte copies.
__device__ void stage_region_rows(float* smem, const float* __restrict__ frame, int pitch, int rx0,
                                  int ry0, int rx1, int ry1, int rs) {
    const int w = rx1 - rx0 + 1;
    const int h = ry1 - ry0 + 1;
    if (((reinterpret_cast<uintptr_t>(frame) & 7) | (pitch & 1) | (rx0 & 1)) == 0) {
        const int npr = w >> 1, total = h * npr, nt = blockDim.x;
        if (npr > 0) {
            const int row = threadIdx.x / npr;
            int pr = threadIdx.x - row * npr;
            const int dr = nt / npr, dp = nt - dr * npr;
            const float* src = frame + (size_t)(ry0 + row) * pitch + rx0 + 2 * pr;
            unsigned dst = (unsigned)__cvta_generic_to_shared(smem + row * rs + 2 * pr);
            const ptrdiff_t src_step = (ptrdiff_t)dr * pitch + 2 * dp, src_wrap = pitch - 2 * npr;
            const unsigned dst_step = 4u * (dr * rs + 2 * dp), dst_wrap = 4u * (rs - 2 * npr);
            for (int i = threadIdx.x; i < total; i += nt) {
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src)
                             : "memory");
                pr += dp;
                src += src_step;
                dst += dst_step;
                if (pr >= npr) {
                    pr -= npr;
                    src += src_wrap;
                    dst += dst_wrap;
                }
            }
        }
        if (w & 1)
            for (int yy = threadIdx.x; yy < h; yy += nt) {
                const float* src = frame + (size_t)(ry0 + yy) * pitch + rx1;
                const unsigned dst = (unsigned)__cvta_generic_to_shared(smem + yy * rs + (w - 1));
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src)
                             : "memory");
            }
        return;
    }
    const int lane = threadIdx.x & 31;
    for (int yy = threadIdx.x >> 5; yy < h; yy += blockDim.x >> 5) {
        const float* __restrict__ row = frame + (size_t)(ry0 + yy) * pitch + rx0;
        for (int xx = lane; xx < w; xx += 32) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(smem + yy * rs + xx);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(row + xx)
                         : "memory");
        }
    }
}

// windows a block holds at once: the spatial one, or ps_num temporal ones
__host__ __device__ inline int window_slots(const StackJob& job) {
    return job.ps_num > 1 ? job.ps_num : 1;
}

struct SmemPlan {
    int region_floats;     // staged region
    int estride;           // floats per block error table (== 8 mod 32)
    int etab_floats;       // all error tables (also the fused filter's buffers), a multiple of 4
    size_t region_offset;  // bytes from the dynamic shared memory's base to the region
    size_t bytes;
};

// The layout match_tile carves (block state, windows, reference blocks,
// tables, region) keeps the tables' float4 reads and the region's 8-byte
// reads aligned; launchers check it before every launch.
template <int TX, int TY>
__host__ inline bool smem_plan_aligned(const SmemPlan& p) {
    const size_t cur = p.region_offset - sizeof(float) * (size_t(TX * TY) * 64 + p.etab_floats);
    return cur % 16 == 0 && p.region_offset % 16 == 0;
}

__host__ __device__ inline int error_table_floats(const StackJob& job) {
    const int ws = 2 * job.bm_range + 1, wt = 2 * job.ps_range + 1;
    const int spatial = (ws * ws + 3) & ~3;
    const int temporal = job.radius > 0 ? job.ps_num * ((wt * wt + 3) & ~3) : 0;
    return spatial > temporal ? spatial : temporal;
}

// The fused modes' tile accumulator for slice r: every spatial match of the
// tile's blocks lies within bm_range of a block, so its patches cover at most
// (tile + 2 bm_range) pixels per axis (numerators), and their origins that
// less 7 (weights).
template <int TX, int TY>
__host__ __device__ inline int accumulator_floats(const StackJob& job) {
    const int tw = (TX - 1) * job.step + 8 + 2 * job.bm_range;
    const int th = (TY - 1) * job.step + 8 + 2 * job.bm_range;
    const int w = tw < job.width ? tw : job.width, h = th < job.height ? th : job.height;
    return w * h + (w - 7) * (h - 7);
}

template <int TX, int TY>
__host__ __device__ inline SmemPlan smem_plan(const StackJob& job, int mode) {
    constexpr int kGroups = TX * TY;
    SmemPlan p;
    const int reach = job.bm_range + job.radius * job.ps_range;
    const int tile_w = (TX - 1) * job.step + 8, tile_h = (TY - 1) * job.step + 8;
    const int w = tile_w + 2 * reach < job.width ? tile_w + 2 * reach : job.width;
    const int h = tile_h + 2 * reach < job.height ? tile_h + 2 * reach : job.height;
    // rows past the region that masked chunk rows read: at most kMaxK - 1;
    // column-major for the exact scan, row-major for the sliding one, whose
    // region may start one column early (an even first column)
    const int cs = (h + kMaxK - 1) | 1;
    p.region_floats = job.radius >= 3 ? cs * w : row_stride(w + 1) * (h + kMaxK - 1);
    // the exact scan (radius >= 3) selects without error tables; its table
    // area holds the block interleaved by column pairs (64 floats)
    const int tf = error_table_floats(job);
    p.estride = job.radius >= 3 ? 64 : tf + ((8 - tf) & 31);  // the least >= tf that is 8 mod 32
    p.etab_floats = kGroups * p.estride;
    // fused modes: the filter's transposes, then the slice-r accumulator
    const int fused_floats = kGroups * kGroupStride + accumulator_floats<TX, TY>(job);
    if (mode != kTableOnly && p.etab_floats < fused_floats) p.etab_floats = fused_floats;
    // the staged region follows the tables and is read as 8-byte pairs: keep
    // it on a 16-byte boundary
    p.etab_floats = (p.etab_floats + 3) & ~3;
    p.region_offset = sizeof(GroupState) * kGroups + sizeof(Window) * kGroups * window_slots(job) +
                      sizeof(float) * (size_t(kGroups) * 64 + size_t(p.etab_floats));
    p.bytes = p.region_offset + sizeof(float) * p.region_floats;
    return p;
}

// The body of one tile: matching of its TX x TY blocks, then (fused modes)
// filtering of their groups. Shared memory: block state, windows, reference
// blocks, error tables (the fused filter's buffers afterwards), then the
// staged region. Every thread of the CTA calls it.
template <int TX, int TY, int kMode, bool kExact = false, int kLanes = 8>
__device__ __forceinline__ void match_tile(const StackJob& job, int tile,
                                           unsigned char* smem_raw) {
    static_assert(kLanes == 8 || (kLanes == 16 && kMode == kTableOnly && !kExact),
                  "16 lanes per block: the sliding scan writing match tables");
    constexpr int kGroups = TX * TY;
    const SmemPlan plan = smem_plan<TX, TY>(job, kMode);
    GroupState* gs_all = reinterpret_cast<GroupState*>(smem_raw);
    Window* win_all = reinterpret_cast<Window*>(gs_all + kGroups);
    float* cur_all = reinterpret_cast<float*>(win_all + kGroups * window_slots(job));
    float* etab_all = cur_all + kGroups * 64;
    float* region = etab_all + (size_t)plan.etab_floats;

    // kLanes lanes per block (group); a warp holds kGpw groups. Lane `sub`
    // of a group holds entry sub & 7 of the block's match list (lanes 8..15
    // of a 16-lane group mirror lanes 0..7: every list operation runs in
    // 8-lane segments)
    constexpr int kGpw = 32 / kLanes;
    const int lane = threadIdx.x & 31;
    const int sub = lane & (kLanes - 1);
    const int ent = sub & 7;
    const int g = threadIdx.x / kLanes;     // group in the CTA
    const int wrp = g / kGpw, gi = g % kGpw;  // warp, group in the warp
    const unsigned gmask = (kLanes == 8 ? 0xffu : 0xffffu) << (lane & ~(kLanes - 1));
    const int tiles_x = (job.nbx + TX - 1) / TX;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    const int bx0 = tx * TX, by0 = ty * TY;
    const int bx_last = min(bx0 + TX - 1, job.nbx - 1);
    const int by_last = min(by0 + TY - 1, job.nby - 1);
    // warp wrp: block row wrp / (TX/kGpw), block columns o + (TX/kGpw) * gi
    constexpr int kWarpsPerRow = TX / kGpw;
    const int bxr = bx0 + (wrp % kWarpsPerRow) + kWarpsPerRow * gi;
    const int byr = by0 + wrp / kWarpsPerRow;
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
    const bool probe = job.probe_tile == tile + 1;

    float* cur_s = cur_all + g * 64;
    float* E = etab_all + (size_t)g * plan.estride;
    Window* win = win_all + g * window_slots(job);
    GroupState* gs = gs_all + g;
    const float* fc = job.slice_frame[r];
    if (sub < 8) {
#pragma unroll
        for (int i = 0; i < 8; ++i) cur_s[sub * 8 + i] = __ldg(fc + (size_t)(y + i) * pitch + x + sub);
    }
    __syncwarp(gmask);
    float c7[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) c7[i] = cur_s[56 + i];
    if (kExact) {
        // block column c at pair c & 3, half c >> 2 (scan_chunk_exact)
#pragma unroll
        for (int i = 0; i < 8; ++i) E[2 * (8 * (sub & 3) + i) + (sub >> 2)] = cur_s[sub * 8 + i];
        __syncwarp(gmask);
    }

    // The staged region of a search phase: the tile +- reach, clamped.
    auto region_of = [&](int reach) {
        Region s;
        const int rx0 = max(tile_x0 - reach, 0);
        const int rx1 = min(tile_x1 + reach, W - 8) + 7;
        const int ry0 = max(tile_y0 - reach, 0);
        const int ry1 = min(tile_y1 + reach, H - 8) + 7;
        // column: the region's rows plus the rows masked chunk rows may read
        // (a chunk starts at or above the window's last row and reads K + 6
        // rows below its start: at most kMaxK - 1 past the region)
        s.cs = (ry1 - ry0 + 1 + kMaxK - 1) | 1;
        // the sliding scan's region starts on an even column, so that its
        // rows are staged as column pairs (stage_region_rows)
        const int rxs = kExact ? rx0 : (rx0 & ~1);
        s.rs = row_stride(rx1 - rxs + 1);
        s.rx0 = rxs;
        s.ry0 = ry0;
        s.rx1 = rx1;
        s.ry1 = ry1;
        s.smem = region;
        return s;
    };
    // Issues the copies of a region (every thread; no wait).
    auto issue = [&](const float* frame, const Region& s) {
        if (kExact)
            stage_region(region, frame, pitch, s.rx0, s.ry0, s.rx1, s.ry1, s.cs);
        else
            stage_region_rows(region, frame, pitch, s.rx0, s.ry0, s.rx1, s.ry1, s.rs);
    };
    auto wait_region = [] {
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
    };
    // The search phases: the spatial one (phase 0, frame r), then per
    // direction dir = -1, +1 the temporal steps t = 1..r (frame r + dir t,
    // reach R + t Q). Sliding scan: once every warp of the CTA has scanned
    // phase p, the region is free, so the next phase's copies are issued
    // then and land while the warps select and update their lists (the
    // region does not depend on the predictors); the next scan waits for
    // them (1.776 against 1.813 ms per 1080p radius-2 stack). The exact
    // scan's selection is a short merge, so it stages each phase at its
    // start (overlapping cost it 0.6%).
    Region next{};
    auto stage_next = [&](int dir, int t) {
        return [&, dir, t] {
            if (kExact || t == 0) return;  // staged at the phase's start / no next phase
            __syncthreads();               // every warp has scanned: the region is free
            next = region_of(R + t * Q);
            issue(job.slice_frame[r + dir * t], next);
        };
    };

    float ge = kFltMax;
    uint32_t gxy = 0u;
    int gz = 0;

    // spatial search (src/bm3d.comp:479-538)
    __syncthreads();  // a previous tile of this CTA has finished with the region
    Region s = region_of(R);
    issue(fc, s);
    wait_region();
    {
        if (sub == 0) win[0] = make_window(x, y, R, W, H, 0, 0);
        __syncwarp(gmask);
        search_windows<kExact, kLanes>(s, cur_s, c7, win, 1, E, gs, gmask, job.status, probe,
                                       stage_next(-1, r >= 1 ? 1 : 0));
        const uint64_t k = gs->top[ent];
        const uint32_t xy = key_xy<kExact>(k, win, 0);
        // the global match list: lane `sub` holds entry sub & 7
        ge = key_err(k);
        gxy = xy;
        gz = r;
        if (sub < 8) gs->sxy[sub] = xy;
        __syncwarp(gmask);
    }

    // temporal predictive search (src/bm3d.comp:540-637)
    const int area = (2 * Q + 1) * (2 * Q + 1);
    for (int dir = -1; dir <= 1; dir += 2) {
        if (sub < 8) gs->pxy[sub] = gs->sxy[sub];
        __syncwarp(gmask);
        for (int t = 1; t <= r; ++t) {
            const int z = r + dir * t;
            if (kExact) {
                __syncthreads();  // the previous phase has finished with the region
                next = region_of(R + t * Q);
                issue(job.slice_frame[z], next);
            }
            wait_region();
            s = next;
            if (sub == 0) {
                int eoff = 0;
                for (int i = 0; i < P; ++i) {
                    const uint32_t p = gs->pxy[i];
                    win[i] = make_window(int(p & 0xffffu), int(p >> 16), Q, W, H, i * area, eoff);
                    eoff += (win[i].rw * win[i].h + 3) & ~3;  // tables start 4-aligned
                }
            }
            __syncwarp(gmask);
            // the next phase: (dir, t + 1), or (+1, 1) after the last step of
            // dir = -1, or none
            const int ndir = t < r ? dir : 1;
            const int nt = t < r ? t + 1 : (dir < 0 ? 1 : 0);
            search_windows<kExact, kLanes>(s, cur_s, c7, win, P, E, gs, gmask, job.status, probe,
                                           stage_next(ndir, nt));
            // the frame's first P matches enter the global list in order with
            // the reference's strict < (src/bm3d.comp:304-322): an entry goes
            // after the ones it does not beat; the group's lanes shift in
            // parallel
            for (int i = 0; i < P; ++i) {
                const uint64_t k = gs->top[i];
                const uint32_t fxy = key_xy<kExact>(k, win, area);
                const float err = key_err(k);
                const float e7 = __shfl_sync(gmask, ge, 7, 8);
                const unsigned below = __ballot_sync(gmask, ge <= err);
                const float pe = __shfl_up_sync(gmask, ge, 1, 8);
                const uint32_t pxy = __shfl_up_sync(gmask, gxy, 1, 8);
                const int pz = __shfl_up_sync(gmask, gz, 1, 8);
                if (err < e7) {
                    const int pos = __popc((below >> (lane & ~7)) & 0xffu);
                    if (ent > pos) {
                        ge = pe;
                        gxy = pxy;
                        gz = pz;
                    } else if (ent == pos) {
                        ge = err;
                        gxy = fxy;
                        gz = z;
                    }
                }
                if (sub == 0) gs->pxy[i] = fxy;
            }
            __syncwarp(gmask);
        }
    }

    // forced self-match (src/bm3d.comp:639-663): when (x, y, r) is not among
    // the 8, the list shifts right and it enters at slot 0
    {
        const uint32_t self_xy = uint32_t(x) | (uint32_t(y) << 16);
        const bool has_self = __any_sync(gmask, gxy == self_xy && gz == r);
        const uint32_t pxy = __shfl_up_sync(gmask, gxy, 1, 8);
        const int pz = __shfl_up_sync(gmask, gz, 1, 8);
        if (!has_self) {
            gxy = ent == 0 ? self_xy : pxy;
            gz = ent == 0 ? r : pz;
        }
        const uint32_t zp = __reduce_or_sync(gmask, sub < 8 ? uint32_t(gz) << (4 * sub) : 0u);
        if (sub < 8) gs->gxy[sub] = gxy;
        if (sub == 0) gs->gz[0] = int(zp);
        if (valid && kMode != kFused && sub < 8) {
            const size_t b = (size_t)by * job.nbx + bx;
            job.match_xy[b * 8 + sub] = gxy;
            if (sub == 0) job.match_z[b] = zp;
        }
    }

    if (kMode != kTableOnly) {
        __syncwarp(gmask);
        uint32_t mxy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) mxy[k] = gs->gxy[k];
        const uint32_t zp = uint32_t(gs->gz[0]);
        // the filter's transposes and the tile's accumulator for slice r
        // (TileAccumulator) reuse the error tables: every group of the CTA
        // must be done selecting
        TileAccumulator acc;
        acc.z = job.slice_dst[r] ? r : -1;
        acc.fx0 = max(tile_x0 - R, 0);
        acc.fy0 = max(tile_y0 - R, 0);
        acc.w = min(tile_x1 + R, W - 8) + 8 - acc.fx0;
        acc.h = min(tile_y1 + R, H - 8) + 8 - acc.fy0;
        acc.num = etab_all + (size_t)kGroups * kGroupStride;
        acc.org = acc.num + acc.w * acc.h;
        const int nacc = acc.w * acc.h + (acc.w - 7) * (acc.h - 7);
        __syncthreads();
        if (acc.z >= 0)
            for (int e = threadIdx.x; e < nacc; e += blockDim.x) acc.num[e] = 0.0f;
        __syncthreads();
        const int b = by * job.nbx + bx;
        filter_group<kMode == kFusedSave>(job, b, valid, mxy, zp, sub,
                                           etab_all + (size_t)g * kGroupStride, &acc);
        __syncthreads();
        // flush: one atomic per covered pixel and per weighted origin (zero
        // sums are skipped; adding +0.0 changes nothing)
        if (acc.z >= 0) {
            float* num = job.slice_dst[r];
            const int dp = job.dst_pitch;
            for (int e = threadIdx.x; e < acc.w * acc.h; e += blockDim.x) {
                const float v = acc.num[e];
                const int rr = e / acc.w, cc = e - rr * acc.w;
                if (v != 0.0f) red_add_global(num + (size_t)(acc.fy0 + rr) * dp + acc.fx0 + cc, v);
            }
            const int ow = acc.w - 7;
            for (int e = threadIdx.x; e < ow * (acc.h - 7); e += blockDim.x) {
                const float v = acc.org[e];
                const int rr = e / ow, cc = e - rr * ow;
                if (v != 0.0f)
                    red_add_global(num + job.dst_plane + (size_t)(acc.fy0 + rr) * dp + acc.fx0 + cc, v);
            }
        }
    }
}

template <int TX, int TY, int kMode, int kLanes = 8>
__global__ void __launch_bounds__(TX * TY * kLanes, 1) bm3d_match_sliding_kernel(const StackJob job) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    match_tile<TX, TY, kMode, false, kLanes>(job, blockIdx.x, smem_raw);
}

// radius >= 3: the same tile body with the exact scan (match table only);
// two CTAs per SM (128 registers, ~100 KB of shared memory each)
template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY * 8, 2) bm3d_match_exact_kernel(const StackJob job) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    match_tile<TX, TY, kTableOnly, true>(job, blockIdx.x, smem_raw);
}

// Persistent form: every CTA pulls (stack, tile) items from the queue.
// Thread 0 claims the next item while the current one runs (the atomic's
// latency hides behind the tile), and the item's StackJob is copied to
// shared memory only when the item belongs to another stack than the last.
template <int TX, int TY, int kMode, int kLanes = 8>
__global__ void __launch_bounds__(TX * TY * kLanes, 1) bm3d_batch_tile_kernel(const BatchWork work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StackJob s_job;
    __shared__ int s_item, s_job_index, s_first, s_end;
    const int total = work.tile_first[work.njobs];
    if (threadIdx.x == 0) {
        s_item = atomicAdd(work.counter, 1);
        s_first = 0;
        s_end = 0;  // no job cached
    }
    for (;;) {
        __syncthreads();  // s_item is set; the previous item is done with s_job
        const int item = s_item;
        if (item >= total) break;
        if (item < s_first || item >= s_end) {  // another stack: look it up
            __syncthreads();                     // all threads read s_first/s_end
            if (threadIdx.x == 0) {
                int lo = 0, hi = work.njobs - 1;
                while (lo < hi) {  // last job whose first tile is <= item
                    const int mid = (lo + hi + 1) >> 1;
                    if (work.tile_first[mid] <= item)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                s_job_index = lo;
                s_first = work.tile_first[lo];
                s_end = work.tile_first[lo + 1];
            }
            __syncthreads();
            const int* src = reinterpret_cast<const int*>(work.jobs + s_job_index);
            int* dst = reinterpret_cast<int*>(&s_job);
            for (int i = threadIdx.x; i < int(sizeof(StackJob) / sizeof(int)); i += blockDim.x)
                dst[i] = src[i];
            __syncthreads();
        }
        int next = 0;
        if (threadIdx.x == 0) next = atomicAdd(work.counter, 1);
        match_tile<TX, TY, kMode, false, kLanes>(s_job, item - s_first, smem_raw);
        __syncthreads();  // every thread has read s_item and s_first
        if (threadIdx.x == 0) s_item = next;
    }
}

// ---------------------------------------------------------------------------
// Launch templates, instantiated once per tile shape (bm3d_match_<shape>.cu).

template <int TX, int TY, int kMode, int kLanes = 8>
cudaError_t launch_grid(const StackJob& job, size_t smem, cudaStream_t stream) {
    auto* fn = bm3d_match_sliding_kernel<TX, TY, kMode, kLanes>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int tiles = ((job.nbx + TX - 1) / TX) * ((job.nby + TY - 1) / TY);
    fn<<<tiles, TX * TY * kLanes, smem, stream>>>(job);
    return cudaGetLastError();
}

template <int TX, int TY>
cudaError_t launch_grid_mode(const StackJob& job, TileMode mode, cudaStream_t stream) {
    const SmemPlan plan = smem_plan<TX, TY>(job, mode);
    if (!smem_plan_aligned<TX, TY>(plan)) return cudaErrorMisalignedAddress;
    const size_t smem = plan.bytes;
    if (job.radius >= 3) {
        if (mode != kTableOnly) return cudaErrorInvalidValue;
        auto* fn = bm3d_match_exact_kernel<TX, TY>;
        cudaError_t e =
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int tiles = ((job.nbx + TX - 1) / TX) * ((job.nby + TY - 1) / TY);
        fn<<<tiles, TX * TY * 8, smem, stream>>>(job);
        return cudaGetLastError();
    }
    switch (mode) {
        case kTableOnly:
            return job.lanes == 16 ? launch_grid<TX, TY, kTableOnly, 16>(job, smem, stream)
                                   : launch_grid<TX, TY, kTableOnly>(job, smem, stream);
        case kFused: return launch_grid<TX, TY, kFused>(job, smem, stream);
        default: return launch_grid<TX, TY, kFusedSave>(job, smem, stream);
    }
}

// CTAs of the persistent kernel that one SM holds at once (with `smem`
// bytes of dynamic shared memory): the persistent grid is this many per SM.
template <int TX, int TY>
int batch_ctas_per_sm(TileMode mode, int lanes, size_t smem) {
    auto* fn = mode == kFused ? bm3d_batch_tile_kernel<TX, TY, kFused>
                              : (lanes == 16 ? bm3d_batch_tile_kernel<TX, TY, kTableOnly, 16>
                                             : bm3d_batch_tile_kernel<TX, TY, kTableOnly>);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, TX * TY * lanes, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

template <int TX, int TY>
cudaError_t launch_batch(const BatchWork& work, TileMode mode, int lanes, size_t smem, int grid,
                         cudaStream_t stream) {
    // (the batch's jobs were checked one by one when it was built:
    // tile_smem_bytes refuses a misaligned plan)
    auto* fn = mode == kFused ? bm3d_batch_tile_kernel<TX, TY, kFused>
                              : (lanes == 16 ? bm3d_batch_tile_kernel<TX, TY, kTableOnly, 16>
                                             : bm3d_batch_tile_kernel<TX, TY, kTableOnly>);
    if (mode == kFused && lanes != 8) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<grid, TX * TY * lanes, smem, stream>>>(work);
    return cudaGetLastError();
}

}  // namespace

}  // namespace vsfeel
