// TEST INFRASTRUCTURE: the CPU oracle of the BM3Dv2 basic estimate.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// this library, and only as the checker or the timed CPU baseline. The
// product path (vapoursynth-feel_b200/csrc) never links or calls it.
//
// It restates the reference's hard-thresholding pass on the CPU, one
// function per reference step, keeping the float operation order wherever
// the GPU kernels must reproduce bits:
//   frame / window mapping ............ src/bm3d.comp:57-81, src/bm3d.cpp:369-371
//   block positions .................... src/bm3d.comp:445-458
//   8-point DCT pair ................... src/bm3d.comp:91-181  (explicit fma kept)
//   3D transform sequence .............. src/bm3d.comp:183-236, 384-399
//   SSD (exact and sliding scans) ...... src/bm3d.comp:253-282, 479-526
//   per-lane top-8 + merge ............. src/bm3d.comp:284-356, 527-537
//   temporal predictive search ......... src/bm3d.comp:540-637
//   forced self-match .................. src/bm3d.comp:639-663
//   hard threshold + weight ............ src/bm3d.comp:358-382
//   extractor-biased scatter ........... src/bm3d.comp:697-715
//   FP64 normalisation ................. src/bm3d_agg.comp:36-52, src/bm3d.cpp:628-696
//   sigma / extractor scaling .......... src/bm3d.cpp:1103-1113, 1188-1190
//
// Contraction rule (GLSL leaves it to the driver): the two multiply-add
// statements the shader writes without fma -- the SSD accumulation
// `e += d*d` and the extractor bias `w*p + E` -- are evaluated as one fused
// multiply-add, as a contracting GPU compiler emits them. Everything else is
// unfused; build with -ffp-contract=off so the compiler adds no other fusion.
//
// Parity pin: tests/test_oracle_ref.py checks this restatement bit for bit
// against the reference's own shader source compiled for the CPU
// (oracle/build_ref.py), and tests/golden/ holds vectors produced that way.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Params {
    int width, height, stride, nframes;
    double thr;        // SIGMA_Y: sigma * the pass's factor, src/bm3d.cpp:1103-1113
    int step, bm_range, radius, ps_num, ps_range;
    double extractor;  // ldexp(1, exp) or 0, src/bm3d.cpp:1188-1190
    bool final_pass;   // Wiener pass with a "ref" clip, src/bm3d.cpp:1062-1083
};

inline int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

// --------------------------------------------------------------------------
// 8-point DCT-II (x4 orthonormal) and its transpose, src/bm3d.comp:91-181.
// The statements follow the reference's order; every fma there is an fma here
// and every other product and sum is rounded on its own.
template <class T>
void dct8_fwd(T v[8]) {
    const T c414 = T(0.414213562373095048801688724209698078569671875);
    const T c1847 = T(1.847759065022573512256366378793576573644833252);
    const T c198 = T(0.198912367379658006911597622644676228597850501);
    const T c1961 = T(1.961570560806460898252364472268478073947867462);
    const T c1414 = T(1.414213562373095048801688724209698078569671875);
    const T c668 = T(0.668178637919298919997757686523080761552472251);
    const T c1662 = T(1.662939224605090474157576755235811513477121624);
    const T c707 = T(0.707106781186547524400844362104849039284835938);

    const T d07 = v[0] - v[7], s07 = v[0] + v[7];
    const T d43 = v[4] - v[3], s43 = v[4] + v[3];
    const T d25 = v[2] - v[5];
    const T d16 = v[1] - v[6];
    const T a = d25 + d16;
    const T s16 = v[1] + v[6];
    const T b = d25 - d16;
    const T s25 = v[2] + v[5];
    const T p = std::fma(-c707, a, d07);
    const T q = std::fma(-c707, b, d43);
    v[3] = c1662 * std::fma(c668, q, p);
    v[5] = -(c1662 * std::fma(-c668, p, q));
    const T e0 = s07 + s43, e1 = s25 + s16;
    v[4] = c1414 * (e0 - e1);
    v[0] = c1414 * (e0 + e1);
    const T h = std::fma(c707, a, d07);
    const T i = std::fma(c707, b, d43);
    v[1] = c1961 * std::fma(-c198, i, h);
    v[7] = c1961 * std::fma(c198, h, i);
    const T l = s07 - s43, o = s25 - s16;
    v[2] = c1847 * std::fma(-c414, o, l);
    v[6] = c1847 * std::fma(c414, l, o);
}

template <class T>
void dct8_inv(T v[8]) {
    const T c1662 = T(1.662939224605090474157576755235811513477121624);
    const T c668 = T(0.668178637919298919997757686523080761552472251);
    const T c1961 = T(1.961570560806460898252364472268478073947867462);
    const T c198 = T(0.198912367379658006911597622644676228597850501);
    const T c1847 = T(1.847759065022573512256366378793576573644833252);
    const T c707 = T(0.707106781186547524400844362104849039284835938);
    const T c414 = T(0.414213562373095048801688724209698078569671875);
    const T c1414 = T(1.414213562373095048801688724209698078569671875);

    const T dc = v[0] * c1414;
    const T a = std::fma(c1414, v[4], dc);
    const T b = std::fma(-c1414, v[4], dc);
    const T c = std::fma(c414, v[6], v[2]);
    const T d = std::fma(c414, v[2], -v[6]);
    const T s53 = v[5] + v[3];
    const T d35 = v[3] - v[5];
    const T e = std::fma(c707, s53, v[1]);
    const T f = std::fma(-c707, d35, v[7]);
    const T g = std::fma(c707, d35, v[7]);
    const T h = std::fma(-c707, s53, v[1]);
    const T t0 = std::fma(c1847, c, a);
    const T t1 = std::fma(c198, g, e);
    const T o7 = std::fma(-c1961, t1, t0);
    const T o0 = std::fma(c1961, t1, t0);
    const T t2 = std::fma(-c1847, d, b);
    const T t3 = std::fma(c668, h, f);
    const T o5 = std::fma(-c1662, t3, t2);
    const T o2 = std::fma(c1662, t3, t2);
    const T t4 = std::fma(-c1847, c, a);
    const T t5 = std::fma(-c198, e, g);
    const T o3 = std::fma(-c1961, t5, t4);
    const T o4 = std::fma(c1961, t5, t4);
    const T t6 = std::fma(c1847, d, b);
    const T t7 = std::fma(-c668, f, h);
    const T o6 = std::fma(-c1662, t7, t6);
    const T o1 = std::fma(c1662, t7, t6);
    v[0] = o0; v[1] = o1; v[2] = o2; v[3] = o3;
    v[4] = o4; v[5] = o5; v[6] = o6; v[7] = o7;
}

// --------------------------------------------------------------------------
// Block matching

template <class T>
struct LaneList {  // one lane's sorted top-8, src/bm3d.comp:284-302
    T e[8];
    int x[8], y[8], s[8];
    void reset() {
        for (int k = 0; k < 8; ++k) {
            e[k] = T(FLT_MAX);
            x[k] = 0;
            y[k] = 0;
            s[k] = INT_MAX;
        }
    }
    // strict `<` keeps an earlier candidate ahead of an equal later one
    void insert(T err, int cx, int cy, int seq) {
        if (!(err < e[7])) return;
        int pos = 7;
        while (pos > 0 && err < e[pos - 1]) {
            e[pos] = e[pos - 1];
            x[pos] = x[pos - 1];
            y[pos] = y[pos - 1];
            s[pos] = s[pos - 1];
            --pos;
        }
        e[pos] = err;
        x[pos] = cx;
        y[pos] = cy;
        s[pos] = seq;
    }
};

template <class T>
struct Match8 {
    T e[8];
    int x[8], y[8], s[8];
};

// 8-way merge of the lanes' lists by (error, seq), src/bm3d.comp:324-356
template <class T>
Match8<T> merge8(const LaneList<T> lanes[8]) {
    Match8<T> m;
    int head[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 8; ++k) {
        int bl = 0, bh = 0;
        T be = T(FLT_MAX);
        int bs = INT_MAX;
        bool found = false;
        for (int l = 0; l < 8; ++l) {
            const int hv = head[l];
            const bool valid = hv < 8;
            const T e = valid ? lanes[l].e[hv] : T(FLT_MAX);
            const int sq = valid ? lanes[l].s[hv] : INT_MAX;
            const bool better = valid && (!found || e < be || (e == be && sq < bs));
            if (better) {
                bl = l;
                bh = hv;
                be = e;
                bs = sq;
            }
            found = found || valid;
        }
        m.e[k] = be;
        m.x[k] = lanes[bl].x[bh];
        m.y[k] = lanes[bl].y[bh];
        m.s[k] = bs;
        head[bl] += 1;
    }
    return m;
}

// cur[c*8 + i] = pixel (row i, column c) of the reference block
template <class T>
T column_ssd(const T cur[64], const float* f, int stride, int cy, int X, int c) {
    T ev = T(0), od = T(0);
    for (int i = 0; i < 8; i += 2) {
        const T d0 = cur[c * 8 + i] - T(f[(size_t)(cy + i) * stride + X]);
        ev = std::fma(d0, d0, ev);
        const T d1 = cur[c * 8 + i + 1] - T(f[(size_t)(cy + i + 1) * stride + X]);
        od = std::fma(d1, d1, od);
    }
    return ev + od;
}

template <class T>
inline T tree8(const T col[8]) {
    return ((col[0] + col[1]) + (col[2] + col[3])) + ((col[4] + col[5]) + (col[6] + col[7]));
}

// Scan one search window into the 8 lane lists with the reference's lane
// partition: the sliding column scan below radius 3, the stride-8 full-SSD
// scan otherwise (src/bm3d.comp:493-526, 582-611). The sliding scan keeps the
// reference's column bookkeeping exactly: after the shift, slot c holds the
// column SSD of source column cx+c against block column min(c + cx-left, 7).
template <class T>
void scan_window(const Params& P, const T cur[64], const float* f, int left, int right,
                 int top, int bottom, int seq_base, LaneList<T> lanes[8]) {
    const int rw = right - left + 1;
    const int stride = P.stride;
    if (P.radius < 3) {
        for (int s = 0; s < 8; ++s) {
            for (int cy = top + s; cy <= bottom; cy += 8) {
                T col[8];
                for (int c = 0; c < 8; ++c) col[c] = column_ssd(cur, f, stride, cy, left + c, c);
                lanes[s].insert(tree8(col), left, cy, seq_base + (cy - top) * rw);
                for (int cx = left + 1; cx <= right; ++cx) {
                    for (int c = 0; c < 7; ++c) col[c] = col[c + 1];
                    col[7] = column_ssd(cur, f, stride, cy, cx + 7, 7);
                    lanes[s].insert(tree8(col), cx, cy, seq_base + (cy - top) * rw + (cx - left));
                }
            }
        }
    } else {
        const int total = (bottom - top + 1) * rw;
        for (int s = 0; s < 8; ++s) {
            for (int idx = s; idx < total; idx += 8) {
                const int cy = top + idx / rw;
                const int cx = left + idx % rw;
                T col[8];
                for (int c = 0; c < 8; ++c) col[c] = column_ssd(cur, f, stride, cy, cx + c, c);
                lanes[s].insert(tree8(col), cx, cy, seq_base + idx);
            }
        }
    }
}

// global-list insertion of a temporal match, src/bm3d.comp:304-322
template <class T>
void ginsert8(T ge[8], int gx[8], int gy[8], int gz[8], T err, int cx, int cy, int cz) {
    if (!(err < ge[7])) return;
    int pos = 7;
    while (pos > 0 && err < ge[pos - 1]) {
        ge[pos] = ge[pos - 1];
        gx[pos] = gx[pos - 1];
        gy[pos] = gy[pos - 1];
        gz[pos] = gz[pos - 1];
        --pos;
    }
    ge[pos] = err;
    gx[pos] = cx;
    gy[pos] = cy;
    gz[pos] = cz;
}

struct Frames {
    const float* base;  // the search clip: nframes planes of height*stride floats
    size_t plane;
    int nframes;
    const float* input = nullptr;  // the denoised clip in the final pass (else base)
    const float* at(int f) const { return base + (size_t)f * plane; }
    const float* input_at(int f) const { return (input ? input : base) + (size_t)f * plane; }
};

// The 8 matches (x, y, z) of the reference block at (x, y) of stack m,
// src/bm3d.comp:460-663. z is the slice index: frame clamp(m - r + z).
template <class T>
void match_block(const Params& P, const Frames& F, int m, int x, int y, int out[8][3]) {
    const int r = P.radius;
    auto frame_of = [&](int z) { return F.at(clampi(m - r + z, 0, P.nframes - 1)); };
    const float* fc = frame_of(r);
    T cur[64];
    for (int c = 0; c < 8; ++c)
        for (int i = 0; i < 8; ++i) cur[c * 8 + i] = T(fc[(size_t)(y + i) * P.stride + x + c]);

    T ge[8];
    int gx[8], gy[8], gz[8];
    {
        LaneList<T> lanes[8];
        for (auto& l : lanes) l.reset();
        const int left = std::max(x - P.bm_range, 0);
        const int right = std::min(x + P.bm_range, P.width - 8);
        const int top = std::max(y - P.bm_range, 0);
        const int bottom = std::min(y + P.bm_range, P.height - 8);
        scan_window(P, cur, fc, left, right, top, bottom, 0, lanes);
        const Match8<T> mm = merge8(lanes);
        for (int k = 0; k < 8; ++k) {
            ge[k] = mm.e[k];
            gx[k] = mm.x[k];
            gy[k] = mm.y[k];
            gz[k] = r;
        }
    }

    int sx[8], sy[8];
    for (int k = 0; k < 8; ++k) {
        sx[k] = gx[k];
        sy[k] = gy[k];
    }
    const int Q = P.ps_range;
    const int win_area = (2 * Q + 1) * (2 * Q + 1);
    for (int dir = -1; dir <= 1; dir += 2) {
        int px[8], py[8];
        for (int k = 0; k < 8; ++k) {
            px[k] = sx[k];
            py[k] = sy[k];
        }
        for (int t = 1; t <= r; ++t) {
            const int z = r + dir * t;
            const float* ft = frame_of(z);
            LaneList<T> lanes[8];
            for (auto& l : lanes) l.reset();
            for (int i = 0; i < P.ps_num; ++i) {
                const int left = std::max(px[i] - Q, 0);
                const int right = std::min(px[i] + Q, P.width - 8);
                const int top = std::max(py[i] - Q, 0);
                const int bottom = std::min(py[i] + Q, P.height - 8);
                scan_window(P, cur, ft, left, right, top, bottom, i * win_area, lanes);
            }
            const Match8<T> fm = merge8(lanes);
            for (int i = 0; i < P.ps_num; ++i) ginsert8(ge, gx, gy, gz, fm.e[i], fm.x[i], fm.y[i], z);
            for (int k = 0; k < 8; ++k) {
                px[k] = fm.x[k];
                py[k] = fm.y[k];
            }
        }
    }

    int self = 0;
    for (int k = 0; k < 8; ++k) self += (gx[k] == x && gy[k] == y && gz[k] == r) ? 1 : 0;
    if (self == 0) {
        for (int k = 7; k >= 1; --k) {
            gx[k] = gx[k - 1];
            gy[k] = gy[k - 1];
            gz[k] = gz[k - 1];
        }
        gx[0] = x;
        gy[0] = y;
        gz[0] = r;
    }
    for (int k = 0; k < 8; ++k) {
        out[k][0] = gx[k];
        out[k][1] = gy[k];
        out[k][2] = gz[k];
    }
}

// --------------------------------------------------------------------------
// Collaborative hard thresholding, src/bm3d.comp:358-399.
// X[k][a][b]: group member k, row a, column b. The 1-D transforms run in the
// reference's order: rows-of-columns, columns-of-rows, then along the group;
// the inverse runs in the same axis order.
// keep (optional): receives the keep bits, word b (horizontal frequency),
// bit 8*k + a (group frequency k, vertical frequency a).
template <class T>
T filter_group(const Params& P, T X[8][8][8], uint64_t* keep_bits = nullptr) {
    T v[8];
    for (int k = 0; k < 8; ++k)
        for (int b = 0; b < 8; ++b) {
            for (int a = 0; a < 8; ++a) v[a] = X[k][a][b];
            dct8_fwd(v);
            for (int a = 0; a < 8; ++a) X[k][a][b] = v[a];
        }
    for (int k = 0; k < 8; ++k)
        for (int a = 0; a < 8; ++a) dct8_fwd(X[k][a]);
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            for (int k = 0; k < 8; ++k) v[k] = X[k][a][b];
            dct8_fwd(v);
            for (int k = 0; k < 8; ++k) X[k][a][b] = v[k];
        }

    const T thr = T(P.thr);
    int kept = 0;
    if (keep_bits)
        for (int b = 0; b < 8; ++b) keep_bits[b] = 0;
    for (int k = 0; k < 8; ++k)
        for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) {
                const T val = X[k][a][b];
                const T t = (k == 0 && a == 0 && b == 0) ? T(0) : thr;
                const bool keep = std::fabs(val) >= t;
                kept += keep ? 1 : 0;
                if (keep_bits && keep) keep_bits[b] |= uint64_t(1) << (8 * k + a);
                X[k][a][b] = keep ? val * (T(1) / T(4096)) : T(0);
            }
    const T weight = T(1) / T(kept);

    for (int k = 0; k < 8; ++k)
        for (int b = 0; b < 8; ++b) {
            for (int a = 0; a < 8; ++a) v[a] = X[k][a][b];
            dct8_inv(v);
            for (int a = 0; a < 8; ++a) X[k][a][b] = v[a];
        }
    for (int k = 0; k < 8; ++k)
        for (int a = 0; a < 8; ++a) dct8_inv(X[k][a]);
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            for (int k = 0; k < 8; ++k) v[k] = X[k][a][b];
            dct8_inv(v);
            for (int k = 0; k < 8; ++k) X[k][a][b] = v[k];
        }
    return weight;
}

// Collaborative Wiener filtering, the final pass (src/bm3d.comp:401-443):
// the 3D transform of the group (X) and of the basic estimate's group at the
// same positions (Xr), coefficient r^2 / (r^2 + SIGMA_Y^2) per coefficient
// (1 at DC), the product scaled by 1/4096, weight 1 / sum(coefficient^2),
// inverse transform of X. Per coefficient, rr = r*r and SS = SIGMA_Y*SIGMA_Y
// are rounded products and rr + SS is an unfused sum (SIGMA_Y is a
// specialisation constant, so a shader compiler folds SS), while the
// accumulation ks += coeff*coeff is fused like the other "a += b*c"
// statements. The sums of the squared coefficients follow the reference's
// order: per horizontal frequency b, four partial sums by vertical frequency
// mod 4 over (group frequency, vertical frequency), then
// (ks0 + ks1) + (ks2 + ks3), then the pairwise tree over b
// (src/bm3d.comp:238-246).
template <class T>
void transform3(T X[8][8][8], bool inverse) {
    T v[8];
    for (int k = 0; k < 8; ++k)
        for (int b = 0; b < 8; ++b) {
            for (int a = 0; a < 8; ++a) v[a] = X[k][a][b];
            inverse ? dct8_inv(v) : dct8_fwd(v);
            for (int a = 0; a < 8; ++a) X[k][a][b] = v[a];
        }
    for (int k = 0; k < 8; ++k)
        for (int a = 0; a < 8; ++a) inverse ? dct8_inv(X[k][a]) : dct8_fwd(X[k][a]);
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            for (int k = 0; k < 8; ++k) v[k] = X[k][a][b];
            inverse ? dct8_inv(v) : dct8_fwd(v);
            for (int k = 0; k < 8; ++k) X[k][a][b] = v[k];
        }
}

template <class T>
T wiener_group(const Params& P, T X[8][8][8], T Xr[8][8][8]) {
    transform3(X, false);
    transform3(Xr, false);
    const T sy = T(P.thr);
    const T ss = sy * sy;
    T lane_k[8];
    for (int b = 0; b < 8; ++b) {
        T ks[4] = {T(0), T(0), T(0), T(0)};
        for (int k = 0; k < 8; ++k)
            for (int a = 0; a < 8; ++a) {
                const T r = Xr[k][a][b];
                const T rr = r * r;
                T coeff = rr / (rr + ss);
                if (k == 0 && a == 0 && b == 0) coeff = T(1);
                const T val = X[k][a][b] * coeff;
                ks[a % 4] = std::fma(coeff, coeff, ks[a % 4]);
                X[k][a][b] = val * (T(1) / T(4096));
            }
        lane_k[b] = (ks[0] + ks[1]) + (ks[2] + ks[3]);
    }
    const T k = ((lane_k[0] + lane_k[1]) + (lane_k[2] + lane_k[3])) +
                ((lane_k[4] + lane_k[5]) + (lane_k[6] + lane_k[7]));
    transform3(X, true);
    return T(1) / k;
}

template <class T>
struct BlockResult {
    int match[8][3];
    T X[8][8][8];
    T Xr[8][8][8];  // final pass: the basic estimate's group
    T weight;
    uint64_t keep[8];
};

int count_blocks(int extent, int step) { return (extent - 9 + 2 * step) / step; }

// One stack m: matching, filtering and the scatter into its 2*TW slices
// (slice z: numerator plane 2z, weight plane 2z+1). The scatter follows the
// reference's accumulation order for a serial dispatch: block rows, block
// columns, then lane (block column), member, row.
template <class T>
void run_stack(const Params& P, const Frames& F, int m, T* slices, int nthreads,
               int32_t* match_out, uint64_t* keep_out = nullptr) {
    const int nbx = count_blocks(P.width, P.step);
    const int nby = count_blocks(P.height, P.step);
    const size_t plane = (size_t)P.height * P.stride;
    const T E = T(P.extractor);
    const int r = P.radius;
    const int chunk_rows = std::max(1, std::min(nby, 4 * std::max(nthreads, 1)));
    std::vector<BlockResult<T>> res((size_t)chunk_rows * nbx);

    for (int by0 = 0; by0 < nby; by0 += chunk_rows) {
        const int rows = std::min(chunk_rows, nby - by0);
        std::atomic<int> next{0};
        auto worker = [&]() {
            for (;;) {
                const int ry = next.fetch_add(1);
                if (ry >= rows) break;
                const int y = std::min((by0 + ry) * P.step, P.height - 8);
                for (int bx = 0; bx < nbx; ++bx) {
                    const int x = std::min(bx * P.step, P.width - 8);
                    BlockResult<T>& br = res[(size_t)ry * nbx + bx];
                    match_block<T>(P, F, m, x, y, br.match);
                    for (int k = 0; k < 8; ++k) {
                        const int fk = clampi(m - r + br.match[k][2], 0, P.nframes - 1);
                        const float* f = F.input_at(fk);
                        const float* fr = F.at(fk);
                        for (int a = 0; a < 8; ++a)
                            for (int b = 0; b < 8; ++b) {
                                const size_t o =
                                    (size_t)(br.match[k][1] + a) * P.stride + br.match[k][0] + b;
                                br.X[k][a][b] = T(f[o]);
                                if (P.final_pass) br.Xr[k][a][b] = T(fr[o]);
                            }
                    }
                    br.weight = P.final_pass ? wiener_group<T>(P, br.X, br.Xr)
                                             : filter_group<T>(P, br.X, br.keep);
                }
            }
        };
        const int nt = std::max(1, std::min(nthreads, rows));
        if (nt == 1) {
            worker();
        } else {
            std::vector<std::thread> th;
            for (int t = 0; t < nt; ++t) th.emplace_back(worker);
            for (auto& t : th) t.join();
        }
        for (int ry = 0; ry < rows; ++ry) {
            for (int bx = 0; bx < nbx; ++bx) {
                const BlockResult<T>& br = res[(size_t)ry * nbx + bx];
                if (match_out) {
                    int32_t* mo = match_out + ((size_t)(by0 + ry) * nbx + bx) * 24;
                    for (int k = 0; k < 8; ++k)
                        for (int q = 0; q < 3; ++q) mo[k * 3 + q] = br.match[k][q];
                }
                if (keep_out)
                    for (int b = 0; b < 8; ++b)
                        keep_out[((size_t)(by0 + ry) * nbx + bx) * 8 + b] = br.keep[b];
                if (!slices) continue;
                const T wv = (br.weight + E) - E;
                for (int b = 0; b < 8; ++b)
                    for (int k = 0; k < 8; ++k) {
                        const int z = br.match[k][2];
                        T* num = slices + (size_t)(2 * z) * plane;
                        T* den = num + plane;
                        const size_t o = (size_t)br.match[k][1] * P.stride + br.match[k][0] + b;
                        for (int a = 0; a < 8; ++a) {
                            num[o + (size_t)a * P.stride] += std::fma(br.weight, br.X[k][a][b], E) - E;
                            den[o + (size_t)a * P.stride] += wv;
                        }
                    }
            }
        }
    }
}

// src/bm3d.cpp:369-371
int agg_z(int i, int n, int nframes, int radius) {
    return std::min(std::max(2 * radius - i, n - nframes + 1 + radius), n + radius);
}

template <class T, class O>
int run_clip(const Params& P, const float* frames, int out_first, int out_count, int nthreads, O* out,
             const float* ref = nullptr) {
    const int N = P.nframes, r = P.radius, tw = 2 * r + 1;
    const size_t plane = (size_t)P.height * P.stride;
    // the final pass searches (and takes its coefficients from) the ref clip
    // and denoises the source clip
    Frames F{P.final_pass ? ref : frames, plane, N, P.final_pass ? frames : nullptr};
    const int m_lo = clampi(out_first - r, 0, N - 1);
    const int m_hi = clampi(out_first + out_count - 1 + r, 0, N - 1);
    std::vector<T> stacks((size_t)(m_hi - m_lo + 1) * 2 * tw * plane, T(0));
    for (int m = m_lo; m <= m_hi; ++m)
        run_stack<T>(P, F, m, stacks.data() + (size_t)(m - m_lo) * 2 * tw * plane, nthreads, nullptr);
    for (int q = 0; q < out_count; ++q) {
        const int n = out_first + q;
        for (int yy = 0; yy < P.height; ++yy)
            for (int xx = 0; xx < P.width; ++xx) {
                const size_t o = (size_t)yy * P.stride + xx;
                double acc = 0.0, acw = 0.0;
                for (int i = 0; i < tw; ++i) {
                    const int mi = clampi(n - r + i, 0, N - 1);
                    const int z = (r == 0) ? 0 : agg_z(i, n, N, r);
                    const T* s = stacks.data() + ((size_t)(mi - m_lo) * 2 * tw + 2 * z) * plane;
                    acc += double(s[o]);
                    acw += double(s[o + plane]);
                }
                out[(size_t)q * P.height * P.width + (size_t)yy * P.width + xx] = O(acc / acw);
            }
    }
    return 0;
}

bool make_params(Params& P, int nframes, int width, int height, float sigma, int block_step,
                 int bm_range, int radius, int ps_num, int ps_range, int extractor_exp,
                 bool final_pass = false) {
    if (nframes <= 0 || width < 8 || height < 8) return false;
    if (sigma < 0.0f || block_step < 1 || block_step > 8 || bm_range <= 0 || radius < 0 ||
        radius > 4 || ps_num < 1 || ps_num > 8 || ps_range <= 0)
        return false;
    // sigma factor of the pass, src/bm3d.cpp:1103-1113
    uint32_t bits = final_pass ? 0x3e40c0c1u : 0x3f021bb6u;
    float factor;
    std::memcpy(&factor, &bits, 4);
    P.width = width;
    P.height = height;
    P.stride = width;
    P.nframes = nframes;
    P.thr = double(sigma * factor);  // rounded to float, as the shader's SIGMA_Y
    P.step = block_step;
    P.bm_range = bm_range;
    P.radius = radius;
    P.ps_num = ps_num;
    P.ps_range = ps_range;
    P.extractor = extractor_exp != 0 ? double(std::ldexp(1.0f, extractor_exp)) : 0.0;
    P.final_pass = final_pass;
    return true;
}

}  // namespace

extern "C" {

int oracle_block_count(int width, int height, int block_step) {
    return count_blocks(width, block_step) * count_blocks(height, block_step);
}

int oracle_agg_z(int i, int n, int nframes, int radius) { return agg_z(i, n, nframes, radius); }

void oracle_dct8_fwd_f32(float* v) { dct8_fwd<float>(v); }
void oracle_dct8_inv_f32(float* v) { dct8_inv<float>(v); }
void oracle_dct8_fwd_f64(double* v) { dct8_fwd<double>(v); }
void oracle_dct8_inv_f64(double* v) { dct8_inv<double>(v); }

float oracle_threshold(float sigma) {
    Params P;
    make_params(P, 1, 8, 8, sigma, 8, 1, 0, 1, 1, 0);
    return float(P.thr);
}

// Full clip, FP32 restatement: frames are nframes x height x width floats;
// out receives out_count frames starting at out_first. Returns 0 or -1.
int oracle_bm3d_f32(const float* frames, int nframes, int width, int height, float sigma,
                    int block_step, int bm_range, int radius, int ps_num, int ps_range,
                    int extractor_exp, int out_first, int out_count, int nthreads, float* out) {
    Params P;
    if (!make_params(P, nframes, width, height, sigma, block_step, bm_range, radius, ps_num,
                     ps_range, extractor_exp))
        return -1;
    if (out_first < 0 || out_count < 0 || out_first + out_count > nframes) return -1;
    return run_clip<float, float>(P, frames, out_first, out_count, nthreads, out);
}

// The same algorithm evaluated in double precision end to end.
int oracle_bm3d_f64(const float* frames, int nframes, int width, int height, float sigma,
                    int block_step, int bm_range, int radius, int ps_num, int ps_range,
                    int extractor_exp, int out_first, int out_count, int nthreads, double* out) {
    Params P;
    if (!make_params(P, nframes, width, height, sigma, block_step, bm_range, radius, ps_num,
                     ps_range, extractor_exp))
        return -1;
    if (out_first < 0 || out_count < 0 || out_first + out_count > nframes) return -1;
    return run_clip<double, double>(P, frames, out_first, out_count, nthreads, out);
}

// The final (Wiener) pass: frames is the clip to denoise, ref the basic
// estimate it is matched on. FP32 or (fp64 != 0) FP64 output.
int oracle_bm3d_final(const float* frames, const float* ref, int nframes, int width, int height,
                      float sigma, int block_step, int bm_range, int radius, int ps_num,
                      int ps_range, int extractor_exp, int out_first, int out_count, int nthreads,
                      int fp64, void* out) {
    Params P;
    if (!ref || !make_params(P, nframes, width, height, sigma, block_step, bm_range, radius,
                             ps_num, ps_range, extractor_exp, true))
        return -1;
    if (out_first < 0 || out_count < 0 || out_first + out_count > nframes) return -1;
    if (fp64)
        return run_clip<double, double>(P, frames, out_first, out_count, nthreads,
                                        static_cast<double*>(out), ref);
    return run_clip<float, float>(P, frames, out_first, out_count, nthreads,
                                  static_cast<float*>(out), ref);
}

// Match table of stack m: nblocks x 8 x (x, y, z), blocks in raster order.
int oracle_bm3d_matches_f32(const float* frames, int nframes, int width, int height, float sigma,
                            int block_step, int bm_range, int radius, int ps_num, int ps_range,
                            int m, int nthreads, int32_t* table) {
    Params P;
    if (!make_params(P, nframes, width, height, sigma, block_step, bm_range, radius, ps_num,
                     ps_range, 0))
        return -1;
    if (m < 0 || m >= nframes) return -1;
    Frames F{frames, (size_t)height * width, nframes};
    run_stack<float>(P, F, m, nullptr, nthreads, table);
    return 0;
}

// Frozen state of stack m for the differentiable form's tests: the match
// table (as oracle_bm3d_matches_f32) and the keep bits of every group,
// nblocks x 8 words (word = horizontal frequency, bit 8 * group frequency +
// vertical frequency), in FP32 or FP64 arithmetic.
int oracle_bm3d_frozen_state(const float* frames, int nframes, int width, int height, float sigma,
                             int block_step, int bm_range, int radius, int ps_num, int ps_range,
                             int m, int fp64, int nthreads, int32_t* table, uint64_t* keep) {
    Params P;
    if (!make_params(P, nframes, width, height, sigma, block_step, bm_range, radius, ps_num,
                     ps_range, 0))
        return -1;
    if (m < 0 || m >= nframes) return -1;
    Frames F{frames, (size_t)height * width, nframes};
    if (fp64)
        run_stack<double>(P, F, m, nullptr, nthreads, table, keep);
    else
        run_stack<float>(P, F, m, nullptr, nthreads, table, keep);
    return 0;
}

// Stack m's 2*TW accumulated slices (numerator, weight per slice).
int oracle_bm3d_stack_f32(const float* frames, int nframes, int width, int height, float sigma,
                          int block_step, int bm_range, int radius, int ps_num, int ps_range,
                          int extractor_exp, int m, int nthreads, float* slices) {
    Params P;
    if (!make_params(P, nframes, width, height, sigma, block_step, bm_range, radius, ps_num,
                     ps_range, extractor_exp))
        return -1;
    if (m < 0 || m >= nframes) return -1;
    Frames F{frames, (size_t)height * width, nframes};
    std::memset(slices, 0, sizeof(float) * (size_t)2 * (2 * radius + 1) * height * width);
    run_stack<float>(P, F, m, slices, nthreads, nullptr);
    return 0;
}

}  // extern "C"
