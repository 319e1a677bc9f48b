// Batched form: many clips of uneven sizes and settings in one run (the
// vsfeel_bm3d_batch_* entry points of include/vsfeel_bm3d.h). It has no
// counterpart in the reference, whose concurrency is num_streams Vulkan
// queues working on frames of one clip (src/bm3d.cpp:698-1028).
//
// Layout. Every clip of a chunk keeps, per output frame n, the TW
// (numerator, weight) plane pairs of its contributing stacks (the plain
// path's slot, without the ring reuse), so that all stacks of a chunk can be
// in flight at once. Chunks run one after another (and classes one after
// another), so every chunk of every class uses the same accumulator buffer
// and the same match-table buffer, sized for the largest chunk.
// Shape classes group the clips whose stacks share a tiled-kernel
// configuration. Per class:
//   * jobs[]: one StackJob per (clip, stack), largest clips first, with the
//     prefix sums of their tile counts -- the persistent kernel's queue;
//   * norm[]: one NormalizeJob per output frame, with the prefix sums of
//     their 32x8 tiles;
//   * a match table per stack;
//   * a CUDA graph: per chunk, clear its accumulators, the persistent
//     matching launch (as many CTAs as the SMs hold) over its queue, one filter launch over
//     every block of its stacks, one normalise launch. (The
//     filter stays a separate kernel: inside the matcher's one CTA per SM
//     its atomics run slower than at the filter kernel's occupancy.)
//     Classes whose stacks no tile shape fits record the direct-read match
//     and filter kernels per stack instead.
// Classes are cut into chunks of whole clips (at least ~16 waves of tiles
// each), matched, filtered and normalised chunk after chunk, so a chunk's
// frames and accumulators are still in L2 when its filter and normalisation
// run. A run replays the class graphs one after another on the caller's
// stream.
#include "bm3d_device.cuh"
#include "vsfeel_bm3d.h"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

namespace vsfeel {
int parse_to_info(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                  vsfeel_bm3d_info* info, int plane = 0);
int set_error(int code, const char* msg);
}  // namespace vsfeel

namespace {

using namespace vsfeel;

int error(int code, const std::string& msg) { return set_error(code, msg.c_str()); }

struct Fail {
    int code;
    std::string msg;
};

void check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
        throw Fail{VSFEEL_E_MEMORY, std::string("out of device memory (") + what + ")"};
    throw Fail{VSFEEL_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e) + " (" + what + ")"};
}

int64_t timeout_ms() {
    const char* s = std::getenv("VSFEEL_TIMEOUT_MS");
    if (s && *s) {
        const long long v = std::atoll(s);
        if (v > 0) return v;
    }
    return 120000;
}

// Bounded wait for a stream.
int wait_stream(cudaStream_t s) {
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t limit = timeout_ms();
    for (int spins = 0;; ++spins) {
        const cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return VSFEEL_OK;
        if (e != cudaErrorNotReady)
            return error(VSFEEL_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - t0)
                            .count();
        if (ms >= limit)
            return error(VSFEEL_E_TIMEOUT,
                         "timed out after " + std::to_string(ms) + " ms waiting for the GPU");
        if (spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// Bounded wait for an event (the end of the last run).
int wait_event(cudaEvent_t ev) {
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t limit = timeout_ms();
    for (int spins = 0;; ++spins) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return VSFEEL_OK;
        if (e != cudaErrorNotReady)
            return error(VSFEEL_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - t0)
                            .count();
        if (ms >= limit)
            return error(VSFEEL_E_TIMEOUT,
                         "timed out after " + std::to_string(ms) + " ms waiting for the GPU");
        if (spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

template <class T>
struct Dev {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
        n = count;
    }
    void upload(const std::vector<T>& v) {
        alloc(v.size());
        if (!v.empty()) check(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice),
                              "cudaMemcpy");
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

inline int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

struct Clip {
    vsfeel_bm3d_batch_clip desc;
    vsfeel_bm3d_info info;
    int acc_pitch = 0;
    size_t plane = 0;      // floats per accumulator plane
    size_t acc_off = 0;    // floats from the shared accumulator base (within its chunk)
    size_t table_off = 0;  // blocks from the shared match-table base (within its chunk)
    // Output n's slot starts at plane pair pair0[n] (pair0[N]: all pairs).
    // An interior output of a clip without the extractor has one merged
    // (numerator, weight-origin) pair that all its stacks scatter into; the
    // others keep one pair per contributing stack (the plain path's rule,
    // vsfeel_bm3d::merged in bm3d_engine.cu).
    std::vector<size_t> pair0;
    bool merged_slots = false;
    int tw() const { return 2 * info.radius + 1; }
    bool merged(int n) const {
        const int r = info.radius;
        return merged_slots && n - r >= 0 && n + r <= info.num_frames - 1;
    }
    void plan_slots(bool allow_merge) {
        merged_slots = allow_merge && info.extractor == 0.0f && info.radius > 0;
        pair0.assign((size_t)info.num_frames + 1, 0);
        for (int n = 0; n < info.num_frames; ++n)
            pair0[n + 1] = pair0[n] + (merged(n) ? 1 : tw());
    }
    // First float of output n's slot pair j (j = 0 for a merged slot).
    size_t pair_floats(int n, int j) const {
        return (pair0[n] + (merged(n) ? 0 : j)) * 2 * plane;
    }
    size_t acc_floats() const { return pair0.back() * 2 * plane; }
};

using ClassKey = std::tuple<int, int, int, int, int>;  // radius, step, R, P, Q

struct Class {
    ClassKey key;
    std::vector<int> clips;
    std::vector<StackJob> jobs;
    int tile_shape = -1;
    int lanes = 8;                       // lanes per reference block of the matcher
    double tuned_ms[kTileShapes] = {};   // autotuner's times, 8 lanes
    double tuned_ms_16[kTileShapes] = {};  // and 16 lanes
    int64_t tiles = 0;
    size_t smem = 0;
    Dev<StackJob> d_jobs;
    Dev<int> d_tile_first;
    Dev<NormalizeJob> d_norm;
    Dev<int> d_norm_first;
    int norm_tiles = 0;
    int nnorm = 0;
    Dev<int> d_filter_first;
    int filter_items = 0;
    Dev<int> counter;
    // chunks of whole clips, each matched, filtered and normalised in turn
    struct Chunk {
        int job0, njobs, norm0, nnorm;     // ranges in jobs[] and norm[]
        int first_off, ffirst_off, nfirst_off;  // chunk-relative prefix arrays
        int tiles, filter_items, norm_tiles;
        size_t acc0, acc_floats;           // accumulator range
        int buf;                           // which of the two buffer sets (overlapped graphs)
    };
    std::vector<Chunk> chunks;
    std::vector<std::vector<int>> chunk_clips;  // the clips of each chunk, in queue order
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;        // the filter branch of an overlapped graph
    std::vector<cudaEvent_t> ev_matched, ev_filtered;
    cudaEvent_t done = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

struct vsfeel_bm3d_batch {
    int device = 0;
    int sms = 0;
    std::vector<Clip> clips;
    std::vector<Class> classes;
    Dev<int> status;
    cudaEvent_t start = nullptr;  // recorded after each run's last graph
    int64_t device_bytes = 0;
    // Shared by every chunk of every class (they run one after another);
    // overlapped graphs alternate two sets, chunk k using set k & 1, so that
    // chunk k+1's matching writes while chunk k's filter still reads
    Dev<float> acc;
    Dev<uint32_t> match_xy, match_z;
    size_t acc_need = 0, table_need = 0;  // floats / blocks of the largest chunk
    // Overlapped class graphs (VSFEEL_BATCH_OVERLAP=1): chunk k's filter and
    // normalisation run on a second branch of lower priority beside chunk
    // k+1's persistent matching, in 8-group filter CTAs small enough to share
    // an SM with a matcher CTA. Measured +0.6% on the 64-clip workload (2,187
    // against 2,173 Mpx/s) for twice the buffers (11.2 against 5.6 GB), so
    // it is off by default.
    bool overlap = false;

    ~vsfeel_bm3d_batch() {
        if (start) wait_event(start);
        for (Class& c : classes) {
            if (c.stream) wait_stream(c.stream);
            if (c.exec) cudaGraphExecDestroy(c.exec);
            if (c.graph) cudaGraphDestroy(c.graph);
            if (c.done) cudaEventDestroy(c.done);
            for (cudaEvent_t e : c.ev_matched) cudaEventDestroy(e);
            for (cudaEvent_t e : c.ev_filtered) cudaEventDestroy(e);
            if (c.stream2) cudaStreamDestroy(c.stream2);
            if (c.stream) cudaStreamDestroy(c.stream);
            c.d_jobs.release();
            c.d_tile_first.release();
            c.d_norm.release();
            c.d_norm_first.release();
            c.d_filter_first.release();
            c.counter.release();
        }
        if (start) cudaEventDestroy(start);
        status.release();
        acc.release();
        match_xy.release();
        match_z.release();
    }

    // The StackJob of stack m of clip c, scattering into the class's
    // accumulators (slice_dst null when `silent`).
    StackJob make_job(const Clip& c, float* acc_base, int m, bool silent) const {
        const vsfeel_bm3d_info& in = c.info;
        const int r = in.radius, N = in.num_frames, tw = c.tw();
        StackJob job{};
        for (int z = 0; z < tw; ++z) {
            const int n = clampi(m - r + z, 0, N - 1);
            job.slice_frame[z] = c.desc.src + (size_t)n * c.desc.src_frame_stride;
            job.slice_dst[z] = nullptr;
            if (silent || slice_reads(m, z, N, r) == 0) continue;
            job.slice_dst[z] = acc_base + c.acc_off + c.pair_floats(n, m - (n - r));
        }
        job.dst_plane = (int64_t)c.plane;
        job.pitch = (int)c.desc.src_row_stride;
        job.dst_pitch = c.acc_pitch;
        job.width = in.width;
        job.height = in.height;
        job.radius = r;
        job.step = in.block_step;
        job.bm_range = in.bm_range;
        job.ps_num = in.ps_num;
        job.ps_range = in.ps_range;
        job.nbx = in.blocks_x;
        job.nby = in.blocks_y;
        job.thr = in.threshold;
        job.extractor = in.extractor;
        job.status = status.p;
        return job;
    }
};

namespace {

// Times every fitting tile shape with each allowed lane count (lanes_mask:
// bit 0, 8 lanes; bit 1, 16 lanes) on one stack of the class (no scatter);
// returns the fastest shape and sets cls.lanes to its lane count.
int autotune(vsfeel_bm3d_batch* b, Class& cls, const StackJob& sample_in, const bool fits[],
             int lanes_mask) {
    // the sample writes its match table into scratch of its own
    StackJob sample = sample_in;
    Dev<uint32_t> xy, zz;
    xy.alloc((size_t)sample.nbx * sample.nby * 8);
    zz.alloc((size_t)sample.nbx * sample.nby);
    sample.match_xy = xy.p;
    sample.match_z = zz.p;
    Dev<StackJob> job;
    job.upload(std::vector<StackJob>{sample});
    Dev<int> first, counter;
    first.alloc(2);
    counter.alloc(1);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct Cleanup {  // frees the tuning scratch on every exit
        std::function<void()> fn;
        ~Cleanup() { fn(); }
    } cleanup{[&] {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        xy.release();
        zz.release();
        job.release();
        first.release();
        counter.release();
    }};
    check(cudaEventCreate(&e0), "cudaEventCreate");
    check(cudaEventCreate(&e1), "cudaEventCreate");
    int best = -1;
    double best_ms = 0.0;
    for (int s = 0; s < kTileShapes; ++s) {
        if (!fits[s]) continue;
        const int tiles = tile_count(sample, TileShape(s));
        const int h_first[2] = {0, tiles};
        check(cudaMemcpy(first.p, h_first, sizeof(h_first), cudaMemcpyHostToDevice), "cudaMemcpy");
        const size_t smem = tile_smem_bytes(sample, TileShape(s), kTableOnly);
        const BatchWork work{job.p, first.p, 1, counter.p};
        for (const int lanes : {8, 16}) {
            if (!(lanes_mask & (lanes == 8 ? 1 : 2))) continue;
            // as many CTAs as the SMs hold at once (two per SM for the
            // 16-block shapes, whose plans take ~115 KB)
            const int grid =
                std::min(b->sms * batch_ctas_per_sm(TileShape(s), kTableOnly, lanes, smem), tiles);
            float best_rep = 0.0f;
            for (int rep = 0; rep < 4; ++rep) {
                check(cudaMemsetAsync(counter.p, 0, sizeof(int), cls.stream), "cudaMemsetAsync");
                check(cudaEventRecord(e0, cls.stream), "cudaEventRecord");
                check(launch_batch_tiles(work, TileShape(s), kTableOnly, lanes, smem, grid,
                                         cls.stream),
                      "autotune launch");
                check(cudaEventRecord(e1, cls.stream), "cudaEventRecord");
                if (wait_stream(cls.stream) != VSFEEL_OK)
                    throw Fail{VSFEEL_E_TIMEOUT, "timed out while autotuning"};
                float ms = 0.0f;
                check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                if (rep > 0 && (rep == 1 || ms < best_rep)) best_rep = ms;  // first run warms up
            }
            (lanes == 8 ? cls.tuned_ms : cls.tuned_ms_16)[s] = best_rep;
            if (best < 0 || best_rep < best_ms) {
                best = s;
                best_ms = best_rep;
                cls.lanes = lanes;
            }
        }
    }
    return best;
}

// Chooses the class's tile shape (autotuning it when asked) and cuts its
// clips into chunks, recording each chunk's accumulator and match-table
// needs; nothing is allocated for the class yet.
void plan_class(vsfeel_bm3d_batch* b, Class& cls, bool tune, int forced, int lanes_mask) {
    check(cudaStreamCreateWithFlags(&cls.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreateWithFlags(&cls.done, cudaEventDisableTiming), "cudaEventCreate");
    // largest clips first: the queue's tail is made of small tiles
    std::stable_sort(cls.clips.begin(), cls.clips.end(), [&](int a, int c) {
        const auto& A = b->clips[a].info;
        const auto& C = b->clips[c].info;
        return (int64_t)A.width * A.height > (int64_t)C.width * C.height;
    });

    // which tile shapes fit every stack of the class
    bool fits[kTileShapes];
    for (int s = 0; s < kTileShapes; ++s) fits[s] = true;
    for (int ci : cls.clips) {
        const Clip& c = b->clips[ci];
        const StackJob probe = b->make_job(c, nullptr, 0, true);
        // the persistent kernel runs the sliding scan (radius < 3)
        for (int s = 0; s < kTileShapes; ++s)
            fits[s] = fits[s] && c.info.radius < 3 &&
                      tile_shape_fits(probe, TileShape(s), kTableOnly);
    }
    int shape = -1;
    cls.lanes = (lanes_mask & 1) ? 8 : 16;
    if (forced >= 0 && forced < kTileShapes && fits[forced]) {
        shape = forced;
        if (tune && lanes_mask == 3) {  // the shape is given: tune the lanes only
            bool only[kTileShapes] = {};
            only[forced] = true;
            const Clip& big = b->clips[cls.clips.front()];
            autotune(b, cls, b->make_job(big, nullptr, big.info.num_frames / 2, true), only, 3);
        }
    } else if (tune) {
        const Clip& big = b->clips[cls.clips.front()];
        const StackJob sample = b->make_job(big, nullptr, big.info.num_frames / 2, true);
        bool any = false;
        for (int s = 0; s < kTileShapes; ++s) any = any || fits[s];
        if (any) shape = autotune(b, cls, sample, fits, lanes_mask);
    } else {
        const TileShape order[] = {kTile8x4, kTile16x2, kTile8x2, kTile4x4};
        for (TileShape s : order)
            if (fits[s]) {
                shape = s;
                break;
            }
    }
    cls.tile_shape = shape;

    // Chunks of whole clips of at least kChunkTiles queue items (about 16
    // waves): a chunk's frames and accumulators are still in L2 when its
    // filter and normalisation run, while the persistent launch keeps small
    // clips together. Without a tile shape every clip is a chunk of its own
    // (its stacks run one after another and share one match table).
    const int64_t kChunkTiles = (int64_t)b->sms * 16;
    std::vector<int> cur;
    size_t acc = 0, blocks = 0;
    int64_t tiles = 0;
    auto close = [&] {
        cls.chunk_clips.push_back(cur);
        b->acc_need = std::max(b->acc_need, acc);
        b->table_need = std::max(b->table_need, blocks);
        cur.clear();
        acc = blocks = 0;
        tiles = 0;
    };
    for (int ci : cls.clips) {
        Clip& c = b->clips[ci];
        const size_t nb = (size_t)c.info.blocks_x * c.info.blocks_y;
        c.acc_off = acc;
        c.table_off = blocks;
        acc += (c.acc_floats() + 63) & ~size_t(63);
        blocks += shape >= 0 ? nb * c.info.num_frames : nb;
        if (shape >= 0)
            tiles += (int64_t)c.info.num_frames *
                     tile_count(b->make_job(c, nullptr, 0, true), TileShape(shape));
        cur.push_back(ci);
        if (shape < 0 || tiles >= kChunkTiles) close();
    }
    if (!cur.empty()) close();
}

// Builds the class's queue, filter and normalisation lists against the
// shared accumulators and match tables, uploads them and records the
// class's graph.
void finish_class(vsfeel_bm3d_batch* b, Class& cls) {
    const int shape = cls.tile_shape;
    const bool two = b->overlap && shape >= 0;  // direct-read classes stay on one stream
    const int fgroups = two ? 8 : 16;           // filter groups per CTA
    std::vector<int> first, nfirst, ffirst;  // chunk-relative prefix sums, chunk after chunk
    std::vector<NormalizeJob> norm;
    for (const std::vector<int>& members : cls.chunk_clips) {
        Class::Chunk ch{};
        ch.buf = two ? (int)(cls.chunks.size() & 1) : 0;
        float* acc_base = b->acc.p + (size_t)ch.buf * b->acc_need;
        uint32_t* xy_base = b->match_xy.p + (size_t)ch.buf * b->table_need * 8;
        uint32_t* z_base = b->match_z.p + (size_t)ch.buf * b->table_need;
        ch.job0 = (int)cls.jobs.size();
        ch.norm0 = (int)norm.size();
        ch.first_off = (int)first.size();
        ch.ffirst_off = (int)ffirst.size();
        ch.nfirst_off = (int)nfirst.size();
        ch.acc0 = 0;
        first.push_back(0);
        ffirst.push_back(0);
        nfirst.push_back(0);
        size_t acc_end = 0;
        for (int ci : members) {
            const Clip& c = b->clips[ci];
            const int N = c.info.num_frames, r = c.info.radius, tw = c.tw();
            const size_t nb = (size_t)c.info.blocks_x * c.info.blocks_y;
            for (int m = 0; m < N; ++m) {
                StackJob job = b->make_job(c, acc_base, m, false);
                // every stack of a tiled chunk is in flight at once: a match
                // table each; the direct-read kernels run stack after stack
                const size_t toff = c.table_off + (shape >= 0 ? (size_t)m * nb : 0);
                job.match_xy = xy_base + toff * 8;
                job.match_z = z_base + toff;
                if (shape >= 0) {
                    job.lanes = cls.lanes;
                    cls.smem = std::max(cls.smem, tile_smem_bytes(job, TileShape(shape), kTableOnly));
                    const int64_t t = (int64_t)first.back() + tile_count(job, TileShape(shape));
                    const int64_t fi = (int64_t)ffirst.back() + filter_items((int)nb, fgroups);
                    if (t > INT32_MAX || fi > INT32_MAX)
                        throw Fail{VSFEEL_E_ARG, "batch too large for one launch"};
                    first.push_back((int)t);
                    ffirst.push_back((int)fi);
                }
                cls.jobs.push_back(job);
            }
            for (int n = 0; n < N; ++n) {
                NormalizeJob nj{};
                for (int i = 0; i < tw; ++i) {
                    const int m = clampi(n - r + i, 0, N - 1);
                    nj.num[i] = acc_base + c.acc_off + c.pair_floats(n, m - (n - r));
                }
                nj.den_offset = (int64_t)c.plane;
                nj.tw = c.merged(n) ? 1 : tw;
                nj.width = c.info.width;
                nj.height = c.info.height;
                nj.src_pitch = c.acc_pitch;
                nj.out_pitch = (int)c.desc.dst_row_stride;
                nj.out = c.desc.dst + (size_t)n * c.desc.dst_frame_stride;
                norm.push_back(nj);
                const int64_t nt = (int64_t)nfirst.back() + normalize_tiles(nj.width, nj.height);
                if (nt > INT32_MAX) throw Fail{VSFEEL_E_ARG, "batch too large for one normalise launch"};
                nfirst.push_back((int)nt);
            }
            acc_end = c.acc_off + c.acc_floats();
        }
        ch.njobs = (int)cls.jobs.size() - ch.job0;
        ch.nnorm = (int)norm.size() - ch.norm0;
        ch.tiles = first.back();
        ch.filter_items = ffirst.back();
        ch.norm_tiles = nfirst.back();
        ch.acc_floats = acc_end;
        cls.chunks.push_back(ch);
    }
    for (const Class::Chunk& ch : cls.chunks) cls.tiles += ch.tiles;
    if (shape >= 0) {
        cls.d_filter_first.upload(ffirst);
        cls.d_tile_first.upload(first);
    }
    cls.d_jobs.upload(cls.jobs);
    cls.d_norm.upload(norm);
    cls.d_norm_first.upload(nfirst);
    cls.nnorm = (int)norm.size();
    cls.counter.alloc(cls.chunks.size());

    // capture the class's run: per chunk, clear its accumulators, match,
    // filter, normalise. Overlapped: the filter and normalisation of chunk
    // k go to a second stream of the lowest priority (the matching's stream
    // has the highest), after chunk k's matching; chunk k+2, which reuses
    // chunk k's buffer set, waits for them.
    if (two) {
        int least = 0, greatest = 0;
        check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "priority range");
        check(cudaStreamDestroy(cls.stream), "cudaStreamDestroy");
        cls.stream = nullptr;
        check(cudaStreamCreateWithPriority(&cls.stream, cudaStreamNonBlocking, greatest),
              "cudaStreamCreate");
        check(cudaStreamCreateWithPriority(&cls.stream2, cudaStreamNonBlocking, least),
              "cudaStreamCreate");
        for (size_t k = 0; k < cls.chunks.size() + 1; ++k) {
            cudaEvent_t e1, e2;
            check(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming), "cudaEventCreate");
            cls.ev_matched.push_back(e1);
            check(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming), "cudaEventCreate");
            cls.ev_filtered.push_back(e2);
        }
    }
    cudaStream_t ms = cls.stream, fs = two ? cls.stream2 : cls.stream;
    // the persistent grid: as many CTAs as the SMs hold at once
    const int ctas_per_sm =
        shape >= 0 ? batch_ctas_per_sm(TileShape(shape), kTableOnly, cls.lanes, cls.smem) : 1;
    check(cudaStreamBeginCapture(ms, cudaStreamCaptureModeRelaxed), "capture");
    cudaError_t err = cudaMemsetAsync(cls.counter.p, 0, sizeof(int) * cls.chunks.size(), ms);
    if (two && err == cudaSuccess) {
        // the filter branch joins the capture
        err = cudaEventRecord(cls.ev_matched.back(), ms);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(fs, cls.ev_matched.back(), 0);
    }
    for (size_t k = 0; k < cls.chunks.size() && err == cudaSuccess; ++k) {
        const Class::Chunk& ch = cls.chunks[k];
        float* acc_base = b->acc.p + (size_t)ch.buf * b->acc_need;
        if (two && k >= 2) err = cudaStreamWaitEvent(ms, cls.ev_filtered[k - 2], 0);
        if (err == cudaSuccess)
            err = cudaMemsetAsync(acc_base + ch.acc0, 0, ch.acc_floats * sizeof(float), ms);
        if (err == cudaSuccess && shape >= 0) {
            const BatchWork work{cls.d_jobs.p + ch.job0, cls.d_tile_first.p + ch.first_off, ch.njobs,
                                 cls.counter.p + k};
            const int grid = std::min(b->sms * ctas_per_sm, ch.tiles);
            err = launch_batch_tiles(work, TileShape(shape), kTableOnly, cls.lanes, cls.smem, grid,
                                     ms);
            if (err == cudaSuccess && two) {
                err = cudaEventRecord(cls.ev_matched[k], ms);
                if (err == cudaSuccess) err = cudaStreamWaitEvent(fs, cls.ev_matched[k], 0);
            }
            const FilterBatch fw{cls.d_jobs.p + ch.job0, cls.d_filter_first.p + ch.ffirst_off,
                                 ch.njobs};
            if (err == cudaSuccess) err = launch_filter_batch(fw, ch.filter_items, fgroups, fs);
        } else if (err == cudaSuccess) {
            for (int j = ch.job0; j < ch.job0 + ch.njobs && err == cudaSuccess; ++j) {
                err = launch_match(cls.jobs[j], ms);
                if (err == cudaSuccess) err = launch_filter(cls.jobs[j], ms);
            }
        }
        if (err == cudaSuccess) {
            const NormalizeBatch nw{cls.d_norm.p + ch.norm0, cls.d_norm_first.p + ch.nfirst_off,
                                    ch.nnorm};
            err = launch_normalize_batch(nw, ch.norm_tiles, fs);
        }
        if (err == cudaSuccess && two) err = cudaEventRecord(cls.ev_filtered[k], fs);
    }
    if (two && err == cudaSuccess) {
        // the filter branch rejoins the origin stream before the capture ends
        err = cudaEventRecord(cls.ev_filtered.back(), fs);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(ms, cls.ev_filtered.back(), 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(ms, &graph);
    cls.graph = graph;
    check(err, "recording the class's graph");
    check(end, "cudaStreamEndCapture");
    check(cudaGraphInstantiate(&cls.exec, cls.graph, 0), "cudaGraphInstantiate");
}

}  // namespace

extern "C" {

int vsfeel_bm3d_batch_create(const vsfeel_bm3d_batch_clip* clips, int nclips, int device, int flags,
                             vsfeel_bm3d_batch** out) {
    if (!out) return error(VSFEEL_E_ARG, "null output pointer");
    *out = nullptr;
    if (!clips || nclips <= 0) return error(VSFEEL_E_ARG, "no clips");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return error(VSFEEL_E_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return error(VSFEEL_E_ARG, "invalid device ordinal");

    auto* b = new (std::nothrow) vsfeel_bm3d_batch();
    if (!b) return error(VSFEEL_E_MEMORY, "out of host memory");
    b->device = device;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    int rc = VSFEEL_OK;
    try {
        std::map<ClassKey, int> index;
        bool merge_slots = true;  // VSFEEL_MERGED_SLOTS=0: one pair per stack everywhere
        if (const char* v = std::getenv("VSFEEL_MERGED_SLOTS")) merge_slots = v[0] != '0';
        for (int i = 0; i < nclips; ++i) {
            const vsfeel_bm3d_batch_clip& d = clips[i];
            Clip c;
            c.desc = d;
            if (d.args.has_ref)
                throw Fail{VSFEEL_E_UNSUPPORTED, "clip " + std::to_string(i) +
                                                     ": the final (Wiener) pass with \"ref\" is not "
                                                     "supported by this build"};
            vsfeel_bm3d_video_info vi{d.width, d.height, d.num_frames, VSFEEL_CF_GRAY,
                                      VSFEEL_ST_FLOAT, 32, 0, 0};
            if (const int prc = parse_to_info(&d.args, &vi, &c.info); prc != VSFEEL_OK) {
                std::string msg = vsfeel_bm3d_last_error();
                if (msg.rfind("BM3D: ", 0) == 0) msg = msg.substr(6);
                throw Fail{prc, "clip " + std::to_string(i) + ": " + msg};
            }
            if (!d.src || !d.dst) throw Fail{VSFEEL_E_ARG, "clip " + std::to_string(i) + ": null buffer"};
            if (d.src_row_stride < d.width || d.dst_row_stride < d.width ||
                d.src_row_stride > INT32_MAX || d.dst_row_stride > INT32_MAX)
                throw Fail{VSFEEL_E_ARG, "clip " + std::to_string(i) + ": row stride smaller than the width"};
            if (d.src_frame_stride < d.src_row_stride * d.height ||
                d.dst_frame_stride < d.dst_row_stride * d.height)
                throw Fail{VSFEEL_E_ARG, "clip " + std::to_string(i) + ": frame stride smaller than a plane"};
            c.acc_pitch = (d.width + 31) & ~31;
            c.plane = (size_t)d.height * c.acc_pitch;
            c.plan_slots(merge_slots);
            b->clips.push_back(c);
            const ClassKey key{c.info.radius, c.info.block_step, c.info.bm_range, c.info.ps_num,
                               c.info.ps_range};
            auto it = index.find(key);
            if (it == index.end()) {
                it = index.emplace(key, (int)b->classes.size()).first;
                b->classes.emplace_back();
                b->classes.back().key = key;
            }
            b->classes[it->second].clips.push_back(i);
        }
        check(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device), "attribute");
        b->status.alloc(1);
        check(cudaMemset(b->status.p, 0, sizeof(int)), "cudaMemset");
        check(cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming), "cudaEventCreate");
        const int forced = ((flags >> 4) & 15) - 1;
        const int force_lanes = (flags >> 8) & 15;  // 0: tune or default; 1: 8; 2: 16
        const int lanes_mask = force_lanes == 1 ? 1 : (force_lanes == 2 ? 2 : 3);
        for (Class& cls : b->classes)
            plan_class(b, cls, (flags & VSFEEL_BATCH_AUTOTUNE) != 0, forced,
                       (flags & VSFEEL_BATCH_AUTOTUNE) || force_lanes ? lanes_mask : 1);
        if (const char* v = std::getenv("VSFEEL_BATCH_OVERLAP")) b->overlap = v[0] == '1';
        const size_t sets = b->overlap ? 2 : 1;
        b->acc.alloc(b->acc_need * sets);
        b->match_xy.alloc(b->table_need * 8 * sets);
        b->match_z.alloc(b->table_need * sets);
        b->device_bytes = (int64_t)(b->acc.n + b->match_xy.n + b->match_z.n) * 4;
        for (Class& cls : b->classes) finish_class(b, cls);
    } catch (const Fail& f) {
        rc = error(f.code, f.msg);
    } catch (const std::bad_alloc&) {
        rc = error(VSFEEL_E_MEMORY, "out of host memory");
    }
    if (rc != VSFEEL_OK) {
        delete b;
        if (prev >= 0) cudaSetDevice(prev);
        return rc;
    }
    if (prev >= 0) cudaSetDevice(prev);
    *out = b;
    return VSFEEL_OK;
}

int vsfeel_bm3d_batch_run(vsfeel_bm3d_batch* b, void* stream) {
    if (!b) return error(VSFEEL_E_ARG, "null batch");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    int rc = VSFEEL_OK;
    try {
        // classes one after another on the caller's stream: run side by side,
        // their persistent launches compete for SMs and L2 (measured slower)
        cudaStream_t st = (cudaStream_t)stream;
        for (Class& c : b->classes) check(cudaGraphLaunch(c.exec, st), "cudaGraphLaunch");
        check(cudaEventRecord(b->start, st), "cudaEventRecord");
    } catch (const Fail& f) {
        rc = error(f.code, f.msg);
    }
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

int vsfeel_bm3d_batch_finish(vsfeel_bm3d_batch* b) {
    if (!b) return error(VSFEEL_E_ARG, "null batch");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    int rc = wait_event(b->start);
    if (rc == VSFEEL_OK) {
        int word = 0;
        cudaError_t e = cudaMemcpy(&word, b->status.p, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            rc = error(VSFEEL_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
        } else if (word != 0) {
            cudaMemset(b->status.p, 0, sizeof(int));
            rc = error(VSFEEL_E_CUDA, status_text(word));
        }
    }
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

int vsfeel_bm3d_batch_classes(const vsfeel_bm3d_batch* b, int* nclasses, int64_t* device_bytes) {
    if (!b || !nclasses || !device_bytes) return error(VSFEEL_E_ARG, "null argument");
    *nclasses = (int)b->classes.size();
    *device_bytes = b->device_bytes;
    return VSFEEL_OK;
}

int vsfeel_bm3d_batch_class(const vsfeel_bm3d_batch* b, int index,
                            vsfeel_bm3d_batch_class_info* info) {
    if (!b || !info) return error(VSFEEL_E_ARG, "null argument");
    if (index < 0 || index >= (int)b->classes.size()) return error(VSFEEL_E_ARG, "class index out of range");
    const Class& c = b->classes[index];
    std::memset(info, 0, sizeof(*info));
    info->radius = std::get<0>(c.key);
    info->block_step = std::get<1>(c.key);
    info->bm_range = std::get<2>(c.key);
    info->ps_num = std::get<3>(c.key);
    info->ps_range = std::get<4>(c.key);
    info->clips = (int)c.clips.size();
    info->stacks = (int)c.jobs.size();
    info->tiles = c.tiles;
    info->tile_shape = c.tile_shape;
    info->lanes = c.tile_shape >= 0 ? c.lanes : 8;
    for (int s = 0; s < kTileShapes && s < VSFEEL_TILE_SHAPES; ++s) {
        info->tuned_ms[s] = c.tuned_ms[s];
        info->tuned_ms_16[s] = c.tuned_ms_16[s];
    }
    return VSFEEL_OK;
}

void vsfeel_bm3d_batch_free(vsfeel_bm3d_batch* b) {
    if (!b) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    delete b;
    if (prev >= 0) cudaSetDevice(prev);
}

}  // extern "C"
