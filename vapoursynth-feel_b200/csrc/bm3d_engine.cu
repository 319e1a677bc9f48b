// Host side of the B200 BM3Dv2 basic estimate: the C ABI declared in
// include/vsfeel_bm3d.h.
//
// Replaces the reference's Vulkan machinery (src/vsfeel.cpp, src/bm3d.cpp)
// with one CUDA stream per context, device-resident frames and a ring of
// per-output accumulator slots:
//
// * Stack m (the reference blocks of frame m) searches and filters in the
//   slices z = 0..2r, slice z being frame clamp(m - r + z). Output frame n
//   sums, in order i = 0..2r, slice agg_z(i, n) of stack clamp(n - r + i)
//   (src/bm3d.cpp:369-371, 628-696). Each slice is therefore read by at most
//   one output, n = clamp(m - r + z); slices no output reads are dropped.
// * Output n owns a slot of TW (numerator, weight) plane pairs, one per
//   contributing stack m = n - r + j. A stack scatters straight into its
//   outputs' slots, so no per-stack result cache is needed; output n is
//   normalised as soon as stack min(n + r, N - 1) is done, and its slot is
//   reused by output n + 2r + 1.
#include "bm3d_device.cuh"
#include "vsfeel_bm3d.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

using namespace vsfeel;

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = "BM3D: " + msg;
    return code;
}

struct CudaError {
    cudaError_t err;
    const char* what;
};

#define VSF_CUDA(call)                                                       \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) throw CudaError{e_, #call};                   \
    } while (0)

inline int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

int agg_z(int i, int n, int nframes, int radius) {
    return std::min(std::max(2 * radius - i, n - nframes + 1 + radius), n + radius);
}

// sigma factor of the pass, src/bm3d.cpp:1103-1107
float sigma_factor(bool final_pass) {
    const uint32_t bits = final_pass ? 0x3e40c0c1u : 0x3f021bb6u;
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// Test hook (VSFEEL_TEST_PROBE_TILE=k): tile k-1 of every stack's tiled
// matching reports a window outside its staged region, so that the status
// word's path to the caller can be tested without a real fault. Read per
// call; unset or 0 means off.
int probe_tile_from_env() {
    const char* s = std::getenv("VSFEEL_TEST_PROBE_TILE");
    return (s && *s) ? std::max(0, std::atoi(s)) : 0;
}

int64_t timeout_ms() {
    const char* s = std::getenv("VSFEEL_TIMEOUT_MS");
    if (s && *s) {
        const long long v = std::atoll(s);
        if (v > 0) return v;
    }
    return 120000;
}

// Bounded wait on an event: polls until it has fired or the deadline passes.
int wait_event(cudaEvent_t e, int64_t limit_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    int spins = 0;
    for (;;) {
        const cudaError_t q = cudaEventQuery(e);
        if (q == cudaSuccess) return VSFEEL_OK;
        if (q != cudaErrorNotReady)
            return fail(VSFEEL_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(q));
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - t0)
                            .count();
        if (ms >= limit_ms)
            return fail(VSFEEL_E_TIMEOUT, "timed out after " + std::to_string(ms) +
                                              " ms waiting for the GPU");
        if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// Bounded wait on a stream: polls until idle or the deadline passes.
int wait_stream(cudaStream_t s, int64_t limit_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    int spins = 0;
    for (;;) {
        const cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return VSFEEL_OK;
        if (e != cudaErrorNotReady)
            return fail(VSFEEL_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - t0)
                            .count();
        if (ms >= limit_ms)
            return fail(VSFEEL_E_TIMEOUT, "timed out after " + std::to_string(ms) +
                                              " ms waiting for the GPU");
        if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

struct Settings {
    int width = 0, height = 0, nframes = 0;
    bool chroma = false;
    bool final_pass = false;  // a "ref" clip was given: the Wiener pass
    float sigma = 3.0f, thr = 0.0f, extractor = 0.0f;
    int step = 8, bm_range = 9, radius = 0, ps_num = 2, ps_range = 4, num_streams = 4;
};

// Argument parsing and validation in the order and with the messages of
// BM3DCreate (src/bm3d.cpp:1062-1190, 1257-1275). `plane` selects which
// element of the per-plane arrays applies and which plane's dimensions the
// context works on; the reference itself always uses element [0] on luma.
int parse_args(const vsfeel_bm3d_args* a, const vsfeel_bm3d_video_info* vi, Settings& s,
               int plane = 0) {
    if (!a || !vi) return fail(VSFEEL_E_ARG, "null argument");
    if (a->has_ref) {
        const vsfeel_bm3d_video_info* r = a->ref_info;
        if (!r) return fail(VSFEEL_E_ARG, "\"ref\" given without its format");
        if (r->color_family != vi->color_family || r->sample_type != vi->sample_type ||
            r->bits_per_sample != vi->bits_per_sample || r->sub_sampling_w != vi->sub_sampling_w ||
            r->sub_sampling_h != vi->sub_sampling_h)
            return fail(VSFEEL_E_ARG, "\"ref\" must be of the same format as \"clip\"");
        if (r->width != vi->width || r->height != vi->height)
            return fail(VSFEEL_E_ARG, "\"ref\" must be of the same dimensions as \"clip\"");
        if (r->num_frames != vi->num_frames)
            return fail(VSFEEL_E_ARG, "\"ref\" must be of the same number of frames as \"clip\"");
    }
    if (vi->width <= 0 || vi->height <= 0 || vi->sample_type != VSFEEL_ST_FLOAT ||
        vi->bits_per_sample != 32)
        return fail(VSFEEL_E_FORMAT, "only constant format 32 bit float input supported");

    float sigma[3];
    for (int i = 0; i < 3; ++i) {
        if (i < a->sigma_count) {
            sigma[i] = a->sigma[i];
            if (sigma[i] < 0.0f) return fail(VSFEEL_E_ARG, "\"sigma\" must be non-negative");
        } else {
            sigma[i] = i == 0 ? 3.0f : sigma[i - 1];
        }
    }
    int step[3], bmr[3], psn[3], psr[3];
    for (int i = 0; i < 3; ++i) {
        if (i < a->block_step_count) {
            step[i] = a->block_step[i];
            if (step[i] <= 0 || step[i] > 8)
                return fail(VSFEEL_E_ARG, "\"block_step\" must be in range [1, 8]");
        } else {
            step[i] = i == 0 ? 8 : step[i - 1];
        }
    }
    for (int i = 0; i < 3; ++i) {
        if (i < a->bm_range_count) {
            bmr[i] = a->bm_range[i];
            if (bmr[i] <= 0) return fail(VSFEEL_E_ARG, "\"bm_range\" must be positive");
        } else {
            bmr[i] = i == 0 ? 9 : bmr[i - 1];
        }
    }
    s.radius = a->radius_set ? a->radius : 0;
    if (s.radius < 0 || s.radius > kMaxRadius)
        return fail(VSFEEL_E_ARG, "\"radius\" must be in range [0, 4]");
    for (int i = 0; i < 3; ++i) {
        if (i < a->ps_num_count) {
            psn[i] = a->ps_num[i];
            if (psn[i] <= 0 || psn[i] > 8)
                return fail(VSFEEL_E_ARG, "\"ps_num\" must be in range [1, 8]");
        } else {
            psn[i] = i == 0 ? 2 : psn[i - 1];
        }
    }
    for (int i = 0; i < 3; ++i) {
        if (i < a->ps_range_count) {
            psr[i] = a->ps_range[i];
            if (psr[i] <= 0) return fail(VSFEEL_E_ARG, "\"ps_range\" must be positive");
        } else {
            psr[i] = i == 0 ? 4 : psr[i - 1];
        }
    }
    s.num_streams = a->num_streams_set ? a->num_streams : 4;
    if (s.num_streams <= 0) return fail(VSFEEL_E_ARG, "\"num_streams\" must be positive");
    const int ext = a->extractor_exp_set ? a->extractor_exp : 0;

    if (vi->color_family == VSFEEL_CF_GRAY) {
        s.chroma = false;
    } else if (vi->color_family == VSFEEL_CF_YUV) {
        s.chroma = true;
    } else {
        return fail(VSFEEL_E_FORMAT, "only Gray and YUV input are currently supported");
    }
    if (plane < 0 || plane >= (s.chroma ? 3 : 1))
        return fail(VSFEEL_E_ARG, "\"planes\" must name planes of the clip");
    if (plane > 0 && (vi->sub_sampling_w < 0 || vi->sub_sampling_w > 4 ||
                      vi->sub_sampling_h < 0 || vi->sub_sampling_h > 4))
        return fail(VSFEEL_E_FORMAT, "invalid chroma subsampling");

    // a ref-pass threshold uses the same element as the plane's sigma
    // (src/bm3d.cpp:1090-1113 scales all three)
    s.sigma = sigma[plane];
    s.final_pass = a->has_ref != 0;
    s.thr = sigma[plane] * sigma_factor(s.final_pass);
    s.extractor = ext != 0 ? std::ldexp(1.0f, ext) : 0.0f;
    s.step = step[plane];
    s.bm_range = bmr[plane];
    s.ps_num = psn[plane];
    s.ps_range = psr[plane];
    // chroma plane sizes as VapourSynth derives them: width >> ssw
    s.width = plane > 0 ? vi->width >> vi->sub_sampling_w : vi->width;
    s.height = plane > 0 ? vi->height >> vi->sub_sampling_h : vi->height;
    s.nframes = vi->num_frames;

    // The reference reads outside the plane below 8x8; the match table packs
    // coordinates in 16 bits.
    if (s.width < 8 || s.height < 8)
        return fail(VSFEEL_E_FORMAT, plane > 0 ? "chroma planes must be at least 8x8"
                                               : "clip dimensions must be at least 8x8");
    if (s.width > 65535 || s.height > 65535)
        return fail(VSFEEL_E_FORMAT, "clip dimensions must be at most 65535");
    if (s.nframes <= 0) return fail(VSFEEL_E_FORMAT, "clip must have at least one frame");
    return VSFEEL_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void ensure(size_t count) {
        if (count <= n) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        VSF_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

}  // namespace

struct vsfeel_bm3d {
    Settings s;
    int device = 0;
    int nbx = 0, nby = 0, nblocks = 0;
    int acc_pitch = 0;       // floats per accumulator / staged frame row
    size_t acc_plane = 0;    // floats per accumulator plane
    cudaStream_t stream = nullptr;
    std::mutex lock;
    std::atomic<int64_t> launches{0};
    // Match and filter in one tiled launch (the match table stays on chip).
    // Off by default: at the matcher's one CTA of 8 warps per SM the filter
    // runs slower than the standalone filter kernel (2.41 against 1.81 + 0.16
    // ms per 1080p radius-2 stack on B200).
    bool fused = false;
    // Lanes per reference block of the tiled sliding matcher (radius < 3):
    // 8 (256-thread CTAs) or 16 (512-thread CTAs, twice the warps per SM at
    // the same shared memory). VSFEEL_MATCH_LANES overrides the default.
    int match_lanes = 8;
    // The plain path's autotuner (VSFEEL_AUTOTUNE=0 turns it off): on the
    // first call that launches stacks, one table-only matching launch of the
    // call's first stack per fitting (tile shape, lanes) pair, timed with
    // events; a pair replaces the default only when it is at least 2% faster.
    // Every pair gives the same match table.
    bool autotune = true;
    // Merged output slots (VSFEEL_MERGED_SLOTS=0 turns them off): without the
    // extractor, an interior output's 2r+1 contributing stacks scatter into
    // one (numerator, weight-origin) plane pair of its ring slot instead of
    // one pair each, and the normaliser reads that one pair. The reference
    // sums its per-stack slices in FP64 after accumulating each in FP32; the
    // merged FP32 sum differs from that by float rounding only (~1e-7 on the
    // [0, 1] scale), like the reference's own atomic order from run to run.
    // With the extractor the per-stack slices are kept, so that every slice
    // sum stays exactly the reference's. An output within r of a clip end
    // reads a clamped stack's slice more than once (the reference's
    // weighting), so it keeps its per-stack slices too.
    bool merge_slots = true;
    int tuned = 0;           // 0: not tuned yet; 1: tuned (or tuning skipped)
    int tuner_ran = 0;       // 1: the autotuner timed the shapes
    int tuned_shape_plus1 = 0;
    void ensure_tuned(const StackJob& sample_in, cudaStream_t st) {
        if (tuned || !autotune || sample_in.radius >= 3 || sample_in.wiener) {
            tuned = 1;
            return;
        }
        tuned = 1;
        const int def = default_tile_shape(sample_in, kTableOnly);
        if (def < 0) return;
        tuner_ran = 1;
        StackJob sample = sample_in;
        for (int z = 0; z < kMaxTW; ++z) sample.slice_dst[z] = nullptr;  // table only
        cudaEvent_t e0 = next_event(), e1 = next_event();
        auto time_one = [&](int shape, int lanes) -> float {
            sample.tile_shape_plus1 = shape + 1;
            sample.lanes = lanes;
            float best = -1.0f;
            for (int rep = 0; rep < 3; ++rep) {
                VSF_CUDA(cudaEventRecord(e0, st));
                VSF_CUDA(launch_match(sample, st));
                launches += 1;
                VSF_CUDA(cudaEventRecord(e1, st));
                if (wait_event(e1, timeout_ms()) != VSFEEL_OK) return -1.0f;
                float ms = 0.0f;
                VSF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (rep > 0 && (best < 0.0f || ms < best)) best = ms;  // the first warms up
            }
            return best;
        };
        const float base = time_one(def, 8);
        if (base <= 0.0f) return;
        float best = base;
        for (int s = 0; s < kTileShapes; ++s) {
            if (!tile_shape_fits(sample, TileShape(s), kTableOnly)) continue;
            for (const int lanes : {8, 16}) {
                if (s == def && lanes == 8) continue;
                const float t = time_one(s, lanes);
                if (t > 0.0f && t < best && t < 0.98f * base) {
                    best = t;
                    tuned_shape_plus1 = s + 1;
                    match_lanes = lanes;
                }
            }
        }
    }

    DevBuf<float> ring;       // (2r+1) slots x TW x {num, den} planes
    DevBuf<float> gscale;     // the backward's scaled output gradients, a ring of frames
    DevBuf<uint32_t> match_xy;
    DevBuf<uint32_t> match_z;
    DevBuf<float> frames;     // staged input frames (host and frame paths)
    DevBuf<float> outbuf;     // staged output frames (host and frame paths)
    DevBuf<int> status;       // kernels' internal-error word
    // host path: uploads and downloads on streams of their own, ordered
    // against the compute stream by per-frame events
    cudaStream_t up_stream = nullptr, down_stream = nullptr;
    std::vector<cudaEvent_t> frame_events, out_events;

    // The end of the context's last enqueued work, on whatever stream it
    // ran: the next call's streams wait for it first, so calls on different
    // streams, or after a bounded wait gave up, never overlap on the
    // context's buffers.
    cudaEvent_t tail = nullptr;
    bool tail_set = false;
    bool tail_from_request = false;  // set by the per-frame path, which orders its own work
    void after_prior(cudaStream_t st) {
        if (tail_set) VSF_CUDA(cudaStreamWaitEvent(st, tail, 0));
    }
    void mark_tail(cudaStream_t st, bool from_request = false) {
        if (!tail) VSF_CUDA(cudaEventCreateWithFlags(&tail, cudaEventDisableTiming));
        VSF_CUDA(cudaEventRecord(tail, st));
        tail_set = true;
        tail_from_request = from_request;
    }

    void copy_streams(size_t nframes_in, size_t nout) {
        if (!up_stream) VSF_CUDA(cudaStreamCreateWithFlags(&up_stream, cudaStreamNonBlocking));
        if (!down_stream) VSF_CUDA(cudaStreamCreateWithFlags(&down_stream, cudaStreamNonBlocking));
        auto grow = [](std::vector<cudaEvent_t>& v, size_t n) {
            while (v.size() < n) {
                cudaEvent_t e;
                VSF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                v.push_back(e);
            }
        };
        grow(frame_events, nframes_in);
        grow(out_events, nout);
    }

    int* status_word() {
        if (!status.p) {
            status.ensure(1);
            VSF_CUDA(cudaMemset(status.p, 0, sizeof(int)));
        }
        return status.p;
    }

    // Waits for `st` (bounded) and reports an internal error the kernels flagged.
    int finish(cudaStream_t st) {
        const int rc = wait_stream(st, timeout_ms());
        if (rc != VSFEEL_OK || !status.p) return rc;
        int word = 0;
        VSF_CUDA(cudaMemcpy(&word, status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (word != 0) {
            VSF_CUDA(cudaMemset(status.p, 0, sizeof(int)));
            invalidate_stacks();
            return fail(VSFEEL_E_CUDA, status_text(word));
        }
        return VSFEEL_OK;
    }
    // Forgets every cached stack of the per-frame path: after a kernel
    // flagged an internal error, a cached stack may hold a skipped scan.
    void invalidate_stacks() { std::fill(stack_tag.begin(), stack_tag.end(), -1); }
    // recorded after a direct-path upload: the frame is released once it fires
    cudaEvent_t direct_copy = nullptr;
    cudaEvent_t direct_copy_done() {
        if (!direct_copy) VSF_CUDA(cudaEventCreateWithFlags(&direct_copy, cudaEventDisableTiming));
        return direct_copy;
    }
    std::map<int, int> frame_slot;  // frame cache of the per-frame path
    std::vector<int> slot_frame;
    // Stack cache of the per-frame path: slot c holds the TW (numerator,
    // weight) slice pairs of stack stack_tag[c] (-1: empty), last used at
    // request stack_use[c].
    DevBuf<float> stackcache;
    std::vector<int> stack_tag;
    std::vector<int64_t> stack_use;
    int64_t requests = 0;
    int stack_slots() const { return tw() + std::min(s.num_streams, 16); }
    float* stack_slices(int c) { return stackcache.p + (size_t)c * tw() * 2 * acc_plane; }

    // Page-locked staging of the per-frame path, so that requests from
    // several threads overlap their host copies with each other's kernels.
    // Uploads: a fetched frame is copied on the host into one of kUpSlots
    // page-locked planes and released at once; the plane is reused after
    // its device copy has run (up_done). Outputs: each request holds a
    // request slot (device plane, page-locked plane and status word, event)
    // from enqueue until its caller has copied the output out.
    static constexpr int kUpSlots = 8;
    float* up_host = nullptr;
    cudaEvent_t up_done[kUpSlots] = {};
    bool up_used[kUpSlots] = {};
    int up_next = 0;
    struct RequestSlot {
        float* dev = nullptr;
        float* host = nullptr;
        int* status = nullptr;
        cudaEvent_t normalised = nullptr, done = nullptr;
        bool busy = false;
    };
    // per frame-cache slot: recorded after the last stack that read it, so
    // that an upload into the slot on the copy stream waits for that stack
    std::vector<cudaEvent_t> frame_read;
    std::vector<char> frame_read_set;
    std::vector<RequestSlot> req_slots;
    unsigned char* req_host = nullptr;
    DevBuf<float> req_dev;
    std::condition_variable req_cv;
    std::atomic<int> requests_in_flight{0};  // callers inside get_frame
    int request_slots() const { return std::max(2, std::min(s.num_streams, 16)); }
    size_t packed_plane_floats() const { return (size_t)s.width * s.height; }
    void request_staging() {
        if (!up_host) {
            VSF_CUDA(cudaHostAlloc(&up_host, sizeof(float) * packed_plane_floats() * kUpSlots,
                                   cudaHostAllocPortable));
            for (auto& e : up_done) VSF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        if (req_slots.empty()) {
            const int k = request_slots();
            const size_t host_bytes = sizeof(float) * packed_plane_floats() + 64;
            VSF_CUDA(cudaHostAlloc(&req_host, host_bytes * k, cudaHostAllocPortable));
            req_dev.ensure(frame_floats() * k);
            req_slots.resize(k);
            for (int i = 0; i < k; ++i) {
                RequestSlot& r = req_slots[i];
                r.dev = req_dev.p + frame_floats() * i;
                r.host = reinterpret_cast<float*>(req_host + host_bytes * i);
                r.status = reinterpret_cast<int*>(req_host + host_bytes * i +
                                                  sizeof(float) * packed_plane_floats());
                VSF_CUDA(cudaEventCreateWithFlags(&r.normalised, cudaEventDisableTiming));
                VSF_CUDA(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
            }
        }
        copy_streams(0, 0);
    }

    // event trace: (kind, start, stop) per traced launch
    struct Mark {
        int kind;
        cudaEvent_t start, stop;
    };
    bool tracing = false;
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> event_pool;
    size_t events_used = 0;

    cudaEvent_t next_event() {
        if (events_used == event_pool.size()) {
            cudaEvent_t e;
            VSF_CUDA(cudaEventCreate(&e));
            event_pool.push_back(e);
        }
        return event_pool[events_used++];
    }
    // records `launch` between two events when tracing
    template <class F>
    void traced(int kind, cudaStream_t st, F&& launch) {
        if (!tracing) {
            VSF_CUDA(launch());
            return;
        }
        Mark mk{kind, next_event(), next_event()};
        VSF_CUDA(cudaEventRecord(mk.start, st));
        VSF_CUDA(launch());
        VSF_CUDA(cudaEventRecord(mk.stop, st));
        marks.push_back(mk);
    }

    int tw() const { return 2 * s.radius + 1; }
    int clampf(int f) const { return clampi(f, 0, s.nframes - 1); }

    size_t ring_floats() const { return (size_t)tw() * tw() * 2 * acc_plane; }
    // Whether output n's ring slot is one merged plane pair.
    bool merged(int n) const {
        return merge_slots && s.extractor == 0.0f && s.radius > 0 && n - s.radius >= 0 &&
               n + s.radius <= s.nframes - 1;
    }
    // Plane pairs output n's ring slot uses.
    int slot_pairs(int n) const { return merged(n) ? 1 : tw(); }
    float* slot_pair(int n, int j) {
        const int slot = n % tw();
        return ring.p + ((size_t)slot * tw() + j) * 2 * acc_plane;
    }

    // The slice of stack m that output n reads (n = clamp(m - r + z)).
    int read_slice(int n, int m) const {
        const int r = s.radius;
        for (int i = 0; i < tw(); ++i)
            if (clampf(n - r + i) == m) return (r == 0) ? 0 : agg_z(i, n, s.nframes, r);
        return -1;
    }

    // Saved state of the differentiable form: per stack a record of the
    // match table and the keep bits, then the per-output denominators.
    struct SavedLayout {
        int64_t off_xy, off_z, off_mask, stack_bytes, den_offset, den_pitch, bytes;
    };
    SavedLayout saved_layout() const {
        auto al = [](int64_t v) { return (v + 255) & ~int64_t(255); };
        SavedLayout L{};
        L.off_xy = 0;
        L.off_z = al(L.off_xy + 4 * 8 * (int64_t)nblocks);
        L.off_mask = al(L.off_z + 4 * (int64_t)nblocks);
        L.stack_bytes = al(L.off_mask + 8 * 8 * (int64_t)nblocks);
        L.den_offset = L.stack_bytes * s.nframes;
        L.den_pitch = acc_pitch;
        L.bytes = L.den_offset + 4 * (int64_t)s.nframes * s.height * acc_pitch;
        return L;
    }

    // `saved` (the differentiable form): write stack m's match table and keep
    // bits into its record instead of the context's match buffers.
    // frame_ptr: the search clip (the ref clip in the final pass); input_ptr:
    // the clip denoised in the final pass (its frames share frame_ptr's pitch)
    // The StackJob of stack m; its match table goes to (table_xy, table_z)
    // unless `saved` gives the stack's record.
    StackJob stack_job(int m, const std::function<const float*(int)>& frame_ptr, int in_pitch,
                       int out_lo, int out_hi, unsigned char* saved,
                       const std::function<const float*(int)>* input_ptr, float* own_slices,
                       uint32_t* table_xy, uint32_t* table_z) {
        const int r = s.radius;
        StackJob job{};
        for (int z = 0; z < tw(); ++z) {
            job.slice_frame[z] = frame_ptr(clampf(m - r + z));
            job.slice_input[z] = input_ptr ? (*input_ptr)(clampf(m - r + z)) : nullptr;
            const int n = clampf(m - r + z);
            job.slice_dst[z] = nullptr;
            // slice z goes to the output that reads it: into that output's
            // ring slot, or (own_slices) into the stack's own slice z
            if (n >= out_lo && n <= out_hi && read_slice(n, m) == z)
                job.slice_dst[z] = own_slices  ? own_slices + (size_t)z * 2 * acc_plane
                                   : merged(n) ? slot_pair(n, 0)
                                               : slot_pair(n, m - (n - r));
        }
        job.dst_plane = (int64_t)acc_plane;
        job.pitch = in_pitch;
        job.dst_pitch = acc_pitch;
        job.width = s.width;
        job.height = s.height;
        job.radius = r;
        job.step = s.step;
        job.bm_range = s.bm_range;
        job.ps_num = s.ps_num;
        job.ps_range = s.ps_range;
        job.nbx = nbx;
        job.nby = nby;
        job.thr = s.thr;
        job.wiener = (s.final_pass && input_ptr) ? 1 : 0;
        job.extractor = s.extractor;
        job.match_xy = table_xy;
        job.match_z = table_z;
        job.mask_out = nullptr;
        if (saved) {
            const SavedLayout L = saved_layout();
            unsigned char* rec = saved + (size_t)m * L.stack_bytes;
            job.match_xy = reinterpret_cast<uint32_t*>(rec + L.off_xy);
            job.match_z = reinterpret_cast<uint32_t*>(rec + L.off_z);
            job.mask_out = reinterpret_cast<uint64_t*>(rec + L.off_mask);
        }
        job.status = status_word();
        job.probe_tile = probe_tile_from_env();
        job.lanes = match_lanes;
        job.tile_shape_plus1 = tuned_shape_plus1;
        return job;
    }

    void launch_stack(int m, const std::function<const float*(int)>& frame_ptr, int in_pitch,
                      int out_lo, int out_hi, cudaStream_t st, unsigned char* saved = nullptr,
                      bool table_only = false,
                      const std::function<const float*(int)>* input_ptr = nullptr,
                      float* own_slices = nullptr) {
        const StackJob job = stack_job(m, frame_ptr, in_pitch, out_lo, out_hi, saved, input_ptr,
                                       own_slices, match_xy.p, match_z.p);
        // fused: one tiled launch matches and filters (the match table stays
        // on chip); otherwise the match table goes through global memory
        if (table_only) {
            traced(VSFEEL_KERNEL_MATCH, st, [&] { return launch_match(job, st); });
            launches += 1;
            return;
        }
        const TileMode mode = job.mask_out ? kFusedSave : kFused;
        const int shape = (fused && !job.wiener) ? default_tile_shape(job, mode) : -1;
        if (shape >= 0) {
            traced(VSFEEL_KERNEL_MATCH, st,
                   [&] { return launch_match_tiles(job, TileShape(shape), mode, st); });
            launches += 1;
            return;
        }
        traced(VSFEEL_KERNEL_MATCH, st, [&] { return launch_match(job, st); });
        traced(VSFEEL_KERNEL_FILTER, st, [&] { return launch_filter(job, st); });
        launches += 2;
    }

    // stack_slices_of(m): stack m's own slices (the stack cache); by default
    // output n's ring slot
    void launch_normalize(int n, float* out, int out_pitch, cudaStream_t st,
                          unsigned char* saved = nullptr,
                          const std::function<float*(int)>* stack_slices_of = nullptr) {
        const int r = s.radius;
        NormalizeJob job{};
        for (int i = 0; i < tw(); ++i) {
            const int m = clampf(n - r + i);
            job.num[i] = stack_slices_of
                             ? (*stack_slices_of)(m) + (size_t)read_slice(n, m) * 2 * acc_plane
                             : slot_pair(n, m - (n - r));
        }
        job.den_offset = (int64_t)acc_plane;
        job.tw = tw();
        if (!stack_slices_of && merged(n)) {
            job.num[0] = slot_pair(n, 0);
            job.tw = 1;
        }
        job.width = s.width;
        job.height = s.height;
        job.src_pitch = acc_pitch;
        job.out_pitch = out_pitch;
        job.out = out;
        job.den_out = nullptr;
        if (saved) {
            const SavedLayout L = saved_layout();
            job.den_out = reinterpret_cast<float*>(saved + L.den_offset) + (size_t)n * frame_floats();
            job.den_pitch = (int)L.den_pitch;
        }
        traced(VSFEEL_KERNEL_NORMALIZE, st, [&] { return vsfeel::launch_normalize(job, st); });
        launches += 1;
    }

    // Second stream of the overlapped schedule (see run) and its events:
    // ev_match[b] after the matching that wrote table buffer b, ev_filter[b]
    // after the filtering that read it.
    cudaStream_t filter_stream = nullptr, match_stream = nullptr;
    cudaEvent_t ev_match[2] = {}, ev_filter[2] = {}, ev_fork = nullptr, ev_join = nullptr,
                ev_join_match = nullptr;
    DevBuf<uint32_t> match_xy2, match_z2;
    bool overlap = true;  // VSFEEL_OVERLAP_FILTER=0: one stream, as the fused mode
    void overlap_setup() {
        if (filter_stream) return;
        int least = 0, greatest = 0;
        VSF_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        VSF_CUDA(cudaStreamCreateWithPriority(&match_stream, cudaStreamNonBlocking, greatest));
        VSF_CUDA(cudaStreamCreateWithPriority(&filter_stream, cudaStreamNonBlocking, least));
        for (cudaEvent_t* e : {&ev_match[0], &ev_match[1], &ev_filter[0], &ev_filter[1], &ev_fork,
                               &ev_join, &ev_join_match})
            VSF_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }

    // Denoises outputs [first, first+count) from device frames.
    // before_stack(m, s) runs before stack m is launched on stream s,
    // after_output(n, s) after output n's normalisation is enqueued on stream
    // s (the host path's copy overlap). All work is ordered after the prior
    // work of st, and st waits for all of it at the end.
    //
    // Overlapped schedule (the default with separate match and filter
    // kernels): stack m's filtering, the clearing of its outputs' slots and
    // their normalisation run on a second stream, beside stack m+1's
    // matching. The matcher leaves room on each SM for one filter CTA of 8
    // groups (launch_filter_beside_match), so the filter's gathers and
    // atomics overlap the matcher's issue-bound work. The matching runs on a
    // stream of the highest priority and the filtering on one of the lowest,
    // so that an SM a matcher CTA leaves goes to the next matcher CTA, not to
    // more filter CTAs. Match tables alternate between two buffers: stack
    // m+2's matching waits for stack m's filter.
    void run(const std::function<const float*(int)>& frame_ptr, int in_pitch,
             const std::function<float*(int)>& out_ptr, int out_pitch, int first, int count,
             cudaStream_t st, unsigned char* saved = nullptr,
             const std::function<const float*(int)>* input_ptr = nullptr,
             const std::function<void(int, cudaStream_t)>* before_stack = nullptr,
             const std::function<void(int, cudaStream_t)>* after_output = nullptr) {
        if (count <= 0) return;
        const int r = s.radius;
        const int last = first + count - 1;
        ring.ensure(ring_floats());
        match_xy.ensure((size_t)nblocks * 8);
        match_z.ensure((size_t)nblocks);
        const int m_lo = clampf(first - r), m_hi = clampf(last + r);
        int zeroed = first - 1;     // highest output whose slot is zeroed
        int finished = first - 1;   // highest output normalised
        const bool two = overlap && !fused;
        if (!tuned) {
            // the first stack's frames must be resident: the host path
            // uploads them just before the stack that needs them
            if (before_stack) (*before_stack)(m_lo, st);
            ensure_tuned(stack_job(m_lo, frame_ptr, in_pitch, first, last, saved, input_ptr, nullptr,
                                   match_xy.p, match_z.p),
                         st);
        }
        cudaStream_t fs = st;  // filter, slot clearing, normalisation
        cudaStream_t ms = st;  // matching
        if (two) {
            overlap_setup();
            match_xy2.ensure((size_t)nblocks * 8);
            match_z2.ensure((size_t)nblocks);
            fs = filter_stream;
            ms = match_stream;
            VSF_CUDA(cudaEventRecord(ev_fork, st));
            VSF_CUDA(cudaStreamWaitEvent(fs, ev_fork, 0));
            VSF_CUDA(cudaStreamWaitEvent(ms, ev_fork, 0));
        }
        // st waits for both streams on every exit, an error's included, so
        // that no later call's work overlaps this call's
        struct Join {
            vsfeel_bm3d* c;
            bool on;
            cudaStream_t st, fs, ms;
            ~Join() {
                if (!on) return;
                cudaEventRecord(c->ev_join, fs);
                cudaStreamWaitEvent(st, c->ev_join, 0);
                cudaEventRecord(c->ev_join_match, ms);
                cudaStreamWaitEvent(st, c->ev_join_match, 0);
            }
        } join{this, two, st, fs, ms};
        for (int m = m_lo; m <= m_hi; ++m) {
            const int want = std::min(last, m + r);
            if (!two) {
                for (int n = zeroed + 1; n <= want; ++n)
                    VSF_CUDA(cudaMemsetAsync(slot_pair(n, 0), 0,
                                             sizeof(float) * (size_t)slot_pairs(n) * 2 * acc_plane,
                                             st));
                zeroed = std::max(zeroed, want);
                if (before_stack) (*before_stack)(m, st);
                launch_stack(m, frame_ptr, in_pitch, first, last, st, saved, false, input_ptr);
            } else {
                const int b = (m - m_lo) & 1;
                // stack m-2's filter has read this table buffer
                if (m - m_lo >= 2) VSF_CUDA(cudaStreamWaitEvent(ms, ev_filter[b], 0));
                if (before_stack) (*before_stack)(m, ms);
                const StackJob job =
                    stack_job(m, frame_ptr, in_pitch, first, last, saved, input_ptr, nullptr,
                              b ? match_xy2.p : match_xy.p, b ? match_z2.p : match_z.p);
                traced(VSFEEL_KERNEL_MATCH, ms, [&] { return launch_match(job, ms); });
                VSF_CUDA(cudaEventRecord(ev_match[b], ms));
                VSF_CUDA(cudaStreamWaitEvent(fs, ev_match[b], 0));
                for (int n = zeroed + 1; n <= want; ++n)
                    VSF_CUDA(cudaMemsetAsync(slot_pair(n, 0), 0,
                                             sizeof(float) * (size_t)slot_pairs(n) * 2 * acc_plane,
                                             fs));
                zeroed = std::max(zeroed, want);
                traced(VSFEEL_KERNEL_FILTER, fs, [&] { return launch_filter_beside_match(job, fs); });
                VSF_CUDA(cudaEventRecord(ev_filter[b], fs));
                launches += 2;
            }
            const int done = (m == m_hi) ? last : std::min(last, m - r);
            for (int n = finished + 1; n <= done; ++n) {
                launch_normalize(n, out_ptr(n), out_pitch, fs, saved);
                if (after_output) (*after_output)(n, fs);
            }
            finished = std::max(finished, done);
        }
    }

    size_t frame_floats() const { return (size_t)s.height * acc_pitch; }
};

namespace {

template <class F>
int guarded(vsfeel_bm3d* ctx, F&& fn) {
    if (!ctx) return fail(VSFEEL_E_ARG, "null context");
    std::unique_lock<std::mutex> lk(ctx->lock);
    DeviceGuard dg(ctx->device);
    try {
        if constexpr (std::is_invocable_v<F, std::unique_lock<std::mutex>&>)
            return fn(lk);
        else
            return fn();
    } catch (const CudaError& e) {
        if (e.err == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return fail(VSFEEL_E_MEMORY, std::string("out of device memory (") + e.what + ")");
        }
        return fail(VSFEEL_E_CUDA,
                    std::string("CUDA error: ") + cudaGetErrorString(e.err) + " (" + e.what + ")");
    } catch (const std::bad_alloc&) {
        return fail(VSFEEL_E_MEMORY, "out of host memory");
    } catch (const std::exception& e) {
        return fail(VSFEEL_E_ARG, std::string("internal error: ") + e.what());
    }
}

}  // namespace

namespace vsfeel {

// Validates arguments as vsfeel_bm3d_create does and reports the effective
// parameters, without touching the device (used by the allocation-free entry
// point in bm3d_noalloc.cu).
// The tile shape launch_match picks for table-mode matching of this
// configuration: the autotuner's choice (1 + shape, 0: none) where it fits,
// else the largest shape that fits; -1: the direct-read matcher.
int table_tile_shape(const Settings& s, int nbx, int nby, int tuned_plus1) {
    StackJob job{};
    job.width = s.width;
    job.height = s.height;
    job.radius = s.radius;
    job.step = s.step;
    job.bm_range = s.bm_range;
    job.ps_num = s.ps_num;
    job.ps_range = s.ps_range;
    job.nbx = nbx;
    job.nby = nby;
    int shape = default_tile_shape(job, kTableOnly);
    if (shape >= 0 && tuned_plus1 > 0 &&
        tile_shape_fits(job, TileShape(tuned_plus1 - 1), kTableOnly))
        shape = tuned_plus1 - 1;
    return shape;
}

int parse_to_info(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                  vsfeel_bm3d_info* info, int plane) {
    Settings s;
    const int rc = parse_args(args, vi, s, plane);
    if (rc != VSFEEL_OK) return rc;
    std::memset(info, 0, sizeof(*info));
    info->width = s.width;
    info->height = s.height;
    info->num_frames = s.nframes;
    info->radius = s.radius;
    info->block_step = s.step;
    info->bm_range = s.bm_range;
    info->ps_num = s.ps_num;
    info->ps_range = s.ps_range;
    info->num_streams = s.num_streams;
    info->sigma = s.sigma;
    info->threshold = s.thr;
    info->extractor = s.extractor;
    info->blocks_x = block_count(s.width, s.step);
    info->blocks_y = block_count(s.height, s.step);
    info->match_tile_shape = table_tile_shape(s, info->blocks_x, info->blocks_y, 0);
    info->match_lanes = 8;
    info->autotuned = 0;
    return VSFEEL_OK;
}

int set_error(int code, const char* msg) { return fail(code, msg); }

}  // namespace vsfeel

extern "C" {

int vsfeel_bm3d_abi_version(void) { return VSFEEL_BM3D_ABI_VERSION; }

const char* vsfeel_bm3d_last_error(void) { return g_error.c_str(); }

void vsfeel_bm3d_args_init(vsfeel_bm3d_args* a) {
    if (a) std::memset(a, 0, sizeof(*a));
}

int vsfeel_bm3d_create(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi, int device,
                       vsfeel_bm3d** out) {
    return vsfeel_bm3d_create_plane(args, vi, 0, device, out);
}

int vsfeel_bm3d_plane_params(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                             int plane, vsfeel_bm3d_info* info) {
    g_error.clear();
    if (!info) return fail(VSFEEL_E_ARG, "null argument");
    return vsfeel::parse_to_info(args, vi, info, plane);
}

int vsfeel_bm3d_create_plane(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                             int plane, int device, vsfeel_bm3d** out) {
    g_error.clear();
    if (!out) return fail(VSFEEL_E_ARG, "null output pointer");
    *out = nullptr;
    Settings s;
    const int rc = parse_args(args, vi, s, plane);
    if (rc != VSFEEL_OK) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(VSFEEL_E_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(VSFEEL_E_ARG, "invalid device ordinal");
    auto* ctx = new (std::nothrow) vsfeel_bm3d();
    if (!ctx) return fail(VSFEEL_E_MEMORY, "out of host memory");
    ctx->s = s;
    ctx->device = device;
    ctx->nbx = block_count(s.width, s.step);
    ctx->nby = block_count(s.height, s.step);
    ctx->nblocks = ctx->nbx * ctx->nby;
    ctx->acc_pitch = (s.width + 31) & ~31;
    ctx->acc_plane = (size_t)s.height * ctx->acc_pitch;
    if (const char* v = std::getenv("VSFEEL_FUSED_FILTER")) ctx->fused = v[0] == '1';
    if (const char* v = std::getenv("VSFEEL_OVERLAP_FILTER")) ctx->overlap = v[0] != '0';
    if (const char* v = std::getenv("VSFEEL_MATCH_LANES")) {
        ctx->match_lanes = std::atoi(v) == 16 ? 16 : 8;
        ctx->autotune = false;  // an explicit choice is kept
    }
    if (const char* v = std::getenv("VSFEEL_AUTOTUNE")) ctx->autotune = ctx->autotune && v[0] != '0';
    if (const char* v = std::getenv("VSFEEL_MERGED_SLOTS")) ctx->merge_slots = v[0] != '0';
    DeviceGuard dg(device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return fail(VSFEEL_E_CUDA, "could not create a CUDA stream");
    }
    *out = ctx;
    return VSFEEL_OK;
}

void vsfeel_bm3d_free(vsfeel_bm3d* ctx) {
    if (!ctx) return;
    {
        DeviceGuard dg(ctx->device);
        if (ctx->stream) {
            wait_stream(ctx->stream, timeout_ms());
            cudaStreamDestroy(ctx->stream);
        }
        for (cudaStream_t cs : {ctx->up_stream, ctx->down_stream, ctx->filter_stream, ctx->match_stream})
            if (cs) {
                wait_stream(cs, timeout_ms());
                cudaStreamDestroy(cs);
            }
        if (ctx->tail) cudaEventDestroy(ctx->tail);
        if (ctx->direct_copy) cudaEventDestroy(ctx->direct_copy);
        for (cudaEvent_t e : {ctx->ev_match[0], ctx->ev_match[1], ctx->ev_filter[0], ctx->ev_filter[1],
                              ctx->ev_fork, ctx->ev_join, ctx->ev_join_match})
            if (e) cudaEventDestroy(e);
        ctx->match_xy2.release();
        ctx->match_z2.release();
        for (cudaEvent_t e : ctx->frame_events) cudaEventDestroy(e);
        for (cudaEvent_t e : ctx->out_events) cudaEventDestroy(e);
        ctx->ring.release();
        ctx->match_xy.release();
        ctx->match_z.release();
        ctx->gscale.release();
        ctx->frames.release();
        ctx->outbuf.release();
        ctx->stackcache.release();
        for (int i = 0; i < vsfeel_bm3d::kUpSlots; ++i)
            if (ctx->up_done[i]) cudaEventDestroy(ctx->up_done[i]);
        if (ctx->up_host) cudaFreeHost(ctx->up_host);
        for (auto& r : ctx->req_slots) {
            if (r.normalised) cudaEventDestroy(r.normalised);
            if (r.done) cudaEventDestroy(r.done);
        }
        for (cudaEvent_t e : ctx->frame_read) cudaEventDestroy(e);
        if (ctx->req_host) cudaFreeHost(ctx->req_host);
        ctx->req_dev.release();
        ctx->status.release();
        for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    }
    delete ctx;
}

int vsfeel_bm3d_frame_range(const vsfeel_bm3d* ctx, int n, int* first, int* last) {
    if (!ctx || !first || !last) return fail(VSFEEL_E_ARG, "null argument");
    if (n < 0 || n >= ctx->s.nframes) return fail(VSFEEL_E_ARG, "frame index out of range");
    const int r = ctx->s.radius;
    *first = clampi(n - 2 * r, 0, ctx->s.nframes - 1);
    *last = clampi(n + 2 * r, 0, ctx->s.nframes - 1);
    return VSFEEL_OK;
}

int vsfeel_bm3d_get_info(const vsfeel_bm3d* ctx, vsfeel_bm3d_info* info) {
    if (!ctx || !info) return fail(VSFEEL_E_ARG, "null argument");
    const Settings& s = ctx->s;
    info->width = s.width;
    info->height = s.height;
    info->num_frames = s.nframes;
    info->radius = s.radius;
    info->block_step = s.step;
    info->bm_range = s.bm_range;
    info->ps_num = s.ps_num;
    info->ps_range = s.ps_range;
    info->num_streams = s.num_streams;
    info->sigma = s.sigma;
    info->threshold = s.thr;
    info->extractor = s.extractor;
    info->blocks_x = ctx->nbx;
    info->blocks_y = ctx->nby;
    info->device_bytes = (int64_t)(ctx->ring.n + ctx->frames.n + ctx->outbuf.n + ctx->stackcache.n) * 4 +
                         (int64_t)(ctx->match_xy.n + ctx->match_z.n) * 4;
    info->match_tile_shape = vsfeel::table_tile_shape(s, ctx->nbx, ctx->nby, ctx->tuned_shape_plus1);
    info->match_lanes = ctx->match_lanes;
    info->autotuned = ctx->tuner_ran;
    return VSFEEL_OK;
}

int64_t vsfeel_bm3d_launch_count(const vsfeel_bm3d* ctx) { return ctx ? ctx->launches.load() : 0; }

int vsfeel_bm3d_trace(vsfeel_bm3d* ctx, int enable) {
    return guarded(ctx, [&]() -> int {
        ctx->tracing = enable != 0;
        ctx->marks.clear();
        ctx->events_used = 0;
        return VSFEEL_OK;
    });
}

int vsfeel_bm3d_trace_read(vsfeel_bm3d* ctx, double ms[VSFEEL_KERNEL_KINDS],
                           int64_t launches[VSFEEL_KERNEL_KINDS]) {
    return guarded(ctx, [&]() -> int {
        if (!ms || !launches) return fail(VSFEEL_E_ARG, "null argument");
        for (int k = 0; k < VSFEEL_KERNEL_KINDS; ++k) {
            ms[k] = 0.0;
            launches[k] = 0;
        }
        for (const auto& mk : ctx->marks) {
            // bounded wait for the stop event, then read the pair
            const auto t0 = std::chrono::steady_clock::now();
            for (;;) {
                const cudaError_t e = cudaEventQuery(mk.stop);
                if (e == cudaSuccess) break;
                if (e != cudaErrorNotReady) VSF_CUDA(e);
                const auto waited = std::chrono::duration_cast<std::chrono::milliseconds>(
                                        std::chrono::steady_clock::now() - t0)
                                        .count();
                if (waited >= timeout_ms())
                    return fail(VSFEEL_E_TIMEOUT, "timed out waiting for traced kernels");
                std::this_thread::sleep_for(std::chrono::microseconds(50));
            }
            float t = 0.0f;
            VSF_CUDA(cudaEventElapsedTime(&t, mk.start, mk.stop));
            ms[mk.kind] += t;
            launches[mk.kind] += 1;
        }
        return VSFEEL_OK;
    });
}

}  // extern "C"

namespace {

// The pass a call asks for must be the context's: a context created with a
// "ref" clip runs the final pass and needs the ref frames, the others must
// not get any.
int check_pass(const vsfeel_bm3d* ctx, bool with_ref) {
    if (ctx->s.final_pass && !with_ref)
        return fail(VSFEEL_E_ARG,
                    "the context runs the final pass: give the \"ref\" frames (the *_ref entry "
                    "points)");
    if (!ctx->s.final_pass && with_ref)
        return fail(VSFEEL_E_ARG, "no \"ref\" clip was given when the context was created");
    return VSFEEL_OK;
}

int process_device(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                   int64_t src_row_stride, const float* ref, int64_t ref_frame_stride,
                   int64_t ref_row_stride, float* dst, int64_t dst_frame_stride,
                   int64_t dst_row_stride, int first, int count, void* stream) {
    return guarded(ctx, [&]() -> int {
        const Settings& s = ctx->s;
        int rc = check_pass(ctx, ref != nullptr);
        if (rc != VSFEEL_OK) return rc;
        if (!src || !dst) return fail(VSFEEL_E_ARG, "null frame buffer");
        if (first < 0 || count < 0 || first + count > s.nframes)
            return fail(VSFEEL_E_ARG, "output range outside the clip");
        if (src_row_stride < s.width || dst_row_stride < s.width || src_row_stride > INT32_MAX ||
            dst_row_stride > INT32_MAX)
            return fail(VSFEEL_E_ARG, "row stride smaller than the width");
        if (src_frame_stride < src_row_stride * s.height || dst_frame_stride < dst_row_stride * s.height)
            return fail(VSFEEL_E_ARG, "frame stride smaller than a plane");
        if (ref && ref_row_stride != src_row_stride)
            return fail(VSFEEL_E_ARG, "\"ref\" and \"clip\" frames must share a row stride");
        if (ref && ref_frame_stride < ref_row_stride * s.height)
            return fail(VSFEEL_E_ARG, "frame stride smaller than a plane");
        cudaStream_t st = (cudaStream_t)stream;
        ctx->after_prior(st);
        auto src_at = [&](int f) -> const float* { return src + (size_t)f * src_frame_stride; };
        auto out_at = [&](int n) { return dst + (size_t)(n - first) * dst_frame_stride; };
        if (!ref) {
            ctx->run(src_at, (int)src_row_stride, out_at, (int)dst_row_stride, first, count, st);
        } else {
            // the final pass searches the ref clip and denoises the source
            const std::function<const float*(int)> input = src_at;
            ctx->run([&](int f) -> const float* { return ref + (size_t)f * ref_frame_stride; },
                     (int)src_row_stride, out_at, (int)dst_row_stride, first, count, st, nullptr,
                     &input);
        }
        ctx->mark_tail(st);
        return VSFEEL_OK;
    });
}

// Host clip(s) -> staged device frames -> outputs -> host. In the final pass
// the staging buffer holds the source frames, then the ref frames.
int process_host(vsfeel_bm3d* ctx, const float* src, ptrdiff_t src_frame_stride_bytes,
                 ptrdiff_t src_row_stride_bytes, const float* ref, ptrdiff_t ref_frame_stride_bytes,
                 ptrdiff_t ref_row_stride_bytes, float* dst, ptrdiff_t dst_frame_stride_bytes,
                 ptrdiff_t dst_row_stride_bytes, int first, int count) {
    return guarded(ctx, [&]() -> int {
        const Settings& s = ctx->s;
        int rc = check_pass(ctx, ref != nullptr);
        if (rc != VSFEEL_OK) return rc;
        if (!src || !dst) return fail(VSFEEL_E_ARG, "null frame buffer");
        if (first < 0 || count < 0 || first + count > s.nframes)
            return fail(VSFEEL_E_ARG, "output range outside the clip");
        const size_t row_bytes = sizeof(float) * (size_t)s.width;
        if (src_row_stride_bytes < (ptrdiff_t)row_bytes || dst_row_stride_bytes < (ptrdiff_t)row_bytes ||
            (ref && ref_row_stride_bytes < (ptrdiff_t)row_bytes))
            return fail(VSFEEL_E_ARG, "row stride smaller than the width");
        if (count == 0) return VSFEEL_OK;
        const int r = s.radius;
        const int f_lo = ctx->clampf(first - 2 * r), f_hi = ctx->clampf(first + count - 1 + 2 * r);
        const int nin = f_hi - f_lo + 1;
        const size_t ff = ctx->frame_floats();
        ctx->frame_slot.clear();
        ctx->slot_frame.clear();
        ctx->frames.ensure(ff * nin * (ref ? 2 : 1));
        ctx->outbuf.ensure(ff * count);
        cudaStream_t st = ctx->stream;
        ctx->copy_streams((size_t)nin, (size_t)count);
        ctx->after_prior(st);
        ctx->after_prior(ctx->up_stream);
        float* src_base = ctx->frames.p;
        float* ref_base = ctx->frames.p + (size_t)nin * ff;
        // Uploads run on their own stream in frame order, each frame's
        // completion marked by an event; stack m waits only for the last
        // frame it reads, clamp(m + r), so the copies overlap the stacks
        // before it. Frames go up just before the first stack that needs
        // them, so a pageable source (whose copies block the host) still
        // overlaps the work already enqueued.
        int uploaded = f_lo - 1;
        auto upload_to = [&](int f_need) {
            for (int f = uploaded + 1; f <= f_need; ++f) {
                VSF_CUDA(cudaMemcpy2DAsync(src_base + (size_t)(f - f_lo) * ff,
                                           sizeof(float) * ctx->acc_pitch,
                                           (const char*)src + (ptrdiff_t)f * src_frame_stride_bytes,
                                           src_row_stride_bytes, row_bytes, s.height,
                                           cudaMemcpyHostToDevice, ctx->up_stream));
                if (ref)
                    VSF_CUDA(cudaMemcpy2DAsync(ref_base + (size_t)(f - f_lo) * ff,
                                               sizeof(float) * ctx->acc_pitch,
                                               (const char*)ref + (ptrdiff_t)f * ref_frame_stride_bytes,
                                               ref_row_stride_bytes, row_bytes, s.height,
                                               cudaMemcpyHostToDevice, ctx->up_stream));
                VSF_CUDA(cudaEventRecord(ctx->frame_events[f - f_lo], ctx->up_stream));
            }
            uploaded = std::max(uploaded, f_need);
        };
        const std::function<void(int, cudaStream_t)> before = [&](int m, cudaStream_t ms) {
            const int f_need = std::min(ctx->clampf(m + r), f_hi);
            upload_to(f_need);
            VSF_CUDA(cudaStreamWaitEvent(ms, ctx->frame_events[f_need - f_lo], 0));
        };
        // Downloads: into page-locked memory each output goes down as soon as
        // it is normalised; into pageable memory (whose copies would block the
        // host until the output exists) all of them after the last stack.
        cudaPointerAttributes pa{};
        const bool pinned_dst = cudaPointerGetAttributes(&pa, dst) == cudaSuccess &&
                                pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        auto download = [&](int n, cudaStream_t cs) {
            const int q = n - first;
            VSF_CUDA(cudaMemcpy2DAsync((char*)dst + (ptrdiff_t)q * dst_frame_stride_bytes,
                                       dst_row_stride_bytes, ctx->outbuf.p + (size_t)q * ff,
                                       sizeof(float) * ctx->acc_pitch, row_bytes, s.height,
                                       cudaMemcpyDeviceToHost, cs));
        };
        const std::function<void(int, cudaStream_t)> after = [&](int n, cudaStream_t ns) {
            VSF_CUDA(cudaEventRecord(ctx->out_events[n - first], ns));
            VSF_CUDA(cudaStreamWaitEvent(ctx->down_stream, ctx->out_events[n - first], 0));
            download(n, ctx->down_stream);
        };
        auto src_at = [&](int f) -> const float* { return src_base + (size_t)(f - f_lo) * ff; };
        auto out_at = [&](int n) { return ctx->outbuf.p + (size_t)(n - first) * ff; };
        const std::function<void(int, cudaStream_t)>* after_ptr = pinned_dst ? &after : nullptr;
        if (!ref) {
            ctx->run(src_at, ctx->acc_pitch, out_at, ctx->acc_pitch, first, count, st, nullptr,
                     nullptr, &before, after_ptr);
        } else {
            const std::function<const float*(int)> input = src_at;
            ctx->run([&](int f) -> const float* { return ref_base + (size_t)(f - f_lo) * ff; },
                     ctx->acc_pitch, out_at, ctx->acc_pitch, first, count, st, nullptr, &input,
                     &before, after_ptr);
        }
        if (!pinned_dst)
            for (int n = first; n < first + count; ++n) download(n, st);
        // the context's work ends when both the compute and download streams do
        cudaEvent_t down_end = ctx->out_events[count - 1];
        VSF_CUDA(cudaEventRecord(down_end, ctx->down_stream));
        VSF_CUDA(cudaStreamWaitEvent(st, down_end, 0));
        ctx->mark_tail(st);
        const int wrc = wait_stream(ctx->down_stream, timeout_ms());
        if (wrc != VSFEEL_OK) return wrc;
        return ctx->finish(st);
    });
}

// The per-frame request path. fetch(clip, f, &stride) returns frame f of
// the source (clip 0) or the ref clip (1); release(clip, f) hands it back.
// A frame-cache slot holds a frame's source plane and, in the final pass,
// its ref plane after it.
//
// Stacks are cached whole, as the reference's result cache holds them
// (src/bm3d.cpp:380-478): a stack writes each slice that an output reads
// into its own cache slot, and output n is normalised from slice
// agg_z(i, n) of the cached stacks clamp(n - r + i). Requests in any order
// compute a stack once while it stays among the stack_slots() most recently
// used; a request computes only the stacks it misses, fetching frames of
// its frame_range window only.
//
// When other requests are in flight, a request holds the context's lock
// only while it enqueues: frames are copied into page-locked staging on the
// host and released at once, the output comes back into the request's
// page-locked slot, and the caller waits for its own event and copies the
// rows out with the lock released. Requests from several threads
// (fmParallel) thus overlap their host copies with each other's kernels;
// the GPU work stays in request order on the context's stream. A request
// alone in flight copies straight from and to the caller's memory instead
// (the driver pipelines pageable copies faster than a host copy plus DMA).
int get_frame(vsfeel_bm3d* ctx, int n, bool with_ref,
              const std::function<const float*(int, int, ptrdiff_t*)>& fetch,
              const std::function<void(int, int)>& release, float* dst, ptrdiff_t dst_stride_bytes) {
    if (!ctx) return fail(VSFEEL_E_ARG, "null context");
    // counted before the lock, so that callers waiting for it count too
    struct InFlight {
        std::atomic<int>& c;
        explicit InFlight(std::atomic<int>& c_) : c(c_) { ++c; }
        ~InFlight() { --c; }
    } in_flight(ctx->requests_in_flight);
    int slot = -1;
    bool direct = false;  // alone in flight: copies from and to the caller's memory
    auto hand_back = [&] {
        if (slot < 0) return;
        {
            std::lock_guard<std::mutex> lk(ctx->lock);
            ctx->req_slots[slot].busy = false;
        }
        ctx->req_cv.notify_one();
    };
    int rc = guarded(ctx, [&](std::unique_lock<std::mutex>& lk) -> int {
        const Settings& s = ctx->s;
        int rc = check_pass(ctx, with_ref);
        if (rc != VSFEEL_OK) return rc;
        if (!dst) return fail(VSFEEL_E_ARG, "null callback or destination");
        if (n < 0 || n >= s.nframes) return fail(VSFEEL_E_ARG, "frame index out of range");
        const size_t row_bytes = sizeof(float) * (size_t)s.width;
        if (dst_stride_bytes < (ptrdiff_t)row_bytes)
            return fail(VSFEEL_E_ARG, "row stride smaller than the width");
        ctx->request_staging();
        // a free request slot; others are handed back as their callers finish
        auto free_slot = [&] {
            for (size_t i = 0; i < ctx->req_slots.size(); ++i)
                if (!ctx->req_slots[i].busy) return (int)i;
            return -1;
        };
        if (!ctx->req_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms()),
                                  [&] { return free_slot() >= 0; }))
            return fail(VSFEEL_E_TIMEOUT, "timed out waiting for a request slot");
        slot = free_slot();
        ctx->req_slots[slot].busy = true;
        direct = ctx->requests_in_flight.load() == 1;

        const int r = s.radius;
        const int planes = with_ref ? 2 : 1;
        const int f_lo = ctx->clampf(n - 2 * r), f_hi = ctx->clampf(n + 2 * r);
        const int cap = 4 * r + 2;  // window plus one frame of slack
        const int nstack = ctx->stack_slots();
        const size_t ff = ctx->frame_floats();
        const size_t pf = ctx->packed_plane_floats();
        if ((int)ctx->slot_frame.size() != cap) {
            ctx->frame_slot.clear();
            ctx->slot_frame.assign(cap, -1);
        }
        while ((int)ctx->frame_read.size() < cap) {
            cudaEvent_t e;
            VSF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            ctx->frame_read.push_back(e);
            ctx->frame_read_set.push_back(0);
        }
        if ((int)ctx->stack_tag.size() != nstack) {
            ctx->stack_tag.assign(nstack, -1);
            ctx->stack_use.assign(nstack, -1);
        }
        ctx->frames.ensure(ff * cap * planes);
        ctx->stackcache.ensure((size_t)nstack * ctx->tw() * 2 * ctx->acc_plane);
        ctx->match_xy.ensure((size_t)ctx->nblocks * 8);
        ctx->match_z.ensure((size_t)ctx->nblocks);
        const int64_t req = ++ctx->requests;
        cudaStream_t st = ctx->stream;
        // another entry point's work first; the per-frame path's own work is
        // ordered by the events below
        if (!ctx->tail_from_request) {
            ctx->after_prior(st);
            ctx->after_prior(ctx->up_stream);
            ctx->after_prior(ctx->down_stream);
        }
        // evict cached frames outside the window
        for (auto it = ctx->frame_slot.begin(); it != ctx->frame_slot.end();) {
            if (it->first < f_lo || it->first > f_hi) {
                ctx->slot_frame[it->second] = -1;
                it = ctx->frame_slot.erase(it);
            } else {
                ++it;
            }
        }
        // frames lo..hi resident (all inside the window)
        auto stage = [&](int lo, int hi) -> int {
            for (int f = lo; f <= hi; ++f) {
                if (ctx->frame_slot.count(f)) continue;
                int slot_f = 0;
                while (ctx->slot_frame[slot_f] != -1) ++slot_f;
                for (int clip = 0; clip < planes; ++clip) {
                    if (direct) {
                        ptrdiff_t stride = 0;
                        const float* p = fetch(clip, f, &stride);
                        if (!p)
                            return fail(VSFEEL_E_FETCH,
                                        std::string("could not fetch ") +
                                            (clip ? "\"ref\" frame " : "source frame ") +
                                            std::to_string(f));
                        if (stride < (ptrdiff_t)row_bytes) {
                            release(clip, f);
                            return fail(VSFEEL_E_ARG, "source row stride smaller than the width");
                        }
                        VSF_CUDA(cudaMemcpy2DAsync(
                            ctx->frames.p + ((size_t)slot_f * planes + clip) * ff,
                            sizeof(float) * ctx->acc_pitch, p, stride, row_bytes, s.height,
                            cudaMemcpyHostToDevice, st));
                        // the source frame must stay valid until the copy has
                        // run: wait for the copy itself, not for earlier
                        // requests' kernels on the stream. A wait that runs
                        // out leaves the frame with the caller (not released:
                        // the copy may still read it)
                        VSF_CUDA(cudaEventRecord(ctx->direct_copy_done(), st));
                        const int wrc = wait_event(ctx->direct_copy, timeout_ms());
                        if (wrc != VSFEEL_OK) return wrc;
                        release(clip, f);
                        continue;
                    }
                    const int k = ctx->up_next;
                    ctx->up_next = (k + 1) % vsfeel_bm3d::kUpSlots;
                    if (ctx->up_used[k]) {
                        const int wrc = wait_event(ctx->up_done[k], timeout_ms());
                        if (wrc != VSFEEL_OK) return wrc;
                    }
                    ptrdiff_t stride = 0;
                    const float* p = fetch(clip, f, &stride);
                    if (!p)
                        return fail(VSFEEL_E_FETCH, std::string("could not fetch ") +
                                                        (clip ? "\"ref\" frame " : "source frame ") +
                                                        std::to_string(f));
                    if (stride < (ptrdiff_t)row_bytes) {
                        release(clip, f);
                        return fail(VSFEEL_E_ARG, "source row stride smaller than the width");
                    }
                    float* staged = ctx->up_host + pf * k;
                    const unsigned char* row = reinterpret_cast<const unsigned char*>(p);
                    for (int y = 0; y < s.height; ++y)
                        std::memcpy(staged + (size_t)y * s.width, row + (size_t)y * stride, row_bytes);
                    release(clip, f);
                    // on the copy stream, after the last stack that read the
                    // slot's previous frame; the stacks wait for the copy
                    cudaStream_t up = ctx->up_stream;
                    if (ctx->frame_read_set[slot_f])
                        VSF_CUDA(cudaStreamWaitEvent(up, ctx->frame_read[slot_f], 0));
                    VSF_CUDA(cudaMemcpy2DAsync(ctx->frames.p + ((size_t)slot_f * planes + clip) * ff,
                                               sizeof(float) * ctx->acc_pitch, staged, row_bytes,
                                               row_bytes, s.height, cudaMemcpyHostToDevice, up));
                    VSF_CUDA(cudaEventRecord(ctx->up_done[k], up));
                    VSF_CUDA(cudaStreamWaitEvent(st, ctx->up_done[k], 0));
                    ctx->up_used[k] = true;
                }
                ctx->slot_frame[slot_f] = f;
                ctx->frame_slot[f] = slot_f;
            }
            return VSFEEL_OK;
        };
        auto plane_at = [&](int f, int clip) -> const float* {
            return ctx->frames.p + ((size_t)ctx->frame_slot.at(f) * planes + clip) * ff;
        };
        const std::function<const float*(int)> search = [&](int f) {
            return plane_at(f, with_ref ? 1 : 0);
        };
        const std::function<const float*(int)> input = [&](int f) { return plane_at(f, 0); };
        auto slot_of = [&](int m) {
            for (int c = 0; c < nstack; ++c)
                if (ctx->stack_tag[c] == m) return c;
            return -1;
        };

        // the stacks output n reads, each pinned for this request
        const int m_lo = ctx->clampf(n - r), m_hi = ctx->clampf(n + r);
        for (int m = m_lo; m <= m_hi; ++m) {
            const int c = slot_of(m);
            if (c >= 0) ctx->stack_use[c] = req;
        }
        for (int m = m_lo; m <= m_hi; ++m) {
            if (slot_of(m) >= 0) continue;
            // least recently used slot not pinned by this request (the
            // cache holds more than 2r+1 stacks, so one exists)
            int c = -1;
            for (int k = 0; k < nstack; ++k)
                if (ctx->stack_use[k] != req && (c < 0 || ctx->stack_use[k] < ctx->stack_use[c]))
                    c = k;
            ctx->stack_tag[c] = -1;
            rc = stage(ctx->clampf(m - r), ctx->clampf(m + r));
            if (rc != VSFEEL_OK) return rc;
            float* slices = ctx->stack_slices(c);
            if (!ctx->tuned)
                ctx->ensure_tuned(ctx->stack_job(m, search, ctx->acc_pitch, 0, s.nframes - 1, nullptr,
                                                 with_ref ? &input : nullptr, slices,
                                                 ctx->match_xy.p, ctx->match_z.p),
                                  st);
            VSF_CUDA(cudaMemsetAsync(slices, 0, sizeof(float) * (size_t)ctx->tw() * 2 * ctx->acc_plane,
                                     st));
            ctx->launch_stack(m, search, ctx->acc_pitch, 0, s.nframes - 1, st, nullptr, false,
                              with_ref ? &input : nullptr, slices);
            for (int f = ctx->clampf(m - r); f <= ctx->clampf(m + r); ++f) {
                const int fs = ctx->frame_slot.at(f);
                VSF_CUDA(cudaEventRecord(ctx->frame_read[fs], st));
                ctx->frame_read_set[fs] = 1;
            }
            ctx->stack_tag[c] = m;
            ctx->stack_use[c] = req;
        }
        const std::function<float*(int)> slices_of = [&](int m) {
            return ctx->stack_slices(slot_of(m));
        };
        vsfeel_bm3d::RequestSlot& rs = ctx->req_slots[slot];
        ctx->launch_normalize(n, rs.dev, ctx->acc_pitch, st, nullptr, &slices_of);
        if (direct) {
            VSF_CUDA(cudaMemcpy2DAsync(dst, dst_stride_bytes, rs.dev, sizeof(float) * ctx->acc_pitch,
                                       row_bytes, s.height, cudaMemcpyDeviceToHost, st));
            ctx->mark_tail(st, true);
            return ctx->finish(st);
        }
        // the download on the other copy stream, after the normalisation
        cudaStream_t down = ctx->down_stream;
        int* status = ctx->status_word();
        VSF_CUDA(cudaEventRecord(rs.normalised, st));
        VSF_CUDA(cudaStreamWaitEvent(down, rs.normalised, 0));
        VSF_CUDA(cudaMemcpy2DAsync(rs.host, row_bytes, rs.dev, sizeof(float) * ctx->acc_pitch,
                                   row_bytes, s.height, cudaMemcpyDeviceToHost, down));
        VSF_CUDA(cudaMemcpyAsync(rs.status, status, sizeof(int), cudaMemcpyDeviceToHost, down));
        VSF_CUDA(cudaEventRecord(rs.done, down));
        // the download stream has waited for everything this request put on
        // the compute stream, so its end is the end of the request
        ctx->mark_tail(down, true);
        return VSFEEL_OK;
    });
    if (rc != VSFEEL_OK || direct) {
        hand_back();
        return rc;
    }
    // the caller's wait and copy, with the lock released
    const vsfeel_bm3d::RequestSlot& rs = ctx->req_slots[slot];
    {
        DeviceGuard dg(ctx->device);
        rc = wait_event(rs.done, timeout_ms());
    }
    if (rc == VSFEEL_OK && *rs.status != 0) {
        rc = guarded(ctx, [&]() -> int {
            VSF_CUDA(cudaMemsetAsync(ctx->status.p, 0, sizeof(int), ctx->stream));
            ctx->invalidate_stacks();
            return fail(VSFEEL_E_CUDA, status_text(*rs.status));
        });
    }
    if (rc == VSFEEL_OK) {
        const size_t row_bytes = sizeof(float) * (size_t)ctx->s.width;
        unsigned char* out = reinterpret_cast<unsigned char*>(dst);
        for (int y = 0; y < ctx->s.height; ++y)
            std::memcpy(out + (size_t)y * dst_stride_bytes, rs.host + (size_t)y * ctx->s.width,
                        row_bytes);
    }
    hand_back();
    return rc;
}

}  // namespace

extern "C" {

int vsfeel_bm3d_process_device(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                               int64_t src_row_stride, float* dst, int64_t dst_frame_stride,
                               int64_t dst_row_stride, int first, int count, void* stream) {
    return process_device(ctx, src, src_frame_stride, src_row_stride, nullptr, 0, 0, dst,
                          dst_frame_stride, dst_row_stride, first, count, stream);
}

int vsfeel_bm3d_process_device_ref(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                                   int64_t src_row_stride, const float* ref,
                                   int64_t ref_frame_stride, int64_t ref_row_stride, float* dst,
                                   int64_t dst_frame_stride, int64_t dst_row_stride, int first,
                                   int count, void* stream) {
    if (!ref) return fail(VSFEEL_E_ARG, "null \"ref\" buffer");
    return process_device(ctx, src, src_frame_stride, src_row_stride, ref, ref_frame_stride,
                          ref_row_stride, dst, dst_frame_stride, dst_row_stride, first, count,
                          stream);
}

int vsfeel_bm3d_saved_layout(const vsfeel_bm3d* ctx, vsfeel_bm3d_saved_info* out) {
    if (!ctx || !out) return fail(VSFEEL_E_ARG, "null argument");
    const auto L = ctx->saved_layout();
    out->bytes = L.bytes;
    out->stack_bytes = L.stack_bytes;
    out->match_xy_offset = L.off_xy;
    out->match_z_offset = L.off_z;
    out->mask_offset = L.off_mask;
    out->den_offset = L.den_offset;
    out->den_row_stride = L.den_pitch;
    out->den_frame_stride = (int64_t)ctx->frame_floats();
    out->num_blocks = ctx->nblocks;
    return VSFEEL_OK;
}

int vsfeel_bm3d_forward_saved(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                              int64_t src_row_stride, float* dst, int64_t dst_frame_stride,
                              int64_t dst_row_stride, void* saved, void* stream) {
    return guarded(ctx, [&]() -> int {
        const Settings& s = ctx->s;
        if (s.final_pass)
            return fail(VSFEEL_E_UNSUPPORTED,
                        "the differentiable form covers the basic estimate, not the final pass");
        if (!src || !dst || !saved) return fail(VSFEEL_E_ARG, "null buffer");
        if ((reinterpret_cast<uintptr_t>(saved) & 255u) != 0)
            return fail(VSFEEL_E_ARG, "saved-state buffer must be 256-byte aligned");
        if (src_row_stride < s.width || dst_row_stride < s.width || src_row_stride > INT32_MAX ||
            dst_row_stride > INT32_MAX)
            return fail(VSFEEL_E_ARG, "row stride smaller than the width");
        if (src_frame_stride < src_row_stride * s.height || dst_frame_stride < dst_row_stride * s.height)
            return fail(VSFEEL_E_ARG, "frame stride smaller than a plane");
        cudaStream_t st = (cudaStream_t)stream;
        ctx->after_prior(st);
        ctx->run([&](int f) { return src + (size_t)f * src_frame_stride; }, (int)src_row_stride,
                 [&](int n) { return dst + (size_t)n * dst_frame_stride; }, (int)dst_row_stride, 0,
                 s.nframes, st, static_cast<unsigned char*>(saved));
        ctx->mark_tail(st);
        return VSFEEL_OK;
    });
}

int vsfeel_bm3d_backward(vsfeel_bm3d* ctx, const void* saved, const float* grad_out,
                         int64_t go_frame_stride, int64_t go_row_stride, float* grad_in,
                         int64_t gi_frame_stride, int64_t gi_row_stride, void* stream) {
    return guarded(ctx, [&]() -> int {
        const Settings& s = ctx->s;
        if (s.final_pass)
            return fail(VSFEEL_E_UNSUPPORTED,
                        "the differentiable form covers the basic estimate, not the final pass");
        if (!saved || !grad_out || !grad_in) return fail(VSFEEL_E_ARG, "null buffer");
        if ((reinterpret_cast<uintptr_t>(saved) & 255u) != 0)
            return fail(VSFEEL_E_ARG, "saved-state buffer must be 256-byte aligned");
        if (go_row_stride < s.width || gi_row_stride < s.width || go_row_stride > INT32_MAX ||
            gi_row_stride > INT32_MAX)
            return fail(VSFEEL_E_ARG, "row stride smaller than the width");
        if (go_frame_stride < go_row_stride * s.height || gi_frame_stride < gi_row_stride * s.height)
            return fail(VSFEEL_E_ARG, "frame stride smaller than a plane");
        cudaStream_t st = (cudaStream_t)stream;
        ctx->after_prior(st);
        const auto L = ctx->saved_layout();
        const auto* base = static_cast<const unsigned char*>(saved);
        // the input gradient is accumulated: clear it first (rows may be padded)
        const size_t pitch_bytes = sizeof(float) * (size_t)gi_row_stride;
        const size_t row_bytes = sizeof(float) * (size_t)s.width;
        if (gi_frame_stride == gi_row_stride * s.height) {
            VSF_CUDA(cudaMemset2DAsync(grad_in, pitch_bytes, 0, row_bytes,
                                       (size_t)s.height * s.nframes, st));
        } else {
            for (int f = 0; f < s.nframes; ++f)
                VSF_CUDA(cudaMemset2DAsync(grad_in + (size_t)f * gi_frame_stride, pitch_bytes, 0,
                                           row_bytes, (size_t)s.height, st));
        }
        // Stacks go in ranges of about eight waves of adjoint CTAs (three
        // 128-thread CTAs per SM), in order. Before a range, the scaled
        // gradients g / D of the frames it reads that no earlier range read
        // are computed into a ring of count + 2r frame slots: the frames a
        // range reads (its stacks -r .. +r) have distinct slots, and a slot
        // it overwrites held a frame that no later stack reads.
        const int r = s.radius;
        int sms = 0;
        VSF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        // (the adjoint kernel: 128-thread CTAs of 16 groups, three per SM)
        const int64_t target_groups = (int64_t)std::max(sms, 1) * 3 * 16 * 8;
        const int per = (int)std::min<int64_t>(
            s.nframes, std::max<int64_t>(1, (target_groups + ctx->nblocks - 1) / ctx->nblocks));
        const int slots = std::min(s.nframes, per + 2 * r);
        ctx->gscale.ensure((size_t)slots * ctx->frame_floats());
        AdjointJob job{};
        job.saved = base;
        job.stack_bytes = L.stack_bytes;
        job.off_xy = L.off_xy;
        job.off_z = L.off_z;
        job.off_mask = L.off_mask;
        job.gs = ctx->gscale.p;
        job.gs_frame = (int64_t)ctx->frame_floats();
        job.gs_pitch = ctx->acc_pitch;
        job.gs_slots = slots;
        job.grad_in = grad_in;
        job.gi_frame = gi_frame_stride;
        job.gi_pitch = (int)gi_row_stride;
        job.nframes = s.nframes;
        job.radius = r;
        job.nblocks = ctx->nblocks;
        job.width = s.width;
        job.height = s.height;
        const float* den = reinterpret_cast<const float*>(base + L.den_offset);
        int scaled = -1;  // frames 0..scaled have their g / D in the ring
        for (int m0 = 0; m0 < s.nframes; m0 += per) {
            const int count = std::min(per, s.nframes - m0);
            const int need = std::min(m0 + count - 1 + r, s.nframes - 1);
            for (int f = scaled + 1; f <= need; ++f) {
                GradScaleJob gj{};
                gj.go = grad_out + (size_t)f * go_frame_stride;
                gj.den = den + (size_t)f * ctx->frame_floats();
                gj.gs = ctx->gscale.p + (size_t)(f % slots) * ctx->frame_floats();
                gj.go_pitch = (int)go_row_stride;
                gj.den_pitch = (int)L.den_pitch;
                gj.gs_pitch = ctx->acc_pitch;
                gj.width = s.width;
                gj.height = s.height;
                VSF_CUDA(launch_grad_scale(gj, st));
                ctx->launches += 1;
            }
            scaled = std::max(scaled, need);
            job.first_stack = m0;
            job.stack_count = count;
            ctx->traced(VSFEEL_KERNEL_ADJOINT, st, [&] { return launch_adjoint(job, st); });
            ctx->launches += 1;
        }
        ctx->mark_tail(st);
        return VSFEEL_OK;
    });
}

int vsfeel_bm3d_process_host(vsfeel_bm3d* ctx, const float* src, ptrdiff_t src_frame_stride_bytes,
                             ptrdiff_t src_row_stride_bytes, float* dst,
                             ptrdiff_t dst_frame_stride_bytes, ptrdiff_t dst_row_stride_bytes,
                             int first, int count) {
    return process_host(ctx, src, src_frame_stride_bytes, src_row_stride_bytes, nullptr, 0, 0, dst,
                        dst_frame_stride_bytes, dst_row_stride_bytes, first, count);
}

int vsfeel_bm3d_process_host_ref(vsfeel_bm3d* ctx, const float* src,
                                 ptrdiff_t src_frame_stride_bytes, ptrdiff_t src_row_stride_bytes,
                                 const float* ref, ptrdiff_t ref_frame_stride_bytes,
                                 ptrdiff_t ref_row_stride_bytes, float* dst,
                                 ptrdiff_t dst_frame_stride_bytes, ptrdiff_t dst_row_stride_bytes,
                                 int first, int count) {
    if (!ref) return fail(VSFEEL_E_ARG, "null \"ref\" buffer");
    return process_host(ctx, src, src_frame_stride_bytes, src_row_stride_bytes, ref,
                        ref_frame_stride_bytes, ref_row_stride_bytes, dst, dst_frame_stride_bytes,
                        dst_row_stride_bytes, first, count);
}

int vsfeel_bm3d_get_frame(vsfeel_bm3d* ctx, int n, vsfeel_fetch_fn fetch, vsfeel_release_fn release,
                          void* user, float* dst, ptrdiff_t dst_stride_bytes) {
    if (!fetch) return fail(VSFEEL_E_ARG, "null callback or destination");
    return get_frame(
        ctx, n, false, [&](int, int f, ptrdiff_t* stride) { return fetch(user, f, stride); },
        [&](int, int f) {
            if (release) release(user, f);
        },
        dst, dst_stride_bytes);
}

int vsfeel_bm3d_get_frame_ref(vsfeel_bm3d* ctx, int n, vsfeel_fetch2_fn fetch,
                              vsfeel_release2_fn release, void* user, float* dst,
                              ptrdiff_t dst_stride_bytes) {
    if (!fetch) return fail(VSFEEL_E_ARG, "null callback or destination");
    return get_frame(
        ctx, n, true,
        [&](int clip, int f, ptrdiff_t* stride) { return fetch(user, clip, f, stride); },
        [&](int clip, int f) {
            if (release) release(user, clip, f);
        },
        dst, dst_stride_bytes);
}

int vsfeel_bm3d_match_table_device(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                                   int64_t src_row_stride, int m, int32_t* table_host) {
    return guarded(ctx, [&]() -> int {
        const Settings& s = ctx->s;
        if (!src || !table_host) return fail(VSFEEL_E_ARG, "null argument");
        if (m < 0 || m >= s.nframes) return fail(VSFEEL_E_ARG, "stack index out of range");
        if (src_row_stride < s.width || src_row_stride > INT32_MAX)
            return fail(VSFEEL_E_ARG, "row stride smaller than the width");
        ctx->ring.ensure(ctx->ring_floats());
        ctx->match_xy.ensure((size_t)ctx->nblocks * 8);
        ctx->match_z.ensure((size_t)ctx->nblocks);
        cudaStream_t st = ctx->stream;
        ctx->after_prior(st);
        // outputs range empty: the filter runs but every slice is dropped
        ctx->launch_stack(m, [&](int f) { return src + (size_t)f * src_frame_stride; },
                          (int)src_row_stride, 1, 0, st, nullptr, true);
        std::vector<uint32_t> xy((size_t)ctx->nblocks * 8), zz((size_t)ctx->nblocks);
        VSF_CUDA(cudaMemcpyAsync(xy.data(), ctx->match_xy.p, xy.size() * 4, cudaMemcpyDeviceToHost, st));
        VSF_CUDA(cudaMemcpyAsync(zz.data(), ctx->match_z.p, zz.size() * 4, cudaMemcpyDeviceToHost, st));
        ctx->mark_tail(st);
        const int rc = ctx->finish(st);
        if (rc != VSFEEL_OK) return rc;
        for (int b = 0; b < ctx->nblocks; ++b)
            for (int k = 0; k < 8; ++k) {
                const uint32_t v = xy[(size_t)b * 8 + k];
                table_host[((size_t)b * 8 + k) * 3 + 0] = (int32_t)(v & 0xffffu);
                table_host[((size_t)b * 8 + k) * 3 + 1] = (int32_t)(v >> 16);
                table_host[((size_t)b * 8 + k) * 3 + 2] = (int32_t)((zz[b] >> (4 * k)) & 15u);
            }
        return VSFEEL_OK;
    });
}

}  // extern "C"
