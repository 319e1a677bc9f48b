// Allocation-free denoising entry point (vsfeel_bm3d_process_device_noalloc).
//
// Some callers cannot let this library allocate device memory: a host
// process that carves the whole GPU into its own fixed pools up front (a
// serving or editing application with a strict memory budget), where a
// cudaMalloc outside its allocator either fails or breaks its accounting;
// and real-time pipelines that must not pay cudaMalloc/cudaFree's implicit
// device-wide synchronisation in the middle of a stream of work. For them
// this entry point denoises from caller-owned input and output buffers and
// keeps every intermediate -- the match table, the per-output accumulator
// planes and the kernels' status word -- in one file-scope device array of
// kNoAllocScratchBytes (32 MiB). Every GPU that loads the library holds that
// array until the process exits.
//
// The array's name is a host-side stand-in in host code, not a device
// address. The real address belongs to a CUDA context: the first call in
// each context resolves it with cudaGetSymbolAddress while that context is
// current (the device's primary context for runtime-API callers) and caches
// it under the context's unique ID, which CUDA never hands out twice in a
// process. A context the host creates itself with the driver API, or the
// primary context re-created after cudaDeviceReset, therefore resolves its
// own address on its first call instead of reusing a stale one. That first
// call per context should come before any stream capture.
// All calls share the array and it keeps the previous call's contents, so
// each call clears the accumulator planes it uses before the kernels run;
// calls that overlap on the GPU (different streams, or different host
// threads without ordering) race on the array and must be serialised by the
// caller. The call only enqueues work on `stream`; it never waits, so an
// internal error a kernel flags is not reported back.
#include "bm3d_device.cuh"
#include "vsfeel_bm3d.h"

#include <cuda.h>  // driver API types only; the calls are resolved at run time

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>

namespace vsfeel {

int parse_to_info(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                  vsfeel_bm3d_info* info, int plane = 0);
int set_error(int code, const char* msg);

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Resolved addresses, one per CUDA context seen (keyed by the context's
// unique ID); the oldest entry is replaced when all are taken.
constexpr int kCachedContexts = 64;

struct CachedAddress {
    unsigned long long ctx_id;
    unsigned char* ptr;
};

std::mutex g_setup_lock;
CachedAddress g_cache[kCachedContexts] = {};
int g_cache_used = 0, g_cache_next = 0;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// cuCtxGetCurrent and cuCtxGetId through the runtime's driver entry points,
// so that the library does not link the driver library itself (it loads on
// hosts without a GPU). Both exist from CUDA 12.0 on; without them every
// call resolves the address afresh.
struct DriverCalls {
    CtxGetCurrentFn get_current = nullptr;
    CtxGetIdFn get_id = nullptr;
};

const DriverCalls& driver_calls() {
    static const DriverCalls calls = [] {
        DriverCalls d;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            d.get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            d.get_id = reinterpret_cast<CtxGetIdFn>(fn);
        cudaGetLastError();
        return d;
    }();
    return calls;
}

// The unique ID of the current context; false when there is none (nothing
// has made a context current on this thread yet) or it cannot be read.
bool current_context_id(unsigned long long* id) {
    const DriverCalls& d = driver_calls();
    if (!d.get_current || !d.get_id) return false;
    CUcontext ctx = nullptr;
    if (d.get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return d.get_id(ctx, id) == CUDA_SUCCESS;
}

int resolve(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return set_error(VSFEEL_E_CUDA, "could not resolve the scratch array's device address");
    }
    *out = static_cast<unsigned char*>(p);
    return VSFEEL_OK;
}

// The device address of the scratch array in the current context.
int scratch_address(unsigned char** out) {
    unsigned long long id = 0;
    if (!current_context_id(&id)) {
        // no context current yet: the runtime call below makes the current
        // device's primary context current, whose ID is then readable
        const int rc = resolve(out);
        if (rc != VSFEEL_OK || !current_context_id(&id)) return rc;
    }
    std::lock_guard<std::mutex> lk(g_setup_lock);
    for (int i = 0; i < g_cache_used; ++i)
        if (g_cache[i].ctx_id == id) {
            *out = g_cache[i].ptr;
            return VSFEEL_OK;
        }
    const int rc = resolve(out);
    if (rc != VSFEEL_OK) return rc;
    const int slot = g_cache_used < kCachedContexts ? g_cache_used++ : g_cache_next;
    if (g_cache_used == kCachedContexts) g_cache_next = (slot + 1) % kCachedContexts;
    g_cache[slot] = CachedAddress{id, *out};
    return VSFEEL_OK;
}

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
inline int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

int agg_z(int i, int n, int nframes, int radius) {
    return std::min(std::max(2 * radius - i, n - nframes + 1 + radius), n + radius);
}

}  // namespace

}  // namespace vsfeel

extern "C" {

int64_t vsfeel_bm3d_noalloc_scratch_bytes(void) { return (int64_t)vsfeel::kNoAllocScratchBytes; }

int vsfeel_bm3d_process_device_noalloc(const vsfeel_bm3d_args* args,
                                       const vsfeel_bm3d_video_info* vi, const float* src,
                                       int64_t src_frame_stride, int64_t src_row_stride, float* dst,
                                       int64_t dst_frame_stride, int64_t dst_row_stride, int first,
                                       int count, void* stream) {
    using namespace vsfeel;
    vsfeel_bm3d_info inf;
    int rc = parse_to_info(args, vi, &inf);
    if (rc != VSFEEL_OK) return rc;
    if (args->has_ref)
        return set_error(VSFEEL_E_UNSUPPORTED,
                         "the allocation-free entry point runs the basic estimate only");
    const int W = inf.width, H = inf.height, N = inf.num_frames, r = inf.radius;
    if (!src || !dst) return set_error(VSFEEL_E_ARG, "null frame buffer");
    if (first < 0 || count < 0 || first + count > N)
        return set_error(VSFEEL_E_ARG, "output range outside the clip");
    if (src_row_stride < W || dst_row_stride < W || src_row_stride > INT32_MAX ||
        dst_row_stride > INT32_MAX)
        return set_error(VSFEEL_E_ARG, "row stride smaller than the width");
    if (src_frame_stride < src_row_stride * H || dst_frame_stride < dst_row_stride * H)
        return set_error(VSFEEL_E_ARG, "frame stride smaller than a plane");
    if (count == 0) return VSFEEL_OK;

    // scratch layout: status word | match xy | match z | accumulator ring
    const int tw = 2 * r + 1;
    const int nblocks = inf.blocks_x * inf.blocks_y;
    const int acc_pitch = (W + 31) & ~31;
    const size_t acc_plane = (size_t)H * acc_pitch;
    const size_t off_xy = 256;
    const size_t off_z = align256(off_xy + sizeof(uint32_t) * 8 * (size_t)nblocks);
    const size_t off_ring = align256(off_z + sizeof(uint32_t) * (size_t)nblocks);
    const size_t need = off_ring + sizeof(float) * (size_t)tw * tw * 2 * acc_plane;
    if (need > kNoAllocScratchBytes) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "clip too large for the allocation-free entry point: needs %zu bytes of "
                      "scratch, the limit is %zu",
                      need, kNoAllocScratchBytes);
        return set_error(VSFEEL_E_ARG, msg);
    }
    unsigned char* base = nullptr;
    rc = scratch_address(&base);
    if (rc != VSFEEL_OK) return rc;

    cudaStream_t st = (cudaStream_t)stream;
    int* status = reinterpret_cast<int*>(base);
    uint32_t* match_xy = reinterpret_cast<uint32_t*>(base + off_xy);
    uint32_t* match_z = reinterpret_cast<uint32_t*>(base + off_z);
    float* ring = reinterpret_cast<float*>(base + off_ring);
    auto clampf = [&](int f) { return clampi(f, 0, N - 1); };
    // An interior output of a clip without the extractor scatters all its
    // stacks into one merged pair of its slot (the plain path's rule,
    // vsfeel_bm3d::merged in bm3d_engine.cu); the others keep a pair per stack.
    const char* merge_env = std::getenv("VSFEEL_MERGED_SLOTS");
    const bool merge_slots = (merge_env == nullptr || merge_env[0] != '0') &&
                             inf.extractor == 0.0f && r > 0;
    auto merged = [&](int n) { return merge_slots && n - r >= 0 && n + r <= N - 1; };
    auto slot_pair = [&](int n, int j) {
        return ring + ((size_t)(n % tw) * tw + (merged(n) ? 0 : j)) * 2 * acc_plane;
    };
    auto read_slice = [&](int n, int m) {
        for (int i = 0; i < tw; ++i)
            if (clampf(n - r + i) == m) return (r == 0) ? 0 : agg_z(i, n, N, r);
        return -1;
    };
    auto check = [&](cudaError_t e) -> int {
        if (e == cudaSuccess) return VSFEEL_OK;
        char msg[160];
        std::snprintf(msg, sizeof(msg), "CUDA error: %s", cudaGetErrorString(e));
        return set_error(VSFEEL_E_CUDA, msg);
    };

    if ((rc = check(cudaMemsetAsync(status, 0, sizeof(int), st))) != VSFEEL_OK) return rc;
    const int last = first + count - 1;
    const int m_lo = clampf(first - r), m_hi = clampf(last + r);
    int zeroed = first - 1, finished = first - 1;
    for (int m = m_lo; m <= m_hi; ++m) {
        const int want = std::min(last, m + r);
        for (int n = zeroed + 1; n <= want; ++n)
            if ((rc = check(cudaMemsetAsync(slot_pair(n, 0), 0,
                                            sizeof(float) * (size_t)(merged(n) ? 1 : tw) * 2 *
                                                acc_plane,
                                            st))) != VSFEEL_OK)
                return rc;
        zeroed = std::max(zeroed, want);

        StackJob job{};
        for (int z = 0; z < tw; ++z) {
            const int n = clampf(m - r + z);
            job.slice_frame[z] = src + (size_t)n * src_frame_stride;
            job.slice_dst[z] = (n >= first && n <= last && read_slice(n, m) == z)
                                   ? slot_pair(n, m - (n - r))
                                   : nullptr;
        }
        job.dst_plane = (int64_t)acc_plane;
        job.pitch = (int)src_row_stride;
        job.dst_pitch = acc_pitch;
        job.width = W;
        job.height = H;
        job.radius = r;
        job.step = inf.block_step;
        job.bm_range = inf.bm_range;
        job.ps_num = inf.ps_num;
        job.ps_range = inf.ps_range;
        job.nbx = inf.blocks_x;
        job.nby = inf.blocks_y;
        job.thr = inf.threshold;
        job.extractor = inf.extractor;
        job.match_xy = match_xy;
        job.match_z = match_z;
        job.status = status;
        if ((rc = check(launch_match(job, st))) != VSFEEL_OK) return rc;
        if ((rc = check(launch_filter(job, st))) != VSFEEL_OK) return rc;

        const int done = (m == m_hi) ? last : std::min(last, m - r);
        for (int n = finished + 1; n <= done; ++n) {
            NormalizeJob nj{};
            for (int i = 0; i < tw; ++i) nj.num[i] = slot_pair(n, clampf(n - r + i) - (n - r));
            nj.den_offset = (int64_t)acc_plane;
            nj.tw = merged(n) ? 1 : tw;
            nj.width = W;
            nj.height = H;
            nj.src_pitch = acc_pitch;
            nj.out_pitch = (int)dst_row_stride;
            nj.out = dst + (size_t)(n - first) * dst_frame_stride;
            if ((rc = check(launch_normalize(nj, st))) != VSFEEL_OK) return rc;
        }
        finished = std::max(finished, done);
    }
    return VSFEEL_OK;
}

}  // extern "C"
