// TEST INFRASTRUCTURE: runs the reference's own BM3D shaders
// (src/bm3d.comp, src/bm3d_agg.comp, compiled as C++ by build_ref.py) on the
// CPU, driven the way the reference's host drives them. Only the oracle
// tests, the golden-vector generator and the benchmark's reference arm load
// the resulting library.
//
// Host restatement (serial, cache-free form of src/bm3d.cpp):
//   sigma / extractor scaling ........ src/bm3d.cpp:1103-1113, 1188-1190
//   plane stride ..................... src/bm3d.cpp:1257-1275
//   specialization constants ......... src/bm3d.cpp:251-317
//   estimation dispatch per stack .... src/bm3d.cpp:558-601 (zero-fill, push constants, grid :1369-1370)
//   aggregation bases ................ src/bm3d.cpp:628-696, agg_z :369-371, grid :1371-1372
// Every stack is computed once; the reference's caches only decide which
// dispatch computes a stack, never its contents. The source ring holds every
// frame (slot = frame index), which the shader's slot arithmetic accepts.

#include "ref_simt.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

extern "C" {
void ref_bm3d_set_spec(int id, double v);
void ref_bm3d_bind(int binding, void* p);
void ref_bm3d_push(const int32_t* values, int count);
void ref_bm3d_entry();
void ref_bm3d_agg_set_spec(int id, double v);
void ref_bm3d_agg_bind(int binding, void* p);
void ref_bm3d_agg_push(const int32_t* values, int count);
void ref_bm3d_agg_entry();
}

// --------------------------------------------------------------------------
// Coroutine switch: saves the callee-saved registers on the current stack,
// stores the stack pointer to *save and resumes the context at `load`.
extern "C" void simt_swap(void** save, void* load);
asm(R"(
    .text
    .p2align 4
    .globl simt_swap
    .hidden simt_swap
    .type simt_swap,@function
simt_swap:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size simt_swap,.-simt_swap
)");

namespace simt {
namespace {

constexpr size_t kStackBytes = 256 * 1024;

struct Scheduler {
    std::vector<Invocation> inv;
    std::vector<std::unique_ptr<char[]>> stacks;
    void* home = nullptr;
    Entry entry = nullptr;
};

thread_local Scheduler* t_sched = nullptr;
thread_local Invocation* t_cur = nullptr;

[[noreturn]] void trampoline() {
    t_sched->entry();
    t_cur->done = true;
    simt_swap(&t_cur->sp, t_sched->home);
    __builtin_unreachable();
}

}  // namespace

Invocation* current() { return t_cur; }

void barrier() { simt_swap(&t_cur->sp, t_sched->home); }

void run_workgroup(Entry entry, const uint32_t ls[3], const uint32_t gid[3]) {
    thread_local Scheduler s;
    const size_t n = (size_t)ls[0] * ls[1] * ls[2];
    while (s.stacks.size() < n) s.stacks.emplace_back(new char[kStackBytes]);
    s.inv.assign(n, Invocation{});
    for (size_t i = 0; i < n; ++i) {
        Invocation& iv = s.inv[i];
        iv.local[0] = (uint32_t)(i % ls[0]);
        iv.local[1] = (uint32_t)((i / ls[0]) % ls[1]);
        iv.local[2] = (uint32_t)(i / ((size_t)ls[0] * ls[1]));
        for (int d = 0; d < 3; ++d) {
            iv.group[d] = gid[d];
            iv.global[d] = gid[d] * ls[d] + iv.local[d];
        }
        uintptr_t top = (uintptr_t)(s.stacks[i].get() + kStackBytes) & ~(uintptr_t)15;
        uint64_t* sp = (uint64_t*)top;
        *--sp = 0;                              // alignment slot: entry sees rsp % 16 == 8
        *--sp = (uint64_t)(uintptr_t)&trampoline;  // popped by `ret`
        for (int r = 0; r < 6; ++r) *--sp = 0;  // rbp rbx r12 r13 r14 r15
        iv.sp = sp;
    }
    s.entry = entry;
    Scheduler* saved_sched = t_sched;
    Invocation* saved_cur = t_cur;
    t_sched = &s;
    for (;;) {
        bool alive = false;
        for (size_t i = 0; i < n; ++i) {
            Invocation& iv = s.inv[i];
            if (iv.done) continue;
            alive = true;
            t_cur = &iv;
            simt_swap(&s.home, iv.sp);
        }
        if (!alive) break;
    }
    t_sched = saved_sched;
    t_cur = saved_cur;
}

}  // namespace simt

namespace {

inline int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

int agg_z(int i, int n, int nframes, int radius) {
    return std::min(std::max(2 * radius - i, n - nframes + 1 + radius), n + radius);
}

// Runs `entry` over a gx x gy grid of workgroups. With one thread the
// workgroups run in row-major order (x fastest); with more, rows of
// workgroups are shared out and atomic order is no longer fixed.
void dispatch(simt::Entry entry, const uint32_t ls[3], int gx, int gy, int nthreads) {
    std::atomic<int> next{0};
    auto worker = [&]() {
        for (;;) {
            const int y = next.fetch_add(1);
            if (y >= gy) break;
            for (int x = 0; x < gx; ++x) {
                const uint32_t gid[3] = {(uint32_t)x, (uint32_t)y, 0};
                simt::run_workgroup(entry, ls, gid);
            }
        }
    };
    const int nt = std::max(1, std::min(nthreads, gy));
    if (nt == 1) {
        worker();
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
}

struct Setup {
    int W, H, stride, nframes, r, tw;
    size_t pe;
    float thr, E;
    int step;
};

bool setup(Setup& S, int nframes, int W, int H, float sigma, int step, int R, int r, int P,
           int Q, int extractor_exp, bool final_pass = false) {
    if (nframes <= 0 || W < 8 || H < 8 || sigma < 0.0f || step < 1 || step > 8 || R <= 0 ||
        r < 0 || r > 4 || P < 1 || P > 8 || Q <= 0)
        return false;
    uint32_t bits = final_pass ? 0x3e40c0c1u : 0x3f021bb6u;  // src/bm3d.cpp:1103-1107
    float factor;
    std::memcpy(&factor, &bits, 4);
    S.W = W;
    S.H = H;
    S.stride = (W + 3) & ~3;
    S.nframes = nframes;
    S.r = r;
    S.tw = 2 * r + 1;
    S.pe = (size_t)S.stride * H;
    S.thr = sigma * factor;
    S.E = extractor_exp != 0 ? std::ldexp(1.0f, extractor_exp) : 0.0f;
    S.step = step;
    const double spec[14] = {double(W), double(H),    double(S.stride), double(S.thr), double(step),
                             double(R), double(r),    double(P),        double(Q),     double(S.E),
                             0.0,       0.0,          double(nframes),  final_pass ? 1.0 : 0.0};
    for (int id = 0; id < 14; ++id) ref_bm3d_set_spec(id, spec[id]);
    return true;
}

// One stack: zero-fill, then the estimation dispatch (src/bm3d.cpp:558-601),
// restricted to workgroup rows [gy_first, gy_first + gy_count) when gy_count
// is not negative (a timing sample of the dispatch).
void run_stack(const Setup& S, float* res, float* src, int m, size_t res_off, int nthreads,
               int gy_first = 0, int gy_count = -1) {
    std::memset(res + res_off, 0, sizeof(float) * S.tw * 2 * S.pe);
    ref_bm3d_bind(0, res);
    ref_bm3d_bind(1, src);
    const int32_t push[4] = {(int32_t)res_off, m, S.nframes, S.r == 0 ? m : 0};
    ref_bm3d_push(push, 4);
    const uint32_t ls[3] = {32, 1, 1};
    const int gx = (S.W + 4 * S.step - 1) / (4 * S.step);
    const int gy = (S.H + S.step - 1) / S.step;
    if (gy_count < 0) {
        dispatch(&ref_bm3d_entry, ls, gx, gy, nthreads);
        return;
    }
    const int lo = std::min(std::max(gy_first, 0), gy);
    const int hi = std::min(lo + gy_count, gy);
    std::atomic<int> next{lo};
    auto worker = [&]() {
        for (;;) {
            const int y = next.fetch_add(1);
            if (y >= hi) break;
            for (int x = 0; x < gx; ++x) {
                const uint32_t gid[3] = {(uint32_t)x, (uint32_t)y, 0};
                simt::run_workgroup(&ref_bm3d_entry, ls, gid);
            }
        }
    };
    const int nt = std::max(1, std::min(nthreads, hi - lo));
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
}

// The source ring with slot = frame index. In the final pass a slot holds
// [ref][source] (src/bm3d.comp:70-81).
std::vector<float> load_frames(const Setup& S, const float* frames, const float* ref = nullptr) {
    const int per_slot = ref ? 2 : 1;
    std::vector<float> src((size_t)S.nframes * per_slot * S.pe, 0.0f);
    for (int f = 0; f < S.nframes; ++f)
        for (int y = 0; y < S.H; ++y) {
            const size_t slot = (size_t)f * per_slot * S.pe + (size_t)y * S.stride;
            if (ref) {
                std::memcpy(&src[slot], ref + ((size_t)f * S.H + y) * S.W, sizeof(float) * S.W);
                std::memcpy(&src[slot + S.pe], frames + ((size_t)f * S.H + y) * S.W,
                            sizeof(float) * S.W);
            } else {
                std::memcpy(&src[slot], frames + ((size_t)f * S.H + y) * S.W, sizeof(float) * S.W);
            }
        }
    return src;
}

}  // namespace

extern "C" {

// Denoises out_count frames starting at out_first with the reference shaders.
// frames: nframes x H x W floats; out: out_count x H x W. Returns 0 or -1.
// ref (optional): the basic-estimate clip of the final (Wiener) pass.
int ref_bm3d_clip(const float* frames, const float* ref, int nframes, int W, int H, float sigma,
                  int step, int R, int r, int P, int Q, int extractor_exp, int out_first,
                  int out_count, int nthreads, float* out) {
    Setup S;
    if (!setup(S, nframes, W, H, sigma, step, R, r, P, Q, extractor_exp, ref != nullptr)) return -1;
    if (out_first < 0 || out_count < 0 || out_first + out_count > nframes) return -1;
    std::vector<float> src = load_frames(S, frames, ref);
    const int m_lo = clampi(out_first - r, 0, nframes - 1);
    const int m_hi = clampi(out_first + out_count - 1 + r, 0, nframes - 1);
    const size_t stack = (size_t)S.tw * 2 * S.pe;
    std::vector<float> res((size_t)(m_hi - m_lo + 1) * stack, 0.0f);
    for (int m = m_lo; m <= m_hi; ++m) run_stack(S, res.data(), src.data(), m, (m - m_lo) * stack, nthreads);

    const double agg_spec[4] = {double(W), double(H), double(S.stride), double(S.tw)};
    for (int id = 0; id < 4; ++id) ref_bm3d_agg_set_spec(id, agg_spec[id]);
    std::vector<float> dst(S.pe, 0.0f);
    ref_bm3d_agg_bind(0, res.data());
    ref_bm3d_agg_bind(2, dst.data());
    const uint32_t ls[3] = {32, 8, 1};
    for (int q = 0; q < out_count; ++q) {
        const int n = out_first + q;
        int32_t bases[9] = {0};
        for (int i = 0; i < S.tw; ++i) {
            const int mi = clampi(n - r + i, 0, nframes - 1);
            const int z = (r == 0) ? 0 : agg_z(i, n, nframes, r);
            bases[i] = (int32_t)((size_t)(mi - m_lo) * stack + (size_t)z * 2 * S.pe);
        }
        ref_bm3d_agg_push(bases, 9);
        dispatch(&ref_bm3d_agg_entry, ls, (W + 31) / 32, (H + 7) / 8, nthreads);
        for (int y = 0; y < H; ++y)
            std::memcpy(out + ((size_t)q * H + y) * W, &dst[(size_t)y * S.stride], sizeof(float) * W);
    }
    return 0;
}

// The 2*TW accumulated slices of stack m (H x W each, numerator then weight
// per slice), as the reference's estimation kernel leaves them.
int ref_bm3d_stack(const float* frames, int nframes, int W, int H, float sigma, int step, int R,
                   int r, int P, int Q, int extractor_exp, int m, int nthreads, float* slices) {
    Setup S;
    if (!setup(S, nframes, W, H, sigma, step, R, r, P, Q, extractor_exp)) return -1;
    if (m < 0 || m >= nframes) return -1;
    std::vector<float> src = load_frames(S, frames);
    std::vector<float> res((size_t)S.tw * 2 * S.pe, 0.0f);
    run_stack(S, res.data(), src.data(), m, 0, nthreads);
    for (int p = 0; p < 2 * S.tw; ++p)
        for (int y = 0; y < H; ++y)
            std::memcpy(slices + ((size_t)p * H + y) * W, &res[(size_t)p * S.pe + (size_t)y * S.stride],
                        sizeof(float) * W);
    return 0;
}

// Timing sample: the estimation dispatch of stack m over workgroup rows
// [gy_first, gy_first + gy_count) only (gy = block row, block_step pixels
// apart). The slices are discarded. Returns 0 or -1.
int ref_bm3d_stack_rows(const float* frames, int nframes, int W, int H, float sigma, int step, int R,
                        int r, int P, int Q, int extractor_exp, int m, int gy_first, int gy_count,
                        int nthreads) {
    Setup S;
    if (!setup(S, nframes, W, H, sigma, step, R, r, P, Q, extractor_exp)) return -1;
    if (m < 0 || m >= nframes || gy_count < 0) return -1;
    std::vector<float> src = load_frames(S, frames);
    std::vector<float> res((size_t)S.tw * 2 * S.pe, 0.0f);
    run_stack(S, res.data(), src.data(), m, 0, nthreads, gy_first, gy_count);
    return 0;
}

}  // extern "C"
