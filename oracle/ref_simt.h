// TEST INFRASTRUCTURE: a deterministic CPU executor for GLSL compute shaders
// compiled as C++ (see build_ref.py). Only the oracle tests and the
// benchmark's reference arm use it.
//
// A workgroup runs as one coroutine per invocation on the calling thread.
// barrier() switches to the next invocation; the scheduler resumes the
// invocations in local-index order, so between two barriers invocation 0
// runs first, then 1, and so on. Atomic adds therefore land in a fixed order
// when the executor runs on one thread.
#pragma once

#include <atomic>
#include <cstdint>
#include <vector>

namespace simt {

struct Invocation {
    void* sp = nullptr;
    bool done = false;
    uint32_t local[3] = {0, 0, 0};
    uint32_t group[3] = {0, 0, 0};
    uint32_t global[3] = {0, 0, 0};
};

using Entry = void (*)();

// Runs every invocation of one workgroup to completion.
void run_workgroup(Entry entry, const uint32_t local_size[3], const uint32_t group_id[3]);

// The invocation that is executing on this thread.
Invocation* current();

// Switches to the next invocation of the workgroup (GLSL barrier()).
void barrier();

}  // namespace simt

// GLSL built-ins, included inside each translated shader's namespace so that
// unqualified calls resolve to these float/int overloads.
#define SIMT_GLSL_BUILTINS                                                          \
    struct uvec3_ {                                                                 \
        uint32_t x, y, z;                                                           \
    };                                                                              \
    inline uvec3_ local_id_() {                                                     \
        auto* i = simt::current();                                                  \
        return {i->local[0], i->local[1], i->local[2]};                             \
    }                                                                               \
    inline uvec3_ group_id_() {                                                     \
        auto* i = simt::current();                                                  \
        return {i->group[0], i->group[1], i->group[2]};                             \
    }                                                                               \
    inline uvec3_ global_id_() {                                                    \
        auto* i = simt::current();                                                  \
        return {i->global[0], i->global[1], i->global[2]};                          \
    }                                                                               \
    inline int min(int a, int b) { return a < b ? a : b; }                          \
    inline int max(int a, int b) { return a > b ? a : b; }                          \
    inline float min(float a, float b) { return b < a ? b : a; }                    \
    inline float max(float a, float b) { return a < b ? b : a; }                    \
    inline float abs(float a) { return __builtin_fabsf(a); }                        \
    inline int abs(int a) { return a < 0 ? -a : a; }                                \
    inline float fma(float a, float b, float c) { return __builtin_fmaf(a, b, c); } \
    inline float atomicAdd(float& x, float v) {                                     \
        return std::atomic_ref<float>(x).fetch_add(v, std::memory_order_relaxed);   \
    }                                                                               \
    inline void barrier() { simt::barrier(); }

#define gl_LocalInvocationID (local_id_())
#define gl_WorkGroupID (group_id_())
#define gl_GlobalInvocationID (global_id_())
