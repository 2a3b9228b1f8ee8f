// Host stand-in for <cuda_runtime.h>, for running the engine's device code
// (mr_device.cuh) on the CPU in the tests.  One CTA is emulated by THREADS
// cooperative fibers on one host thread (ucontext): __syncthreads waits at a
// barrier over all of them, and the warp-level intrinsics exchange values
// through a barrier over the 32 fibers of the warp; a fiber that waits
// switches to the next one, round-robin.  Only what mr_device.cuh uses is
// provided.
#pragma once
#include <stdint.h>
#include <stdlib.h>
#include <ucontext.h>

#include <stdio.h>

#include <algorithm>
#include <functional>
#include <stdexcept>
#include <vector>

#define __device__
#define __host__
#define __forceinline__ inline
#define __constant__

struct uint4 {
    unsigned x, y, z, w;
};

struct emu_dim3 {
    unsigned x = 0, y = 0, z = 0;
};

// The running fiber's indices (set on every switch).
inline emu_dim3 threadIdx;
inline emu_dim3 blockDim;

namespace emu {

struct Fiber {
    ucontext_t ctx;
    void *stack = nullptr;
    bool done = false;
};

struct Group {
    int size = 0, arrived = 0;
    unsigned long long gen = 0;
};

inline std::vector<Fiber> *fibers = nullptr;
inline std::vector<Group> *groups = nullptr;  // 0: the CTA; 1 + w: warp w
inline std::vector<unsigned long long> *lane_vals = nullptr;
inline const std::function<void()> *body = nullptr;
inline ucontext_t main_ctx;
inline int current = 0;

inline void switch_to(int next) {
    const int prev = current;
    current = next;
    threadIdx.x = (unsigned)next;
    swapcontext(&(*fibers)[prev].ctx, &(*fibers)[next].ctx);
    threadIdx.x = (unsigned)current;
}

// Switches to the next unfinished fiber; false if there is none but this one.
inline bool yield() {
    const int n = (int)fibers->size();
    for (int k = 1; k < n; k++) {
        const int j = (current + k) % n;
        if (!(*fibers)[j].done) {
            switch_to(j);
            return true;
        }
    }
    return false;
}

inline void group_wait(int g) {
    Group &G = (*groups)[g];
    const unsigned long long my = G.gen;
    if (++G.arrived == G.size) {
        G.arrived = 0;
        G.gen++;
        return;
    }
    while (G.gen == my)
        if (!yield()) {
            // every other thread has finished: this barrier can never complete
            fprintf(stderr, "emulated CTA: thread %d waits at a barrier no other thread reaches\n", current);
            abort();
        }
}

inline void fiber_main(int id) {
    (*body)();
    (*fibers)[id].done = true;
    yield();  // to an unfinished fiber, never back here; none left: to the caller
    setcontext(&main_ctx);
}

inline void trampoline(unsigned lo, unsigned hi) {
    (void)hi;
    fiber_main((int)lo);
}

// Runs f once per thread of one CTA of `threads` threads.
inline void run_cta(int threads, const std::function<void()> &f) {
    std::vector<Fiber> fs(threads);
    std::vector<Group> gs(1 + (threads + 31) / 32);
    gs[0].size = threads;
    for (int w = 0; w + 1 < (int)gs.size(); w++) gs[1 + w].size = std::min(32, threads - 32 * w);
    std::vector<unsigned long long> vals(threads);
    fibers = &fs;
    groups = &gs;
    lane_vals = &vals;
    body = &f;
    blockDim.x = (unsigned)threads;
    const size_t stack_bytes = 256 * 1024;
    for (int t = 0; t < threads; t++) {
        Fiber &fb = fs[t];
        fb.stack = malloc(stack_bytes);
        if (!fb.stack) throw std::runtime_error("fiber stack");
        getcontext(&fb.ctx);
        fb.ctx.uc_stack.ss_sp = fb.stack;
        fb.ctx.uc_stack.ss_size = stack_bytes;
        fb.ctx.uc_link = &main_ctx;
        makecontext(&fb.ctx, (void (*)())trampoline, 2, (unsigned)t, 0u);
    }
    current = 0;
    threadIdx.x = 0;
    swapcontext(&main_ctx, &fs[0].ctx);
    for (auto &fb : fs) free(fb.stack);
    fibers = nullptr;
    groups = nullptr;
    lane_vals = nullptr;
    body = nullptr;
}

}  // namespace emu

inline void __syncthreads() { emu::group_wait(0); }

inline unsigned __umulhi(unsigned a, unsigned b) { return (unsigned)(((unsigned long long)a * b) >> 32); }

template <class T>
inline T __ldg(const T *p) { return *p; }

template <class T>
inline T __ldcg(const T *p) { return *p; }

// Every lane of the warp takes part (all calls in the engine are warp-uniform).
inline unsigned __ballot_sync(unsigned, int pred) {
    const unsigned t = threadIdx.x, w = t >> 5, base = w << 5;
    (*emu::lane_vals)[t] = pred ? 1ull : 0ull;
    emu::group_wait(1 + (int)w);
    unsigned r = 0;
    for (unsigned i = 0; i < 32 && base + i < blockDim.x; i++) r |= ((*emu::lane_vals)[base + i] ? 1u : 0u) << i;
    emu::group_wait(1 + (int)w);
    return r;
}

template <class T>
inline T __shfl_up_sync(unsigned, T v, unsigned delta) {
    const unsigned t = threadIdx.x, w = t >> 5, lane = t & 31u;
    (*emu::lane_vals)[t] = (unsigned long long)v;
    emu::group_wait(1 + (int)w);
    const T r = lane >= delta ? (T)(*emu::lane_vals)[t - delta] : v;
    emu::group_wait(1 + (int)w);
    return r;
}
