// Host stand-in for <cuda_runtime.h>, for running the engine's device code
// (mr_device.cuh, sieve_device.cuh) on the CPU in the tests.  One CTA is
// emulated by cooperative fibers on one host thread (ucontext), one per CUDA
// thread: __syncthreads waits at a barrier over all of them, and the
// warp-level intrinsics exchange values through a barrier over the 32 fibers
// of the warp; a fiber that waits switches to the next one, round-robin.  A
// grid runs its CTAs one after another, so atomics need no locking.  Only
// what those headers use is provided.
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
#define __global__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)
#define __constant__
#define __shared__ static  // one CTA at a time: a static is the CTA's shared variable
#define __align__(n) alignas(n)
#define PFB_DYNAMIC_SMEM(T, name) T *name = emu::dynamic_smem<T>()

typedef int cudaError_t;
enum : int { cudaSuccess = 0 };

struct uint4 {
    unsigned x, y, z, w;
};

struct emu_dim3 {
    unsigned x = 0, y = 0, z = 0;
};

// The running fiber's indices (set on every switch) and the grid's.
inline emu_dim3 threadIdx;
inline emu_dim3 blockDim;
inline emu_dim3 blockIdx;
inline emu_dim3 gridDim;

namespace emu {

// Context switch: on x86-64 (without a sanitizer, which must see stack
// switches through swapcontext) a plain switch of the callee-saved registers
// and the stack pointer; elsewhere ucontext.
#if defined(__x86_64__) && !defined(__SANITIZE_ADDRESS__)
#define EMU_FAST_SWITCH 1
extern "C" void emu_switch(void **save_sp, void *load_sp);
asm(R"(
    .text
    .globl emu_switch
    .type emu_switch, @function
emu_switch:
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
    .size emu_switch, .-emu_switch
)");
#endif

struct Fiber {
    ucontext_t ctx;
    void *sp = nullptr;  // saved stack pointer (fast switch)
    void *stack = nullptr;
    bool done = false;
};

struct Group {
    int size = 0, arrived = 0;
    unsigned long long gen = 0;
};

// Dynamic shared memory of the running grid: exactly the bytes the launch
// asked for (so that a sanitizer sees an overrun).
inline unsigned char *dyn_smem = nullptr;
template <class T>
inline T *dynamic_smem() { return reinterpret_cast<T *>(dyn_smem); }

inline std::vector<Fiber> *fibers = nullptr;
inline std::vector<Group> *groups = nullptr;  // 0: the CTA; 1 + w: warp w
inline std::vector<unsigned long long> *lane_vals = nullptr;
inline const std::function<void()> *body = nullptr;
inline ucontext_t main_ctx;
inline void *main_sp = nullptr;
inline int current = 0;

inline void switch_to(int next) {
    const int prev = current;
    current = next;
    threadIdx.x = (unsigned)next;
#ifdef EMU_FAST_SWITCH
    emu_switch(&(*fibers)[prev].sp, (*fibers)[next].sp);
#else
    swapcontext(&(*fibers)[prev].ctx, &(*fibers)[next].ctx);
#endif
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
#ifdef EMU_FAST_SWITCH
    void *dead = nullptr;
    emu_switch(&dead, main_sp);
#else
    setcontext(&main_ctx);
#endif
}

#ifdef EMU_FAST_SWITCH
inline void fiber_entry() { fiber_main(current); }
#endif

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
    static std::vector<void *> stacks;  // reused by every CTA of the process
    while ((int)stacks.size() < threads) {
        void *st = malloc(stack_bytes);
        if (!st) throw std::runtime_error("fiber stack");
        stacks.push_back(st);
    }
    for (int t = 0; t < threads; t++) {
        Fiber &fb = fs[t];
        fb.stack = stacks[t];
#ifdef EMU_FAST_SWITCH
        // initial frame: six register slots, then fiber_entry as the return
        // address, then a null slot so that fiber_entry starts as if called
        void **p = (void **)(((uintptr_t)fb.stack + stack_bytes) & ~(uintptr_t)15);
        *--p = nullptr;
        *--p = (void *)&fiber_entry;
        for (int r = 0; r < 6; r++) *--p = nullptr;
        fb.sp = p;
#else
        getcontext(&fb.ctx);
        fb.ctx.uc_stack.ss_sp = fb.stack;
        fb.ctx.uc_stack.ss_size = stack_bytes;
        fb.ctx.uc_link = &main_ctx;
        makecontext(&fb.ctx, (void (*)())trampoline, 2, (unsigned)t, 0u);
#endif
    }
    current = 0;
    threadIdx.x = 0;
#ifdef EMU_FAST_SWITCH
    emu_switch(&main_sp, fs[0].sp);
#else
    swapcontext(&main_ctx, &fs[0].ctx);
#endif
    fibers = nullptr;
    groups = nullptr;
    lane_vals = nullptr;
    body = nullptr;
}

// Runs f for every thread of a gx x gy grid of CTAs of `threads` threads,
// one CTA after another, with smem bytes of dynamic shared memory.
inline void run_grid(unsigned gx, unsigned gy, int threads, const std::function<void()> &f, size_t smem = 0) {
    std::vector<unsigned char> buf(smem);
    dyn_smem = smem ? buf.data() : nullptr;
    gridDim.x = gx;
    gridDim.y = gy;
    for (unsigned y = 0; y < gy; y++)
        for (unsigned x = 0; x < gx; x++) {
            blockIdx.x = x;
            blockIdx.y = y;
            run_cta(threads, f);
        }
    dyn_smem = nullptr;
}

}  // namespace emu

inline void __syncthreads() { emu::group_wait(0); }

inline unsigned atomicOr(unsigned *p, unsigned v) {
    const unsigned o = *p;
    *p = o | v;
    return o;
}

inline unsigned atomicAdd(unsigned *p, unsigned v) {
    const unsigned o = *p;
    *p = o + v;
    return o;
}

inline int atomicCAS(int *p, int cmp, int v) {
    const int o = *p;
    if (o == cmp) *p = v;
    return o;
}

inline int atomicExch(int *p, int v) {
    const int o = *p;
    *p = v;
    return o;
}

inline void __threadfence() {}

// Barrier of the CTA that also returns whether pred holds on every thread.
inline int __syncthreads_and(int pred) {
    (*emu::lane_vals)[threadIdx.x] = pred ? 1ull : 0ull;
    emu::group_wait(0);
    int all = 1;
    for (unsigned t = 0; t < blockDim.x; t++) all &= (*emu::lane_vals)[t] ? 1 : 0;
    emu::group_wait(0);
    return all;
}

// CUDA's integer min/max (mixed operands convert as in arithmetic).
template <class A, class B>
inline auto min(A a, B b) -> decltype(a + b) {
    return a < b ? a : b;
}
template <class A, class B>
inline auto max(A a, B b) -> decltype(a + b) {
    return a < b ? b : a;
}

inline int __popc(unsigned v) { return __builtin_popcount(v); }
inline int __ffs(int v) { return __builtin_ffs(v); }

inline unsigned long long __umul64hi(unsigned long long a, unsigned long long b) {
    return (unsigned long long)(((unsigned __int128)a * b) >> 64);
}

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
inline T __shfl_xor_sync(unsigned, T v, int lane_mask) {
    const unsigned t = threadIdx.x, w = t >> 5, lane = t & 31u;
    (*emu::lane_vals)[t] = (unsigned long long)v;
    emu::group_wait(1 + (int)w);
    const T r = (T)(*emu::lane_vals)[(w << 5) + (lane ^ (unsigned)lane_mask)];
    emu::group_wait(1 + (int)w);
    return r;
}

template <class T>
inline T __shfl_sync(unsigned, T v, int src) {
    const unsigned t = threadIdx.x, w = t >> 5;
    (*emu::lane_vals)[t] = (unsigned long long)v;
    emu::group_wait(1 + (int)w);
    const T r = (T)(*emu::lane_vals)[(w << 5) + ((unsigned)src & 31u)];
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
