// Work-item emulation shim for compiling the reference's own device kernels
// (pyPaSWAS/Core/cuda/default_main.cu and pyPaSWAS/Core/ocl/default_main_cpu.cl,
// after template expansion by pyPaSWAS/Core/PaSWAS.py) as host C++.
//
// TEST INFRASTRUCTURE ONLY.  This file is part of the oracle: it is used to run
// the reference kernels on the CPU so that golden outputs can be generated and
// the CPU baseline can be timed.  Nothing in the shipped engine includes it.
//
// Execution model
//   * Blocks / work-groups run one after another in linear order (x fastest),
//     or spread over host threads when a launch is started with nthreads > 1
//     (the OpenCL CPU kernels have no work-group local memory, so blocks are
//     independent within a launch).
//   * The work-items of one block run as cooperative fibers on one host thread.
//     A barrier (__syncthreads / barrier()) switches back to the scheduler; the
//     scheduler resumes the fibers in linear thread order (threadIdx.x fastest).
//     Between two barriers every work-item therefore runs to completion in
//     linear order, which is a legal interleaving of the reference kernels
//     (they have no intra-phase races) and pins the atomicAdd order of starting
//     points to linear thread order.
//   * __shared__ variables become function-local statics in thread_local
//     storage: one copy per host thread, shared by the fibers of the block.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <stdlib.h>
#include <stdio.h>
#include <functional>
#include <vector>
#include <thread>
#include <atomic>
#include <algorithm>

struct emu_dim3 { unsigned int x, y, z; };

// Fiber switch: saves the callee-saved registers of the x86-64 System V ABI
// on the current stack, stores the stack pointer in *from and continues on
// `to`.  Unlike swapcontext it makes no system call (no signal mask), so a
// barrier costs a few nanoseconds, as work-item loops of an OpenCL CPU
// runtime do.  The floating-point control state is never changed by the
// kernels, so it is not switched.
extern "C" void emu_ctx_switch(void** from, void* to);
asm(R"(
.text
.globl emu_ctx_switch
.hidden emu_ctx_switch
.type emu_ctx_switch,@function
emu_ctx_switch:
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
.size emu_ctx_switch, .-emu_ctx_switch
)");

namespace emu {

struct Fiber {
    void* sp;
    char* stack;
    bool done;
    emu_dim3 tid;
};

constexpr size_t kFiberStack = 128 * 1024;

// Fiber stacks are allocated once per host thread and reused by every block.
inline char* fiber_stack(unsigned t) {
    static thread_local std::vector<char*> pool;
    while (pool.size() <= t) pool.push_back(static_cast<char*>(malloc(kFiberStack)));
    return pool[t];
}

struct BlockRunner {
    void* sched;
    std::vector<Fiber> fibers;
    int current;
    const std::function<void()>* body;
};

inline thread_local BlockRunner* tl_runner = nullptr;
inline thread_local emu_dim3 tl_threadIdx, tl_blockIdx, tl_blockDim, tl_gridDim;

inline void fiber_entry() {
    BlockRunner* r = tl_runner;
    (*r->body)();
    r->fibers[r->current].done = true;
    emu_ctx_switch(&r->fibers[r->current].sp, r->sched);  // never resumed
}

inline void barrier_yield() {
    BlockRunner* r = tl_runner;
    emu_ctx_switch(&r->fibers[r->current].sp, r->sched);
}

// A fresh fiber's stack: switching to it "returns" into fiber_entry with the
// stack aligned as at a function's entry (rsp + 8 a multiple of 16).
inline void* fiber_start(char* stack) {
    uintptr_t top = ((uintptr_t)(stack + kFiberStack)) & ~(uintptr_t)15;
    void** sp = (void**)top;
    *--sp = nullptr;                                   // fiber_entry's return slot (never used)
    *--sp = (void*)(void (*)())fiber_entry;            // popped by the switch's ret
    for (int k = 0; k < 6; ++k) *--sp = nullptr;       // r15 r14 r13 r12 rbx rbp
    return (void*)sp;
}

// Runs one block: bdx*bdy work-items, each executing `body`.
inline void run_block(unsigned bdx, unsigned bdy, const std::function<void()>& body) {
    BlockRunner r;
    r.body = &body;
    r.current = 0;
    const unsigned n = bdx * bdy;
    r.fibers.resize(n);
    for (unsigned t = 0; t < n; ++t) {
        Fiber& f = r.fibers[t];
        f.stack = fiber_stack(t);
        f.done = false;
        f.tid = emu_dim3{t % bdx, t / bdx, 0};
        f.sp = fiber_start(f.stack);
    }
    BlockRunner* saved = tl_runner;
    tl_runner = &r;
    bool any = true;
    while (any) {
        any = false;
        for (unsigned t = 0; t < n; ++t) {
            if (r.fibers[t].done) continue;
            r.current = (int)t;
            tl_threadIdx = r.fibers[t].tid;
            emu_ctx_switch(&r.sched, r.fibers[t].sp);
            if (!r.fibers[t].done) any = true;
        }
    }
    tl_runner = saved;
}

// Launches a grid.  nthreads > 1 spreads whole blocks over host threads.
inline void launch(unsigned gx, unsigned gy, unsigned bdx, unsigned bdy,
                   const std::function<void()>& body, int nthreads = 1) {
    const unsigned long nblocks = (unsigned long)gx * gy;
    auto run_range = [&](unsigned long b0, unsigned long b1) {
        for (unsigned long b = b0; b < b1; ++b) {
            tl_blockIdx = emu_dim3{(unsigned)(b % gx), (unsigned)(b / gx), 0};
            tl_blockDim = emu_dim3{bdx, bdy, 1};
            tl_gridDim = emu_dim3{gx, gy, 1};
            run_block(bdx, bdy, body);
        }
    };
    if (nthreads <= 1 || nblocks < 2) {
        run_range(0, nblocks);
        return;
    }
    std::atomic<unsigned long> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
        pool.emplace_back([&]() {
            for (;;) {
                unsigned long b = next.fetch_add(16);
                if (b >= nblocks) break;
                run_range(b, std::min(nblocks, b + 16));
            }
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace emu

// ---------------------------------------------------------------- CUDA dialect
#define __global__
#define __device__
#define __constant__
#define __shared__ static thread_local
#define threadIdx (emu::tl_threadIdx)
#define blockIdx (emu::tl_blockIdx)
#define blockDim (emu::tl_blockDim)
#define gridDim (emu::tl_gridDim)
inline void __syncthreads() { emu::barrier_yield(); }
inline float __int_as_float(int v) { float f; memcpy(&f, &v, 4); return f; }
inline int __float_as_int(float f) { int v; memcpy(&v, &f, 4); return v; }
inline unsigned int atomicAdd(unsigned int* p, unsigned int v) {
    return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
// CUDA's max() on floats is fmaxf; on ints the integer max.
inline float max(float a, float b) { return fmaxf(a, b); }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }

// -------------------------------------------------------------- OpenCL dialect
#define __kernel
#define __global
#define __local static thread_local
#define constant
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
inline unsigned get_local_id(int d) { return d == 0 ? emu::tl_threadIdx.x : emu::tl_threadIdx.y; }
inline unsigned get_group_id(int d) { return d == 0 ? emu::tl_blockIdx.x : emu::tl_blockIdx.y; }
inline void barrier(int) { emu::barrier_yield(); }
inline float as_float(int v) { float f; memcpy(&f, &v, 4); return f; }
inline int as_int(float f) { int v; memcpy(&v, &f, 4); return v; }
inline unsigned int atom_inc(volatile unsigned int* p) {
    return __atomic_fetch_add((unsigned int*)p, 1u, __ATOMIC_SEQ_CST);
}
inline int atom_xchg(volatile int* p, int v) {
    return __atomic_exchange_n((int*)p, v, __ATOMIC_SEQ_CST);
}
