/*
 * emu_shim.hpp -- a small SIMT emulator that lets the reference's CUDA kernel
 * sources (src/RPBHKernels.cu, src/RPFA2Kernels.cu) compile as host C++ and run
 * on the CPU, so the oracle can be checked against what those kernels compute.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref); nothing in the engine uses it.
 *
 * Model: one block at a time; each CUDA thread is a cooperative coroutine on
 * its own stack.  A thread runs until it reaches __syncthreads() (a barrier
 * over the block's threads that have not exited, as on Volta and later) or a
 * warp vote (a barrier over the warp's threads that have not exited).  Between
 * two such points the threads of a warp run one after another in lane order,
 * which reproduces the lock-step reads and writes of the reference's
 * warp-shared traversal stack.  A launch can also make every read of blockDim
 * a warp barrier: ForceCalculationKernel reads it in its per-body loop
 * increment, where a real warp is converged, so no lane starts the next body
 * (and re-initialises the shared stack) before its warp has finished the
 * current one.  Atomics are plain read-modify-writes, which is
 * exact because only one coroutine runs at a time.  A spin loop with no
 * barrier in it never yields, so kernels that spin on other threads
 * (SortKernel) must be launched with one thread; the harness does that.
 */
#pragma once
#include <assert.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <functional>
#include <vector>

struct dim3 {
    unsigned x, y, z;
};
struct float2 {
    float x, y;
};

namespace emu {

enum State { RUN, BAR, VOTE, WSYNC, DONE };

struct Thread {
    void *sp;
    dim3 tid;
    State st;
    int vote_in, vote_out;
    char *stack;
};

struct Block {
    dim3 bidx, bdim, gdim;
    std::vector<Thread> th;
    unsigned cur;
    void *sched_sp;
    std::function<void()> body;
    bool sync_on_blockdim;
};

extern Block *B;

void launch(unsigned grid, unsigned block, std::function<void()> body,
            bool sync_on_blockdim = false);
void syncthreads();
int all_sync(int pred);
const dim3 &blockdim_hook();

}  // namespace emu

#define threadIdx (emu::B->th[emu::B->cur].tid)
#define blockIdx (emu::B->bidx)
#define blockDim (emu::blockdim_hook())
#define gridDim (emu::B->gdim)

#define __global__
#define __device__
#define __shared__ static
#define __launch_bounds__(a, b)
#define __syncthreads() emu::syncthreads()
#define __threadfence() ((void)0)
#define __threadfence_block() ((void)0)
#define __activemask() 0xffffffffu
#define __all_sync(mask, pred) emu::all_sync((pred) ? 1 : 0)

inline int atomicCAS(int *a, int cmp, int val) {
    int old = *a;
    if (old == cmp) *a = val;
    return old;
}
inline int atomicSub(int *a, int v) {
    int old = *a;
    *a = old - v;
    return old;
}
inline int atomicMax(int *a, int v) {
    int old = *a;
    if (v > old) *a = v;
    return old;
}
inline unsigned atomicInc(unsigned *a, unsigned v) {
    unsigned old = *a;
    *a = (old >= v) ? 0u : old + 1u;
    return old;
}
inline float atomicAdd(float *a, float v) {
    float old = *a;
    *a = old + v;
    return old;
}
inline int max(int a, int b) { return a > b ? a : b; }
inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
