/*
 * ref_gpu_emu.cpp -- runs the reference's own GPU kernels (src/RPBHKernels.cu,
 * src/RPFA2Kernels.cu, included from the reference tree at build time, never
 * copied) on the CPU through emu_shim.hpp, in the order of
 * CUDAForceAtlas2::doStep (src/RPGPUForceAtlas2.cu:206-248).
 * TEST INFRASTRUCTURE ONLY: it pins the oracle restatement in oracle/.
 *
 * Launch shapes differ from the reference's (one block everywhere); the
 * kernels are written for any shape, with these exceptions honoured here:
 *  - BoundingBoxKernel and SpeedKernel index with THREADS1, so they get 512
 *    threads;
 *  - ForceCalculationKernel gets 256 = THREADS5 threads, so its warps hold the
 *    same 32 consecutive sorted bodies as on a GPU;
 *  - SortKernel spins on other threads and gets one thread (cells are created
 *    after their parents, so one thread walking down never waits);
 *  - SummarizationKernel and ClearKernel2 get 32 threads so that their first
 *    cell, (bottom & -32) + threadIdx, covers [bottom, nnodes] exactly.
 */
#include "emu_shim.hpp"

#include <string.h>

#include <algorithm>

// The reference sources, compiled as host code in this translation unit so
// that their file-static device variables are visible to the harness.
#include "RPBHKernels.cu"
#include "RPFA2Kernels.cu"

namespace emu {

Block *B = nullptr;
static const size_t kStack = 64 * 1024;

extern "C" void emu_swap(void **save_sp, void *load_sp);
// x86-64 SysV: save callee-saved registers on the current stack, switch
// stacks, restore the other context's registers.
asm(R"(
    .text
    .globl emu_swap
    .type emu_swap, @function
emu_swap:
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
    .size emu_swap, .-emu_swap
)");

static void entry() {
    Block *b = B;
    b->body();
    b->th[b->cur].st = DONE;
    emu_swap(&b->th[b->cur].sp, b->sched_sp);
    abort();  // never resumed
}

static void *fresh_stack(char *mem, size_t size) {
    uintptr_t top = (uintptr_t)(mem + size) & ~(uintptr_t)15;
    void **sp = (void **)top;
    *--sp = nullptr;          // fake return address of entry()
    *--sp = (void *)&entry;   // popped by emu_swap's ret
    for (int i = 0; i < 6; ++i) *--sp = nullptr;  // rbp rbx r12..r15
    return sp;
}

void launch(unsigned grid, unsigned block, std::function<void()> body, bool sync_on_blockdim) {
    for (unsigned bx = 0; bx < grid; ++bx) {
        Block blk;
        blk.bidx = {bx, 0, 0};
        blk.bdim = {block, 1, 1};
        blk.gdim = {grid, 1, 1};
        blk.body = body;
        blk.sync_on_blockdim = sync_on_blockdim;
        blk.th.resize(block);
        for (unsigned t = 0; t < block; ++t) {
            blk.th[t].stack = (char *)malloc(kStack);
            blk.th[t].sp = fresh_stack(blk.th[t].stack, kStack);
            blk.th[t].tid = {t, 0, 0};
            blk.th[t].st = RUN;
        }
        B = &blk;
        for (;;) {
            bool progressed = false;
            for (unsigned t = 0; t < block; ++t) {
                if (blk.th[t].st != RUN) continue;
                blk.cur = t;
                emu_swap(&blk.sched_sp, blk.th[t].sp);
                progressed = true;
            }
            unsigned live = 0, at_bar = 0;
            for (unsigned t = 0; t < block; ++t) {
                if (blk.th[t].st != DONE) live++;
                if (blk.th[t].st == BAR) at_bar++;
            }
            if (live == 0) break;
            if (at_bar == live) {
                for (unsigned t = 0; t < block; ++t)
                    if (blk.th[t].st == BAR) blk.th[t].st = RUN;
                progressed = true;
            }
            for (unsigned w = 0; w < block; w += 32) {
                unsigned end = std::min(block, w + 32), wl = 0, wv = 0, ws = 0;
                int all = 1;
                for (unsigned t = w; t < end; ++t) {
                    if (blk.th[t].st != DONE) wl++;
                    if (blk.th[t].st == VOTE) {
                        wv++;
                        all &= blk.th[t].vote_in;
                    }
                    if (blk.th[t].st == WSYNC) ws++;
                }
                if (wl > 0 && wv == wl) {
                    for (unsigned t = w; t < end; ++t)
                        if (blk.th[t].st == VOTE) {
                            blk.th[t].vote_out = all;
                            blk.th[t].st = RUN;
                        }
                    progressed = true;
                }
                if (wl > 0 && ws == wl) {
                    for (unsigned t = w; t < end; ++t)
                        if (blk.th[t].st == WSYNC) blk.th[t].st = RUN;
                    progressed = true;
                }
            }
            if (!progressed) {
                fprintf(stderr, "emu: threads wait on each other without progress\n");
                abort();
            }
        }
        for (unsigned t = 0; t < block; ++t) free(blk.th[t].stack);
        B = nullptr;
    }
}

void syncthreads() {
    Thread &t = B->th[B->cur];
    t.st = BAR;
    emu_swap(&t.sp, B->sched_sp);
}

const dim3 &blockdim_hook() {
    if (B->sync_on_blockdim) {
        Thread &t = B->th[B->cur];
        t.st = WSYNC;
        emu_swap(&t.sp, B->sched_sp);
    }
    return B->bdim;
}

int all_sync(int pred) {
    Thread &t = B->th[B->cur];
    t.vote_in = pred;
    t.st = VOTE;
    emu_swap(&t.sp, B->sched_sp);
    return t.vote_out;
}

}  // namespace emu

namespace {

struct RefGpu {
    int nbodies, nedges, nnodes, tree_threads;
    bool strong_gravity;
    float k_g, k_r, itolsq, epssq;
    std::vector<float> body_mass, node_mass, fx, fy, fxp, fyp;
    std::vector<float2> body_pos, node_pos;
    std::vector<int> sources, targets, child, count, start, sortv;
    std::vector<float> minx, miny, maxx, maxy, swg, etra;
};

}  // namespace

extern "C" {

/* The CUDAForceAtlas2 constructor's host setup (src/RPGPUForceAtlas2.cu:37-162)
 * for a B200 (148 SMs, 1024 threads per block); resets the kernels'
 * file-static state (RPBHKernels.cu:58-62, RPFA2Kernels.cu:29-33). */
void *refgpu_create(int nbodies, int nedges, const float *xy, const float *mass,
                    const int *sources, const int *targets, int strong_gravity, float k_g,
                    float k_r, int tree_threads) {
    RefGpu *g = new RefGpu();
    g->nbodies = nbodies;
    g->nedges = nedges;
    g->strong_gravity = strong_gravity != 0;
    g->k_g = k_g;
    g->k_r = k_r;
    g->tree_threads = tree_threads > 0 ? tree_threads : 1;
    g->itolsq = 1.0f / (1.0f * 1.0f);  // RPForceAtlas2.cpp:45-47 (theta = 1)
    g->epssq = 0.05 * 0.05;
    const int mp_count = 148, max_threads_per_block = 1024;
    int nnodes = std::max(2 * nbodies, mp_count * max_threads_per_block);
    while ((nnodes & (WARPSIZE - 1)) != 0) nnodes++;
    nnodes--;
    g->nnodes = nnodes;
    g->child.assign((size_t)(nnodes + 1) * 4, -1);
    g->body_mass.assign(mass, mass + nbodies);
    g->node_mass.assign(nnodes + 1, 0.0f);
    g->body_pos.resize(nbodies);
    for (int i = 0; i < nbodies; ++i) g->body_pos[i] = {xy[2 * i], xy[2 * i + 1]};
    g->node_pos.assign(nnodes + 1, {0.0f, 0.0f});
    g->count.assign(nnodes + 1, 0);
    g->start.assign(nnodes + 1, 0);
    g->sortv.assign(nnodes + 1, 0);
    g->sources.assign(sources, sources + nedges);
    g->targets.assign(targets, targets + nedges);
    g->fx.assign(nbodies, 0.0f);
    g->fy.assign(nbodies, 0.0f);
    g->fxp.assign(nbodies, 0.0f);
    g->fyp.assign(nbodies, 0.0f);
    g->minx.assign(mp_count * FACTOR1, 0.0f);
    g->miny = g->maxx = g->maxy = g->swg = g->etra = g->minx;
    stepd = -1;
    maxdepthd = 1;
    blkcntd = 0;
    radiusd = 0.0f;
    bottomd = 0;
    global_speedd = 1.0;
    speed_efficiencyd = 1.0;
    jitter_toleranced = 1.0;
    k_s_maxd = 10.0;
    blkcntd_speed_kernel = 0;
    return g;
}

void refgpu_destroy(void *h) { delete (RefGpu *)h; }

/* One doStep (src/RPGPUForceAtlas2.cu:206-248).  Optional outputs:
 * f_ga (2n, after gravity + attraction), f_tot (2n, after the force kernel),
 * sort (n, sortd). */
void refgpu_step(void *h, float *f_ga, float *f_tot, int *sort_out) {
    RefGpu *g = (RefGpu *)h;
    int nb = g->nbodies, nn = g->nnodes, ne = g->nedges;
    float *body_mass = g->body_mass.data(), *node_mass = g->node_mass.data();
    float2 *body_pos = g->body_pos.data(), *node_pos = g->node_pos.data();
    float *fx = g->fx.data(), *fy = g->fy.data(), *fxp = g->fxp.data(), *fyp = g->fyp.data();
    int *child = g->child.data(), *count = g->count.data(), *start = g->start.data();
    int *sortd = g->sortv.data(), *src = g->sources.data(), *dst = g->targets.data();
    float *minx = g->minx.data(), *miny = g->miny.data(), *maxx = g->maxx.data(),
          *maxy = g->maxy.data(), *swg = g->swg.data(), *etra = g->etra.data();
    float k_g = g->k_g, k_r = g->k_r, itolsq = g->itolsq, epssq = g->epssq;
    bool sg = g->strong_gravity;

    emu::launch(1, 1, [=] { GravityKernel(nb, k_g, sg, body_mass, body_pos, fx, fy); });
    emu::launch(1, 1, [=] { AttractiveForceKernel(ne, body_pos, fx, fy, src, dst); });
    if (f_ga)
        for (int i = 0; i < nb; ++i) {
            f_ga[2 * i] = fx[i];
            f_ga[2 * i + 1] = fy[i];
        }
    emu::launch(1, THREADS1, [=] {
        BoundingBoxKernel(nn, nb, start, child, node_mass, body_pos, node_pos, maxx, maxy, minx, miny);
    });
    emu::launch(1, 1, [=] { ClearKernel1(nn, nb, child); });
    emu::launch(1, g->tree_threads, [=] { TreeBuildingKernel(nn, nb, child, body_pos, node_pos); });
    emu::launch(1, 32, [=] { ClearKernel2(nn, start, node_mass); });
    emu::launch(1, 32, [=] {
        SummarizationKernel(nn, nb, count, child, body_mass, node_mass, body_pos, node_pos);
    });
    emu::launch(1, 1, [=] { SortKernel(nn, nb, sortd, count, start, child); });
    emu::launch(1, THREADS5, [=] {
        ForceCalculationKernel(nn, nb, itolsq, epssq, sortd, child, body_mass, node_mass, body_pos,
                               node_pos, fx, fy, k_r);
    }, /*sync_on_blockdim=*/true);
    if (f_tot)
        for (int i = 0; i < nb; ++i) {
            f_tot[2 * i] = fx[i];
            f_tot[2 * i + 1] = fy[i];
        }
    if (sort_out) memcpy(sort_out, sortd, sizeof(int) * nb);
    emu::launch(1, THREADS1, [=] { SpeedKernel(nb, fx, fy, fxp, fyp, body_mass, swg, etra); });
    emu::launch(1, 1, [=] { DisplacementKernel(nb, body_pos, fx, fy, fxp, fyp); });
}

void refgpu_get_positions(void *h, float *xy) {
    RefGpu *g = (RefGpu *)h;
    for (int i = 0; i < g->nbodies; ++i) {
        xy[2 * i] = g->body_pos[i].x;
        xy[2 * i + 1] = g->body_pos[i].y;
    }
}

void refgpu_set_positions(void *h, const float *xy) {
    RefGpu *g = (RefGpu *)h;
    for (int i = 0; i < g->nbodies; ++i) g->body_pos[i] = {xy[2 * i], xy[2 * i + 1]};
}

float refgpu_global_speed(void) { return global_speedd; }
float refgpu_speed_efficiency(void) { return speed_efficiencyd; }
int refgpu_maxdepth(void) { return maxdepthd; }
float refgpu_radius(void) { return radiusd; }
int refgpu_bottom(void) { return bottomd; }
int refgpu_nnodes(void *h) { return ((RefGpu *)h)->nnodes; }

/* Cell data after the last step, for cells [bottom, nnodes]: mass, centre and
 * body count (SummarizationKernel output).  Returns the number of cells. */
int refgpu_cells(void *h, float *mass, float *cx, float *cy, int *count) {
    RefGpu *g = (RefGpu *)h;
    int nc = 0;
    for (int k = bottomd; k <= g->nnodes; ++k, ++nc) {
        if (mass) mass[nc] = g->node_mass[k];
        if (cx) cx[nc] = g->node_pos[k].x;
        if (cy) cy[nc] = g->node_pos[k].y;
        if (count) count[nc] = g->count[k];
    }
    return nc;
}

}  // extern "C"
