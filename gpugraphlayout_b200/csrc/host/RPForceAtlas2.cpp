// RPForceAtlas2.cpp -- include/RPLayoutAlgorithm.hpp, RPForceAtlas2.hpp and
// RPGPUForceAtlas2.hpp.  The GPU class is a shim over the C ABI (fa2b200.h).
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "RPCPUForceAtlas2.hpp"
#include "RPGPUForceAtlas2.hpp"
#include "fa2b200.h"

namespace RPGraph
{
    LayoutAlgorithm::LayoutAlgorithm(GraphLayout &layout) : layout(layout) {}
    LayoutAlgorithm::~LayoutAlgorithm() {}

    // Parameter defaults of src/RPForceAtlas2.cpp:28-55.
    ForceAtlas2::ForceAtlas2(GraphLayout &layout, bool use_barneshut, bool strong_gravity,
                             float gravity, float scale)
        : LayoutAlgorithm(layout), use_barneshut{use_barneshut}, strong_gravity{strong_gravity}
    {
        iteration = 0;
        setGravity(gravity);
        setScale(scale);
        global_speed = 1.0;
        speed_efficiency = 1.0;
        jitter_tolerance = 1.0;
        k_s = 0.1;
        k_s_max = 10.0;
        theta = 1.0;
        epssq = 0.05 * 0.05;
        itolsq = 1.0f / (theta * theta);
        delta = 0.0;
        prevent_overlap = false;
        use_linlog = false;
        layout.randomizePositions();
    }

    ForceAtlas2::~ForceAtlas2() {}

    void ForceAtlas2::doSteps(int n)
    {
        for (int i = 0; i < n; ++i) doStep();
    }

    void ForceAtlas2::setScale(float s) { k_r = s; }
    void ForceAtlas2::setGravity(float g) { k_g = g; }
    float ForceAtlas2::mass(nid_t n) { return layout.graph.degree(n) + 1.0; }

    namespace
    {
        // The reference's cudaCatchError: report and exit (src/RPCommon.hpp:33-41).
        void check(int status, const char *what)
        {
            if (status == FA2_OK) return;
            fprintf(stderr, "error: %s: %s (status %d)\n", what, fa2_status_string(status), status);
            exit(EXIT_FAILURE);
        }
    }

    CUDAForceAtlas2::CUDAForceAtlas2(GraphLayout &layout, bool use_barneshut, bool strong_gravity,
                                     float gravity, float scale)
        : ForceAtlas2(layout, use_barneshut, strong_gravity, gravity, scale), ctx(nullptr)
    {
        std::vector<nid_t> sources, targets;
        layout.graph.edges(sources, targets);
        fa2_graph_desc g;
        g.num_nodes = layout.graph.num_nodes();
        g.num_edges = sources.size();
        g.sources = sources.data();
        g.targets = targets.data();
        g.weights = nullptr;  // UGraph has no edge weights
        fa2_params p;
        fa2_default_params(&p);
        // The reference's GPU step is Barnes-Hut whatever use_barneshut says
        // (src/RPGPUForceAtlas2.cu:206-248); the CLI refuses exact mode earlier.
        p.use_barneshut = 1;
        p.strong_gravity = strong_gravity ? 1 : 0;
        p.gravity = k_g;
        p.scale = k_r;
        p.theta = theta;
        p.epssq = epssq;
        p.jitter_tolerance = jitter_tolerance;
        p.k_s_max = k_s_max;
        p.delta = delta;
        int status = FA2_OK;
        ctx = fa2_create(&g, &p, &status);
        if (status == FA2_ERR_NO_DEVICE) {
            fprintf(stderr, "error: No CUDA devices found.\n");  // src/RPGPUForceAtlas2.cu:44-48
            exit(EXIT_FAILURE);
        }
        check(status, "creating the GPU layout");
        applied_k_r = k_r;
        applied_k_g = k_g;
        sendLayoutToGPU();
    }

    CUDAForceAtlas2::~CUDAForceAtlas2() { fa2_destroy(ctx); }

    void CUDAForceAtlas2::push_params()
    {
        // use_linlog is public in ForceAtlas2; the reference's GPU path
        // ignores it, this engine honours it (linear-log attraction)
        if (use_linlog != applied_linlog)
        {
            check(fa2_set_linlog(ctx, use_linlog ? 1 : 0), "setting linlog");
            applied_linlog = use_linlog;
        }
        if (k_r == applied_k_r && k_g == applied_k_g) return;
        check(fa2_set_force_params(ctx, k_r, k_g), "setting scale/gravity");
        applied_k_r = k_r;
        applied_k_g = k_g;
    }

    void CUDAForceAtlas2::doStep()
    {
        push_params();
        check(fa2_step(ctx, 1), "doStep");
        iteration++;
    }

    void CUDAForceAtlas2::doStepsBatched(int n)
    {
        push_params();
        check(fa2_step(ctx, n), "doStep");
        iteration += n;
    }

    void CUDAForceAtlas2::sendLayoutToGPU()
    {
        check(fa2_set_positions(ctx, layout.data()), "sending the layout");
    }

    void CUDAForceAtlas2::retrieveLayoutFromGPU()
    {
        check(fa2_get_positions(ctx, layout.data()), "retrieving the layout");
    }

    void CUDAForceAtlas2::sync_layout() { retrieveLayoutFromGPU(); }

    CPUForceAtlas2::CPUForceAtlas2(GraphLayout &layout, bool use_barneshut, bool strong_gravity,
                                   float gravity, float scale)
        : ForceAtlas2(layout, use_barneshut, strong_gravity, gravity, scale)
    {
        fprintf(stderr, "error: this build provides the GPU (CUDAForceAtlas2) path only.\n");
        exit(EXIT_FAILURE);
    }
    CPUForceAtlas2::~CPUForceAtlas2() {}
    void CPUForceAtlas2::doStep() {}
    void CPUForceAtlas2::sync_layout() {}
}
