/*
 * RPGPUForceAtlas2.hpp -- the GPU ForceAtlas2 (drop-in for the reference's
 * src/RPGPUForceAtlas2.hpp:30-68).  Same constructor, doStep() and
 * sync_layout(); underneath it drives the B200 engine through the C ABI of
 * fa2b200.h.  As in the reference, a CUDA failure prints a message and exits
 * the process (src/RPCommon.hpp:33-41); Barnes-Hut is required
 * (src/graph_viewer.cpp:93-97).
 */
#ifndef RPGPUForceAtlas2_hpp
#define RPGPUForceAtlas2_hpp
#include "RPForceAtlas2.hpp"

struct fa2_ctx;

namespace RPGraph
{
    class CUDAForceAtlas2: public ForceAtlas2
    {
    public:
        CUDAForceAtlas2(GraphLayout &layout, bool use_barneshut,
                        bool strong_gravity, float gravity, float scale);
        ~CUDAForceAtlas2();
        void doStep() override;
        void sync_layout() override;

        // n iterations in one call, one device synchronisation at the end.
        void doStepsBatched(int n);

    private:
        fa2_ctx *ctx;
        float applied_k_r, applied_k_g;
        bool applied_linlog = false;
        void push_params();
        void sendLayoutToGPU();
        void retrieveLayoutFromGPU();
    };
};

#endif
