/*
 * RPCPUForceAtlas2.hpp -- the reference's CPU layout class name (src/
 * RPCPUForceAtlas2.hpp:31-55), declared so that code written against the
 * reference interface compiles unchanged.  This engine provides the GPU path
 * only: constructing a CPUForceAtlas2 prints an error and exits, as the
 * reference's CLI does for an unavailable backend (src/graph_viewer.cpp:112-118).
 */
#ifndef RPCPUForceAtlas2_hpp
#define RPCPUForceAtlas2_hpp

#include "RPForceAtlas2.hpp"

namespace RPGraph
{
    class CPUForceAtlas2 : public ForceAtlas2
    {
    public:
        CPUForceAtlas2(GraphLayout &layout, bool use_barneshut,
                       bool strong_gravity, float gravity, float scale);
        ~CPUForceAtlas2();
        void doStep() override;
        void sync_layout() override;
    };
}
#endif
