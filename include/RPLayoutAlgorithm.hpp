/*
 * RPLayoutAlgorithm.hpp -- base of layout algorithms (drop-in for the
 * reference's src/RPLayoutAlgorithm.hpp:31-39).
 */
#ifndef RPLayoutAlgorithm_hpp
#define RPLayoutAlgorithm_hpp

#include "RPGraphLayout.hpp"

namespace RPGraph
{
    class LayoutAlgorithm
    {
    public:
        LayoutAlgorithm(GraphLayout &layout);
        virtual ~LayoutAlgorithm();
        GraphLayout &layout;

        virtual void sync_layout() = 0; // write current layout to `layout'.
    };
}

#endif
