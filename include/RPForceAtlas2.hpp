/*
 * RPForceAtlas2.hpp -- ForceAtlas2 parameters and stepping interface
 * (drop-in for the reference's src/RPForceAtlas2.hpp:32-60 and its
 * constructor defaults in src/RPForceAtlas2.cpp:28-55: theta 1, epssq 0.05^2,
 * k_s 0.1, k_s_max 10, speed/efficiency/jitter 1; the constructor randomizes
 * the layout's positions).
 */
#ifndef RPForceAtlas2_hpp
#define RPForceAtlas2_hpp

#include "RPLayoutAlgorithm.hpp"

namespace RPGraph
{
    class ForceAtlas2 : public LayoutAlgorithm
    {
        public:
            ForceAtlas2(GraphLayout &layout, bool use_barneshut,
                        bool strong_gravity, float gravity, float scale);
            virtual ~ForceAtlas2();

            virtual void doStep() = 0;
            void doSteps(int n);
            void setScale(float s);
            void setGravity(float s);
            float mass(nid_t n);
            bool prevent_overlap, use_barneshut, use_linlog, strong_gravity;

        protected:
            int iteration;
            float k_r, k_g;
            float delta;
            float global_speed;

            float speed_efficiency, jitter_tolerance;
            float k_s, k_s_max;

            float theta;
            float epssq;
            float itolsq;
    };
}
#endif
