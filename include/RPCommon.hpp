/*
 * RPCommon.hpp -- small helpers of the RPGraph interface (drop-in for the
 * reference's src/RPCommon.hpp): file checks, libc-random floats and the 2-D
 * vector/coordinate types used by GraphLayout.  Same names and signatures as
 * the reference so code written against it compiles unchanged.
 */
#ifndef RPCommonUtils_hpp
#define RPCommonUtils_hpp
#include <string>

bool is_file_exists(std::string filepath);
std::string basename(std::string filepath);

namespace RPGraph
{
    // lowerbound + (upperbound-lowerbound) * random()/RAND_MAX, in float
    // (reference src/RPCommon.cpp:50-53); seeded by srandom().
    float get_random(float lowerbound, float upperbound);

    class Real2DVector
    {
    public:
        Real2DVector(float x, float y);
        float x, y;
        float magnitude();
        float distance(Real2DVector to);

        Real2DVector operator*(float b);
        Real2DVector operator/(float b);
        Real2DVector operator+(Real2DVector b);
        Real2DVector operator-(Real2DVector b);
        void operator+=(Real2DVector b);

        Real2DVector getNormalized();
        Real2DVector normalize();
    };

    class Coordinate
    {
    public:
        float x, y;
        Coordinate(float x, float y);

        Coordinate operator+(float b);
        Coordinate operator*(float b);
        Coordinate operator/(float b);
        Coordinate operator+(Real2DVector b);
        Coordinate operator-(Coordinate b);
        bool operator==(Coordinate b);
        void operator/=(float b);
        void operator+=(Coordinate b);
        void operator+=(RPGraph::Real2DVector b);

        int quadrant();
        float distance(Coordinate to);
        float distance2(Coordinate to);
    };

    float distance(Coordinate from, Coordinate to);
    float distance2(Coordinate from, Coordinate to);

    Real2DVector normalizedDirection(Coordinate from, Coordinate to);
    Real2DVector direction(Coordinate from, Coordinate to);
}

#endif
