// RPCommon.cpp -- helpers of include/RPCommon.hpp.
#include "RPCommon.hpp"

#include <stdlib.h>
#include <sys/stat.h>

#include <cmath>
#include <vector>

bool is_file_exists(std::string filepath) {
    struct stat sb;
    return stat(filepath.c_str(), &sb) == 0;
}

// GNU basename: the text after the last '/' (empty for a trailing '/').
std::string basename(std::string filepath) {
    const size_t slash = filepath.rfind('/');
    return slash == std::string::npos ? filepath : filepath.substr(slash + 1);
}

namespace RPGraph
{
    float get_random(float lowerbound, float upperbound)
    {
        // float arithmetic in the reference's order (src/RPCommon.cpp:50-53)
        const float r = static_cast<float>(random());
        return lowerbound + (upperbound - lowerbound) * r / static_cast<float>(RAND_MAX);
    }

    Real2DVector::Real2DVector(float x, float y) : x(x), y(y) {}
    float Real2DVector::magnitude() { return std::sqrt(x * x + y * y); }
    float Real2DVector::distance(Real2DVector to)
    {
        // as the reference defines it (src/RPCommon.cpp:65-70)
        const float dx = (x - to.x) * (x - to.x);
        const float dy = (y - to.y) * (y - to.y);
        return std::sqrt(dx * dx + dy * dy);
    }
    Real2DVector Real2DVector::operator*(float b) { return Real2DVector(x * b, y * b); }
    Real2DVector Real2DVector::operator/(float b) { return Real2DVector(x / b, y / b); }
    Real2DVector Real2DVector::operator+(Real2DVector b) { return Real2DVector(x + b.x, y + b.y); }
    Real2DVector Real2DVector::operator-(Real2DVector b) { return Real2DVector(x - b.x, y - b.y); }
    void Real2DVector::operator+=(Real2DVector b) { x += b.x; y += b.y; }
    Real2DVector Real2DVector::getNormalized() { const float m = magnitude(); return Real2DVector(x / m, y / m); }
    Real2DVector Real2DVector::normalize()
    {
        const float m = magnitude();
        x /= m;
        y /= m;
        return *this;
    }

    Coordinate::Coordinate(float x, float y) : x(x), y(y) {}
    Coordinate Coordinate::operator+(float b) { return Coordinate(x + b, y + b); }
    Coordinate Coordinate::operator*(float b) { return Coordinate(x * b, y * b); }
    Coordinate Coordinate::operator/(float b) { return Coordinate(x / b, y / b); }
    Coordinate Coordinate::operator+(Real2DVector b) { return Coordinate(x + b.x, y + b.y); }
    Coordinate Coordinate::operator-(Coordinate b) { return Coordinate(x - b.x, y - b.y); }
    bool Coordinate::operator==(Coordinate b) { return x == b.x && y == b.y; }
    void Coordinate::operator/=(float b) { x /= b; y /= b; }
    void Coordinate::operator+=(Coordinate b) { x += b.x; y += b.y; }
    void Coordinate::operator+=(Real2DVector b) { x += b.x; y += b.y; }
    int Coordinate::quadrant()
    {
        // quadrants 0..3 clockwise from the upper left (src/RPCommon.cpp:175-188)
        if (x <= 0) return y >= 0 ? 0 : 3;
        return y >= 0 ? 1 : 2;
    }
    float Coordinate::distance(Coordinate to) { return RPGraph::distance(*this, to); }
    float Coordinate::distance2(Coordinate to) { return RPGraph::distance2(*this, to); }

    float distance(Coordinate from, Coordinate to) { return std::sqrt(distance2(from, to)); }
    float distance2(Coordinate from, Coordinate to)
    {
        const float dx = from.x - to.x, dy = from.y - to.y;
        return dx * dx + dy * dy;
    }
    Real2DVector normalizedDirection(Coordinate from, Coordinate to)
    {
        const float dx = from.x - to.x, dy = from.y - to.y;
        const float len = std::sqrt(dx * dx + dy * dy);
        return Real2DVector(dx / len, dy / len);
    }
    Real2DVector direction(Coordinate from, Coordinate to)
    {
        return Real2DVector(from.x - to.x, from.y - to.y);
    }
}
