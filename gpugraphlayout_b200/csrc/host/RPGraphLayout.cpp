// RPGraphLayout.cpp -- include/RPGraphLayout.hpp.
#include "RPGraphLayout.hpp"
#include "fa2b200.h"

#include <stdio.h>
#include <stdlib.h>

#include <cmath>
#include <algorithm>
#include <fstream>
#include <limits>

namespace RPGraph
{
    GraphLayout::GraphLayout(UGraph &graph, float width, float height)
        : coordinates(graph.num_nodes(), Coordinate(0.0f, 0.0f)), width(width), height(height),
          graph(graph)
    {
    }

    GraphLayout::~GraphLayout() {}

    void GraphLayout::randomizePositions()
    {
        // bounds are double expressions passed to float parameters, x then y
        // per node (src/RPGraphLayout.cpp:45-52)
        for (nid_t i = 0; i < graph.num_nodes(); ++i) {
            setX(i, get_random(-width / 2.0, width / 2.0));
            setY(i, get_random(-height / 2.0, height / 2.0));
        }
    }

    float GraphLayout::getX(nid_t node_id) { return coordinates[node_id].x; }
    float GraphLayout::getY(nid_t node_id) { return coordinates[node_id].y; }

    // The extrema start from numeric_limits<float>::max() and ::min() (the
    // smallest positive float), as in src/RPGraphLayout.cpp:64-104.
    float GraphLayout::minX()
    {
        float v = std::numeric_limits<float>::max();
        for (const Coordinate &c : coordinates) if (c.x < v) v = c.x;
        return v;
    }
    float GraphLayout::maxX()
    {
        float v = std::numeric_limits<float>::min();
        for (const Coordinate &c : coordinates) if (c.x > v) v = c.x;
        return v;
    }
    float GraphLayout::minY()
    {
        float v = std::numeric_limits<float>::max();
        for (const Coordinate &c : coordinates) if (c.y < v) v = c.y;
        return v;
    }
    float GraphLayout::maxY()
    {
        float v = std::numeric_limits<float>::min();
        for (const Coordinate &c : coordinates) if (c.y > v) v = c.y;
        return v;
    }

    float GraphLayout::getXRange() { return maxX() - minX(); }
    float GraphLayout::getYRange() { return maxY() - minY(); }
    float GraphLayout::getSpan() { return ceil(fmaxf(getXRange(), getYRange())); }

    float GraphLayout::getDistance(nid_t n1, nid_t n2)
    {
        const float dx = getX(n1) - getX(n2), dy = getY(n1) - getY(n2);
        return std::sqrt(dx * dx + dy * dy);
    }

    Real2DVector GraphLayout::getDistanceVector(nid_t n1, nid_t n2)
    {
        return Real2DVector(getX(n2) - getX(n1), getY(n2) - getY(n1));
    }

    Real2DVector GraphLayout::getNormalizedDistanceVector(nid_t n1, nid_t n2)
    {
        const float dx = getX(n2) - getX(n1), dy = getY(n2) - getY(n1);
        const float len = std::sqrt(dx * dx + dy * dy);
        return Real2DVector(dx / len, dy / len);
    }

    Coordinate GraphLayout::getCoordinate(nid_t node_id) { return coordinates[node_id]; }

    Coordinate GraphLayout::getCenter()
    {
        float x = minX() + getXRange() / 2.0;
        float y = minY() + getYRange() / 2.0;
        return Coordinate(x, y);
    }

    void GraphLayout::setX(nid_t node_id, float x_value) { coordinates[node_id].x = x_value; }
    void GraphLayout::setY(nid_t node_id, float y_value) { coordinates[node_id].y = y_value; }

    void GraphLayout::moveNode(nid_t n, Real2DVector v)
    {
        setX(n, getX(n) + v.x);
        setY(n, getY(n) + v.y);
    }

    void GraphLayout::setCoordinates(nid_t node_id, Coordinate c)
    {
        setX(node_id, c.x);
        setY(node_id, c.y);
    }

    // src/RPGraphLayout.cpp:170-207: rendered on the GPU (fa2_render_rgb) and
    // written by this library's PNG encoder; errors print and exit, as the
    // reference's library calls do.
    void GraphLayout::writeToPNG(const int image_w, const int image_h, std::string path)
    {
        std::vector<nid_t> s, t;
        graph.edges(s, t);
        std::vector<uint32_t> su(s.begin(), s.end()), tu(t.begin(), t.end());
        std::vector<uint8_t> rgb((size_t)std::max(image_w, 0) * (size_t)std::max(image_h, 0) * 3);
        int st = fa2_render_rgb(graph.num_nodes(), su.size(), su.data(), tu.data(), data(),
                                image_w, image_h, 0, rgb.data());
        if (st == FA2_OK) st = fa2_png_encode(rgb.data(), image_w, image_h, path.c_str());
        if (st != FA2_OK)
        {
            fprintf(stderr, "error: writing %s: %s\n", path.c_str(), fa2_status_string(st));
            exit(EXIT_FAILURE);
        }
    }

    void GraphLayout::writeToCSV(std::string path)
    {
        if (is_file_exists(path)) {  // src/RPGraphLayout.cpp:211-215
            printf("Error: File exists at %s\n", path.c_str());
            exit(EXIT_FAILURE);
        }
        std::ofstream out_file(path);
        for (nid_t n = 0; n < graph.num_nodes(); ++n)
            out_file << graph.original_id(n) << "," << getX(n) << "," << getY(n) << "\n";
    }

    void GraphLayout::writeToBin(std::string path)
    {
        if (is_file_exists(path)) {
            printf("Error: File exists at %s\n", path.c_str());
            exit(EXIT_FAILURE);
        }
        std::ofstream out_file(path, std::ofstream::binary);
        for (nid_t n = 0; n < graph.num_nodes(); ++n) {
            const nid_t id = graph.original_id(n);
            const float x = getX(n), y = getY(n);
            out_file.write(reinterpret_cast<const char *>(&id), sizeof(id));
            out_file.write(reinterpret_cast<const char *>(&x), sizeof(x));
            out_file.write(reinterpret_cast<const char *>(&y), sizeof(y));
        }
    }

    float *GraphLayout::data() { return reinterpret_cast<float *>(coordinates.data()); }
}
