/*
 * RPGraphLayout.hpp -- 2-D positions of a UGraph's nodes (drop-in for the
 * reference's src/RPGraphLayout.hpp:31-67).  Writers produce the reference's
 * formats: CSV "id,x,y" and binary {uint32 id, float x, float y} per node, in
 * UGraph id order with edge-list ids.  writeToPNG renders the reference's
 * picture (node discs and edge lines blended black on white) on the GPU and
 * writes it with this library's own PNG encoder (fa2_render_rgb,
 * fa2_png_encode in fa2b200.h): pngwriter and libpng are not used.
 */
#ifndef RPGraphLayout_hpp
#define RPGraphLayout_hpp

#include <string>
#include <vector>

#include "RPCommon.hpp"
#include "RPGraph.hpp"

namespace RPGraph
{
    class GraphLayout
    {
    private:
        std::vector<Coordinate> coordinates;

    protected:
        float width, height;
        float minX(), minY(), maxX(), maxY();

    public:
        GraphLayout(RPGraph::UGraph &graph,
                    float width = 10000, float height = 10000);
        ~GraphLayout();

        UGraph &graph;

        // Uniform in [-width/2, width/2] x [-height/2, height/2] from libc
        // random(), x then y per node (reference src/RPGraphLayout.cpp:45-52).
        void randomizePositions();

        float getX(nid_t node_id), getY(nid_t node_id);
        float getXRange(), getYRange(), getSpan();
        float getDistance(nid_t n1, nid_t n2);
        Real2DVector getDistanceVector(nid_t n1, nid_t n2);
        Real2DVector getNormalizedDistanceVector(nid_t n1, nid_t n2);
        Coordinate getCoordinate(nid_t node_id);
        Coordinate getCenter();

        void setX(nid_t node_id, float x_value), setY(nid_t node_id, float y_value);
        void moveNode(nid_t, Real2DVector v);
        void setCoordinates(nid_t node_id, Coordinate c);
        void writeToPNG(const int image_w, const int image_h, std::string path);
        void writeToCSV(std::string path);
        void writeToBin(std::string path);

        // Interleaved x,y of all nodes (engine upload/download).
        float *data();
    };
}

#endif
