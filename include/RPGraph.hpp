/*
 * RPGraph.hpp -- undirected graph read from an edge list (drop-in for the
 * reference's src/RPGraph.hpp:31-81).
 *
 * Same public interface and results as the reference's UGraph: node ids are
 * assigned in order of first appearance in the file, self-loops and repeated
 * undirected edges are dropped, neighbors_with_geq_id(n) lists the larger
 * endpoints of n's edges in file order.  The loader is O(E) (hash set of
 * edges) where the reference's has_edge copies a neighbour list per line.
 */
#ifndef RPGraph_hpp
#define RPGraph_hpp
#include <stdint.h>

#include <string>
#include <unordered_map>
#include <vector>

namespace RPGraph
{
    typedef uint32_t nid_t;
    typedef uint32_t eid_t;

    class Graph
    {
        public:
            virtual ~Graph() {}
            virtual nid_t num_nodes() = 0;
            virtual nid_t num_edges() = 0;
            virtual nid_t degree(nid_t nid) = 0;
            virtual nid_t in_degree(nid_t nid) = 0;
            virtual nid_t out_degree(nid_t nid) = 0;
            virtual std::vector<nid_t> neighbors_with_geq_id(nid_t nid) = 0;
    };

    class UGraph : public Graph
    {
    private:
        nid_t node_count, edge_count;
        std::vector<nid_t> degrees_;       // per mapped id
        std::vector<uint64_t> adj_off_;    // CSR of neighbors_with_geq_id
        std::vector<nid_t> adj_;
        void build(const std::vector<nid_t> &src, const std::vector<nid_t> &dst);

    public:
        // Reads `edgelist_path`: one "s t" pair per line, lines starting with
        // '#' skipped.  Lines without two unsigned integers are skipped (the
        // reference leaves their ids uninitialised).  A file that cannot be
        // read gives an empty graph, as the reference's std::fstream does.
        UGraph(std::string edgelist_path);
        // The same graph from (s, t) pairs already in memory, in file order.
        UGraph(const std::vector<nid_t> &src, const std::vector<nid_t> &dst);

        std::unordered_map<nid_t, nid_t> node_map;   // edge-list id -> UGraph id
        std::unordered_map<nid_t, nid_t> node_map_r; // UGraph id -> edge-list id

        virtual nid_t num_nodes() override;
        virtual nid_t num_edges() override;
        virtual nid_t degree(nid_t nid) override;
        virtual nid_t in_degree(nid_t nid) override;
        virtual nid_t out_degree(nid_t nid) override;
        std::vector<nid_t> neighbors_with_geq_id(nid_t nid) override;

        // Fast access for the engine: edge-list id of UGraph id n, and the
        // COO of all edges in CUDAForceAtlas2's order (src/RPGPUForceAtlas2.cu:77-84).
        nid_t original_id(nid_t n) const;
        void edges(std::vector<nid_t> &sources, std::vector<nid_t> &targets) const;
    };
}

#endif
