// RPGraph.cpp -- O(E) edge-list loader behind include/RPGraph.hpp.
//
// Results equal the reference's UGraph (src/RPGraph.cpp:35-131): ids by first
// appearance (s before t), self-loops and repeated undirected edges dropped,
// neighbors_with_geq_id in file order.  Where the reference looks an edge up
// by copying and scanning a neighbour list per line, this loader keeps an
// open-addressing hash set of (min, max) pairs.
#include "RPGraph.hpp"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <memory>

namespace
{
    // Open-addressing hash map uint64 -> uint32, linear probing, never shrinks.
    class HashMap
    {
    public:
        explicit HashMap(uint64_t expected)
        {
            uint64_t cap = 1024;
            while (cap < expected * 2) cap <<= 1;
            keys_.assign(cap, kEmpty);
            vals_.resize(cap);
            mask_ = cap - 1;
        }
        // Inserts key -> val if absent; returns the stored value and whether it
        // was inserted.
        uint32_t insert(uint64_t key, uint32_t val, bool *inserted)
        {
            if ((count_ + 1) * 2 > keys_.size()) grow();
            uint64_t h = mix(key) & mask_;
            for (;;) {
                if (keys_[h] == key) {
                    *inserted = false;
                    return vals_[h];
                }
                if (keys_[h] == kEmpty) {
                    keys_[h] = key;
                    vals_[h] = val;
                    ++count_;
                    *inserted = true;
                    return val;
                }
                h = (h + 1) & mask_;
            }
        }

    private:
        static constexpr uint64_t kEmpty = ~0ull;
        std::vector<uint64_t> keys_;
        std::vector<uint32_t> vals_;
        uint64_t mask_ = 0, count_ = 0;

        static uint64_t mix(uint64_t k)
        {
            k ^= k >> 31;
            k *= 0x7fb5d329728ea185ull;
            k ^= k >> 27;
            k *= 0x81dadef4bc2dd44dull;
            k ^= k >> 33;
            return k;
        }
        void grow()
        {
            std::vector<uint64_t> ok;
            std::vector<uint32_t> ov;
            ok.swap(keys_);
            ov.swap(vals_);
            keys_.assign(ok.size() * 2, kEmpty);
            vals_.resize(ok.size() * 2);
            mask_ = keys_.size() - 1;
            count_ = 0;
            for (size_t i = 0; i < ok.size(); ++i) {
                if (ok[i] == kEmpty) continue;
                bool ins;
                insert(ok[i], ov[i], &ins);
            }
        }
    };

    inline bool is_space(char c)
    {
        return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
    }

    // Unsigned decimal after optional blanks, as `istream >> uint32_t` reads
    // it; false if there is none or it does not fit.
    inline bool parse_u32(const char *&p, const char *end, uint32_t &out)
    {
        while (p < end && is_space(*p)) ++p;
        if (p < end && *p == '+') ++p;
        if (p >= end || *p < '0' || *p > '9') return false;
        uint64_t v = 0;
        while (p < end && *p >= '0' && *p <= '9') {
            v = v * 10 + (uint64_t)(*p - '0');
            if (v > 0xffffffffull) return false;
            ++p;
        }
        out = (uint32_t)v;
        return true;
    }
}

namespace RPGraph
{
    UGraph::UGraph(std::string edgelist_path) : node_count(0), edge_count(0)
    {
        std::vector<nid_t> src, dst;
        FILE *f = fopen(edgelist_path.c_str(), "rb");
        if (f) {
            const size_t kChunk = 1 << 24;
            std::unique_ptr<char[]> buf(new char[kChunk + 1]);
            std::string carry;
            size_t got;
            auto parse_line = [&](const char *p, const char *end) {
                if (p < end && *p == '#') return;  // src/RPGraph.cpp:46
                uint32_t s, t;
                if (parse_u32(p, end, s) && parse_u32(p, end, t)) {
                    src.push_back(s);
                    dst.push_back(t);
                }
            };
            while ((got = fread(buf.get(), 1, kChunk, f)) > 0) {
                const char *p = buf.get(), *end = buf.get() + got;
                const char *nl = (const char *)memchr(p, '\n', end - p);
                if (!carry.empty()) {
                    if (!nl) {
                        carry.append(p, end);
                        continue;
                    }
                    carry.append(p, nl);
                    parse_line(carry.data(), carry.data() + carry.size());
                    carry.clear();
                    p = nl + 1;
                }
                while (p < end) {
                    nl = (const char *)memchr(p, '\n', end - p);
                    if (!nl) {
                        carry.assign(p, end);
                        break;
                    }
                    parse_line(p, nl);
                    p = nl + 1;
                }
            }
            if (!carry.empty()) parse_line(carry.data(), carry.data() + carry.size());
            fclose(f);
        }
        build(src, dst);
    }

    UGraph::UGraph(const std::vector<nid_t> &src, const std::vector<nid_t> &dst)
        : node_count(0), edge_count(0)
    {
        build(src, dst);
    }

    void UGraph::build(const std::vector<nid_t> &src, const std::vector<nid_t> &dst)
    {
        const size_t n_pairs = src.size() < dst.size() ? src.size() : dst.size();
        HashMap nodes(n_pairs / 4 + 16), edges(n_pairs + 16);
        std::vector<nid_t> map_r;
        std::vector<nid_t> lo, hi;
        lo.reserve(n_pairs);
        hi.reserve(n_pairs);
        for (size_t e = 0; e < n_pairs; ++e) {
            const nid_t s = src[e], t = dst[e];
            if (s == t) continue;  // src/RPGraph.cpp:52
            bool ins;
            const nid_t sm = nodes.insert(s, (uint32_t)map_r.size(), &ins);
            if (ins) map_r.push_back(s);
            const nid_t tm = nodes.insert(t, (uint32_t)map_r.size(), &ins);
            if (ins) map_r.push_back(t);
            const nid_t a = sm < tm ? sm : tm, b = sm < tm ? tm : sm;
            edges.insert(((uint64_t)a << 32) | b, 0, &ins);
            if (!ins) continue;
            lo.push_back(a);
            hi.push_back(b);
        }
        node_count = (nid_t)map_r.size();
        edge_count = (nid_t)lo.size();
        degrees_.assign(node_count, 0);
        adj_off_.assign((size_t)node_count + 1, 0);
        for (size_t e = 0; e < lo.size(); ++e) {
            degrees_[lo[e]]++;
            degrees_[hi[e]]++;
            adj_off_[lo[e] + 1]++;
        }
        for (nid_t n = 0; n < node_count; ++n) adj_off_[n + 1] += adj_off_[n];
        adj_.resize(lo.size());
        std::vector<uint64_t> fill(adj_off_.begin(), adj_off_.end() - 1);
        for (size_t e = 0; e < lo.size(); ++e) adj_[fill[lo[e]]++] = hi[e];
        node_map.reserve(node_count);
        node_map_r.reserve(node_count);
        for (nid_t n = 0; n < node_count; ++n) {
            node_map[map_r[n]] = n;
            node_map_r[n] = map_r[n];
        }
    }

    nid_t UGraph::num_nodes() { return node_count; }
    nid_t UGraph::num_edges() { return edge_count; }
    nid_t UGraph::degree(nid_t nid) { return nid < node_count ? degrees_[nid] : 0; }
    nid_t UGraph::in_degree(nid_t nid) { return degree(nid); }
    nid_t UGraph::out_degree(nid_t nid) { return degree(nid); }

    std::vector<nid_t> UGraph::neighbors_with_geq_id(nid_t nid)
    {
        if (nid >= node_count) return std::vector<nid_t>();
        return std::vector<nid_t>(adj_.begin() + adj_off_[nid], adj_.begin() + adj_off_[nid + 1]);
    }

    nid_t UGraph::original_id(nid_t n) const
    {
        auto it = node_map_r.find(n);
        return it == node_map_r.end() ? 0 : it->second;
    }

    void UGraph::edges(std::vector<nid_t> &sources, std::vector<nid_t> &targets) const
    {
        sources.resize(adj_.size());
        targets.resize(adj_.size());
        for (nid_t n = 0; n < node_count; ++n)
            for (uint64_t q = adj_off_[n]; q < adj_off_[n + 1]; ++q) {
                sources[q] = n;
                targets[q] = adj_[q];
            }
    }
}
