// fa2_host_capi.cpp -- the host graph layer of include/fa2b200.h: UGraph and
// GraphLayout behind plain C, for FFI callers (ctypes, cgo, JNI).
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "RPGraphLayout.hpp"
#include "fa2b200.h"

struct fa2_ugraph {
    RPGraph::UGraph *g;
};

extern "C" {

fa2_ugraph *fa2_ugraph_load(const char *path, int *status) {
    int dummy;
    if (!status) status = &dummy;
    if (!path || !is_file_exists(path)) {
        *status = FA2_ERR_IO;
        return nullptr;
    }
    fa2_ugraph *h = new fa2_ugraph{new RPGraph::UGraph(std::string(path))};
    *status = FA2_OK;
    return h;
}

fa2_ugraph *fa2_ugraph_from_pairs(const uint32_t *s, const uint32_t *t, uint64_t n_pairs,
                                  int *status) {
    int dummy;
    if (!status) status = &dummy;
    if (n_pairs && (!s || !t)) {
        *status = FA2_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    std::vector<RPGraph::nid_t> src(s, s + n_pairs), dst(t, t + n_pairs);
    fa2_ugraph *h = new fa2_ugraph{new RPGraph::UGraph(src, dst)};
    *status = FA2_OK;
    return h;
}

void fa2_ugraph_free(fa2_ugraph *h) {
    if (!h) return;
    delete h->g;
    delete h;
}

uint32_t fa2_ugraph_num_nodes(const fa2_ugraph *h) { return h ? h->g->num_nodes() : 0; }
uint64_t fa2_ugraph_num_edges(const fa2_ugraph *h) { return h ? h->g->num_edges() : 0; }

int fa2_ugraph_node_map_r(const fa2_ugraph *h, uint32_t *out) {
    if (!h || (!out && h->g->num_nodes())) return FA2_ERR_INVALID_ARGUMENT;
    for (RPGraph::nid_t n = 0; n < h->g->num_nodes(); ++n) out[n] = h->g->original_id(n);
    return FA2_OK;
}

int fa2_ugraph_degrees(const fa2_ugraph *h, uint32_t *out) {
    if (!h || (!out && h->g->num_nodes())) return FA2_ERR_INVALID_ARGUMENT;
    for (RPGraph::nid_t n = 0; n < h->g->num_nodes(); ++n) out[n] = h->g->degree(n);
    return FA2_OK;
}

int fa2_ugraph_edges(const fa2_ugraph *h, uint32_t *sources, uint32_t *targets) {
    if (!h || ((!sources || !targets) && h->g->num_edges())) return FA2_ERR_INVALID_ARGUMENT;
    std::vector<RPGraph::nid_t> s, t;
    h->g->edges(s, t);
    for (size_t e = 0; e < s.size(); ++e) {
        sources[e] = s[e];
        targets[e] = t[e];
    }
    return FA2_OK;
}

void fa2_random_positions(uint32_t n, float width, float height, uint32_t seed, float *xy) {
    if (!xy) return;
    srandom(seed);
    for (uint32_t i = 0; i < n; ++i) {
        xy[2 * i] = RPGraph::get_random(-width / 2.0, width / 2.0);
        xy[2 * i + 1] = RPGraph::get_random(-height / 2.0, height / 2.0);
    }
}

int fa2_write_layout(const fa2_ugraph *h, const float *xy, const char *path, int binary) {
    if (!h || !path || (!xy && h->g->num_nodes())) return FA2_ERR_INVALID_ARGUMENT;
    if (is_file_exists(path)) return FA2_ERR_IO;
    RPGraph::GraphLayout layout(*h->g);
    for (RPGraph::nid_t n = 0; n < h->g->num_nodes(); ++n) {
        layout.setX(n, xy[2 * n]);
        layout.setY(n, xy[2 * n + 1]);
    }
    if (binary)
        layout.writeToBin(path);
    else
        layout.writeToCSV(path);
    return is_file_exists(path) ? FA2_OK : FA2_ERR_IO;
}

int fa2_write_png(const fa2_ugraph *h, const float *xy, int32_t image_w, int32_t image_h,
                  const char *path) {
    if (!h || !path || (!xy && h->g->num_nodes())) return FA2_ERR_INVALID_ARGUMENT;
    std::vector<RPGraph::nid_t> s, t;
    h->g->edges(s, t);
    std::vector<uint32_t> su(s.begin(), s.end()), tu(t.begin(), t.end());
    std::vector<uint8_t> rgb((size_t)std::max(image_w, 0) * (size_t)std::max(image_h, 0) * 3);
    int st = fa2_render_rgb(h->g->num_nodes(), su.size(), su.data(), tu.data(), xy, image_w,
                            image_h, 0, rgb.data());
    if (st) return st;
    return fa2_png_encode(rgb.data(), image_w, image_h, path);
}

}  // extern "C"
