// Graph loading shared by the drivers around the reference's library (oracle/ref_driver.cpp,
// oracle/adapter_check.cpp).  TEST INFRASTRUCTURE ONLY.
//
// edges.bin: int32 V, int64 n, int32 src[n], int32 dst[n].
#pragma once
#include <cstdio>
#include <vector>

#include "graph.hpp"
#include "utils.hpp"

inline bool read_edges(const char* path, int& V, std::vector<int>& src, std::vector<int>& dst) {
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    int64_t n = 0;
    bool ok = fread(&V, 4, 1, f) == 1 && fread(&n, 8, 1, f) == 1;
    src.resize(n);
    dst.resize(n);
    ok = ok && fread(src.data(), 4, n, f) == (size_t)n && fread(dst.data(), 4, n, f) == (size_t)n;
    fclose(f);
    return ok;
}

// Graph(out_neighbors, in_neighbors, V, E, self_edges) as the reference's tests build it
// (test/toy_example.hpp), E counted like Graph::load_text (src/graph.cpp:132-135).
inline Graph make_graph(int V, const std::vector<int>& src, const std::vector<int>& dst) {
    NeighborList out_neighbors, in_neighbors;
    std::vector<bool> self_edges(V, false);
    for (size_t i = 0; i < src.size(); ++i) {
        utils::insert_nodup(out_neighbors, src[i], dst[i]);
        utils::insert_nodup(in_neighbors, dst[i], src[i]);
        if (src[i] == dst[i]) self_edges[src[i]] = true;
    }
    while ((int)out_neighbors.size() < V) out_neighbors.push_back(std::vector<int>());
    while ((int)in_neighbors.size() < V) in_neighbors.push_back(std::vector<int>());
    int E = 0;
    for (const auto& nb : out_neighbors) E += (int)nb.size();
    Graph g(out_neighbors, in_neighbors, V, E, self_edges);
#ifdef SBP_REPLAY_H
    // the replay build logs the degree split the hybrid schedule will use
    sbp_replay::on_split(g.high_degree_vertices(), g.low_degree_vertices());
#endif
    return g;
}

