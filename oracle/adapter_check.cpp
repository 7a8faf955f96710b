// Runs the reference-facing C++ adapter (include/sbp_b200_reference.hpp) from a program built
// against the reference's own headers and Graph / Blockmodel sources, as a maintainer of the
// reference would call it.  TEST INFRASTRUCTURE ONLY (tests/test_reference_adapter.py).
//
//   adapter_check <edges.bin> <assignment.bin> <out.bin> <seed>
//
// Steps, each through the adapter on the reference's own Blockmodel object:
//   gibbs  = finetune::asynchronous_gibbs from the given assignment
//   merge  = block_merge::merge_blocks down to half the blocks
//   hybrid = finetune::hybrid_mcmc
//   sbp    = sbp::stochastic_block_partition of the graph
// out.bin: int32 n_high, high[], n_low, low[] (the reference's degree split), then per step
// int32 B, V, b[V], d_out[B], d_in[B], d[B], M[B*B] (read through blockmatrix()->get), float64
// entropy::mdl.  Prints one JSON line; on an engine error prints {"error": ...} and exits 3.
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpi_data.hpp"
#include "ref_graph.hpp"
#include "sbp_b200_reference.hpp"

MPI_t mpi;
Args args;

static void put_ints(FILE* f, const std::vector<int>& v) {
    const int32_t n = (int32_t)v.size();
    fwrite(&n, 4, 1, f);
    if (n) fwrite(v.data(), 4, n, f);
}

static void dump(FILE* f, const Blockmodel& bm, const Graph& graph) {
    const int32_t B = bm.getNum_blocks(), V = graph.num_vertices();
    fwrite(&B, 4, 1, f);
    fwrite(&V, 4, 1, f);
    fwrite(bm.block_assignment().data(), 4, V, f);
    fwrite(bm.degrees_out().data(), 4, B, f);
    fwrite(bm.degrees_in().data(), 4, B, f);
    fwrite(bm.degrees().data(), 4, B, f);
    std::vector<int32_t> M((size_t)B * B);
    for (int r = 0; r < B; ++r)
        for (int c = 0; c < B; ++c) M[(size_t)r * B + c] = bm.blockmatrix()->get(r, c);
    fwrite(M.data(), 4, M.size(), f);
    const double mdl = sbp_b200::entropy::mdl(bm, graph.num_vertices(), graph.num_edges());
    fwrite(&mdl, 8, 1, f);
}

int main(int argc, char** argv) {
    if (argc < 5) return 2;
    mpi.rank = 0;
    mpi.num_processes = 1;
    args.transpose = true;
    args.undirected = false;
    args.nodelta = false;
    args.algorithm = "async_gibbs";
    args.batches = 10;
    args.approximate = true;
    args.asynciterations = std::numeric_limits<int>::max();
    args.threads = 1;
    int V;
    std::vector<int> src, dst;
    if (!read_edges(argv[1], V, src, dst)) return 2;
    FILE* fa = fopen(argv[2], "rb");
    int B = 0;
    std::vector<int> a(V);
    const bool ok = fa && fread(&B, 4, 1, fa) == 1 && fread(a.data(), 4, V, fa) == (size_t)V;
    if (fa) fclose(fa);
    if (!ok) return 2;
    const uint64_t seed = std::stoull(argv[4]);
    std::ostringstream sink;
    std::streambuf* saved = std::cout.rdbuf(sink.rdbuf());
    Graph graph = make_graph(V, src, dst);
    FILE* f = fopen(argv[3], "wb");
    if (!f) return 2;
    put_ints(f, graph.high_degree_vertices());
    put_ints(f, graph.low_degree_vertices());
    try {
        Blockmodel bm(B, graph, 0.5, a);
        BlockmodelTriplet triplet;
        sbp_b200::finetune::asynchronous_gibbs(bm, graph, triplet, seed);
        dump(f, bm, graph);
        bm.setNum_blocks_to_merge(bm.getNum_blocks() / 2);
        sbp_b200::block_merge::merge_blocks(bm, graph, graph.num_edges(), seed);
        dump(f, bm, graph);
        sbp_b200::finetune::hybrid_mcmc(bm, graph, triplet, seed);
        dump(f, bm, graph);
        Blockmodel part = sbp_b200::sbp::stochastic_block_partition(graph, args, seed);
        dump(f, part, graph);
        fclose(f);
        std::cout.rdbuf(saved);
        printf("{\"steps\": 4, \"final_blocks\": %d, \"mcmc_iterations\": %d}\n", part.getNum_blocks(),
               finetune::MCMC_iterations);
        return 0;
    } catch (const std::exception& e) {
        fclose(f);
        std::cout.rdbuf(saved);
        std::string msg = e.what();
        for (char& ch : msg)
            if (ch == '"' || ch == '\\') ch = '\'';
        printf("{\"error\": \"%s\"}\n", msg.c_str());
        return 3;
    }
}
