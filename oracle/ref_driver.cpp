// Driver around the reference's own library (vtsynergy/Hybrid-Stochastic-Block-Partitioning built
// from its sources by oracle/build_reference.py).  TEST INFRASTRUCTURE ONLY: it times the
// reference's CPU path for the benchmark's baseline arm and runs it for parity checks.
//
//   ref_driver finetune <edges.bin> <algo> <assignment.bin> <batches> <threads>
//   ref_driver sbp      <edges.bin> <algo> <batches> <threads> <approximate> <assignment_out.bin>
//   ref_driver merge    <edges.bin> <assignment.bin> <num_blocks_to_merge> <threads> <approximate>
//
// edges.bin: int32 V, int64 n, int32 src[n], int32 dst[n]; assignment.bin: int32 B, int32 b[V].
// Prints one JSON line.  The reference's own progress output is discarded.
#include <omp.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "args.hpp"
#include "blockmodel/blockmodel.hpp"
#include "blockmodel/blockmodel_triplet.hpp"
#include "block_merge.hpp"
#include "entropy.hpp"
#include "finetune.hpp"
#include "graph.hpp"
#include "mpi_data.hpp"
#include "sbp.hpp"
#include "utils.hpp"
#include "ref_graph.hpp"

MPI_t mpi;
Args args;

static long long visits_per_sweep(const Graph& g, const std::string& algo, int batches) {
    const int V = g.num_vertices();
    if (algo == "metropolis_hastings") return V;
    if (algo == "async_gibbs") {
        int bs = int(ceil(V / double(batches)));
        return (long long)(V / bs) * bs;
    }
    int nl = (int)g.low_degree_vertices().size();
    int bs = int(ceil(nl / double(batches)));
    long long low = bs > 0 ? (long long)(nl / bs) * bs : 0;
    return (long long)g.high_degree_vertices().size() + low;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::string mode = argv[1];
    mpi.rank = 0;
    mpi.num_processes = 1;
    args.transpose = true;   // every reference run script passes --transpose
    args.undirected = false;
    args.nodelta = false;
    args.asynciterations = std::numeric_limits<int>::max();
    int V;
    std::vector<int> src, dst;
    if (argc < 3 || !read_edges(argv[2], V, src, dst)) {
        fprintf(stderr, "cannot read edges\n");
        return 2;
    }
    std::ostringstream sink;
    std::streambuf* saved = std::cout.rdbuf(sink.rdbuf());
    if (mode == "finetune" && argc >= 7) {
        std::string algo = argv[3];
        args.algorithm = algo;
        args.batches = atoi(argv[5]);
        args.threads = atoi(argv[6]);
        omp_set_num_threads(args.threads);
        FILE* f = fopen(argv[4], "rb");
        int B = 0;
        std::vector<int> a(V);
        bool ok = f && fread(&B, 4, 1, f) == 1 && fread(a.data(), 4, V, f) == (size_t)V;
        if (f) fclose(f);
        if (!ok) return 2;
        Graph graph = make_graph(V, src, dst);
        Blockmodel bm(B, graph, 0.5, a);
        BlockmodelTriplet triplet;
        auto t0 = std::chrono::steady_clock::now();
        if (algo == "metropolis_hastings") bm = finetune::metropolis_hastings(bm, graph, triplet);
        else if (algo == "hybrid_mcmc") bm = finetune::hybrid_mcmc(bm, graph, triplet);
        else bm = finetune::asynchronous_gibbs(bm, graph, triplet);
        auto t1 = std::chrono::steady_clock::now();
        std::cout.rdbuf(saved);
        const double secs = std::chrono::duration<double>(t1 - t0).count();
        const long long visits = (long long)finetune::MCMC_iterations * visits_per_sweep(graph, algo, args.batches);
        printf("{\"seconds\": %.6f, \"sweeps\": %d, \"visits\": %lld, \"mdl\": %.6f, \"threads\": %d, \"V\": %d, "
               "\"E\": %d, \"B\": %d}\n",
               secs, finetune::MCMC_iterations, visits, (double)bm.getOverall_entropy(), args.threads, V,
               graph.num_edges(), B);
        return 0;
    }
    if (mode == "merge" && argc >= 7) {
        args.threads = atoi(argv[5]);
        args.approximate = atoi(argv[6]) != 0;
        omp_set_num_threads(args.threads);
        FILE* f = fopen(argv[3], "rb");
        int B = 0;
        std::vector<int> a(V);
        bool ok = f && fread(&B, 4, 1, f) == 1 && fread(a.data(), 4, V, f) == (size_t)V;
        if (f) fclose(f);
        if (!ok) return 2;
        Graph graph = make_graph(V, src, dst);
        Blockmodel bm(B, graph, 0.5, a);
        bm.setNum_blocks_to_merge(atoi(argv[4]));
        auto t0 = std::chrono::steady_clock::now();
        bm = block_merge::merge_blocks(bm, graph, graph.num_edges());
        auto t1 = std::chrono::steady_clock::now();
        std::cout.rdbuf(saved);
        printf("{\"seconds\": %.6f, \"num_blocks\": %d, \"threads\": %d, \"V\": %d, \"E\": %d}\n",
               std::chrono::duration<double>(t1 - t0).count(), bm.getNum_blocks(), args.threads, V, graph.num_edges());
        return 0;
    }
    if (mode == "sbp" && argc >= 8) {
        args.algorithm = argv[3];
        args.batches = atoi(argv[4]);
        args.threads = atoi(argv[5]);
        args.approximate = atoi(argv[6]) != 0;
        Graph graph = make_graph(V, src, dst);
        auto t0 = std::chrono::steady_clock::now();
        Blockmodel bm = sbp::stochastic_block_partition(graph, args);
        auto t1 = std::chrono::steady_clock::now();
        std::cout.rdbuf(saved);
        FILE* f = fopen(argv[7], "wb");
        if (f) {
            int B = bm.getNum_blocks();
            fwrite(&B, 4, 1, f);
            fwrite(bm.block_assignment().data(), 4, V, f);
            fclose(f);
        }
        printf("{\"seconds\": %.6f, \"mcmc_seconds\": %.6f, \"sweeps\": %d, \"mdl\": %.6f, \"num_blocks\": %d, "
               "\"threads\": %d, \"V\": %d, \"E\": %d}\n",
               std::chrono::duration<double>(t1 - t0).count(), finetune::MCMC_time, finetune::MCMC_iterations,
               (double)bm.getOverall_entropy(), bm.getNum_blocks(), args.threads, V, graph.num_edges());
        return 0;
    }
    std::cout.rdbuf(saved);
    fprintf(stderr, "bad arguments\n");
    return 2;
}
