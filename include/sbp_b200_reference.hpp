/*
 * sbp_b200_reference.hpp -- the reference's C++ API (vtsynergy/Hybrid-Stochastic-Block-
 * Partitioning) on the B200 engine, for code compiled against the reference's own headers.
 *
 * Each function has the argument list of the reference function it stands in for and runs it on
 * the GPU through the C ABI of sbp_b200.h:
 *
 *   sbp_b200::sbp::stochastic_block_partition(Graph&, Args&)           src/sbp.cpp:61-98
 *   sbp_b200::finetune::metropolis_hastings(Blockmodel&, const Graph&, BlockmodelTriplet&)
 *                                                                       src/finetune.cpp:412-444
 *   sbp_b200::finetune::asynchronous_gibbs(...)                         src/finetune.cpp:31-89
 *   sbp_b200::finetune::hybrid_mcmc(...)                                src/finetune.cpp:342-410
 *   sbp_b200::block_merge::merge_blocks(Blockmodel&, const Graph&, int) src/block_merge.cpp:278-311
 *   sbp_b200::entropy::mdl(const Blockmodel&, int, int)                 src/entropy.cpp:584-589
 *
 * A caller switches by qualifying its calls with sbp_b200:: (or with a using-declaration at the
 * call site).  The reference's Blockmodel stays the caller's object: a finetune or merge call
 * uploads its assignment (and the finetune its block degrees d, which drift as the reference
 * updates them), runs on the device and writes the result back into it -- assignment, block
 * count, block matrix (rebuilt by the reference's own Blockmodel::initialize_edge_counts, so
 * blockmatrix()->get and the degree accessors read the engine's state), d and the overall
 * entropy -- and returns it, as the reference's functions do.  finetune::MCMC_iterations and
 * finetune::MCMC_time advance as in the reference.  stochastic_block_partition returns the
 * blockmodel of the final assignment built by the reference's constructor (its d is the rebuilt
 * one, without the drift of the finetune that produced it).
 *
 * Random numbers: the engine's Philox stream, keyed by `seed`; successive calls use successive
 * stream words.  The flags come from the reference's Args (algorithm, batches, approximate,
 * asynciterations).  Errors throw std::runtime_error carrying sbp_last_error().
 *
 * Link with -lsbp_b200 (hybrid-stochastic-block-partitioning_b200/libsbp_b200.so), together with
 * the reference's graph and blockmodel sources that define Graph and Blockmodel.
 */
#ifndef SBP_B200_REFERENCE_HPP
#define SBP_B200_REFERENCE_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "sbp_b200.h"

#include "args.hpp"
#include "blockmodel/blockmodel.hpp"
#include "blockmodel/blockmodel_triplet.hpp"
#include "finetune.hpp"
#include "graph.hpp"

namespace sbp_b200 {
namespace detail {

inline void check(SbpStatus st, const char *what) {
    if (st != SBP_OK) throw std::runtime_error(std::string("sbp_b200 ") + what + ": " + sbp_last_error());
}

/* Stream word 2 of the engine's Philox counter for the next call (one per call). */
inline uint32_t next_call() {
    static thread_local uint32_t call = 0;
    return call++;
}

/* Owns one engine handle for the duration of a call. */
struct DeviceGraph {
    SbpGraph *h = nullptr;
    /* The reference graph's edges in its own adjacency order, and its high/low degree split in
     * the order Graph::sort_vertices left it (the hybrid schedule visits vertices in that order). */
    explicit DeviceGraph(const Graph &graph) {
        std::vector<int32_t> src, dst;
        src.reserve(graph.num_edges());
        dst.reserve(graph.num_edges());
        for (int v = 0; v < graph.num_vertices(); ++v)
            for (int u : graph.out_neighbors(v)) {
                src.push_back(v);
                dst.push_back(u);
            }
        check(sbp_graph_create(graph.num_vertices(), (int64_t)src.size(), src.data(), dst.data(), &h), "graph");
        const std::vector<int> &hi = graph.high_degree_vertices(), &lo = graph.low_degree_vertices();
        if (hi.size() + lo.size() == (size_t)graph.num_vertices())
            check(sbp_graph_set_split(h, (int32_t)hi.size(), hi.data(), (int32_t)lo.size(), lo.data()), "split");
    }
    ~DeviceGraph() {
        if (h) sbp_graph_destroy(h);
    }
    DeviceGraph(const DeviceGraph &) = delete;
    DeviceGraph &operator=(const DeviceGraph &) = delete;
};

struct DeviceBlockmodel {
    SbpBlockmodel *h = nullptr;
    DeviceBlockmodel(const DeviceGraph &g, const Blockmodel &bm, bool with_degrees) {
        const std::vector<int> &a = bm.block_assignment();
        check(sbp_blockmodel_create(g.h, bm.getNum_blocks(), a.data(), &h), "blockmodel");
        if (with_degrees && (int)bm.degrees().size() == bm.getNum_blocks())
            check(sbp_set_degrees(h, bm.degrees().data()), "degrees");
    }
    ~DeviceBlockmodel() {
        if (h) sbp_blockmodel_destroy(h);
    }
    DeviceBlockmodel(const DeviceBlockmodel &) = delete;
    DeviceBlockmodel &operator=(const DeviceBlockmodel &) = delete;
};

/* Write the engine's blockmodel back into the reference object. */
inline void mirror(Blockmodel &bm, const Graph &graph, const DeviceBlockmodel &dbm, double entropy) {
    int32_t B = 0;
    check(sbp_blockmodel_num_blocks(dbm.h, &B), "num_blocks");
    std::vector<int32_t> a(graph.num_vertices()), d_out(B), d_in(B), d(B);
    check(sbp_get_assignment(dbm.h, a.data()), "assignment");
    check(sbp_get_degrees(dbm.h, d_out.data(), d_in.data(), d.data()), "degrees");
    bm.setNum_blocks(B);
    bm.set_block_assignment(std::vector<int>(a.begin(), a.end()));
    bm.initialize_edge_counts(graph);
    bm.degrees(std::vector<int>(d.begin(), d.end()));
    bm.setOverall_entropy(entropy);
}

inline int algorithm_of(const std::string &name) {
    if (name == "metropolis_hastings") return SBP_METROPOLIS_HASTINGS;
    if (name == "hybrid_mcmc") return SBP_HYBRID_MCMC;
    return SBP_ASYNC_GIBBS;
}

inline Blockmodel &run_finetune(int algorithm, Blockmodel &blockmodel, const Graph &graph,
                                BlockmodelTriplet &blockmodels, uint64_t seed) {
    if (blockmodel.getNum_blocks() == 1) return blockmodel;   // src/finetune.cpp:33-35
    DeviceGraph g(graph);
    DeviceBlockmodel bm(g, blockmodel, true);
    SbpFinetuneOptions opt{args.batches, blockmodels.get(2).empty ? 0 : 1, 0, next_call(), seed};
    SbpStats st{};
    check(sbp_finetune(bm.h, g.h, algorithm, &opt, nullptr, &st), "finetune");
    ::finetune::MCMC_iterations += st.sweeps;
    mirror(blockmodel, graph, bm, st.mdl);
    return blockmodel;
}

}  // namespace detail

namespace finetune {
inline Blockmodel &metropolis_hastings(Blockmodel &blockmodel, const Graph &graph, BlockmodelTriplet &blockmodels,
                                       uint64_t seed = 0) {
    return detail::run_finetune(SBP_METROPOLIS_HASTINGS, blockmodel, graph, blockmodels, seed);
}
inline Blockmodel &asynchronous_gibbs(Blockmodel &blockmodel, const Graph &graph, BlockmodelTriplet &blockmodels,
                                      uint64_t seed = 0) {
    return detail::run_finetune(SBP_ASYNC_GIBBS, blockmodel, graph, blockmodels, seed);
}
inline Blockmodel &hybrid_mcmc(Blockmodel &blockmodel, const Graph &graph, BlockmodelTriplet &blockmodels,
                               uint64_t seed = 0) {
    return detail::run_finetune(SBP_HYBRID_MCMC, blockmodel, graph, blockmodels, seed);
}
}  // namespace finetune

namespace block_merge {
/* num_edges is the graph's (the engine reads it from the graph, as the reference's callers pass
 * graph.num_edges()). */
inline Blockmodel &merge_blocks(Blockmodel &blockmodel, const Graph &graph, int num_edges, uint64_t seed = 0) {
    (void)num_edges;
    detail::DeviceGraph g(graph);
    detail::DeviceBlockmodel bm(g, blockmodel, false);
    detail::check(sbp_blockmodel_set_num_blocks_to_merge(bm.h, blockmodel.getNum_blocks_to_merge()), "merge count");
    SbpMergeOptions opt{args.approximate ? 1 : 0, detail::next_call(), seed};
    SbpStats st{};
    detail::check(sbp_merge_blocks(bm.h, g.h, &opt, nullptr, nullptr, nullptr, &st), "merge");
    detail::mirror(blockmodel, graph, bm, blockmodel.getOverall_entropy());
    return blockmodel;
}
}  // namespace block_merge

namespace entropy {
inline double mdl(const Blockmodel &blockmodel, int num_vertices, int num_edges) {
    const Indices nz = blockmodel.blockmatrix()->nonzero();
    const std::vector<int> values = blockmodel.blockmatrix()->values();
    double out = 0.0;
    detail::check(sbp_mdl_of_cells(blockmodel.getNum_blocks(), (int64_t)values.size(), nz.rows.data(), nz.cols.data(),
                                   values.data(), blockmodel.degrees_out().data(), blockmodel.degrees_in().data(),
                                   num_vertices, num_edges, &out),
                  "mdl");
    return out;
}
}  // namespace entropy

namespace sbp {
inline Blockmodel stochastic_block_partition(Graph &graph, Args &args, uint64_t seed = 0) {
    detail::DeviceGraph g(graph);
    SbpOptions opt{detail::algorithm_of(args.algorithm), args.batches, args.approximate ? 1 : 0, args.asynciterations,
                   seed};
    std::vector<int32_t> out(graph.num_vertices());
    SbpStats st{};
    detail::check(sbp_partition(g.h, &opt, out.data(), &st), "partition");
    ::finetune::MCMC_iterations += st.sweeps;
    ::finetune::MCMC_time += st.mcmc_seconds;
    std::vector<int> a(out.begin(), out.end());
    Blockmodel bm(st.num_blocks, graph, float(BLOCK_REDUCTION_RATE), a);
    bm.setOverall_entropy(st.mdl);
    return bm;
}
}  // namespace sbp

}  // namespace sbp_b200

#endif  // SBP_B200_REFERENCE_HPP
