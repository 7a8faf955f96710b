/* Replay hooks compiled into a patched copy of the reference (vtsynergy/Hybrid-Stochastic-Block-
 * Partitioning) by oracle/build_reference.py.  TEST INFRASTRUCTURE ONLY.
 *
 * The patched copy records, for every vertex visit of a finetune call, the proposed block and
 * the accept uniform it drew, and for every merge proposal the proposed block, together with
 * the blockmodel state at the start and at the end of every finetune / merge call.  The GPU
 * engine replays that stream (sbp_finetune_replayed / sbp_merge_blocks_replayed) and must reach
 * the same states.  Included into every translation unit of the patched build (-include).
 *
 * Patch sites (all in the copy; the reference checkout is never written):
 *   P1 seeded engines      include/common.hpp:25-26 (std::random_device -> seed())
 *   P1 visit records       src/finetune.cpp:494-496, 510-512, 538-540 (on_proposal), :22 (on_uniform)
 *   P1 merge records       src/block_merge.cpp:291 (on_merge_slot), :340-341 (on_merge_proposal),
 *                          :304 (on_merge_scores)
 *   P1 call records        src/finetune.cpp:32, 343, 413 and src/block_merge.cpp:278 (CallScope)
 *   P2 FP64 logs           include/common.hpp:35-44 (cell_entropy), include/utils.hpp:148 (nat_log)
 *   P3 merge tie order     src/block_merge.cpp:342-345 (merge_delta_canonical: the lower block id is
 *                          merged into the higher, so r->s and s->r give the same double, and the
 *                          value is rounded to a multiple of 2^-20 as the engine ranks merges),
 *                          src/blockmodel/blockmodel.cpp:52 (stable order of equal delta-MDLs)
 *   P4 bounded sweeps      include/finetune.hpp:56 (MAX_NUM_ITERATIONS = max_sweeps())
 */
#ifndef SBP_REPLAY_H
#define SBP_REPLAY_H

#include <vector>

class Blockmodel;

namespace sbp_replay {

enum Kind { kMetropolisHastings = 0, kAsyncGibbs = 1, kHybrid = 2, kMerge = 3 };

/* Seed of every per-translation-unit engine (SBP_REF_SEED, default 1). */
unsigned seed();
/* Sweep cap of every finetune call (SBP_REF_MAX_SWEEPS, default 100 = the reference's value). */
int max_sweeps();

/* One finetune or merge call: its start state is logged on construction, its end state on
 * destruction (after the call has produced its result).  `bracket`: 1 when the golden-section
 * bracket is established (finetune's early-stop threshold), -1 for a merge. */
struct CallScope {
    CallScope(int kind, Blockmodel &bm, int bracket = -1);
    ~CallScope();
    int kind;
    int id;
    int sweep0;
    Blockmodel &bm;
};

/* The graph's high- and low-degree vertex lists in the order Graph::sort_vertices left them
 * (std::sort leaves the order of equal degrees to the implementation; the hybrid schedule visits
 * them in this order). */
void on_split(const std::vector<int> &high, const std::vector<int> &low);
/* Finetune visit of `vertex` proposing block `s` (the current block when the vertex stays). */
void on_proposal(int vertex, int s);
/* The accept uniform drawn for the calling thread's current visit. */
void on_uniform(double u);
/* Merge proposal number `i` of `block` is being drawn by the calling thread. */
void on_merge_slot(int block, int i);
void on_merge_proposal(int s);
/* Best proposal and its delta-MDL per block, before the carry-out. */
void on_merge_scores(const std::vector<int> &best, const std::vector<double> &delta);
/* block_merge_delta_mdl of merging r into s, always evaluated in the orientation lower id into
 * higher id with the reference's own functions (the merged blockmodel is the same either way),
 * rounded to a multiple of 2^-20: values that differ only by the rounding of their summation
 * order then rank as ties, which the reference's loops break by proposal order and block index. */
double merge_delta_canonical(int r, int s, int k_out, int k_in, const Blockmodel &bm);
/* utils::sort_indices with equal values kept in index order. */
std::vector<int> stable_sort_indices(const std::vector<double> &values);

}  // namespace sbp_replay

#endif
