// Kernel prototypes shared by the kernel and host translation units.
#pragma once
#include "sbp_device.cuh"

namespace sbpb {

constexpr int kProposalsPerBlock = 10;   // block_merge::NUM_AGG_PROPOSALS_PER_BLOCK (include/block_merge.hpp:24)
constexpr int kMaxIterations = 100;      // finetune::MAX_NUM_ITERATIONS (include/finetune.hpp:56)

struct Csr {
  const int* ptr;
  const int* idx;
  const int* val;
};

__global__ void k_rebuild_global(GraphView g, BlockView bm);
__global__ void k_rebuild_smem(GraphView g, BlockView bm);
__global__ void k_rebuild_degrees(BlockView bm);
__global__ void k_mdl_cells(BlockView bm, double* partial);
__global__ void k_mdl_edges(GraphView g, BlockView bm, const int* __restrict__ out_src, double* partial);
__global__ void k_mdl_final(const double* partial, int n, int V, long long E, int B, double* out);
__global__ void __launch_bounds__(256, 2) k_gibbs_eval(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng,
                             int sweep, int* prop, int* moved_list, int* n_moved, unsigned long long* counters,
                             int cap, int* status);
__global__ void k_apply_edges(GraphView g, BlockView bm, const int* moved_list, const int* n_moved, const int* prop,
                              int* qr, int* qs, unsigned long long* last, unsigned gen);
__global__ void k_apply_finish(BlockView bm, const int* moved_list, const int* n_moved, int* next_n_moved, int* prop,
                               const int* qr, const int* qs, const unsigned long long* last, unsigned gen);
__global__ void k_mh(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                     int cap, double* out, int* status);
__global__ void k_move_vertex(GraphView g, BlockView bm, int v, int s, int cap, int* status);
__global__ void k_eval_list(GraphView g, BlockView bm, const int* verts, int n, const uint4* records, int cap,
                            int* out_s, double* out_dS, double* out_H, int* out_acc, int* status);
__global__ void k_row_nnz(const int* A, int B, int ld, int* cnt);
__global__ void k_excl_scan(const int* in, int* out, int n);
__global__ void k_row_fill(const int* A, int B, int ld, const int* ptr, int* idx, int* val);
__global__ void k_merge_propose(BlockView bm, Csr rows, Csr cols, RngParams rng, int* best_s, double* best_dS,
                                unsigned long long* counters, int* status);
__global__ void k_block_sizes(const int* b, int V, int* size);
__global__ void k_relabel(int* b, int V, const int* map);

// Shared-memory ints per warp table of `cap` slots (keys, out counts, in counts, used list, count).
inline int table_ints(int cap) { return 4 * cap + 32; }

}  // namespace sbpb
