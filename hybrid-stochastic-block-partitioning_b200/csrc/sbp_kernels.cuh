// Kernel prototypes shared by the kernel and host translation units.
#pragma once
#include "sbp_device.cuh"

namespace sbpb {

constexpr int kProposalsPerBlock = 10;   // block_merge::NUM_AGG_PROPOSALS_PER_BLOCK (include/block_merge.hpp:24)
constexpr int kMaxIterations = 100;      // finetune::MAX_NUM_ITERATIONS (include/finetune.hpp:56)

// Device-side state of an asynchronous-Gibbs finetune run as one CUDA graph: the loop over
// sweeps and its early stop are decided on the GPU (k_mdl).  Kernels given a
// control block read the sweep index and the batch generation from it.
struct SweepCtl {
  int sweep;               // index of the sweep being run
  unsigned gen0;           // batch generation before the sweep
  int nbatches;
  int count;               // sweeps finished
  int max_sweeps;
  int bracket;
  int* n_moved;            // the blockmodel's two moved-count slots
  double initial;          // the call's first MDL, as stored (float) by the reference
  double deltas[kMaxIterations];
};

struct Csr {
  const int* ptr;
  const int* idx;
  const int* val;
};

__global__ void k_rebuild_global(GraphView g, BlockView bm);
__global__ void k_rebuild_smem(GraphView g, BlockView bm);
__global__ void k_rebuild_degrees(BlockView bm);
// entropy::mdl of host-supplied nonzero cells (row, col, count) and block degrees: the per-cell
// form count * log(count / (d_out[row] * d_in[col])) of Blockmodel::log_posterior_probability.
__global__ void k_mdl_cells_list(const int* __restrict__ rows, const int* __restrict__ cols,
                                 const int* __restrict__ counts, long long nnz, const int* __restrict__ d_out,
                                 const int* __restrict__ d_in, double* partial);
__global__ void k_mdl_cells_list_final(const double* partial, int n, int V, long long E, int B, double* out);
__global__ void k_mdl(GraphView g, BlockView bm, const int* __restrict__ out_src, int cells, double* partial,
                      unsigned* done, double* out, SweepCtl* ctl, cudaGraphConditionalHandle loop);
// Asynchronous-Gibbs evaluation compiled for one storage of the block matrix.
__global__ void __launch_bounds__(256, 2)
    k_gibbs_eval_dense(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                       int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap, int* status,
                       const SweepCtl* ctl, int batch);
__global__ void __launch_bounds__(256, 2)
    k_gibbs_eval_hashed(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                        int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap, int* status,
                        const SweepCtl* ctl, int batch);
__global__ void __launch_bounds__(256, 3)
    k_gibbs_eval_dense_occ3(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                            int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap,
                            int* status, const SweepCtl* ctl, int batch);
using GibbsEvalKernel = void (*)(GraphView, BlockView, const int* __restrict__, int, RngParams, int, int*, int*, int*,
                                 unsigned long long*, int, int*, const SweepCtl*, int);
// Dense blockmodels up to this many blocks take the three-CTAs-per-SM build of the evaluation
// (measured on the 200,000-vertex graph: 10-17 % shorter launches up to 11,771 blocks, 5 % longer
// at 39,366, where the cells come from DRAM and more warps in flight only add misses).
constexpr int kEvalOcc3MaxB = 16384;
inline GibbsEvalKernel gibbs_eval_kernel(bool hashed, int B) {
  return hashed ? k_gibbs_eval_hashed : B <= kEvalOcc3MaxB ? k_gibbs_eval_dense_occ3 : k_gibbs_eval_dense;
}
// Asynchronous-Gibbs evaluation of light vertices on dense storage (sbp_eval_small.cu): groups of
// kSmallGroup lanes per vertex; neighbour-block histograms direct-indexed (B <= kSmallB) or in
// per-group hash tables of `cap` slots (hashed_table), in dynamic shared memory of
// gibbs_eval_group_smem bytes.
constexpr int kSmallB = 128;
constexpr int kSmallThreads = 256;
constexpr int kSmallGroup = 8;
constexpr int kGroupMaxK = 128;   // largest degree of a vertex on hashed group tables (256 slots)
using GibbsEvalGroupKernel = void (*)(GraphView, BlockView, const int* __restrict__, int, RngParams, int, int*, int*,
                                      int*, unsigned long long*, int, int*, const SweepCtl*, int);
GibbsEvalGroupKernel gibbs_eval_group_kernel(bool hashed_table);
size_t gibbs_eval_group_smem(bool hashed_table, int cap);
// Metropolis-Hastings rounds of kMhGroupThreads / kSmallGroup vertices (one CTA, dense storage).
constexpr int kMhGroupThreads = 512;
using MhGroupKernel = void (*)(GraphView, BlockView, const int* __restrict__, int, RngParams, int, int, double*, int*);
MhGroupKernel mh_group_kernel(bool hashed_table);
size_t mh_group_smem(bool hashed_table, int cap);
__global__ void k_apply_edges(GraphView g, BlockView bm, const int* moved_list, const int* n_moved, const int* prop,
                              int* qr, int* qs, unsigned long long* last, unsigned gen, const SweepCtl* ctl, int batch);
__global__ void k_apply_finish(BlockView bm, const int* moved_list, const int* n_moved, int* next_n_moved, int* prop,
                               const int* qr, const int* qs, const unsigned long long* last, unsigned gen,
                               const SweepCtl* ctl, int batch);
__global__ void k_mh(GraphView g, BlockView bm, const int* __restrict__ verts, int n, int start, RngParams rng,
                     int sweep, int cap, double* out, int* status);
__global__ void k_move_vertex(GraphView g, BlockView bm, int v, int s, int cap, int* status);
__global__ void k_eval_list(GraphView g, BlockView bm, const int* verts, int n, const uint4* records, int cap,
                            int* out_s, double* out_dS, double* out_H, int* out_acc, int* status);
__global__ void k_row_nnz(const int* A, int B, int ld, int* cnt);
__global__ void k_excl_scan(const int* in, int* out, int n);
__global__ void k_row_fill(const int* A, int B, int ld, const int* ptr, int* idx, int* val);
__global__ void k_merge_propose(BlockView bm, Csr rows, Csr cols, RngParams rng, int* best_s, double* best_dS,
                                unsigned long long* counters, int* status);
__global__ void k_block_sizes(const int* b, int V, int* size);
// Integer block statistics: out[0] = sum_b M[b,b], out[1] = sum_b d_in[b], out[2] = sum_b
// d_out[b] * d_in[b] (the interblock-edge fraction and the modularity of a partition).
__global__ void k_block_stats(BlockView bm, unsigned long long* out);
__global__ void k_relabel(int* b, int V, const int* map);

// row-hashed block matrix (sbp_sparse.cu)
__global__ void k_edge_keys(GraphView g, const int* __restrict__ b, const int* __restrict__ out_src, int B,
                            unsigned long long* keys, unsigned long long* keysT);
__global__ void k_unique_rows(const unsigned long long* __restrict__ ukeys, long long n, int B, unsigned* rowcnt);
__global__ void k_row_caps(const unsigned* __restrict__ rowcnt, int B, unsigned factor, unsigned* cap, int* mask);
__global__ void k_fill_empty(int2* slot, long long n);
__global__ void k_fill_rows(const long long* __restrict__ rowptr, const unsigned long long* __restrict__ ukeys,
                            const long long* __restrict__ heads, long long nu, long long nedges, int B,
                            const long long* __restrict__ base, const int* __restrict__ mask, int2* slot,
                            int* csr_ptr, int* csr_idx, int* csr_val);
__global__ void k_block_degrees(GraphView g, const int* __restrict__ b, int* d_out, int* d_in);
__global__ void k_fill_csr(const long long* __restrict__ rowptr, const unsigned long long* __restrict__ ukeys,
                           const long long* __restrict__ heads, long long nu, long long nedges, int B, int* csr_ptr,
                           int* csr_idx, int* csr_val);
__global__ void k_recover_assign(int* b, const int* moved, const int* n_moved, const int* prop, int* old_block);
__global__ void k_regrow_alloc(const int* __restrict__ full, const int* __restrict__ deg, int B, long long top,
                               long long limit, unsigned long long* used, unsigned long long* nrows, long long* base,
                               int* mask, int* list, unsigned long long* no_room);
__global__ void k_regrow_clear(const int* __restrict__ list, int n, const long long* __restrict__ base,
                               const int* __restrict__ mask, int2* slot);
__global__ void k_regrow_fill(GraphView g, BlockView bm, const int* __restrict__ out_src);
// sbp_ingest.cu
__global__ void k_ingest_first(const int* __restrict__ src, const int* __restrict__ dst, long long n, int V,
                               unsigned long long* keys, int* first, int tbits, int* bad);
__global__ void k_ingest_keep(const int* __restrict__ src, const int* __restrict__ dst, long long n, int V,
                              const unsigned long long* __restrict__ keys, const int* __restrict__ first, int tbits,
                              int ib, unsigned long long* out_keys, unsigned long long* in_keys,
                              unsigned long long* ctr, unsigned* out_cnt, unsigned* in_cnt, unsigned char* self);
__global__ void k_ingest_fill(const unsigned long long* __restrict__ sorted, long long m, int ib,
                              const int* __restrict__ other, int* idx, int* srcs);
__global__ void k_ingest_ptr(const long long* __restrict__ in, int* out, long long n);
__global__ void k_iota(int* out, int n);
__global__ void k_recover_finish(BlockView bm, const int* moved_list, const int* n_moved, int* next_n_moved,
                                 int* prop, const int* old_block, const int* qr, const int* qs,
                                 const unsigned long long* last, unsigned gen);
__global__ void k_fix_move_degrees(BlockView bm, int r, int s, int d_rr, int d_ss);
__global__ void k_hashed_to_dense(const long long* __restrict__ base, const int* __restrict__ mask,
                                  const int2* __restrict__ slot, int B, int row0, int rows, int* dense);

// Shared-memory ints per warp table of `cap` slots (keys, out counts, in counts, used list, count).
inline int table_ints(int cap) { return 4 * cap + 64; }   // keys, counts, list; count, 31 spare, 32 walk bins

}  // namespace sbpb
