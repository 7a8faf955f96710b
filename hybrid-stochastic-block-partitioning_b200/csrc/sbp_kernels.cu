// CUDA kernels of the B200 stochastic block partitioning engine.
//
// Kernel map (reference function each one stands in for):
//   k_rebuild_*        Blockmodel::initialize_edge_counts     src/blockmodel/blockmodel.cpp:187-255
//   k_mdl              entropy::mdl / log_posterior_probability src/entropy.cpp:584-589, blockmodel.cpp:267-285
//   k_gibbs_eval_*     asynchronous_gibbs evaluation half     src/finetune.cpp:49-57, 531-545
//   k_apply_*          asynchronous_gibbs apply half          src/finetune.cpp:58-71 + Blockmodel::move_vertex
//   k_mh               metropolis_hastings sweep              src/finetune.cpp:412-444, 446-501
//   k_row_nnz/fill     ISparseMatrix row/column views for the merge phase
//   k_merge_propose    merge_blocks proposal scoring          src/block_merge.cpp:278-301, 335-368
//   k_relabel          carry-out relabel                      src/blockmodel/blockmodel.cpp:71-76
#include "sbp_kernels.cuh"
#include "sbp_steps.cuh"

namespace sbpb {

// ------------------------------------------------------------------------------------------
// Rebuild: M, MT, d_out, d_in from the assignment; d = d_out + d_in - M[x,x].
// ------------------------------------------------------------------------------------------
__global__ void k_rebuild_global(GraphView g, BlockView bm) {
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < g.V; v += stride) {
    const int bv = bm.b[v];
    const int o0 = g.out_ptr[v], o1 = g.out_ptr[v + 1];
    for (int e = o0; e < o1; ++e) {
      const int bu = bm.b[__ldg(g.out_idx + e)];
      atomicAdd(bm.M + (size_t)bv * bm.ld + bu, 1);
      atomicAdd(bm.MT + (size_t)bu * bm.ld + bv, 1);
      chunk_add(bm.CS, bm.nch, bv, bu, 1);
      chunk_add(bm.CST, bm.nch, bu, bv, 1);
    }
    atomicAdd(bm.d_out + bv, o1 - o0);
    atomicAdd(bm.d_in + bv, (g.in_ptr[v + 1] - g.in_ptr[v]) + g.self[v]);
  }
}

// Small-B variant: a CTA-private B x B histogram in shared memory, flushed once.
__global__ void k_rebuild_smem(GraphView g, BlockView bm) {
  extern __shared__ int hist[];   // B*B
  const int BB = bm.B * bm.B;
  for (int i = threadIdx.x; i < BB; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < g.V; v += stride) {
    const int bv = bm.b[v];
    const int o0 = g.out_ptr[v], o1 = g.out_ptr[v + 1];
    for (int e = o0; e < o1; ++e) atomicAdd(hist + bv * bm.B + bm.b[__ldg(g.out_idx + e)], 1);
    atomicAdd(bm.d_out + bv, o1 - o0);
    atomicAdd(bm.d_in + bv, (g.in_ptr[v + 1] - g.in_ptr[v]) + g.self[v]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < BB; i += blockDim.x) {
    const int c = hist[i];
    if (c) {
      const int row = i / bm.B, col = i - row * bm.B;
      atomicAdd(bm.M + (size_t)row * bm.ld + col, c);
      atomicAdd(bm.MT + (size_t)col * bm.ld + row, c);
      chunk_add(bm.CS, bm.nch, row, col, c);
      chunk_add(bm.CST, bm.nch, col, row, c);
    }
  }
}

__global__ void k_rebuild_degrees(BlockView bm) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < bm.B) bm.d[x] = bm.d_out[x] + bm.d_in[x] - bm_get(bm, x, x);
}
// ------------------------------------------------------------------------------------------
// Asynchronous Gibbs: evaluate a list of vertices against the frozen state.  Accepted moves
// go to prop[v] and the moved list; counters: [0] visits [1] proposals_moved [2] accepted.
// ------------------------------------------------------------------------------------------
template <Store ST>
__device__ __forceinline__ void gibbs_eval_body(GraphView g, BlockView bm, const int* __restrict__ verts, int n,
                                                RngParams rng, int sweep, int* prop, int* moved_list, int* n_moved,
                                                unsigned long long* counters, int cap, int* status,
                                                const SweepCtl* ctl, int batch) {
  extern __shared__ int smem[];
  if (ctl) {
    sweep = ctl->sweep;
    n_moved = ctl->n_moved + ((ctl->gen0 + (unsigned)batch) & 1u);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  unsigned long long c_visit = 0, c_moved = 0, c_acc = 0;
  for (int i = blockIdx.x * wpb + warp; i < n; i += gridDim.x * wpb) {
    const int v = verts[i];
    const uint4 x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * g.V + v, status);
    int r, k_out, k_in;
    const EvalResult res = evaluate_vertex<ST>(g, bm, v, x, t, lane, status, &r, &k_out, &k_in, rng.moves != 0);
    c_visit++;
    if (res.s != r) c_moved++;
    if (res.accepted) {
      c_acc++;
      if (lane == 0) {
        prop[v] = res.s;
        moved_list[atomicAdd(n_moved, 1)] = v;
      }
    }
    table_reset(t, lane);
  }
  if (lane == 0 && c_visit) {
    atomicAdd(counters + 0, c_visit);
    atomicAdd(counters + 1, c_moved);
    atomicAdd(counters + 2, c_acc);
  }
}

__global__ void __launch_bounds__(256, 2)
    k_gibbs_eval_dense(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                       int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap, int* status,
                       const SweepCtl* ctl, int batch) {
  gibbs_eval_body<Store::kDenseFrozen>(g, bm, verts, n, rng, sweep, prop, moved_list, n_moved, counters, cap, status,
                                       ctl, batch);
}
// The same with registers capped for three CTAs per SM (a few spilled values): more vertices in
// flight, which pays while the block matrix is small enough for its cells to hit in L2.
__global__ void __launch_bounds__(256, 3)
    k_gibbs_eval_dense_occ3(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                            int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap,
                            int* status, const SweepCtl* ctl, int batch) {
  gibbs_eval_body<Store::kDenseFrozen>(g, bm, verts, n, rng, sweep, prop, moved_list, n_moved, counters, cap, status,
                                       ctl, batch);
}
__global__ void __launch_bounds__(256, 2)
    k_gibbs_eval_hashed(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                        int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap, int* status,
                        const SweepCtl* ctl, int batch) {
  gibbs_eval_body<Store::kHashed>(g, bm, verts, n, rng, sweep, prop, moved_list, n_moved, counters, cap, status, ctl,
                                  batch);
}


// Apply accepted moves of one batch.  Every edge incident to a moved vertex moves once from
// its old cell to its new cell; the result equals the reference's one-by-one application.
// qr/qs keep the reference's diagonal delta of each move as seen at its turn in vertex order,
// which Blockmodel::move_vertex folds into d[r], d[s] (blockmodel.cpp:348-359).
// Every edge incident to a moved vertex moves once from its old cell to its new cell; the
// result equals the reference's one-by-one application.  qr/qs keep the reference's diagonal
// delta of each move as seen at its turn in vertex order, which Blockmodel::move_vertex folds
// into d[r], d[s] (blockmodel.cpp:348-359); last[x] keeps (batch generation, last mover of x).
__global__ void k_apply_edges(GraphView g, BlockView bm, const int* moved_list, const int* n_moved, const int* prop,
                              int* qr, int* qs, unsigned long long* last, unsigned gen, const SweepCtl* ctl, int batch) {
  if (ctl) {
    gen = ctl->gen0 + (unsigned)batch + 1u;
    n_moved = ctl->n_moved + ((gen - 1u) & 1u);
  }
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int n = *n_moved;
  for (int i = wid; i < n; i += nw) apply_moved_vertex(g, bm, moved_list[i], prop, qr, qs, last, gen, lane);
}

// d[r], d[s] from the last mover of each block, then the new assignment; clears the other
// moved-count slot for the next batch.
__global__ void k_apply_finish(BlockView bm, const int* moved_list, const int* n_moved, int* next_n_moved, int* prop,
                               const int* qr, const int* qs, const unsigned long long* last, unsigned gen,
                               const SweepCtl* ctl, int batch) {
  if (ctl) {
    gen = ctl->gen0 + (unsigned)batch + 1u;
    n_moved = ctl->n_moved + ((gen - 1u) & 1u);
    next_n_moved = ctl->n_moved + (gen & 1u);
  }
  const int n = *n_moved;
  if (blockIdx.x == 0 && threadIdx.x == 0) *next_n_moved = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    finish_moved_vertex(bm, moved_list[i], prop, qr, qs, last, gen);
}

// End of one sweep of a graph-run finetune: record delta = MDL - first MDL (the asynchronous-
// Gibbs rule, src/finetune.cpp:40,74) and apply finetune::early_stop (src/finetune.cpp:144-162)
// in the host's arithmetic; the loop continues while it does not stop.
__device__ __forceinline__ void sweep_control(SweepCtl* ctl, double mdl, cudaGraphConditionalHandle loop) {
  const int it = ctl->count;
  ctl->deltas[it] = mdl - ctl->initial;
  ctl->count = it + 1;
  bool stop;
  if (ctl->deltas[it] == 0.0) {
    stop = true;
  } else if (it < 3) {
    stop = false;
  } else {
    double average = ctl->deltas[it] + ctl->deltas[it - 1] + ctl->deltas[it - 2];
    average /= -3.0;
    const double threshold = ctl->bracket ? 1e-4 * ctl->initial : 5e-4 * ctl->initial;
    stop = average < threshold;
  }
  if (ctl->count >= ctl->max_sweeps) stop = true;
  ctl->sweep = it + 1;
  ctl->gen0 += (unsigned)ctl->nbatches;
  cudaGraphSetConditional(loop, stop ? 0u : 1u);
}

// entropy::mdl (src/entropy.cpp:584-589) in one launch.  Every CTA writes its partial sum (cell
// form when B*B <= 4E on dense storage, else the edge form); the CTA that finishes last (a
// counter taken after a memory fence) sums the partials in a fixed order and applies the
// formula.  With a graph-run sweep (ctl) it then records the sweep and sets the loop condition.
__global__ void k_mdl(GraphView g, BlockView bm, const int* __restrict__ out_src, int cells, double* partial,
                      unsigned* done, double* out, SweepCtl* ctl, cudaGraphConditionalHandle loop) {
  __shared__ double red[32];
  __shared__ int s_last;
  const double t = cells ? mdl_cells_part(bm, blockIdx.x, gridDim.x, red)
                         : mdl_edges_part(g, bm, out_src, blockIdx.x, gridDim.x, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = t;
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const double v = mdl_final_value(partial, gridDim.x, g.V, g.E, bm.B, red);
  if (threadIdx.x == 0) {
    *out = v;
    *done = 0u;
    if (ctl) sweep_control(ctl, v, loop);
  }
}

// entropy::mdl (src/entropy.cpp:584-589) from a list of nonzero cells, each term as
// Blockmodel::log_posterior_probability (src/blockmodel/blockmodel.cpp:267-285) forms it.
// Deterministic: grid-stride partials per CTA, then one CTA sums them in order.
__global__ void k_mdl_cells_list(const int* __restrict__ rows, const int* __restrict__ cols,
                                 const int* __restrict__ counts, long long nnz, const int* __restrict__ d_out,
                                 const int* __restrict__ d_in, double* partial) {
  __shared__ double red[32];
  double acc = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += stride) {
    const double m = counts[i];
    acc += m * log(m / ((double)d_out[rows[i]] * (double)d_in[cols[i]]));
  }
  const double t = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

__global__ void k_mdl_cells_list_final(const double* partial, int n, int V, long long E, int B, double* out) {
  __shared__ double red[32];
  const double v = mdl_final_value(partial, n, V, E, B, red);
  if (threadIdx.x == 0) *out = v;
}

// ------------------------------------------------------------------------------------------
// Metropolis-Hastings over a vertex list, exact sequential semantics, one CTA.
// Round: the W warps evaluate the next W vertices against the current state; the first
// accepted one (in list order) is applied by the warp that evaluated it, everything before it
// was rejected against the true state, everything after it is re-evaluated next round.  The
// random record of a visit depends only on (vertex, sweep), so re-evaluation is idempotent.
// out: [0] visits [1] proposals_moved [2] accepted (as doubles), [3] sum of accepted dS.
// ------------------------------------------------------------------------------------------
__global__ void k_mh(GraphView g, BlockView bm, const int* __restrict__ verts, int n, int start, RngParams rng,
                     int sweep, int cap, double* out, int* status) {
  extern __shared__ int smem[];
  __shared__ int s_acc[32], s_moved[32], s_r[32], s_s[32], s_t[32], s_commit[32];
  __shared__ double s_dS[32];
  __shared__ int s_stop, s_upto;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int W = blockDim.x >> 5;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  long long visits = 0, moved = 0, accepted = 0;
  double sum_dS = 0.0;
  int pos = start;
  if (threadIdx.x == 0) {
    s_stop = 0;
    out[4] = 0.0;
  }
  __syncthreads();
  while (pos < n) {
    const int i = pos + warp;
    int r = -1, k_out = 0, k_in = 0, v = -1;
    EvalResult res;
    res.accepted = 0;
    res.s = -1;
    res.dS = 0.0;
    if (i < n) {
      v = verts[i];
      const uint4 x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * g.V + v, status);
      res = evaluate_vertex(g, bm, v, x, t, lane, status, &r, &k_out, &k_in, rng.moves != 0);
    }
    if (lane == 0) {
      s_acc[warp] = (i < n) ? res.accepted : 0;
      s_moved[warp] = (i < n && res.s != r) ? 1 : 0;
      s_dS[warp] = res.dS;
      s_r[warp] = r;
      s_s[warp] = res.s;
      s_t[warp] = res.t;
      s_commit[warp] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int first;
      s_upto = mh_round_commits(bm, smem, cap, min(W, n - pos), s_acc, s_r, s_s, s_t, s_commit, &first);
    }
    __syncthreads();
    const int upto_round = s_upto;
    // a hashed row can run out of room only on row-hashed storage, where the round commits its
    // first accepted vertex alone: the stop position is pos + first
    if (s_commit[warp]) mh_apply_move(g, bm, t, v, r, res.s, k_out, k_in, lane, pos + warp, out, &s_stop);
    if (threadIdx.x == 0) {
      for (int w = 0; w < upto_round; ++w) {
        moved += s_moved[w];
        if (s_commit[w]) {   // accepted moves in vertex order
          accepted++;
          sum_dS += s_dS[w];
        }
      }
      visits += upto_round;
    }
    pos += upto_round;
    table_reset(t, lane);
    __syncthreads();
    if (s_stop) break;
  }
  if (threadIdx.x == 0) {
    out[0] = (double)visits;
    out[1] = (double)moved;
    out[2] = (double)accepted;
    out[3] = sum_dS;
  }
}

// Blockmodel::move_vertex(vertex, delta, proposal) (src/blockmodel/blockmodel.cpp:344-360) for
// one vertex: a single warp builds the neighbour-block table and applies the move, including
// the reference's d[r], d[s] update from the already-updated diagonal.
__global__ void k_move_vertex(GraphView g, BlockView bm, int v, int s, int cap, int* status) {
  extern __shared__ int smem[];
  const int lane = threadIdx.x & 31;
  WarpTable t = carve_table(smem, cap, 0);
  init_table(t, lane);
  const int r = bm.b[v];
  if (r == s) return;
  build_table(g, bm, v, r, t, lane, status);
  const int self = g.self[v];
  const int k_out = g.out_ptr[v + 1] - g.out_ptr[v];
  const int k_in = g.in_ptr[v + 1] - g.in_ptr[v];
  const MoveCounts mc = corner_counts(t, r, s);
  const int nl = *t.nlist;
  for (int j = lane; j < nl; j += kWarp) {
    const int h = t.list[j];
    const int u = t.keys[h], co = t.cout[h], ci = t.cin[h];
    if (u == r || u == s) continue;
    cell_add_owned(bm, r, u, -co);
    cell_add_owned(bm, s, u, co);
    cell_add_owned(bm, u, r, -ci);
    cell_add_owned(bm, u, s, ci);
  }
  __syncwarp();
  if (lane == 0) {
    const int d_rr = -mc.co_r - mc.ci_r - self, d_rs = -mc.co_s + mc.ci_r;
    const int d_sr = mc.co_r - mc.ci_s, d_ss = mc.co_s + mc.ci_s + self;
    cell_add_owned(bm, r, r, d_rr);
    cell_add_owned(bm, r, s, d_rs);
    cell_add_owned(bm, s, r, d_sr);
    cell_add_owned(bm, s, s, d_ss);
    bm.b[v] = s;
    bm.d_out[r] -= k_out;
    bm.d_out[s] += k_out;
    bm.d_in[r] -= k_in + self;
    bm.d_in[s] += k_in + self;
    __threadfence_block();
    if (!*bm.overflow) {
      bm.d[r] = bm.d_out[r] + bm.d_in[r] - (bm_get(bm, r, r) + d_rr);
      bm.d[s] = bm.d_out[s] + bm.d_in[s] - (bm_get(bm, s, s) + d_ss);
    }
    status[1] = d_rr;   // kept for the d fix-up after a row-capacity rebuild
    status[2] = d_ss;
  }
}

// Evaluate (without moving) a list of vertices with caller-supplied records.
__global__ void k_eval_list(GraphView g, BlockView bm, const int* verts, int n, const uint4* records, int cap,
                            int* out_s, double* out_dS, double* out_H, int* out_acc, int* status) {
  extern __shared__ int smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  for (int i = blockIdx.x * wpb + warp; i < n; i += gridDim.x * wpb) {
    const int v = verts[i];
    int r, k_out, k_in;
    const EvalResult res = evaluate_vertex(g, bm, v, records[i], t, lane, status, &r, &k_out, &k_in);
    if (lane == 0) {
      out_s[i] = res.s;
      out_dS[i] = res.dS;
      out_H[i] = res.H;
      out_acc[i] = res.accepted;
    }
    table_reset(t, lane);
  }
}

// ------------------------------------------------------------------------------------------
// Merge phase: compressed rows of M (out_blocks) and of MT (in_blocks), ascending.
// ------------------------------------------------------------------------------------------
__global__ void k_row_nnz(const int* A, int B, int ld, int* cnt) {
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int row = wid; row < B; row += nw) {
    int c = 0;
    const int* p = A + (size_t)row * ld;
    for (int col = lane; col < B; col += kWarp) c += (p[col] != 0);
    c = warp_sum_int(c);
    if (lane == 0) cnt[row] = c;
  }
}

// Exclusive scan of n ints (single CTA of 1024 threads).
__global__ void k_excl_scan(const int* in, int* out, int n) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      int t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, t, o);
        if (lane >= o) t += y;
      }
      warp_tot[lane] = t;
    }
    __syncthreads();
    const int before = carry + (w > 0 ? warp_tot[w - 1] : 0);
    if (i < n) out[i] = before + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_row_fill(const int* A, int B, int ld, const int* ptr, int* idx, int* val) {
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int row = wid; row < B; row += nw) {
    int pos = ptr[row];
    const int* p = A + (size_t)row * ld;
    for (int base = 0; base < B; base += kWarp) {
      const int col = base + lane;
      const int x = col < B ? p[col] : 0;
      const unsigned m = __ballot_sync(kFull, x != 0);
      if (x != 0) {
        const int o = pos + __popc(m & ((1u << lane) - 1));
        idx[o] = col;
        val[o] = x;
      }
      pos += __popc(m);
    }
  }
}

// Merge proposal for block r (common::propose_new_block with block_merge = true, canonical
// order) and the merge delta-MDL in closed form:
//   dS = sum_c g(M[r,c]) + sum_{c!=r} g(M[c,r]) + sum_{c not in r,s} [g(M[s,c]) - g(M[s,c]+M[r,c])]
//      + sum_{c not in r,s} [g(M[c,s]) - g(M[c,s]+M[c,r])] + g(M[s,s]) - g(M[s,s]+M[r,r]+M[r,s]+M[s,r])
//      - [g(do_r)+g(do_s)-g(do_r+do_s)] - [g(di_r)+g(di_s)-g(di_r+di_s)]
// which equals entropy::block_merge_delta_mdl (src/entropy.cpp:127-180).
__device__ double merge_delta(const BlockView& bm, const Csr& rows, const Csr& cols, int r, int s, int lane) {
  double dS = 0.0;
  for (int j = rows.ptr[r] + lane; j < rows.ptr[r + 1]; j += kWarp) {
    const int c = rows.idx[j], m = rows.val[j];
    dS += xlogx((double)m);
    if (c != r && c != s) {
      const int msc = bm_get(bm, s, c);
      dS += dxlogx((double)msc, (double)(msc + m));
    }
  }
  for (int j = cols.ptr[r] + lane; j < cols.ptr[r + 1]; j += kWarp) {
    const int c = cols.idx[j], m = cols.val[j];
    if (c == r) continue;
    dS += xlogx((double)m);
    if (c != s) {
      const int mcs = bm_getT(bm, s, c);
      dS += dxlogx((double)mcs, (double)(mcs + m));
    }
  }
  dS = warp_sum(dS);
  const int M_rr = bm_get(bm, r, r), M_rs = bm_get(bm, r, s);
  const int M_sr = bm_get(bm, s, r), M_ss = bm_get(bm, s, s);
  dS += dxlogx((double)M_ss, (double)(M_ss + M_rr + M_rs + M_sr));
  const double dor = bm.d_out[r], dos = bm.d_out[s], dir = bm.d_in[r], dis = bm.d_in[s];
  dS -= xlogx(dor) + xlogx(dos) - xlogx(dor + dos);
  dS -= xlogx(dir) + xlogx(dis) - xlogx(dir + dis);
  return dS;
}

__global__ void k_merge_propose(BlockView bm, Csr rows, Csr cols, RngParams rng, int* best_s, double* best_dS,
                                unsigned long long* counters, int* status) {
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int B = bm.B;
  for (int r = wid; r < B; r += nw) {
    int seen[kProposalsPerBlock];
    int nseen = 0;
    int best = -1;
    double bdS = 1.79769313486231570815e+308;
    int avoided = 0;
    const long long k_out = bm.d_out[r], k = k_out + bm.d_in[r];
    for (int i = 0; i < kProposalsPerBlock; ++i) {
      const uint4 x = draw_record(rng, (uint32_t)r, (uint32_t)i, 1u, (long long)r * kProposalsPerBlock + i, status);
      int s;
      if (rng.moves) {   // a replayed proposal
        s = (int)x.x;
        if (s < 0 || s >= B || s == r) {
          if (lane == 0) atomicOr(status, kErrReplay);
          s = r == 0 ? 1 : 0;
        }
      } else if (k == 0) {
        s = random_block(r, B, x.y);
      } else {
        const long long target = scale32(x.x, k);
        int t;
        if (target < k_out) t = warp_select_sparse(rows.idx + rows.ptr[r], rows.val + rows.ptr[r],
                                                   rows.ptr[r + 1] - rows.ptr[r], target, -1, lane);
        else t = warp_select_sparse(cols.idx + cols.ptr[r], cols.val + cols.ptr[r], cols.ptr[r + 1] - cols.ptr[r],
                                    target - k_out, -1, lane);
        if (t < 0) {
          if (lane == 0) atomicOr(status, kErrScan);
          t = r;
        }
        const long long m_tr = bm_get(bm, t, r), m_rt = bm_get(bm, r, t);
        const long long rowpart = (long long)bm.d_out[t] - m_tr;
        const long long total = rowpart + (long long)bm.d_in[t] - m_rt;
        if (total == 0) {
          s = random_block(r, B, x.y);
        } else {
          const long long tg = scale32(x.y, total);
          if (tg < rowpart) s = warp_select_sparse(rows.idx + rows.ptr[t], rows.val + rows.ptr[t],
                                                   rows.ptr[t + 1] - rows.ptr[t], tg, r, lane);
          else s = warp_select_sparse(cols.idx + cols.ptr[t], cols.val + cols.ptr[t], cols.ptr[t + 1] - cols.ptr[t],
                                      tg - rowpart, r, lane);
          if (s < 0) {
            if (lane == 0) atomicOr(status, kErrScan);
            s = random_block(r, B, x.y);
          }
        }
      }
      bool dup = false;
      for (int j = 0; j < nseen; ++j) dup |= (seen[j] == s);
      if (dup) {
        avoided++;
        continue;
      }
      seen[nseen++] = s;
      // same value for r->s and s->r; one fixed orientation makes mutual pairs tie exactly
      const double dS = merge_score(merge_delta(bm, rows, cols, min(r, s), max(r, s), lane));
      if (dS < bdS) {
        bdS = dS;
        best = s;
      }
    }
    if (lane == 0) {
      best_s[r] = best;
      best_dS[r] = bdS;
      atomicAdd(counters + 0, (unsigned long long)kProposalsPerBlock);
      atomicAdd(counters + 1, (unsigned long long)avoided);
    }
  }
}

__global__ void k_block_sizes(const int* b, int V, int* size) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) atomicAdd(size + b[v], 1);
}

__global__ void k_block_stats(BlockView bm, unsigned long long* out) {
  unsigned long long tr = 0, din = 0, prod = 0;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < bm.B; x += gridDim.x * blockDim.x) {
    tr += (unsigned long long)bm_get(bm, x, x);
    din += (unsigned long long)bm.d_in[x];
    prod += (unsigned long long)bm.d_out[x] * (unsigned long long)bm.d_in[x];
  }
  atomicAdd(out + 0, tr);
  atomicAdd(out + 1, din);
  atomicAdd(out + 2, prod);
}

__global__ void k_relabel(int* b, int V, const int* map) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) b[v] = map[b[v]];
}

}  // namespace sbpb
