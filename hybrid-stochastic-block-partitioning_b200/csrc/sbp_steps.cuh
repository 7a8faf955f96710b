// Per-element steps of the finetune apply and of entropy::mdl, shared by the single-graph
// kernels (sbp_kernels.cu) and the batched persistent kernel (sbp_batched.cu) so both run the
// same arithmetic in the same order.
#pragma once
#include "sbp_device.cuh"

namespace sbpb {

// Sum over the CTA's threads (deterministic: warp butterflies, then warps in order); the total
// is returned to thread 0.
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  __syncthreads();
  return t;
}

// M[row,col] += delta with the transpose kept in step: dense cells and both chunk sums, or the
// two hashed rows (atomic).
__device__ __forceinline__ void cell_add(const BlockView& bm, int row, int col, int delta) {
  if (bm.sparse) {
    hashed_add(bm.rbase, bm.rmask, bm.rslot, row, col, delta, bm.overflow, bm.overflow + 1);
    hashed_add(bm.cbase, bm.cmask, bm.cslot, col, row, delta, bm.overflow, bm.overflow + 1 + bm.B);
    return;
  }
  atomicAdd(bm.M + (size_t)row * bm.ld + col, delta);
  atomicAdd(bm.MT + (size_t)col * bm.ld + row, delta);
  chunk_add(bm.CS, bm.nch, row, col, delta);
  chunk_add(bm.CST, bm.nch, col, row, delta);
}

// Same for a dense cell owned by one thread (plain update of M/MT, atomic chunk sums, which
// lanes share); hashed rows are always updated atomically (lanes share their slots).
__device__ __forceinline__ void cell_add_owned(const BlockView& bm, int row, int col, int delta) {
  if (!delta) return;
  if (bm.sparse) {
    cell_add(bm, row, col, delta);
    return;
  }
  bm.M[(size_t)row * bm.ld + col] += delta;
  bm.MT[(size_t)col * bm.ld + row] += delta;
  chunk_add(bm.CS, bm.nch, row, col, delta);
  chunk_add(bm.CST, bm.nch, col, row, delta);
}

// Commit rule of a sequential Metropolis-Hastings round (finetune::metropolis_hastings,
// src/finetune.cpp:412-444, run speculatively): warps 0 .. avail-1 of the CTA evaluated list
// positions pos .. pos+avail-1 against the same state, with warp w's neighbour-block table in
// the CTA's shared tables.  The first accepted vertex (in list order) commits; everything
// before it was rejected against the true state.  On dense storage a later vertex keeps its
// result while no commit of the round could have touched what it read: a commit c changes
// cells in rows / columns r_c, s_c towards its neighbour blocks, and the degrees and d of r_c
// and s_c.  Vertex w read its neighbours' blocks (a neighbour that moved puts r_c among them),
// the row and column of its proposal's block t_w (-1: none), cells towards r_w, s_w and its
// neighbour blocks, and their degrees.  Marks s_commit; returns the number of positions the
// round visited.  Called by one thread.
__device__ __forceinline__ int mh_round_commits(const BlockView& bm, int* smem, int cap, int avail, const int* s_acc,
                                                const int* s_r, const int* s_s, const int* s_t, int* s_commit,
                                                int* first_out) {
  int first = -1;
  for (int w = 0; w < avail; ++w)
    if (s_acc[w]) {
      first = w;
      break;
    }
  int upto = first >= 0 ? first + 1 : avail;
  if (first >= 0) s_commit[first] = 1;
  if (first >= 0 && !bm.sparse) {
    int ncommit = 1;
    int cw[32];
    cw[0] = first;
    for (int w = first + 1; w < avail; ++w) {
      const WarpTable tw = carve_table(smem, cap, w);
      bool indep = true;
      for (int q = 0; q < ncommit && indep; ++q) {
        const int c = cw[q];
        const WarpTable tc = carve_table(smem, cap, c);
        const int rc = s_r[c], sc = s_s[c];
        const int rw = s_r[w], sw = s_s[w], tb = s_t[w];
        if (rc == rw || rc == sw || rc == tb || sc == rw || sc == sw || sc == tb) indep = false;
        else if (table_find(tw, rc) >= 0 || table_find(tw, sc) >= 0) indep = false;
        else if ((tb >= 0 && table_find(tc, tb) >= 0) || table_find(tc, rw) >= 0 || table_find(tc, sw) >= 0)
          indep = false;
      }
      if (!indep) break;
      upto = w + 1;
      if (s_acc[w]) {
        s_commit[w] = 1;
        cw[ncommit++] = w;
      }
    }
  }
  *first_out = first;
  return upto;
}

// One warp applies the committed move of v from r to s (Blockmodel::move_vertex,
// src/blockmodel/blockmodel.cpp:344-360) with the counts still in its table: lanes own distinct
// non-corner cells, lane 0 the four corner cells (r,r) (r,s) (s,r) (s,s), the assignment and
// the degrees.  When a hashed row runs out of room, lane 0 sets *stop and records in out[4..9]
// where the round stopped (list position stop_pos) and the move's diagonal deltas: the host
// rebuilds the rows with more room, sets d[r], d[s] from the rebuilt diagonal and these deltas,
// and resumes at stop_pos + 1.
__device__ __forceinline__ void mh_apply_move(const GraphView& g, const BlockView& bm, const WarpTable& t, int v, int r,
                                              int s, int k_out, int k_in, int lane, int stop_pos, double* out,
                                              int* stop) {
  const int self = g.self[v];
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
    const int d_rr = -mc.co_r - mc.ci_r - self;
    const int d_rs = -mc.co_s + mc.ci_r;
    const int d_sr = mc.co_r - mc.ci_s;
    const int d_ss = mc.co_s + mc.ci_s + self;
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
    if (*bm.overflow) {
      *stop = 1;
      out[4] = 1.0;
      out[5] = (double)stop_pos;
      out[6] = (double)r;
      out[7] = (double)s;
      out[8] = (double)d_rr;
      out[9] = (double)d_ss;
    } else {
      // Blockmodel::move_vertex reads the already-updated diagonal and adds the delta again
      bm.d[r] = bm.d_out[r] + bm.d_in[r] - (bm_get(bm, r, r) + d_rr);
      bm.d[s] = bm.d_out[s] + bm.d_in[s] - (bm_get(bm, s, s) + d_ss);
    }
  }
}

// Apply of one accepted move v: r -> prop[v] (Blockmodel::move_vertex, src/blockmodel/
// blockmodel.cpp:344-360, for a batch of simultaneous moves): M, MT and the chunk sums by edge,
// d_out / d_in, the quirk terms qr/qs of d[r], d[s] (the neighbours that are counted in the
// reference's sequential apply) and the batch's last mover of r and s.  One warp per vertex;
// lanes whose edges change the same cell add their count with one atomic.
__device__ __forceinline__ void apply_moved_vertex(const GraphView& g, const BlockView& bm, int v, const int* prop,
                                                   int* qr, int* qs, unsigned long long* last, unsigned gen,
                                                   int lane) {
  const int r = bm.b[v], s = prop[v];
  const int self = g.self[v];
  int cr = 0, cs = 0;
  const int o0 = g.out_ptr[v], o1 = g.out_ptr[v + 1];
  const int i0 = g.in_ptr[v], i1 = g.in_ptr[v + 1];
  const int k_out = o1 - o0, k = k_out + (i1 - i0);
  // One pass over the virtual neighbour list (out-edges, then in-edges), two elements per lane
  // in flight.  Out-edge v -> u (not the self loop): (r, b_u) -= 1 and (s, b'_u) += 1, b'_u the
  // block u moves to in this batch.  In-edge u -> v of a u that stays: (b_u, r) -= 1 and
  // (b_u, s) += 1 (a moving u's own out-edge covers the cell otherwise).
  for (int base = 0; base < k; base += 2 * kWarp) {
    int u[2], bo[2], pu[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = base + h * kWarp + lane;
      u[h] = j < k ? (j < k_out ? __ldg(g.out_idx + o0 + j) : __ldg(g.in_idx + i0 + (j - k_out))) : -1;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      bo[h] = u[h] >= 0 ? bm.b[u[h]] : -1;
      pu[h] = u[h] >= 0 ? prop[u[h]] : -1;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = base + h * kWarp + lane;
      const bool out_edge = j < k_out;
      int ko = -1, kn = -1, ks = -1;
      if (u[h] >= 0 && !(out_edge && u[h] == v)) {
        if (out_edge) {
          ko = bo[h];
          kn = pu[h] >= 0 ? pu[h] : bo[h];
        } else if (pu[h] < 0) {
          ks = bo[h];
        }
        const int ba = (pu[h] >= 0 && u[h] < v) ? pu[h] : bo[h];
        cr += (ba == r);
        cs += (ba == s);
      }
      const unsigned po = __match_any_sync(kFull, ko);
      if (ko >= 0 && (__ffs(po) - 1) == lane) cell_add(bm, r, ko, -__popc(po));
      const unsigned pn = __match_any_sync(kFull, kn);
      if (kn >= 0 && (__ffs(pn) - 1) == lane) cell_add(bm, s, kn, __popc(pn));
      const unsigned pb = __match_any_sync(kFull, ks);
      if (ks >= 0 && (__ffs(pb) - 1) == lane) {
        const int c = __popc(pb);
        cell_add(bm, ks, r, -c);
        cell_add(bm, ks, s, c);
      }
    }
  }
  cr = warp_sum_int(cr);
  cs = warp_sum_int(cs);
  if (lane == 0) {
    if (self) {
      cell_add(bm, r, r, -1);
      cell_add(bm, s, s, 1);
    }
    const int k_in_self = (i1 - i0) + self;
    atomicAdd(bm.d_out + r, -k_out);
    atomicAdd(bm.d_out + s, k_out);
    atomicAdd(bm.d_in + r, -k_in_self);
    atomicAdd(bm.d_in + s, k_in_self);
    qr[v] = -(cr + self);
    qs[v] = cs + self;
    const unsigned long long key = ((unsigned long long)gen << 32) | (unsigned)v;
    atomicMax(last + r, key);
    atomicMax(last + s, key);
  }
}

// d[r], d[s] from the last mover of each block, then the new assignment of v.
__device__ __forceinline__ void finish_moved_vertex(const BlockView& bm, int v, int* prop, const int* qr,
                                                    const int* qs, const unsigned long long* last, unsigned gen) {
  const int r = bm.b[v], s = prop[v];
  const unsigned long long key = ((unsigned long long)gen << 32) | (unsigned)v;
  if (last[r] == key) bm.d[r] = bm.d_out[r] + bm.d_in[r] - bm_get(bm, r, r) - qr[v];
  if (last[s] == key) bm.d[s] = bm.d_out[s] + bm.d_in[s] - bm_get(bm, s, s) - qs[v];
  bm.b[v] = s;
  prop[v] = -1;
}

// MDL: L = sum_cells g(M) - sum g(d_out) - sum g(d_in); mdl = E h(B^2/E) + V log B - L.
// Deterministic two-pass reduction: partial cta of ncta CTAs of 256 threads (elements in
// grid-stride order), then the partials summed in a fixed order.
__device__ __forceinline__ double mdl_cells_part(const BlockView& bm, int cta, int ncta, double* red) {
  double acc = 0.0;
  const long long BB = (long long)bm.B * bm.B;
  const long long stride = (long long)ncta * blockDim.x;
  for (long long i = (long long)cta * blockDim.x + threadIdx.x; i < BB; i += stride) {
    const int row = (int)(i / bm.B), col = (int)(i - (long long)row * bm.B);
    const int m = bm.M[(size_t)row * bm.ld + col];
    if (m > 0) acc += xlogx((double)m);
  }
  for (long long x = (long long)cta * blockDim.x + threadIdx.x; x < bm.B; x += stride)
    acc -= xlogx((double)bm.d_out[x]) + xlogx((double)bm.d_in[x]);
  return block_sum(acc, red);
}

// Edge form: sum_cells M log M = sum over edges of log M[b_src, b_dst].
__device__ __forceinline__ double mdl_edges_part(const GraphView& g, const BlockView& bm, const int* out_src, int cta,
                                                 int ncta, double* red) {
  double acc = 0.0;
  const long long stride = (long long)ncta * blockDim.x;
  for (long long e = (long long)cta * blockDim.x + threadIdx.x; e < g.E; e += stride) {
    const int bv = bm.b[__ldg(out_src + e)], bu = bm.b[__ldg(g.out_idx + e)];
    acc += log((double)bm_get(bm, bv, bu));
  }
  for (long long x = (long long)cta * blockDim.x + threadIdx.x; x < bm.B; x += stride)
    acc -= xlogx((double)bm.d_out[x]) + xlogx((double)bm.d_in[x]);
  return block_sum(acc, red);
}

__device__ __forceinline__ double mdl_final_value(const double* partial, int n, int V, long long E, int B,
                                                  double* red) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += __ldcg(partial + i);
  const double L = block_sum(acc, red);
  const double x = pow((double)B, 2) / (double)E;
  const double h = ((1 + x) * log(1 + x)) - (x * log(x));
  return ((double)E * h) + ((double)V * log((double)B)) - L;
}

}  // namespace sbpb
