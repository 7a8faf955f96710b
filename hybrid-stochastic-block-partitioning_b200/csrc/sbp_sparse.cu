// Kernels of the row-hashed (sparse) block matrix used when B is large: rebuild from the edge
// list (Blockmodel::initialize_edge_counts, src/blockmodel/blockmodel.cpp:187-255, through a
// sort of (b_src, b_dst) keys), and the repair steps after a hashed row ran out of room.
#include "sbp_kernels.cuh"

namespace sbpb {

// (b[src], b[dst]) and (b[dst], b[src]) keys of every edge.
__global__ void k_edge_keys(GraphView g, const int* __restrict__ b, const int* __restrict__ out_src, int B,
                            unsigned long long* keys, unsigned long long* keysT) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.E; e += stride) {
    const unsigned long long bs = (unsigned)b[__ldg(out_src + e)], bd = (unsigned)b[__ldg(g.out_idx + e)];
    keys[e] = bs * (unsigned long long)B + bd;
    keysT[e] = bd * (unsigned long long)B + bs;
  }
}

// Non-zero cells per row from the unique sorted keys.
__global__ void k_unique_rows(const unsigned long long* __restrict__ ukeys, long long n, int B, unsigned* rowcnt) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
    atomicAdd(rowcnt + (ukeys[j] / (unsigned long long)B), 1u);
}

// Row capacity: a power of two of at least factor * cells + 4 factor slots (room to grow: at
// large B most moves add cells, and a full row has to be regrown).  Rows of more than 128
// cells get at most factor 2: the hashed walk reads a row's whole region, and for long rows
// that costs more than the occasional regrowth.
__global__ void k_row_caps(const unsigned* __restrict__ rowcnt, int B, unsigned factor, unsigned* cap, int* mask) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < B; r += gridDim.x * blockDim.x) {
    const unsigned f = rowcnt[r] > 128u && factor > 2u ? 2u : factor;
    unsigned want = f * rowcnt[r] + 4u * f, c = 8u;
    while (c < want) c <<= 1;
    cap[r] = c;
    mask[r] = (int)c - 1;
  }
}

__global__ void k_fill_empty(int2* slot, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    slot[i] = make_int2(-1, 0);
}

// One thread per row inserts its cells in ascending column order, so the slot layout of a
// rebuilt row is the same on every run.  Also writes the compressed (sorted) row.
__global__ void k_fill_rows(const long long* __restrict__ rowptr, const unsigned long long* __restrict__ ukeys,
                            const long long* __restrict__ heads, long long nu, long long nedges, int B,
                            const long long* __restrict__ base, const int* __restrict__ mask, int2* slot,
                            int* csr_ptr, int* csr_idx, int* csr_val) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < B; r += gridDim.x * blockDim.x) {
    const long long j0 = rowptr[r], j1 = (r + 1 < B) ? rowptr[r + 1] : nu;
    csr_ptr[r] = (int)j0;
    if (r == B - 1) csr_ptr[B] = (int)nu;
    const long long b0 = base[r];
    const int m = mask[r];
    for (long long j = j0; j < j1; ++j) {
      const int col = (int)(ukeys[j] % (unsigned long long)B);
      const int cnt = (int)(((j + 1 < nu) ? heads[j + 1] : nedges) - heads[j]);
      csr_idx[j] = col;
      csr_val[j] = cnt;
      unsigned h = slot_hash(col) & (unsigned)m;
      while (slot[b0 + h].x != -1) h = (h + 1) & (unsigned)m;   // capacity >= 2 * count + 8
      slot[b0 + h] = make_int2(col, cnt);
    }
  }
}

// Compressed rows only (no hashed slots): the merge step of a large dense blockmodel, whose B x B
// matrix is too large to scan for its non-zero cells.
__global__ void k_fill_csr(const long long* __restrict__ rowptr, const unsigned long long* __restrict__ ukeys,
                           const long long* __restrict__ heads, long long nu, long long nedges, int B, int* csr_ptr,
                           int* csr_idx, int* csr_val) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < B; r += gridDim.x * blockDim.x) {
    const long long j0 = rowptr[r], j1 = (r + 1 < B) ? rowptr[r + 1] : nu;
    csr_ptr[r] = (int)j0;
    if (r == B - 1) csr_ptr[B] = (int)nu;
    for (long long j = j0; j < j1; ++j) {
      csr_idx[j] = (int)(ukeys[j] % (unsigned long long)B);
      csr_val[j] = (int)(((j + 1 < nu) ? heads[j + 1] : nedges) - heads[j]);
    }
  }
}

// Regrowth of the hashed rows that ran out of room (one side: rows of M or of MT).  A flagged
// row x gets a region of the power of two at least twice its old room and at least
// 2 min(deg[x], B) + 16 slots, taken after the `top` slots in use; with no room left below
// `limit` the step reports it and changes nothing for that row.
__global__ void k_regrow_alloc(const int* __restrict__ full, const int* __restrict__ deg, int B, long long top,
                               long long limit, unsigned long long* used, unsigned long long* nrows, long long* base,
                               int* mask, int* list, unsigned long long* no_room) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < B; x += gridDim.x * blockDim.x) {
    if (!full[x]) continue;
    const long long need = 2LL * (long long)min(deg[x], B) + 16;
    long long cap = 2LL * ((long long)mask[x] + 1);
    while (cap < need) cap <<= 1;
    const unsigned long long off = atomicAdd(used, (unsigned long long)cap);
    if (cap > (1LL << 30) || top + (long long)off + cap > limit) {
      atomicOr(no_room, 1ull);
      continue;
    }
    base[x] = top + (long long)off;
    mask[x] = (int)(cap - 1);
    list[atomicAdd(nrows, 1ull)] = x;
  }
}

// Empty slots in the new regions (one CTA per listed row).
__global__ void k_regrow_clear(const int* __restrict__ list, int n, const long long* __restrict__ base,
                               const int* __restrict__ mask, int2* slot) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int x = list[i];
    const long long b0 = base[x];
    const int cap = mask[x] + 1;
    for (int j = threadIdx.x; j < cap; j += blockDim.x) slot[b0 + j] = make_int2(-1, 0);
  }
}

// Recount the regrown rows: every edge (b_src, b_dst) adds one to row b_src of M when that row
// is flagged and to row b_dst of MT when that one is (the new regions cannot run out of room).
__global__ void k_regrow_fill(GraphView g, BlockView bm, const int* __restrict__ out_src) {
  const int* full_r = bm.overflow + 1;
  const int* full_c = bm.overflow + 1 + bm.B;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.E; e += stride) {
    const int bs = bm.b[__ldg(out_src + e)], bd = bm.b[__ldg(g.out_idx + e)];
    if (full_r[bs]) hashed_add(bm.rbase, bm.rmask, bm.rslot, bs, bd, 1, bm.overflow, bm.overflow + 1);
    if (full_c[bd]) hashed_add(bm.cbase, bm.cmask, bm.cslot, bd, bs, 1, bm.overflow, bm.overflow + 1 + bm.B);
  }
}

// Block degrees from the vertices (out-degree; in-degree with the self loop).
__global__ void k_block_degrees(GraphView g, const int* __restrict__ b, int* d_out, int* d_in) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < g.V; v += gridDim.x * blockDim.x) {
    const int bv = b[v];
    atomicAdd(d_out + bv, g.out_ptr[v + 1] - g.out_ptr[v]);
    atomicAdd(d_in + bv, (g.in_ptr[v + 1] - g.in_ptr[v]) + g.self[v]);
  }
}

// Gibbs batch whose apply overflowed a row: move the assignment now (keeping the old block),
// so the rows can be rebuilt from it before the degree step.
__global__ void k_recover_assign(int* b, const int* moved, const int* n_moved, const int* prop, int* old_block) {
  const int n = *n_moved;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = moved[i];
    old_block[v] = b[v];
    b[v] = prop[v];
  }
}

// The degree step of k_apply_finish on the rebuilt rows.
__global__ void k_recover_finish(BlockView bm, const int* moved_list, const int* n_moved, int* next_n_moved,
                                 int* prop, const int* old_block, const int* qr, const int* qs,
                                 const unsigned long long* last, unsigned gen) {
  const int n = *n_moved;
  if (blockIdx.x == 0 && threadIdx.x == 0) *next_n_moved = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = moved_list[i];
    const int r = old_block[v], s = prop[v];
    const unsigned long long key = ((unsigned long long)gen << 32) | (unsigned)v;
    if (last[r] == key) bm.d[r] = bm.d_out[r] + bm.d_in[r] - bm_get(bm, r, r) - qr[v];
    if (last[s] == key) bm.d[s] = bm.d_out[s] + bm.d_in[s] - bm_get(bm, s, s) - qs[v];
    prop[v] = -1;
  }
}

// d[r], d[s] of one move (Blockmodel::move_vertex) after its rows were rebuilt.
__global__ void k_fix_move_degrees(BlockView bm, int r, int s, int d_rr, int d_ss) {
  if (threadIdx.x || blockIdx.x) return;
  bm.d[r] = bm.d_out[r] + bm.d_in[r] - (bm_get(bm, r, r) + d_rr);
  bm.d[s] = bm.d_out[s] + bm.d_in[s] - (bm_get(bm, s, s) + d_ss);
}

// Dense dump of the hashed rows of M (for sbp_get_block_matrix): one thread per slot.
__global__ void k_hashed_to_dense(const long long* __restrict__ base, const int* __restrict__ mask,
                                  const int2* __restrict__ slot, int B, int row0, int rows, int* dense) {
  for (int r = row0 + blockIdx.x; r < row0 + rows && r < B; r += gridDim.x) {
    const long long b0 = base[r];
    const int cap = mask[r] + 1;
    for (int i = threadIdx.x; i < cap; i += blockDim.x) {
      const int2 e = slot[b0 + i];
      if (e.x >= 0) dense[(size_t)(r - row0) * B + e.x] = e.y;
    }
  }
}

}  // namespace sbpb
