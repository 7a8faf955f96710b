// Host side of the B200 stochastic block partitioning engine: device-resident graph and
// blockmodel handles, the finetune / merge / partition drivers and the C ABI declared in
// include/sbp_b200.h.  Control flow mirrors the reference driver (src/sbp.cpp:61-112,
// src/blockmodel/blockmodel_triplet.cpp:3-100, src/finetune.cpp:31-162,342-444,
// src/block_merge.cpp:123-311); all per-vertex and per-block work runs in the kernels of
// sbp_kernels.cu.  No CPU fallback: every compute entry point needs a CUDA device.
#include "sbp_engine.cuh"


namespace sbpb {

static thread_local char g_last_error[512];

void set_last_error(const char* msg) {
  std::snprintf(g_last_error, sizeof g_last_error, "%s", msg ? msg : "");
}
const char* last_error() { return g_last_error; }

// Scratch of the sparse rebuild (grow-only, shared by all blockmodels).
struct SortScratch {
  DevBuf<unsigned long long> keys, keysT, tmp, ukeys, partial;
  DevBuf<unsigned> hist, flags, rowcnt, caps;
  DevBuf<long long> pos, heads, rowptr;
};
static thread_local SortScratch g_sort;   // per host thread (the batched partitioner merges on several)

// 0..n-1 ordered by key ascending, equal keys by index: the order of std::stable_sort on the
// indices with `key[a] < key[b]`, from an LSD radix sort (16-bit digits) of order-preserving
// 64-bit images of the keys (-0.0 taken as +0.0, which compares equal).  With a NaN key (no
// strict weak order) it is std::stable_sort itself.  A 200,000-key sort takes a few ms instead
// of about 20.
static std::vector<int> stable_order_by(const std::vector<double>& key) {
  const size_t n = key.size();
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::vector<unsigned long long> img(n);
  for (size_t i = 0; i < n; ++i) {
    double x = key[i];
    if (std::isnan(x)) {
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
      return order;
    }
    if (x == 0.0) x = 0.0;
    unsigned long long bits;
    std::memcpy(&bits, &x, sizeof bits);
    img[i] = (bits >> 63) ? ~bits : (bits | (1ull << 63));
  }
  std::vector<int> tmp(n);
  std::vector<unsigned> count(1u << 16);
  for (int shift = 0; shift < 64; shift += 16) {
    std::fill(count.begin(), count.end(), 0u);
    for (size_t i = 0; i < n; ++i) count[(img[i] >> shift) & 0xffff]++;
    if (n > 0 && count[(img[0] >> shift) & 0xffff] == n) continue;   // one digit value: order unchanged
    unsigned run = 0;
    for (auto& c : count) {
      const unsigned k = c;
      c = run;
      run += k;
    }
    for (size_t i = 0; i < n; ++i) {
      const int o = order[i];
      tmp[count[(img[o] >> shift) & 0xffff]++] = o;
    }
    order.swap(tmp);
  }
  return order;
}

static int key_bits(int B) {
  const unsigned long long maxkey = (unsigned long long)B * (unsigned long long)B;
  int bits = 1;
  while (bits < 64 && (1ull << bits) < maxkey) ++bits;
  return bits;
}

// One orientation of the sparse rebuild: sort keys, unique them, size the rows, fill them.
static void rebuild_hashed_side(SbpBlockmodel& bm, long long E, unsigned long long* keys, DevBuf<long long>& base,
                                DevBuf<int>& mask, DevBuf<int2>& slot, DevBuf<int>& cptr, DevBuf<int>& cidx,
                                DevBuf<int>& cval, long long* top, long long* limit) {
  Context& c = Context::get();
  const int B = bm.B;
  long long nu = 0;
  unsigned long long* sorted = keys;
  if (E > 0) {
    radix_sort_u64(keys, g_sort.tmp.p, E, key_bits(B), g_sort.hist.p, g_sort.partial.p, c.num_sms, c.stream, &sorted);
    rle(sorted, E, g_sort.flags.p, g_sort.pos.p, g_sort.ukeys.p, g_sort.heads.p, g_sort.partial.p, c.num_sms, c.stream);
    long long lastpos = 0;
    unsigned lastflag = 0;
    SBP_CUDA(SBP_COPY_ASYNC(&lastpos, g_sort.pos.p + E - 1, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(&lastflag, g_sort.flags.p + E - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
    SBP_CHECK_LAUNCH();
    c.sync();
    nu = lastpos + lastflag;
  }
  SBP_CUDA(cudaMemsetAsync(g_sort.rowcnt.p, 0, B * sizeof(unsigned), c.stream));
  if (nu > 0) {
    k_unique_rows<<<grid_for(nu, 256, 8 * c.num_sms), 256, 0, c.stream>>>(g_sort.ukeys.p, nu, B, g_sort.rowcnt.p);
    SBP_CHECK_LAUNCH();
  }
  exclusive_scan_u32(g_sort.rowcnt.p, g_sort.rowptr.p, B, g_sort.partial.p, c.num_sms, c.stream);
  k_row_caps<<<grid_for(B, 256, 8 * c.num_sms), 256, 0, c.stream>>>(g_sort.rowcnt.p, B, (unsigned)g_hashed_row_factor,
                                                                   g_sort.caps.p, mask.p);
  exclusive_scan_u32(g_sort.caps.p, base.p, B, g_sort.partial.p, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  long long lastbase = 0;
  unsigned lastcap = 0;
  SBP_CUDA(SBP_COPY_ASYNC(&lastbase, base.p + B - 1, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(&lastcap, g_sort.caps.p + B - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  const long long total = lastbase + lastcap;
  // half as many slots again stay free for rows that outgrow their region (regrow_hashed)
  slot.reserve(total + total / 2 + 4096);
  *top = total;
  *limit = (long long)slot.n;
  cptr.reserve(B + 1);
  cidx.reserve(std::max(nu, 1LL));
  cval.reserve(std::max(nu, 1LL));
  k_fill_empty<<<grid_for(total, 256, 16 * c.num_sms), 256, 0, c.stream>>>(slot.p, total);
  k_fill_rows<<<grid_for(B, 128, 16 * c.num_sms), 128, 0, c.stream>>>(g_sort.rowptr.p, g_sort.ukeys.p, g_sort.heads.p,
                                                                     nu, E, B, base.p, mask.p, slot.p, cptr.p,
                                                                     cidx.p, cval.p);
  SBP_CHECK_LAUNCH();
}

// Compressed rows of M (or of MT, keys of the transposed edges) from the sorted (b_src, b_dst)
// keys of the edges, ascending by column: the merge step's outgoing / incoming edge views of a
// dense blockmodel too large to scan cell by cell.
static void sorted_rows(const SbpBlockmodel& bm, long long E, unsigned long long* keys, DevBuf<int>& cptr,
                        DevBuf<int>& cidx, DevBuf<int>& cval) {
  Context& c = Context::get();
  const int B = bm.B;
  long long nu = 0;
  if (E > 0) {
    unsigned long long* sorted = keys;
    radix_sort_u64(keys, g_sort.tmp.p, E, key_bits(B), g_sort.hist.p, g_sort.partial.p, c.num_sms, c.stream, &sorted);
    rle(sorted, E, g_sort.flags.p, g_sort.pos.p, g_sort.ukeys.p, g_sort.heads.p, g_sort.partial.p, c.num_sms, c.stream);
    long long lastpos = 0;
    unsigned lastflag = 0;
    SBP_CUDA(SBP_COPY_ASYNC(&lastpos, g_sort.pos.p + E - 1, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(&lastflag, g_sort.flags.p + E - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
    SBP_CHECK_LAUNCH();
    c.sync();
    nu = lastpos + lastflag;
  }
  SBP_CUDA(cudaMemsetAsync(g_sort.rowcnt.p, 0, B * sizeof(unsigned), c.stream));
  if (nu > 0) {
    k_unique_rows<<<grid_for(nu, 256, 8 * c.num_sms), 256, 0, c.stream>>>(g_sort.ukeys.p, nu, B, g_sort.rowcnt.p);
    SBP_CHECK_LAUNCH();
  }
  exclusive_scan_u32(g_sort.rowcnt.p, g_sort.rowptr.p, B, g_sort.partial.p, c.num_sms, c.stream);
  cptr.reserve(B + 1);
  cidx.reserve(std::max(nu, 1LL));
  cval.reserve(std::max(nu, 1LL));
  k_fill_csr<<<grid_for(B, 128, 16 * c.num_sms), 128, 0, c.stream>>>(g_sort.rowptr.p, g_sort.ukeys.p, g_sort.heads.p,
                                                                    nu, E, B, cptr.p, cidx.p, cval.p);
  SBP_CHECK_LAUNCH();
}

static void reserve_sort_scratch(long long E, int B) {
  Context& c = Context::get();
  g_sort.keys.reserve(std::max(E, 1LL));
  g_sort.keysT.reserve(std::max(E, 1LL));
  g_sort.tmp.reserve(std::max(E, 1LL));
  g_sort.ukeys.reserve(std::max(E, 1LL));
  g_sort.flags.reserve(std::max(E, 1LL));
  g_sort.pos.reserve(std::max(E, 1LL));
  g_sort.heads.reserve(std::max(E, 1LL));
  g_sort.hist.reserve(radix_hist_capacity(std::max(E, 1LL), c.num_sms));
  g_sort.partial.reserve(scan_partial_capacity(c.num_sms));
  g_sort.rowcnt.reserve(B);
  g_sort.caps.reserve(B);
  g_sort.rowptr.reserve(B);
}

// Sparse Blockmodel::initialize_edge_counts: rows of M and MT from sorted (b_src, b_dst) keys.
static void rebuild_sparse(SbpBlockmodel& bm, const SbpGraph& g, bool recompute_d) {
  Context& c = Context::get();
  const long long E = g.E;
  const int B = bm.B;
  reserve_sort_scratch(E, B);
  SBP_CUDA(cudaMemsetAsync(bm.d_out.p, 0, B * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.d_in.p, 0, B * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.overflow.p, 0, (1 + 2 * (size_t)B) * sizeof(int), c.stream));
  k_block_degrees<<<grid_for(g.V, 256, 8 * c.num_sms), 256, 0, c.stream>>>(g.view(), bm.b.p, bm.d_out.p, bm.d_in.p);
  if (E > 0)
    k_edge_keys<<<grid_for(E, 256, 16 * c.num_sms), 256, 0, c.stream>>>(g.view(), bm.b.p, g.out_src.p, B,
                                                                       g_sort.keys.p, g_sort.keysT.p);
  SBP_CHECK_LAUNCH();
  rebuild_hashed_side(bm, E, g_sort.keys.p, bm.rbase, bm.rmask, bm.rslot, bm.csr_rptr, bm.csr_ridx, bm.csr_rval,
                      &bm.rtop, &bm.rlimit);
  rebuild_hashed_side(bm, E, g_sort.keysT.p, bm.cbase, bm.cmask, bm.cslot, bm.csr_cptr, bm.csr_cidx, bm.csr_cval,
                      &bm.ctop, &bm.climit);
  if (recompute_d) {
    k_rebuild_degrees<<<grid_for(B, 256, 1 << 20), 256, 0, c.stream>>>(bm.view());
    SBP_CHECK_LAUNCH();
  }
}

// Blockmodel::initialize_edge_counts (src/blockmodel/blockmodel.cpp:187-255).  recompute_d =
// false keeps d (the reference's drifting block degree) when only the storage is rebuilt.
void rebuild(SbpBlockmodel& bm, const SbpGraph& g, bool recompute_d) {
  if (bm.sparse) {
    rebuild_sparse(bm, g, recompute_d);
    return;
  }
  Context& c = Context::get();
  const size_t cells = (size_t)bm.B * (size_t)bm.ld;
  SBP_CUDA(cudaMemsetAsync(bm.M.p, 0, cells * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.MT.p, 0, cells * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.CS.p, 0, (size_t)bm.B * bm.nch * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.CST.p, 0, (size_t)bm.B * bm.nch * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.d_out.p, 0, bm.B * sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm.d_in.p, 0, bm.B * sizeof(int), c.stream));
  if (g.V > 0) {
    if (bm.B <= kSmemRebuildMaxB) {   // B*B ints fit the default 48 KB of shared memory
      k_rebuild_smem<<<grid_for(g.V, 256, c.num_sms), 256, (size_t)bm.B * bm.B * sizeof(int), c.stream>>>(
          g.view(), bm.view());
    } else {
      k_rebuild_global<<<grid_for(g.V, 256, 8 * c.num_sms), 256, 0, c.stream>>>(g.view(), bm.view());
    }
    SBP_CHECK_LAUNCH();
  }
  k_rebuild_degrees<<<grid_for(bm.B, 256, 1 << 20), 256, 0, c.stream>>>(bm.view());
  SBP_CHECK_LAUNCH();
}

// A Gibbs apply ran out of room in some hashed rows (their flags are set): give each such row
// a new region after the slots in use, sized from its block's degree (a row of M has at most
// min(d_out, B) cells, a row of MT at most min(d_in, B)), and recount it from the edges and the
// assignment, which already carries the batch's moves.  Rows that did not run out of room took
// every update of the batch and stay as they are.  Costs one pass over the edges instead of a
// full rebuild; returns false (and changes nothing) when the slot arrays have no room left.
static thread_local DevBuf<int> g_regrow_list;
static thread_local DevBuf<unsigned long long> g_regrow_ctr;   // [0, 1] slots taken per side, [2, 3] rows per side, [4] no room

static bool regrow_hashed(SbpBlockmodel& bm, const SbpGraph& g) {
  Context& c = Context::get();
  const int B = bm.B;
  g_regrow_list.reserve(2 * (size_t)B);
  g_regrow_ctr.reserve(5);
  SBP_CUDA(cudaMemsetAsync(g_regrow_ctr.p, 0, 5 * sizeof(unsigned long long), c.stream));
  int* full_r = bm.overflow.p + 1;
  int* full_c = bm.overflow.p + 1 + B;
  const int grid = grid_for(B, 256, 16 * c.num_sms);
  k_regrow_alloc<<<grid, 256, 0, c.stream>>>(full_r, bm.d_out.p, B, bm.rtop, bm.rlimit, g_regrow_ctr.p,
                                             g_regrow_ctr.p + 2, bm.rbase.p, bm.rmask.p, g_regrow_list.p,
                                             g_regrow_ctr.p + 4);
  k_regrow_alloc<<<grid, 256, 0, c.stream>>>(full_c, bm.d_in.p, B, bm.ctop, bm.climit, g_regrow_ctr.p + 1,
                                             g_regrow_ctr.p + 3, bm.cbase.p, bm.cmask.p, g_regrow_list.p + B,
                                             g_regrow_ctr.p + 4);
  SBP_CHECK_LAUNCH();
  unsigned long long h[5];
  SBP_CUDA(SBP_COPY_ASYNC(h, g_regrow_ctr.p, sizeof h, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  if (h[4]) return false;
  bm.rtop += (long long)h[0];
  bm.ctop += (long long)h[1];
  if (h[2]) k_regrow_clear<<<4 * c.num_sms, 256, 0, c.stream>>>(g_regrow_list.p, (int)h[2], bm.rbase.p, bm.rmask.p,
                                                                 bm.rslot.p);
  if (h[3]) k_regrow_clear<<<4 * c.num_sms, 256, 0, c.stream>>>(g_regrow_list.p + B, (int)h[3], bm.cbase.p,
                                                                 bm.cmask.p, bm.cslot.p);
  if (g.E > 0)
    k_regrow_fill<<<grid_for(g.E, 256, 16 * c.num_sms), 256, 0, c.stream>>>(g.view(), bm.view(), g.out_src.p);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(cudaMemsetAsync(bm.overflow.p, 0, (1 + 2 * (size_t)B) * sizeof(int), c.stream));
  return true;
}

// After a sweep in which hashed rows were regrown: rebuild every row from the assignment
// (keeping d), which drops the cells whose count went back to 0 and sizes each row for its
// current cells again.  Regrowth alone keeps a batch going; without this the rows fill up with
// dead cells, probe chains grow and nearly every batch overflows.
void tidy_hashed(SbpBlockmodel& bm, const SbpGraph& g, long long overflows_before) {
  if (bm.sparse && g_overflow_rebuilds > overflows_before) rebuild(bm, g, false);
}

// entropy::mdl (src/entropy.cpp:584-589).
double mdl(SbpBlockmodel& bm, const SbpGraph& g) {
  Context& c = Context::get();
  const int cells = !bm.sparse && (long long)bm.B * bm.B <= 4LL * g.E;
  k_mdl<<<c.npartial, 256, 0, c.stream>>>(g.view(), bm.view(), g.out_src.p, cells, c.partial, c.done, c.scalar,
                                         nullptr, 0);
  SBP_CHECK_LAUNCH();
  double out = 0.0;
  SBP_CUDA(SBP_COPY_ASYNC(&out, c.scalar, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return out;
}

// finetune::early_stop (src/finetune.cpp:144-162).
bool early_stop(int iteration, bool bracket, double initial_entropy, const std::vector<double>& deltas) {
  const size_t last = deltas.size() - 1;
  if (deltas[last] == 0.0) return true;
  if (iteration < 3) return false;
  double average = deltas[last] + deltas[last - 1] + deltas[last - 2];
  average /= -3.0;
  const double threshold = bracket ? 1e-4 * initial_entropy : 5e-4 * initial_entropy;
  return average < threshold;
}

int mh_cap(int max_k) {
  int cap = pow2_at_least(std::max(2 * max_k, kLightCap));
  if (cap > kMaxCap) throw Error(SBP_ERR_UNSUPPORTED, "vertex degree too large for the Metropolis-Hastings kernel");
  return cap;
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes` (never lowers it: another host
// thread may be about to launch the kernel with a larger request).
void set_smem_limit(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::unordered_map<const void*, size_t> limit;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[fn];
  if (bytes <= cur) return;
  SBP_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
}

// One sequential Metropolis-Hastings pass over verts (device list of n vertices).
MhResult mh_pass(SbpBlockmodel& bm, const SbpGraph& g, const int* verts, int n, int max_k, RngParams rng,
                        int sweep) {
  Context& c = Context::get();
  MhResult res;
  if (n == 0) return res;
  if (use_group_kernel(bm) && (bm.B <= kSmallB || 2 * max_k <= g.light_cap)) {
    // rounds of one vertex per lane group (every vertex of the list fits the group tables)
    const bool hashed_table = bm.B > kSmallB;
    const int cap = g.light_cap;
    const size_t smem = mh_group_smem(hashed_table, cap);
    if (smem <= kSmemBudget) {
      const MhGroupKernel k = mh_group_kernel(hashed_table);
      set_smem_limit((const void*)k, smem);
      k<<<1, kMhGroupThreads, smem, c.stream>>>(g.view(), bm.view(), verts, n, rng, sweep, cap, c.mh_out, c.status);
      SBP_CHECK_LAUNCH();
      double out[4];
      SBP_CUDA(SBP_COPY_ASYNC(out, c.mh_out, sizeof(out), cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      res.visits = (long long)out[0];
      res.moved = (long long)out[1];
      res.accepted = (long long)out[2];
      res.sum_dS = out[3];
      return res;
    }
  }
  const int cap = mh_cap(max_k);
  const size_t per_warp = (size_t)table_ints(cap) * sizeof(int);
  int W = (int)std::min<size_t>(16, kSmemBudget / per_warp);
  if (W < 1) throw Error(SBP_ERR_UNSUPPORTED, "vertex degree too large for the Metropolis-Hastings kernel");
  const size_t smem = per_warp * W;
  set_smem_limit((const void*)k_mh, smem);
  int start = 0;
  while (start < n) {
    k_mh<<<1, W * 32, smem, c.stream>>>(g.view(), bm.view(), verts, n, start, rng, sweep, cap, c.mh_out, c.status);
    SBP_CHECK_LAUNCH();
    double out[10];
    SBP_CUDA(SBP_COPY_ASYNC(out, c.mh_out, sizeof(out), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    res.visits += (long long)out[0];
    res.moved += (long long)out[1];
    res.accepted += (long long)out[2];
    res.sum_dS += out[3];
    if (out[4] == 0.0) break;
    // a hashed row ran out of room at list position out[5]: rebuild the rows with more room
    // (keeping d), finish that move's d[r], d[s] and resume after it
    rebuild(bm, g, false);
    ++g_overflow_rebuilds;
    k_fix_move_degrees<<<1, 1, 0, c.stream>>>(bm.view(), (int)out[6], (int)out[7], (int)out[8], (int)out[9]);
    SBP_CHECK_LAUNCH();
    start = (int)out[5] + 1;
  }
  return res;
}

// One asynchronous-Gibbs batch: evaluate every vertex of the batch, then apply the moves.
void gibbs_batch(SbpBlockmodel& bm, const SbpGraph& g, const BatchPlan& plan, int bt, RngParams rng,
                        int sweep) {
  Context& c = Context::get();
  const int nl = plan.light_n[bt], nh = plan.heavy_n[bt];
  int* n_cur = bm.n_moved.p + (bm.gen & 1);
  const GibbsEvalKernel k_eval = gibbs_eval_kernel(bm.sparse, bm.B);
  if (nl > 0) {
    const bool small = use_group_kernel(bm);
    const size_t smem = (size_t)table_ints(g.light_cap) * sizeof(int) * kLightWarps;
    set_smem_limit((const void*)k_eval, smem);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (g_prof.on) {
      e0 = g_prof.get();
      e1 = g_prof.get();
      SBP_CUDA(cudaEventRecord(e0, c.stream));
    }
    if (small) {
      // direct-indexed tables take every light vertex; hashed ones those of k <= kGroupMaxK, the
      // warp kernel the rest
      const int ng = bm.B <= kSmallB ? nl : plan.group_n[bt];
      if (ng > 0)
        launch_group_eval(g, bm, plan.order.p + plan.light_begin[bt], ng, rng, sweep, n_cur, nullptr, 0, c.stream);
      if (nl > ng)
        k_eval<<<grid_for(nl - ng, kLightWarps, 64 * c.num_sms), kLightWarps * 32, smem, c.stream>>>(
            g.view(), bm.view(), plan.order.p + plan.light_begin[bt] + ng, nl - ng, rng, sweep, bm.prop.p,
            bm.moved.p, n_cur, c.counters, g.light_cap, c.status, nullptr, 0);
    } else {
      k_eval<<<grid_for(nl, kLightWarps, 64 * c.num_sms), kLightWarps * 32, smem, c.stream>>>(
          g.view(), bm.view(), plan.order.p + plan.light_begin[bt], nl, rng, sweep, bm.prop.p, bm.moved.p, n_cur,
          c.counters, g.light_cap, c.status, nullptr, 0);
    }
    SBP_CHECK_LAUNCH();
    if (g_prof.on) {
      SBP_CUDA(cudaEventRecord(e1, c.stream));
      g_prof.add(e0, e1, nl, plan.light_bytes[bt]);
    }
  }
  if (nh > 0) {
    const size_t smem = (size_t)table_ints(g.heavy_cap) * sizeof(int);
    set_smem_limit((const void*)k_eval, std::max(smem, (size_t)table_ints(g.light_cap) * sizeof(int) * kLightWarps));
    k_eval<<<grid_for(nh, 1, 64 * c.num_sms), 32, smem, c.stream>>>(
        g.view(), bm.view(), plan.order.p + plan.heavy_begin[bt], nh, rng, sweep, bm.prop.p, bm.moved.p, n_cur,
        c.counters, g.heavy_cap, c.status, nullptr, 0);
    SBP_CHECK_LAUNCH();
  }
  gibbs_apply(bm, g, nl + nh);
}

void gibbs_apply(SbpBlockmodel& bm, const SbpGraph& g, int batch) {
  Context& c = Context::get();
  const int slot = bm.gen & 1;
  int* n_cur = bm.n_moved.p + slot;
  int* n_next = bm.n_moved.p + (slot ^ 1);
  const unsigned gen = ++bm.gen;
  const int gw = grid_for((long long)batch * 32, 256, 64 * c.num_sms);
  k_apply_edges<<<gw, 256, 0, c.stream>>>(g.view(), bm.view(), bm.moved.p, n_cur, bm.prop.p, bm.qr.p, bm.qs.p,
                                          bm.last.p, gen, nullptr, 0);
  SBP_CHECK_LAUNCH();
  if (bm.sparse) {
    int ovf = 0;
    SBP_CUDA(SBP_COPY_ASYNC(&ovf, bm.overflow.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (ovf) {
      // a hashed row ran out of room: move the assignment, rebuild the rows with more room
      // (keeping d) and run the degree step on the rebuilt rows
      k_recover_assign<<<grid_for(batch, 256, 64 * c.num_sms), 256, 0, c.stream>>>(bm.b.p, bm.moved.p, n_cur,
                                                                                    bm.prop.p, bm.old_block.p);
      SBP_CHECK_LAUNCH();
      if (!regrow_hashed(bm, g)) rebuild(bm, g, false);
      ++g_overflow_rebuilds;
      k_recover_finish<<<grid_for(batch, 256, 64 * c.num_sms), 256, 0, c.stream>>>(
          bm.view(), bm.moved.p, n_cur, n_next, bm.prop.p, bm.old_block.p, bm.qr.p, bm.qs.p, bm.last.p, gen);
      SBP_CHECK_LAUNCH();
      return;
    }
  }
  k_apply_finish<<<grid_for(batch, 256, 64 * c.num_sms), 256, 0, c.stream>>>(
      bm.view(), bm.moved.p, n_cur, n_next, bm.prop.p, bm.qr.p, bm.qs.p, bm.last.p, gen, nullptr, 0);
  SBP_CHECK_LAUNCH();
}


// Asynchronous-Gibbs sweeps of one finetune call as ONE CUDA graph launch: a conditional while
// node whose body is a sweep (every batch's evaluation, apply and degree step, then the MDL,
// whose last CTA applies the early stop on the GPU and sets the loop condition).
// Same kernels, same order and the same early-stop arithmetic as the host loop, so the chain
// and the sweep count are the host loop's.  Returns the sweeps run.
static thread_local DevBuf<SweepCtl> g_ctl;

static int gibbs_sweeps_graph(SbpBlockmodel& bm, const SbpGraph& g, const BatchPlan& plan, RngParams rng,
                              int max_sweeps, bool bracket, double initial_entropy) {
  Context& c = Context::get();
  const int nb = (int)plan.light_n.size();
  g_ctl.reserve(1);
  SweepCtl h;
  std::memset(&h, 0, sizeof h);
  h.sweep = 0;
  h.gen0 = bm.gen;
  h.nbatches = nb;
  h.count = 0;
  h.max_sweeps = max_sweeps;
  h.bracket = bracket ? 1 : 0;
  h.n_moved = bm.n_moved.p;
  h.initial = initial_entropy;
  SBP_CUDA(SBP_COPY_ASYNC(g_ctl.p, &h, sizeof h, cudaMemcpyHostToDevice, c.stream));
  const size_t smem_light = (size_t)table_ints(g.light_cap) * sizeof(int) * kLightWarps;
  const size_t smem_heavy = (size_t)table_ints(g.heavy_cap) * sizeof(int);
  const GibbsEvalKernel k_eval = gibbs_eval_kernel(false, bm.B);   // the graph runs dense storage only
  set_smem_limit((const void*)k_eval, std::max(smem_light, smem_heavy));
  const bool cells = (long long)bm.B * bm.B <= 4LL * g.E;
  const int mdl_grid = c.npartial;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  struct Guard {
    cudaGraph_t* g;
    cudaGraphExec_t* e;
    ~Guard() {
      if (*e) cudaGraphExecDestroy(*e);
      if (*g) cudaGraphDestroy(*g);
    }
  } guard{&graph, &exec};
  SBP_CUDA(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle loop;
  SBP_CUDA(cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault));
  // cudaGraphNodeParams holds a union of non-trivial members: build it in zeroed storage
  alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)] = {};
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_storage);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = loop;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  SBP_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  SBP_CUDA(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int launches = 0;
  for (int bt = 0; bt < nb; ++bt) {
    const int nl = plan.light_n[bt], nh = plan.heavy_n[bt];
    if (nl > 0) {
      const int ng = !use_group_kernel(bm) ? 0 : bm.B <= kSmallB ? nl : plan.group_n[bt];
      if (ng > 0) {
        launch_group_eval(g, bm, plan.order.p + plan.light_begin[bt], ng, rng, 0, nullptr, g_ctl.p, bt, c.stream);
        ++launches;
      }
      if (nl > ng) {
        k_eval<<<grid_for(nl - ng, kLightWarps, 64 * c.num_sms), kLightWarps * 32, smem_light, c.stream>>>(
            g.view(), bm.view(), plan.order.p + plan.light_begin[bt] + ng, nl - ng, rng, 0, bm.prop.p, bm.moved.p,
            nullptr, c.counters, g.light_cap, c.status, g_ctl.p, bt);
        ++launches;
      }
    }
    if (nh > 0) {
      k_eval<<<grid_for(nh, 1, 64 * c.num_sms), 32, smem_heavy, c.stream>>>(
          g.view(), bm.view(), plan.order.p + plan.heavy_begin[bt], nh, rng, 0, bm.prop.p, bm.moved.p, nullptr,
          c.counters, g.heavy_cap, c.status, g_ctl.p, bt);
      ++launches;
    }
    const int batch = nl + nh;
    k_apply_edges<<<grid_for((long long)batch * 32, 256, 64 * c.num_sms), 256, 0, c.stream>>>(
        g.view(), bm.view(), bm.moved.p, nullptr, bm.prop.p, bm.qr.p, bm.qs.p, bm.last.p, 0u, g_ctl.p, bt);
    k_apply_finish<<<grid_for(batch, 256, 64 * c.num_sms), 256, 0, c.stream>>>(
        bm.view(), bm.moved.p, nullptr, nullptr, bm.prop.p, bm.qr.p, bm.qs.p, bm.last.p, 0u, g_ctl.p, bt);
    launches += 2;
  }
  k_mdl<<<mdl_grid, 256, 0, c.stream>>>(g.view(), bm.view(), g.out_src.p, cells ? 1 : 0, c.partial, c.done,
                                       c.scalar, g_ctl.p, loop);
  launches += 1;
  const cudaError_t ce = cudaStreamEndCapture(c.stream, &body);
  SBP_CUDA(ce);
  SBP_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  SBP_CUDA(cudaGraphLaunch(exec, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(&h, g_ctl.p, sizeof h, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  g_launches += (long long)launches * h.count;
  bm.gen += (unsigned)(nb * h.count);
  return h.count;
}

// finetune::{metropolis_hastings, asynchronous_gibbs, hybrid_mcmc}.
void finetune(SbpBlockmodel& bm, SbpGraph& g, int algo, const SbpFinetuneOptions& opt, const SbpReplay* replay,
              SbpStats& st, const SbpMoveReplay* moves) {
  Context& c = Context::get();
  std::memset(&st, 0, sizeof st);
  st.num_blocks = bm.B;
  if (algo < 0 || algo > 2) throw Error(SBP_ERR_INVALID_ARGUMENT, "unknown finetune algorithm");
  if (opt.batches <= 0 && algo != SBP_METROPOLIS_HASTINGS) throw Error(SBP_ERR_INVALID_ARGUMENT, "batches must be >= 1");
  if (bm.B == 1) {   // src/finetune.cpp:33-35: nothing to do, entropy left as it was
    st.mdl = bm.overall_entropy;
    return;
  }
  SBP_CUDA(cudaEventRecord(c.ev0, c.stream));
  ReplayDev rp;
  rp.upload(replay);
  rp.upload_moves(moves);
  RngParams rng;
  rng.seed = opt.seed;
  rng.replay = rp.records ? rp.buf.p : nullptr;
  rng.replay_records = rp.records;
  rng.call = opt.call;
  rng.moves = rp.moves;
  const int max_sweeps = (opt.max_sweeps <= 0 || opt.max_sweeps > kMaxIterations) ? kMaxIterations : opt.max_sweeps;
  const bool bracket = opt.bracket_established != 0;
  SBP_CUDA(cudaMemsetAsync(c.counters, 0, 8 * sizeof(unsigned long long), c.stream));
  const long long ovf0 = g_overflow_rebuilds;
  bm.overall_entropy = (float)mdl(bm, g);
  const double initial_entropy = bm.overall_entropy;
  std::vector<double> deltas;
  long long mh_visits = 0, mh_moved = 0, mh_acc = 0;
  const BatchPlan* plan = nullptr;
  if (algo != SBP_METROPOLIS_HASTINGS) plan = &g.plan(algo, opt.batches);
  if (algo == SBP_ASYNC_GIBBS && g_graph_sweeps && !bm.sparse && !g_prof.on && !plan->light_n.empty()) {
    st.sweeps = gibbs_sweeps_graph(bm, g, *plan, rng, max_sweeps, bracket, initial_entropy);
    c.check_status();
  } else
  for (int it = 0; it < max_sweeps; ++it) {
    if (algo == SBP_METROPOLIS_HASTINGS) {
      const MhResult r = mh_pass(bm, g, g.identity.p, g.V, g.max_k, rng, it);
      mh_visits += r.visits;
      mh_moved += r.moved;
      mh_acc += r.accepted;
      deltas.push_back(r.sum_dS);
      st.sweeps++;
      c.check_status();
      if (early_stop(it, bracket, (double)bm.overall_entropy, deltas)) break;
    } else {
      if (algo == SBP_HYBRID_MCMC && !g.high.empty()) {
        const MhResult r = mh_pass(bm, g, g.high_dev.p, (int)g.high.size(), g.max_k_of(g.high), rng, it);
        mh_visits += r.visits;
        mh_moved += r.moved;
        mh_acc += r.accepted;
      }
      const long long ovf_sweep = g_overflow_rebuilds;
      for (size_t bt = 0; bt < plan->light_n.size(); ++bt) gibbs_batch(bm, g, *plan, (int)bt, rng, it);
      tidy_hashed(bm, g, ovf_sweep);
      const double entropy = mdl(bm, g);
      deltas.push_back(entropy - initial_entropy);   // last_iteration_entropy is never updated
      st.sweeps++;
      c.check_status();
      if (early_stop(it, bracket, initial_entropy, deltas)) break;
    }
  }
  bm.overall_entropy = (float)mdl(bm, g);
  unsigned long long cnt[8];
  SBP_CUDA(SBP_COPY_ASYNC(cnt, c.counters, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(cudaEventRecord(c.ev1, c.stream));
  c.sync();
  c.check_status();
  float ms = 0.f;
  SBP_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  st.visits = (long long)cnt[0] + mh_visits;
  st.proposals_moved = (long long)cnt[1] + mh_moved;
  st.accepted = (long long)cnt[2] + mh_acc;
  st.mdl = bm.overall_entropy;
  st.mcmc_seconds = ms * 1e-3;
  st.num_blocks = bm.B;
  st.overflow_rebuilds = (int)(g_overflow_rebuilds - ovf0);
  g_mcmc_iterations += st.sweeps;
  g_mcmc_time += st.mcmc_seconds;
}

// ------------------------------------------------------------------------------------------
// Block merge
// ------------------------------------------------------------------------------------------
struct MergeScratch {
  DevBuf<int> rcnt, rptr, ridx, rval, ccnt, cptr, cidx, cval, best_s, sizes, map;
  DevBuf<double> best_dS;
};

// block_map of the reference's carry-out loops: block_map[x] is the current name of x's group,
// and merging `from` into `to` renames every entry equal to `from` (src/blockmodel/blockmodel.cpp:
// 61-66).  Member lists make a rename cost the size of the renamed group instead of O(B).
struct GroupMap {
  std::vector<int> name;                    // block -> group name
  std::vector<std::vector<int>> members;    // group name -> blocks carrying it
  explicit GroupMap(int B) : name(B), members(B) {
    for (int i = 0; i < B; ++i) {
      name[i] = i;
      members[i].push_back(i);
    }
  }
  void rename(int from, int to) {
    auto& src = members[from];
    auto& dst = members[to];
    for (int x : src) name[x] = to;
    dst.insert(dst.end(), src.begin(), src.end());
    std::vector<int>().swap(src);
  }
};

// block_merge::carry_out_best_merges_advanced (src/block_merge.cpp:123-217) on a host copy
// of the sparse matrix (serial by construction); heap order (dS, block).
static void carry_out_advanced(int B, int to_merge, const std::vector<int>& rptr, const std::vector<int>& ridx,
                               const std::vector<int>& rval, std::vector<int> d_out, std::vector<int> d_in,
                               const std::vector<double>& dS, const std::vector<int>& best, std::vector<int>& block_map) {
  std::vector<std::unordered_map<int, int>> rows(B), cols(B);
  for (int r = 0; r < B; ++r)
    for (int j = rptr[r]; j < rptr[r + 1]; ++j) {
      rows[r][ridx[j]] = rval[j];
      cols[ridx[j]][r] = rval[j];
    }
  auto get = [&](int r, int c) {
    auto it = rows[r].find(c);
    return it == rows[r].end() ? 0 : it->second;
  };
  auto g = [](double x) { return x > 0 ? x * std::log(x) : 0.0; };
  // closed-form merge delta (matches entropy::block_merge_delta_mdl)
  auto delta = [&](int r, int s) {
    double v = 0.0;
    for (auto& kv : rows[r]) {
      v += g(kv.second);
      if (kv.first != r && kv.first != s) {
        const double m = get(s, kv.first);
        v += g(m) - g(m + kv.second);
      }
    }
    for (auto& kv : cols[r]) {
      if (kv.first == r) continue;
      v += g(kv.second);
      if (kv.first != s) {
        const double m = get(kv.first, s);
        v += g(m) - g(m + kv.second);
      }
    }
    const double mss = get(s, s);
    v += g(mss) - g(mss + get(r, r) + get(r, s) + get(s, r));
    v -= g(d_out[r]) + g(d_out[s]) - g((double)d_out[r] + d_out[s]);
    v -= g(d_in[r]) + g(d_in[s]) - g((double)d_in[r] + d_in[s]);
    return merge_score(v);
  };
  struct Item {
    int from, to;
    double dS;
  };
  auto cmp = [](const Item& a, const Item& b) {   // min-heap on (dS, from)
    if (a.dS != b.dS) return a.dS > b.dS;
    return a.from > b.from;
  };
  std::vector<Item> heap;
  for (int i = 0; i < B; ++i) heap.push_back({i, best[i], dS[i]});
  std::make_heap(heap.begin(), heap.end(), cmp);
  GroupMap gm(B);
  int merged = 0;
  while (merged < to_merge && !heap.empty()) {
    std::pop_heap(heap.begin(), heap.end(), cmp);
    Item m = heap.back();
    heap.pop_back();
    if (m.to < 0) continue;
    const int from = m.from, to = gm.name[m.to];
    if (from == to) continue;
    const double actual = delta(std::min(from, to), std::max(from, to));
    if (!heap.empty() && actual > heap.front().dS) {
      m.dS = actual;
      heap.push_back(m);
      std::push_heap(heap.begin(), heap.end(), cmp);
      continue;
    }
    gm.rename(from, to);
    // move row/col `from` into `to`
    std::vector<std::pair<int, int>> rf(rows[from].begin(), rows[from].end());
    std::vector<std::pair<int, int>> cf(cols[from].begin(), cols[from].end());
    auto add = [&](int r, int c, int v) {
      if (!v) return;
      int& x = rows[r][c];
      x += v;
      cols[c][r] = x;
      if (x == 0) {
        rows[r].erase(c);
        cols[c].erase(r);
      }
    };
    for (auto& kv : rf) {
      add(from, kv.first, -kv.second);
      add(to, (kv.first == from || kv.first == to) ? to : kv.first, kv.second);
    }
    for (auto& kv : cf) {
      if (kv.first == from) continue;
      add(kv.first, from, -kv.second);
      add(kv.first == to ? to : kv.first, to, kv.second);
    }
    d_out[to] += d_out[from];
    d_out[from] = 0;
    d_in[to] += d_in[from];
    d_in[from] = 0;
    merged++;
  }
  block_map = gm.name;
}

void merge_blocks(SbpBlockmodel& bm, SbpGraph& g, const SbpMergeOptions& opt, const SbpReplay* replay,
                  int* best_out, double* dS_out, SbpStats& st, const SbpMoveReplay* moves) {
  Context& c = Context::get();
  const int B = bm.B;
  if (B < 2) throw Error(SBP_ERR_INVALID_ARGUMENT, "block merge needs at least two blocks");
  SBP_CUDA(cudaEventRecord(c.ev0, c.stream));
  MergeScratch ms;
  ReplayDev rp;
  rp.upload(replay);
  rp.upload_moves(moves);
  int nnz[2] = {0, 0};
  Csr rows, cols;
  if (bm.sparse) {
    // the sorted rows come with a rebuild (which also folds in any finetune updates)
    rebuild(bm, g, true);
    rows = Csr{bm.csr_rptr.p, bm.csr_ridx.p, bm.csr_rval.p};
    cols = Csr{bm.csr_cptr.p, bm.csr_cidx.p, bm.csr_cval.p};
  } else if ((long long)B * bm.ld > 8LL * g.E) {
    // compressed rows from the sorted edge keys: fewer bytes than scanning B x ld cells twice
    reserve_sort_scratch(g.E, B);
    if (g.E > 0)
      k_edge_keys<<<grid_for(g.E, 256, 16 * c.num_sms), 256, 0, c.stream>>>(g.view(), bm.b.p, g.out_src.p, B,
                                                                            g_sort.keys.p, g_sort.keysT.p);
    SBP_CHECK_LAUNCH();
    sorted_rows(bm, g.E, g_sort.keys.p, ms.rptr, ms.ridx, ms.rval);
    sorted_rows(bm, g.E, g_sort.keysT.p, ms.cptr, ms.cidx, ms.cval);
    rows = Csr{ms.rptr.p, ms.ridx.p, ms.rval.p};
    cols = Csr{ms.cptr.p, ms.cidx.p, ms.cval.p};
  } else {
  // compressed rows of M and of MT (outgoing_edges / incoming_edges views)
  ms.rcnt.reserve(B);
  ms.ccnt.reserve(B);
  ms.rptr.reserve(B + 1);
  ms.cptr.reserve(B + 1);
  const int gw = grid_for((long long)B * 32, 256, 64 * c.num_sms);
  k_row_nnz<<<gw, 256, 0, c.stream>>>(bm.M.p, B, bm.ld, ms.rcnt.p);
  k_row_nnz<<<gw, 256, 0, c.stream>>>(bm.MT.p, B, bm.ld, ms.ccnt.p);
  k_excl_scan<<<1, 1024, 0, c.stream>>>(ms.rcnt.p, ms.rptr.p, B);
  k_excl_scan<<<1, 1024, 0, c.stream>>>(ms.ccnt.p, ms.cptr.p, B);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(SBP_COPY_ASYNC(&nnz[0], ms.rptr.p + B, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(&nnz[1], ms.cptr.p + B, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  ms.ridx.reserve(nnz[0]);
  ms.rval.reserve(nnz[0]);
  ms.cidx.reserve(nnz[1]);
  ms.cval.reserve(nnz[1]);
  k_row_fill<<<gw, 256, 0, c.stream>>>(bm.M.p, B, bm.ld, ms.rptr.p, ms.ridx.p, ms.rval.p);
  k_row_fill<<<gw, 256, 0, c.stream>>>(bm.MT.p, B, bm.ld, ms.cptr.p, ms.cidx.p, ms.cval.p);
  SBP_CHECK_LAUNCH();
  rows = Csr{ms.rptr.p, ms.ridx.p, ms.rval.p};
  cols = Csr{ms.cptr.p, ms.cidx.p, ms.cval.p};
  }
  const int gw = grid_for((long long)B * 32, 256, 64 * c.num_sms);
  RngParams rng;
  rng.seed = opt.seed;
  rng.replay = rp.records ? rp.buf.p : nullptr;
  rng.replay_records = rp.records;
  rng.call = opt.call;
  rng.moves = rp.moves;
  ms.best_s.reserve(B);
  ms.best_dS.reserve(B);
  SBP_CUDA(cudaMemsetAsync(c.counters, 0, 8 * sizeof(unsigned long long), c.stream));
  k_merge_propose<<<gw, 256, 0, c.stream>>>(bm.view(), rows, cols, rng, ms.best_s.p, ms.best_dS.p, c.counters,
                                            c.status);
  SBP_CHECK_LAUNCH();
  ms.sizes.reserve(B);
  SBP_CUDA(cudaMemsetAsync(ms.sizes.p, 0, B * sizeof(int), c.stream));
  k_block_sizes<<<grid_for(bm.V, 256, 8 * c.num_sms), 256, 0, c.stream>>>(bm.b.p, bm.V, ms.sizes.p);
  SBP_CHECK_LAUNCH();
  std::vector<int> best(B), sizes(B);
  std::vector<double> dS(B);
  unsigned long long cnt[8];
  SBP_CUDA(SBP_COPY_ASYNC(best.data(), ms.best_s.p, B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(dS.data(), ms.best_dS.p, B * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(sizes.data(), ms.sizes.p, B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(cnt, c.counters, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  c.check_status();
  st.merge_proposals += (long long)cnt[0];
  st.merge_avoided += (long long)cnt[1];
  if (best_out) std::memcpy(best_out, best.data(), B * sizeof(int));
  if (dS_out) std::memcpy(dS_out, dS.data(), B * sizeof(double));

  std::vector<int> block_map(B);
  const int to_merge = bm.num_blocks_to_merge;
  if (opt.approximate) {
    // Blockmodel::carry_out_best_merges (src/blockmodel/blockmodel.cpp:50-78); sort ties by index
    const std::vector<int> order = stable_order_by(dS);
    GroupMap gm(B);
    int merged = 0, counter = 0;
    while (merged < to_merge) {
      if (counter >= B) throw Error(SBP_ERR_DEVICE, "not enough mergeable blocks for num_blocks_to_merge");
      const int from = order[counter++];
      if (best[from] < 0) continue;
      const int to = gm.name[best[from]];
      if (to != from) {
        gm.rename(from, to);
        merged++;
      }
    }
    block_map = gm.name;
  } else {
    std::vector<int> rptr(B + 1), dout(B), din(B);
    SBP_CUDA(SBP_COPY_ASYNC(rptr.data(), rows.ptr, (B + 1) * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    nnz[0] = rptr[B];
    std::vector<int> ridx(std::max(nnz[0], 1)), rval(std::max(nnz[0], 1));
    SBP_CUDA(SBP_COPY_ASYNC(ridx.data(), rows.idx, nnz[0] * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(rval.data(), rows.val, nnz[0] * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(dout.data(), bm.d_out.p, B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(din.data(), bm.d_in.p, B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    carry_out_advanced(B, to_merge, rptr, ridx, rval, dout, din, dS, best, block_map);
  }
  // Blockmodel::build_mapping over the labels the vertices carry, then relabel
  std::vector<char> present(B, 0);
  for (int x = 0; x < B; ++x)
    if (sizes[x] > 0) present[block_map[x]] = 1;
  std::vector<int> rank(B, -1), map(B, 0);
  int counter = 0;
  for (int x = 0; x < B; ++x)
    if (present[x]) rank[x] = counter++;
  for (int x = 0; x < B; ++x) map[x] = sizes[x] > 0 ? rank[block_map[x]] : 0;
  ms.map.reserve(B);
  SBP_CUDA(SBP_COPY_ASYNC(ms.map.p, map.data(), B * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  k_relabel<<<grid_for(bm.V, 256, 8 * c.num_sms), 256, 0, c.stream>>>(bm.b.p, bm.V, ms.map.p);
  SBP_CHECK_LAUNCH();
  c.sync();   // host vectors above must outlive the async copy
  bm.set_blocks(B - to_merge);
  rebuild(bm, g);
  SBP_CUDA(cudaEventRecord(c.ev1, c.stream));
  c.sync();
  float ms_time = 0.f;
  SBP_CUDA(cudaEventElapsedTime(&ms_time, c.ev0, c.ev1));
  st.merge_seconds += ms_time * 1e-3;
  st.num_blocks = bm.B;
}

Snapshot snapshot(SbpBlockmodel& bm) {
  Context& c = Context::get();
  Snapshot x;
  x.empty = false;
  x.B = bm.B;
  x.entropy = bm.overall_entropy;
  x.b.resize(bm.V);
  SBP_CUDA(SBP_COPY_ASYNC(x.b.data(), bm.b.p, bm.V * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return x;
}

void restore(SbpBlockmodel& bm, SbpGraph& g, const Snapshot& x) {
  Context& c = Context::get();
  SBP_CUDA(SBP_COPY_ASYNC(bm.b.p, x.b.data(), bm.V * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  bm.set_blocks(x.B);
  bm.overall_entropy = x.entropy;
  rebuild(bm, g);
  c.sync();
}

// entropy::null_mdl_v1 / null_mdl_v2 (src/entropy.cpp:567-583).
static double null_mdl_v1(long long E) {
  const double lp = (double)E * std::log(1.0 / (double)E);
  const double x = 1.0 / (double)E;
  const double h = ((1 + x) * std::log(1 + x)) - (x * std::log(x));
  return ((double)E * h) - lp;
}
static double null_mdl_v2(long long V, long long E) {
  const double lp = (double)E * std::log(1.0 / (double)E);
  const double x = std::pow((double)V, 2) / (double)E;
  const double h = ((1 + x) * std::log(1 + x)) - (x * std::log(x));
  return ((double)E * h) + ((double)V * std::log((double)V)) - lp;
}

// sbp::add_intermediate (src/sbp.cpp:36-59) with Blockmodel::interblock_edges
// (src/blockmodel/blockmodel.cpp:257-261), Blockmodel::block_size_variation (blockmodel.cpp:9-27)
// and, for the final record, Graph::modularity (src/graph.cpp:142-163) in its block form
// (sum_b M[b,b] - sum_b d_out[b] d_in[b] / E) / E.
void add_intermediate(PartitionState& ps, const SbpGraph& g, float iteration, double mdl, bool modularity) {
  Context& c = Context::get();
  SbpBlockmodel& bm = ps.bm;
  DevBuf<unsigned long long> stats;
  DevBuf<int> sizes;
  stats.reserve(3);
  sizes.reserve(bm.B);
  SBP_CUDA(cudaMemsetAsync(stats.p, 0, 3 * sizeof(unsigned long long), c.stream));
  SBP_CUDA(cudaMemsetAsync(sizes.p, 0, bm.B * sizeof(int), c.stream));
  k_block_stats<<<grid_for(bm.B, 256, 4 * c.num_sms), 256, 0, c.stream>>>(bm.view(), stats.p);
  k_block_sizes<<<grid_for(g.V, 256, 8 * c.num_sms), 256, 0, c.stream>>>(bm.b.p, g.V, sizes.p);
  SBP_CHECK_LAUNCH();
  unsigned long long st[3];
  std::vector<int> sz(bm.B);
  SBP_CUDA(SBP_COPY_ASYNC(st, stats.p, sizeof st, cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(sz.data(), sizes.p, bm.B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  cudaEvent_t now;
  SBP_CUDA(cudaEventCreate(&now));
  SBP_CUDA(cudaEventRecord(now, c.stream));
  c.sync();
  float ms = 0.f;
  if (ps.t_start) SBP_CUDA(cudaEventElapsedTime(&ms, ps.t_start, now));
  cudaEventDestroy(now);
  SbpIntermediate r;
  std::memset(&r, 0, sizeof r);
  r.iteration = iteration;
  r.num_blocks = bm.B;
  r.mdl = mdl;
  r.normalized_mdl_v1 = mdl / null_mdl_v1(g.E);
  r.normalized_mdl_v2 = mdl / null_mdl_v2(g.V, g.E);
  const double E = (double)g.E;
  r.modularity = modularity ? ((double)st[0] - (double)st[2] / E) / E : -1.0;
  r.interblock_edges = ((double)st[1] - (double)st[0]) / (double)st[1];
  double total = 0.0, mn = std::numeric_limits<double>::max(), mx = std::numeric_limits<double>::min();
  for (int x : sz) total += x;
  const double mean = total / double(bm.B);
  double var = 0.0;
  for (int x : sz) {
    mn = std::min(mn, (double)x);
    mx = std::max(mx, (double)x);
    var += double(x - mean) * double(x - mean);
  }
  var /= double(bm.B);
  r.block_size_variation = float(var / ((double(mx - mn) * double(mx - mean)) / 4.0));
  r.mcmc_iterations = (int32_t)g_mcmc_iterations;
  r.mcmc_time = g_mcmc_time;
  r.visits = ps.st.visits;
  r.seconds = ms * 1e-3;
  g_intermediates.push_back(r);
}

// sbp::stochastic_block_partition (src/sbp.cpp:61-98) as a per-graph state machine: the
// single-graph driver below and the batched driver (sbp_batched.cu) run the same steps.
void partition_begin(PartitionState& ps, SbpGraph& g) {
  Context& c = Context::get();
  std::memset(&ps.st, 0, sizeof ps.st);
  SbpBlockmodel& bm = ps.bm;
  bm.init_vertex_scratch(g.V);
  std::vector<int> ident(g.V);
  std::iota(ident.begin(), ident.end(), 0);
  SBP_CUDA(SBP_COPY_ASYNC(bm.b.p, ident.data(), g.V * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  bm.set_blocks(g.V);
  bm.num_blocks_to_merge = (int)(g.V * 0.5f);
  rebuild(bm, g);
  c.sync();
  if (ps.record) add_intermediate(ps, g, 0.f, mdl(bm, g), false);
}

int partition_merge(PartitionState& ps, SbpGraph& g, const SbpOptions& opt, SbpFinetuneOptions* fo) {
  SbpMergeOptions mo;
  mo.approximate = opt.approximate;
  mo.call = ps.call;
  mo.seed = opt.seed;
  merge_blocks(ps.bm, g, mo, nullptr, nullptr, nullptr, ps.st, ps.take_replay());
  if (ps.replays) ps.block_counts.push_back(ps.bm.B);
  if (ps.record && ps.iteration < 1) add_intermediate(ps, g, 0.5f, mdl(ps.bm, g), false);
  int algo = opt.algorithm;
  if (algo == SBP_ASYNC_GIBBS && !(ps.iteration < (float)opt.asynciterations)) algo = SBP_METROPOLIS_HASTINGS;
  fo->batches = opt.batches;
  fo->bracket_established = !ps.t.s[2].empty;
  fo->max_sweeps = ps.max_sweeps;
  fo->call = ps.call;
  fo->seed = opt.seed;
  return algo;
}

void partition_finish_round(PartitionState& ps, SbpGraph& g, const SbpStats& fs, int* out) {
  SbpStats& st = ps.st;
  st.visits += fs.visits;
  st.proposals_moved += fs.proposals_moved;
  st.accepted += fs.accepted;
  st.sweeps += fs.sweeps;
  st.mcmc_seconds += fs.mcmc_seconds;
  st.learned_sweeps += fs.learned_sweeps;
  ++ps.iteration;
  if (ps.record) add_intermediate(ps, g, ps.iteration, ps.bm.overall_entropy, false);
  ++ps.call;
  st.outer_iterations++;
  int to_merge = 0;
  const Snapshot nxt = ps.t.next(snapshot(ps.bm), &to_merge);
  if (ps.t.optimal) {
    std::memcpy(out, nxt.b.data(), g.V * sizeof(int));
    st.mdl = nxt.entropy;
    st.num_blocks = nxt.B;
    ps.done = true;
    if (ps.record) {   // the final record is taken on the blockmodel the partition returns
      restore(ps.bm, g, nxt);
      add_intermediate(ps, g, -1.f, nxt.entropy, true);
    }
    return;
  }
  restore(ps.bm, g, nxt);
  ps.bm.num_blocks_to_merge = to_merge;
}

void partition(SbpGraph& g, const SbpOptions& opt, int* out, SbpStats& st, const FinetuneStep* step,
               PartitionReplay* replay) {
  Context& c = Context::get();
  cudaEvent_t t0, t1;
  SBP_CUDA(cudaEventCreate(&t0));
  SBP_CUDA(cudaEventCreate(&t1));
  SBP_CUDA(cudaEventRecord(t0, c.stream));
  PartitionState ps;
  ps.record = step == nullptr && replay == nullptr;
  ps.t_start = t0;
  if (replay) {
    ps.replays = replay->calls;
    ps.nreplays = replay->num_calls;
    ps.max_sweeps = replay->max_sweeps;
  }
  partition_begin(ps, g);
  while (!ps.done) {
    SbpFinetuneOptions fo;
    const int algo = partition_merge(ps, g, opt, &fo);
    SbpStats fs;
    if (step) (*step)(ps.bm, g, algo, fo, fs);
    else finetune(ps.bm, g, algo, fo, nullptr, fs, ps.take_replay());
    if (ps.replays) ps.block_counts.push_back(ps.bm.B);
    partition_finish_round(ps, g, fs, out);
  }
  if (replay) {
    replay->calls_made = ps.next_replay;
    replay->block_counts = ps.block_counts;
  }
  st = ps.st;
  SBP_CUDA(cudaEventRecord(t1, c.stream));
  c.sync();
  float ms = 0.f;
  SBP_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  st.total_seconds = ms * 1e-3;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
}

}  // namespace sbpb

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
#define SBP_API_BEGIN try {
#define SBP_API_END                                        \
  return SBP_OK;                                           \
  }                                                        \
  catch (const Error& e) {                                 \
    set_last_error(e.what());                               \
    return e.code;                                         \
  }                                                        \
  catch (const std::bad_alloc&) {                          \
    set_last_error("host allocation failed");               \
    return SBP_ERR_OUT_OF_MEMORY;                          \
  }                                                        \
  catch (const std::exception& e) {                        \
    set_last_error(e.what());                               \
    return SBP_ERR_CUDA;                                   \
  }

#define SBP_REQUIRE(cond, msg) \
  if (!(cond)) throw Error(SBP_ERR_INVALID_ARGUMENT, msg)

extern "C" {

const char* sbp_last_error(void) { return sbpb::last_error(); }

int32_t sbp_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

SbpStatus sbp_get_stream(void** out) {
  SBP_API_BEGIN
  SBP_REQUIRE(out, "out is NULL");
  *out = (void*)Context::get().stream;
  SBP_API_END
}

SbpStatus sbp_release_cached_memory(void) {
  SBP_API_BEGIN
  DeviceCache::get().release_all();
  SBP_API_END
}

SbpStatus sbp_profile_enable(int32_t on) {
  SBP_API_BEGIN
  Context::get();
  g_prof.on = on != 0;
  SBP_API_END
}

SbpStatus sbp_profile_read(SbpProfile* out, int32_t reset) {
  SBP_API_BEGIN
  SBP_REQUIRE(out, "out is NULL");
  g_prof.resolve();
  out->launches = g_launches;
  out->eval_launches = g_prof.launches;
  out->eval_visits = g_prof.visits;
  out->eval_ms = g_prof.ms;
  out->eval_bytes = g_prof.bytes;
  out->h2d_bytes = g_h2d;
  out->d2h_bytes = g_d2h;
  if (reset) {
    g_prof.launches = g_prof.visits = 0;
    g_prof.ms = g_prof.bytes = 0.0;
  }
  SBP_API_END
}

SbpStatus sbp_set_option(const char* name, int64_t value) {
  SBP_API_BEGIN
  SBP_REQUIRE(name, "NULL option name");
  const std::string n(name);
  if (n == "dense_max_blocks") {
    SBP_REQUIRE(value >= 1 && value <= (1 << 30), "dense_max_blocks out of range");
    g_dense_max_blocks = (int)value;
  } else if (n == "hashed_row_factor") {
    SBP_REQUIRE(value >= 2 && value <= 64, "hashed_row_factor must be in [2, 64]");
    g_hashed_row_factor = (int)value;
  } else if (n == "graph_sweeps") {
    SBP_REQUIRE(value == 0 || value == 1, "graph_sweeps must be 0 or 1");
    g_graph_sweeps = (int)value;
  } else if (n == "dense_max_memory_pct") {
    SBP_REQUIRE(value >= 1 && value <= 90, "dense_max_memory_pct must be in [1, 90]");
    g_dense_max_memory_pct = (int)value;
  } else if (n == "group_kernel") {
    SBP_REQUIRE(value >= 0 && value <= 2, "group_kernel must be 0, 1 or 2");
    g_group_kernel = (int)value;
  } else if (n == "batched_wait_limit") {
    SBP_REQUIRE(value >= 16 && value <= (1LL << 30), "batched_wait_limit must be in [16, 2^30]");
    g_batched_wait_limit = value;
  } else if (n == "batched_stall_graph") {
    SBP_REQUIRE(value >= -1 && value < (1LL << 30), "batched_stall_graph must be -1 or a graph index");
    g_batched_stall_graph = (int)value;
  } else if (n == "batched_threads") {
    SBP_REQUIRE(value >= 1 && value <= 64, "batched_threads must be in [1, 64]");
    g_batched_threads = (int)value;
  } else if (n == "batched_overlap") {
    SBP_REQUIRE(value >= 0 && value <= 1024, "batched_overlap must be in [0, 1024]");
    g_batched_overlap = (int)value;
  } else {
    throw Error(SBP_ERR_INVALID_ARGUMENT, "unknown option: " + n);
  }
  SBP_API_END
}

SbpStatus sbp_graph_create(int32_t V, int64_t n, const int32_t* src, const int32_t* dst, SbpGraph** out) {
  SBP_API_BEGIN
  SBP_REQUIRE(out, "out is NULL");
  *out = nullptr;
  SBP_REQUIRE(V > 0, "num_vertices must be positive");
  SBP_REQUIRE(n >= 0 && (n == 0 || (src && dst)), "edge arrays are NULL");
  SBP_REQUIRE(n < 2000000000LL, "more than 2e9 edges are not supported");
  Context& c = Context::get();
  auto g = std::make_unique<SbpGraph>();
  g->V = V;
  // Device ingest (sbp_ingest.cu): first occurrence of each (src, dst) pair, adjacency lists in
  // input order, self loops on the out side only.
  DevBuf<int> d_src, d_dst, first, bad;
  DevBuf<unsigned long long> table, okeys, ikeys, tmp, partial, ctr;
  DevBuf<unsigned> ocnt, icnt, hist;
  DevBuf<long long> optr, iptr;
  g->self.reserve(V);
  ocnt.reserve((size_t)V + 1);
  icnt.reserve((size_t)V + 1);
  SBP_CUDA(cudaMemsetAsync(g->self.p, 0, V, c.stream));
  SBP_CUDA(cudaMemsetAsync(ocnt.p, 0, ((size_t)V + 1) * sizeof(unsigned), c.stream));
  SBP_CUDA(cudaMemsetAsync(icnt.p, 0, ((size_t)V + 1) * sizeof(unsigned), c.stream));
  int ib = 1;
  while ((1LL << ib) < n) ++ib;
  int vb = 1;
  while ((1LL << vb) < V) ++vb;
  long long m = 0, mi = 0;
  if (n > 0) {
    d_src.reserve(n);
    d_dst.reserve(n);
    SBP_CUDA(SBP_COPY_ASYNC(d_src.p, src, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(d_dst.p, dst, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    int tbits = 4;
    while ((1LL << tbits) < 2 * n + 16) ++tbits;
    const long long cap = 1LL << tbits;
    table.reserve(cap);
    first.reserve(cap);
    bad.reserve(1);
    ctr.reserve(2);
    okeys.reserve(n);
    ikeys.reserve(n);
    SBP_CUDA(cudaMemsetAsync(table.p, 0xff, cap * sizeof(unsigned long long), c.stream));
    SBP_CUDA(cudaMemsetAsync(first.p, 0x7f, cap * sizeof(int), c.stream));
    SBP_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), c.stream));
    SBP_CUDA(cudaMemsetAsync(ctr.p, 0, 2 * sizeof(unsigned long long), c.stream));
    const int grid = grid_for(n, 256, 16 * c.num_sms);
    k_ingest_first<<<grid, 256, 0, c.stream>>>(d_src.p, d_dst.p, n, V, table.p, first.p, tbits, bad.p);
    k_ingest_keep<<<grid, 256, 0, c.stream>>>(d_src.p, d_dst.p, n, V, table.p, first.p, tbits, ib, okeys.p, ikeys.p,
                                              ctr.p, ocnt.p, icnt.p, g->self.p);
    SBP_CHECK_LAUNCH();
    unsigned long long cnt[2] = {0, 0};
    int any_bad = 0;
    SBP_CUDA(SBP_COPY_ASYNC(cnt, ctr.p, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(&any_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (any_bad) throw Error(SBP_ERR_INVALID_ARGUMENT, "edge endpoint out of range");
    m = (long long)cnt[0];
    mi = (long long)cnt[1];
  }
  g->E = m;
  partial.reserve(scan_partial_capacity(c.num_sms));
  g->out_idx.reserve(m);
  g->out_src.reserve(m);
  g->in_idx.reserve(mi);
  if (m > 0) {
    tmp.reserve(m);
    hist.reserve(radix_hist_capacity(m, c.num_sms));
    unsigned long long* sorted = nullptr;
    radix_sort_u64(okeys.p, tmp.p, m, vb + ib, hist.p, partial.p, c.num_sms, c.stream, &sorted);
    k_ingest_fill<<<grid_for(m, 256, 16 * c.num_sms), 256, 0, c.stream>>>(sorted, m, ib, d_dst.p, g->out_idx.p,
                                                                        g->out_src.p);
    SBP_CHECK_LAUNCH();
  }
  if (mi > 0) {
    unsigned long long* sorted = nullptr;
    radix_sort_u64(ikeys.p, tmp.p, mi, vb + ib, hist.p, partial.p, c.num_sms, c.stream, &sorted);
    k_ingest_fill<<<grid_for(mi, 256, 16 * c.num_sms), 256, 0, c.stream>>>(sorted, mi, ib, d_src.p, g->in_idx.p,
                                                                         nullptr);
    SBP_CHECK_LAUNCH();
  }
  optr.reserve((size_t)V + 1);
  iptr.reserve((size_t)V + 1);
  g->out_ptr.reserve((size_t)V + 1);
  g->in_ptr.reserve((size_t)V + 1);
  exclusive_scan_u32(ocnt.p, optr.p, (long long)V + 1, partial.p, c.num_sms, c.stream);
  k_ingest_ptr<<<grid_for((long long)V + 1, 256, 8 * c.num_sms), 256, 0, c.stream>>>(optr.p, g->out_ptr.p,
                                                                                    (long long)V + 1);
  exclusive_scan_u32(icnt.p, iptr.p, (long long)V + 1, partial.p, c.num_sms, c.stream);
  k_ingest_ptr<<<grid_for((long long)V + 1, 256, 8 * c.num_sms), 256, 0, c.stream>>>(iptr.p, g->in_ptr.p,
                                                                                    (long long)V + 1);
  SBP_CHECK_LAUNCH();
  std::vector<int> op((size_t)V + 1), ip((size_t)V + 1);
  SBP_CUDA(SBP_COPY_ASYNC(op.data(), g->out_ptr.p, ((size_t)V + 1) * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(ip.data(), g->in_ptr.p, ((size_t)V + 1) * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  g->h_k.resize(V);
  for (int v = 0; v < V; ++v) {
    g->h_k[v] = (op[v + 1] - op[v]) + (ip[v + 1] - ip[v]);
    g->max_k = std::max(g->max_k, g->h_k[v]);
  }
  // one table size for every vertex when it stays small; larger degrees go to the 1-warp path
  g->light_cap = std::min(kLightCapMax, std::max(kLightCap, pow2_at_least(2 * g->max_k)));
  g->heavy_cap = std::max(512, pow2_at_least(2 * g->max_k));
  if (g->heavy_cap > kMaxCap) {
    if (V <= kMaxCap) g->heavy_cap = kMaxCap;   // distinct neighbour blocks <= B <= V
    else throw Error(SBP_ERR_UNSUPPORTED, "vertex degree above 4096 is not supported");
  }
  // Graph::sort_vertices: degree = out + in - self, descending; ties by vertex id (a counting
  // sort by degree, vertices in ascending order inside each degree)
  {
    std::vector<int> start((size_t)g->max_k + 2, 0), ord(V);
    for (int v = 0; v < V; ++v) start[(size_t)(g->max_k - g->h_k[v]) + 1]++;
    for (int k = 0; k <= g->max_k; ++k) start[k + 1] += start[k];
    for (int v = 0; v < V; ++v) ord[start[g->max_k - g->h_k[v]]++] = v;
    for (int i = 0; i < V; ++i) {
      if ((double)i < 0.15 * (double)V) g->high.push_back(ord[i]);
      else g->low.push_back(ord[i]);
    }
  }
  g->identity.reserve(V);
  g->high_dev.reserve(g->high.size());
  k_iota<<<grid_for(V, 256, 8 * c.num_sms), 256, 0, c.stream>>>(g->identity.p, V);
  SBP_CHECK_LAUNCH();
  if (!g->high.empty())
    SBP_CUDA(SBP_COPY_ASYNC(g->high_dev.p, g->high.data(), g->high.size() * sizeof(int), cudaMemcpyHostToDevice,
                            c.stream));
  c.sync();
  *out = g.release();
  SBP_API_END
}

SbpStatus sbp_graph_destroy(SbpGraph* g) {
  SBP_API_BEGIN
  delete g;
  SBP_API_END
}

SbpStatus sbp_graph_num_edges(const SbpGraph* g, int64_t* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(g && out, "NULL argument");
  *out = g->E;
  SBP_API_END
}

SbpStatus sbp_graph_get_split(const SbpGraph* g, int32_t* num_high, int32_t* high, int32_t* low) {
  SBP_API_BEGIN
  SBP_REQUIRE(g && num_high, "NULL argument");
  *num_high = (int32_t)g->high.size();
  if (high) std::memcpy(high, g->high.data(), g->high.size() * sizeof(int));
  if (low) std::memcpy(low, g->low.data(), g->low.size() * sizeof(int));
  SBP_API_END
}

SbpStatus sbp_graph_set_split(SbpGraph* g, int32_t nh, const int32_t* high, int32_t nl, const int32_t* low) {
  SBP_API_BEGIN
  SBP_REQUIRE(g, "NULL graph");
  SBP_REQUIRE(nh >= 0 && nl >= 0 && nh + nl == g->V, "split must cover every vertex once");
  std::vector<char> seen(g->V, 0);
  for (int i = 0; i < nh; ++i) {
    SBP_REQUIRE(high[i] >= 0 && high[i] < g->V && !seen[high[i]], "bad vertex in split");
    seen[high[i]] = 1;
  }
  for (int i = 0; i < nl; ++i) {
    SBP_REQUIRE(low[i] >= 0 && low[i] < g->V && !seen[low[i]], "bad vertex in split");
    seen[low[i]] = 1;
  }
  g->high.assign(high, high + nh);
  g->low.assign(low, low + nl);
  g->plans.clear();
  g->high_dev.reserve(std::max(nh, 1));
  if (nh) SBP_CUDA(SBP_COPY(g->high_dev.p, high, nh * sizeof(int), cudaMemcpyHostToDevice));
  SBP_API_END
}

SbpStatus sbp_blockmodel_create(const SbpGraph* g, int32_t B, const int32_t* assignment, SbpBlockmodel** out) {
  SBP_API_BEGIN
  SBP_REQUIRE(g && assignment && out, "NULL argument");
  *out = nullptr;
  SBP_REQUIRE(B >= 1 && B <= g->V, "num_blocks must be in [1, V]");
  for (int v = 0; v < g->V; ++v) SBP_REQUIRE(assignment[v] >= 0 && assignment[v] < B, "block id out of range");
  Context& c = Context::get();
  auto bm = std::make_unique<SbpBlockmodel>();
  bm->graph = g;
  bm->init_vertex_scratch(g->V);
  SBP_CUDA(SBP_COPY_ASYNC(bm->b.p, assignment, g->V * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  bm->set_blocks(B);
  bm->num_blocks_to_merge = (int)(B * 0.5f);
  rebuild(*bm, *g);
  c.sync();
  *out = bm.release();
  SBP_API_END
}

SbpStatus sbp_blockmodel_copy(const SbpBlockmodel* src, SbpBlockmodel** out) {
  SBP_API_BEGIN
  SBP_REQUIRE(src && out, "NULL argument");
  Context& c = Context::get();
  auto bm = std::make_unique<SbpBlockmodel>();
  bm->init_vertex_scratch(src->V);
  bm->set_blocks(src->B);
  bm->graph = src->graph;
  if (src->sparse) {
    SBP_REQUIRE(src->graph, "copying a row-hashed blockmodel needs its graph");
    SBP_CUDA(SBP_COPY_ASYNC(bm->b.p, src->b.p, src->V * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
    bm->graph = src->graph;
    rebuild(*bm, *src->graph, false);
    SBP_CUDA(SBP_COPY_ASYNC(bm->d.p, src->d.p, src->B * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
    bm->overall_entropy = src->overall_entropy;
    bm->num_blocks_to_merge = 0;
    c.sync();
    *out = bm.release();
    return SBP_OK;
  }
  const size_t cells = (size_t)src->B * src->ld;
  SBP_CUDA(SBP_COPY_ASYNC(bm->b.p, src->b.p, src->V * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->M.p, src->M.p, cells * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->MT.p, src->MT.p, cells * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->CS.p, src->CS.p, (size_t)src->B * src->nch * sizeof(int), cudaMemcpyDeviceToDevice,
                          c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->CST.p, src->CST.p, (size_t)src->B * src->nch * sizeof(int), cudaMemcpyDeviceToDevice,
                          c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->d_out.p, src->d_out.p, src->B * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->d_in.p, src->d_in.p, src->B * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bm->d.p, src->d.p, src->B * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  bm->overall_entropy = src->overall_entropy;
  bm->num_blocks_to_merge = 0;
  c.sync();
  *out = bm.release();
  SBP_API_END
}

SbpStatus sbp_blockmodel_destroy(SbpBlockmodel* bm) {
  SBP_API_BEGIN
  delete bm;
  SBP_API_END
}

SbpStatus sbp_blockmodel_num_blocks(const SbpBlockmodel* bm, int32_t* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && out, "NULL argument");
  *out = bm->B;
  SBP_API_END
}

SbpStatus sbp_blockmodel_set_num_blocks_to_merge(SbpBlockmodel* bm, int32_t n) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && n >= 0 && n < bm->B, "num_blocks_to_merge must be in [0, B)");
  bm->num_blocks_to_merge = n;
  SBP_API_END
}

SbpStatus sbp_blockmodel_overall_entropy(const SbpBlockmodel* bm, float* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && out, "NULL argument");
  *out = bm->overall_entropy;
  SBP_API_END
}

SbpStatus sbp_get_assignment(const SbpBlockmodel* bm, int32_t* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && out, "NULL argument");
  Context& c = Context::get();
  SBP_CUDA(SBP_COPY_ASYNC(out, bm->b.p, bm->V * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_get_block_matrix(const SbpBlockmodel* bm, int32_t* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && out, "NULL argument");
  Context& c = Context::get();
  if (bm->sparse) {   // scatter the hashed rows into a dense device band, band by band
    const int B = bm->B;
    const int band = (int)std::max<long long>(1, std::min<long long>(B, (64LL << 20) / B));
    DevBuf<int> dense;
    dense.reserve((size_t)band * B);
    for (int r0 = 0; r0 < B; r0 += band) {
      const int rows = std::min(band, B - r0);
      SBP_CUDA(cudaMemsetAsync(dense.p, 0, (size_t)rows * B * sizeof(int), c.stream));
      k_hashed_to_dense<<<std::min(rows, 4096), 128, 0, c.stream>>>(bm->rbase.p, bm->rmask.p, bm->rslot.p, B, r0,
                                                                   rows, dense.p);
      SBP_CHECK_LAUNCH();
      SBP_CUDA(SBP_COPY_ASYNC(out + (size_t)r0 * B, dense.p, (size_t)rows * B * sizeof(int), cudaMemcpyDeviceToHost,
                              c.stream));
      c.sync();
    }
    return SBP_OK;
  }
  SBP_CUDA(cudaMemcpy2DAsync(out, bm->B * sizeof(int), bm->M.p, bm->ld * sizeof(int), bm->B * sizeof(int), bm->B,
                             cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_get_degrees(const SbpBlockmodel* bm, int32_t* d_out, int32_t* d_in, int32_t* d) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm, "NULL argument");
  Context& c = Context::get();
  if (d_out) SBP_CUDA(SBP_COPY_ASYNC(d_out, bm->d_out.p, bm->B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  if (d_in) SBP_CUDA(SBP_COPY_ASYNC(d_in, bm->d_in.p, bm->B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  if (d) SBP_CUDA(SBP_COPY_ASYNC(d, bm->d.p, bm->B * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_set_degrees(SbpBlockmodel* bm, const int32_t* d) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && d, "NULL argument");
  Context& c = Context::get();
  SBP_CUDA(SBP_COPY_ASYNC(bm->d.p, d, bm->B * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_mdl_of_cells(int32_t num_blocks, int64_t nnz, const int32_t* rows, const int32_t* cols,
                           const int32_t* counts, const int32_t* d_out, const int32_t* d_in, int32_t num_vertices,
                           int64_t num_edges, double* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(out && d_out && d_in && num_blocks > 0 && nnz >= 0 && num_vertices > 0 && num_edges > 0,
              "bad argument");
  SBP_REQUIRE(nnz == 0 || (rows && cols && counts), "NULL cell arrays");
  for (int64_t i = 0; i < nnz; ++i) {
    SBP_REQUIRE(rows[i] >= 0 && rows[i] < num_blocks && cols[i] >= 0 && cols[i] < num_blocks, "cell out of range");
    SBP_REQUIRE(counts[i] > 0 && d_out[rows[i]] > 0 && d_in[cols[i]] > 0,
                "a nonzero cell needs positive counts and degrees (the reference exits on a zero degree)");
  }
  Context& c = Context::get();
  DevBuf<int> dr, dc, dv, ddo, ddi;
  const size_t n = (size_t)std::max<int64_t>(nnz, 1);
  dr.reserve(n);
  dc.reserve(n);
  dv.reserve(n);
  ddo.reserve(num_blocks);
  ddi.reserve(num_blocks);
  if (nnz > 0) {
    SBP_CUDA(SBP_COPY_ASYNC(dr.p, rows, nnz * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(dc.p, cols, nnz * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(dv.p, counts, nnz * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  }
  SBP_CUDA(SBP_COPY_ASYNC(ddo.p, d_out, num_blocks * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(ddi.p, d_in, num_blocks * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  k_mdl_cells_list<<<c.npartial, 256, 0, c.stream>>>(dr.p, dc.p, dv.p, nnz, ddo.p, ddi.p, c.partial);
  k_mdl_cells_list_final<<<1, 256, 0, c.stream>>>(c.partial, c.npartial, num_vertices, num_edges, num_blocks,
                                                  c.scalar);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(SBP_COPY_ASYNC(out, c.scalar, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_mdl(const SbpBlockmodel* bm, const SbpGraph* g, double* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && g && out && bm->V == g->V, "bad argument");
  *out = mdl(const_cast<SbpBlockmodel&>(*bm), *g);
  SBP_API_END
}

SbpStatus sbp_evaluate_vertices(const SbpBlockmodel* cbm, const SbpGraph* g, int32_t n, const int32_t* vertices,
                                const uint32_t* records, int32_t* proposal, double* delta_mdl, double* hastings,
                                int32_t* accepted) {
  SBP_API_BEGIN
  SBP_REQUIRE(cbm && g && cbm->V == g->V && n >= 0, "bad argument");
  if (n == 0) return SBP_OK;
  SBP_REQUIRE(vertices && records && proposal && delta_mdl && hastings && accepted, "NULL buffer");
  for (int i = 0; i < n; ++i) SBP_REQUIRE(vertices[i] >= 0 && vertices[i] < g->V, "vertex out of range");
  SbpBlockmodel& bm = const_cast<SbpBlockmodel&>(*cbm);
  Context& c = Context::get();
  std::vector<int> vv(vertices, vertices + n);
  const int cap = mh_cap(g->max_k_of(vv));
  const size_t per_warp = (size_t)table_ints(cap) * sizeof(int);
  const int W = (int)std::max<size_t>(1, std::min<size_t>(8, kSmemBudget / per_warp));
  DevBuf<int> dv, ds, da;
  DevBuf<double> dd, dh;
  DevBuf<uint4> dr;
  dv.reserve(n);
  ds.reserve(n);
  da.reserve(n);
  dd.reserve(n);
  dh.reserve(n);
  dr.reserve(n);
  SBP_CUDA(SBP_COPY_ASYNC(dv.p, vertices, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(dr.p, records, n * sizeof(uint4), cudaMemcpyHostToDevice, c.stream));
  set_smem_limit((const void*)k_eval_list, per_warp * W);
  k_eval_list<<<grid_for(n, W, 64 * c.num_sms), W * 32, per_warp * W, c.stream>>>(
      g->view(), bm.view(), dv.p, n, dr.p, cap, ds.p, dd.p, dh.p, da.p, c.status);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(SBP_COPY_ASYNC(proposal, ds.p, n * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(delta_mdl, dd.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(hastings, dh.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(accepted, da.p, n * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  c.check_status();
  SBP_API_END
}

SbpStatus sbp_move_vertex(SbpBlockmodel* bm, const SbpGraph* g, int32_t vertex, int32_t block) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && g && bm->V == g->V, "bad argument");
  SBP_REQUIRE(vertex >= 0 && vertex < g->V, "vertex out of range");
  SBP_REQUIRE(block >= 0 && block < bm->B, "block out of range");
  Context& c = Context::get();
  const int cap = mh_cap(g->h_k[vertex]);
  const size_t smem = (size_t)table_ints(cap) * sizeof(int);
  set_smem_limit((const void*)k_move_vertex, smem);
  int r0 = 0;
  SBP_CUDA(SBP_COPY_ASYNC(&r0, bm->b.p + vertex, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  k_move_vertex<<<1, 32, smem, c.stream>>>(g->view(), bm->view(), vertex, block, cap, c.status);
  SBP_CHECK_LAUNCH();
  c.sync();
  if (bm->sparse && r0 != block) {
    int flags[3] = {0, 0, 0};
    SBP_CUDA(SBP_COPY_ASYNC(&flags[0], bm->overflow.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(&flags[1], c.status + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (flags[0]) {   // a hashed row ran out of room: rebuild with more room, keep d, finish d[r], d[s]
      rebuild(*bm, *g, false);
      ++g_overflow_rebuilds;
      k_fix_move_degrees<<<1, 1, 0, c.stream>>>(bm->view(), r0, block, flags[1], flags[2]);
      SBP_CHECK_LAUNCH();
      c.sync();
    }
  }
  c.check_status();
  SBP_API_END
}

SbpStatus sbp_finetune(SbpBlockmodel* bm, const SbpGraph* g, int32_t algorithm, const SbpFinetuneOptions* opt,
                       const SbpReplay* replay, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && g && opt && bm->V == g->V, "bad argument");
  SbpStats st;
  finetune(*bm, const_cast<SbpGraph&>(*g), algorithm, *opt, replay, st);
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_merge_blocks(SbpBlockmodel* bm, const SbpGraph* g, const SbpMergeOptions* opt, const SbpReplay* replay,
                           int32_t* best_merge, double* delta_mdl, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && g && opt && bm->V == g->V, "bad argument");
  SbpStats st;
  std::memset(&st, 0, sizeof st);
  merge_blocks(*bm, const_cast<SbpGraph&>(*g), *opt, replay, best_merge, delta_mdl, st);
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_finetune_replayed(SbpBlockmodel* bm, const SbpGraph* g, int32_t algorithm, const SbpFinetuneOptions* opt,
                                const SbpMoveReplay* replay, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && g && opt && bm->V == g->V, "bad argument");
  SBP_REQUIRE(replay && replay->proposal && replay->uniform && replay->records > 0,
              "a finetune replay needs proposals and uniforms");
  SbpStats st;
  finetune(*bm, const_cast<SbpGraph&>(*g), algorithm, *opt, nullptr, st, replay);
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_merge_blocks_replayed(SbpBlockmodel* bm, const SbpGraph* g, const SbpMergeOptions* opt,
                                    const SbpMoveReplay* replay, int32_t* best_merge, double* delta_mdl,
                                    SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && g && opt && bm->V == g->V, "bad argument");
  SBP_REQUIRE(replay && replay->proposal && replay->records > 0, "a merge replay needs proposals");
  SbpStats st;
  std::memset(&st, 0, sizeof st);
  merge_blocks(*bm, const_cast<SbpGraph&>(*g), *opt, nullptr, best_merge, delta_mdl, st, replay);
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_get_intermediates(SbpIntermediate* out, int32_t capacity, int32_t* count) {
  SBP_API_BEGIN
  SBP_REQUIRE(count && (capacity == 0 || out) && capacity >= 0, "bad argument");
  *count = (int32_t)g_intermediates.size();
  for (int32_t i = 0; i < capacity && i < *count; ++i) out[i] = g_intermediates[i];
  SBP_API_END
}

SbpStatus sbp_clear_intermediates(void) {
  SBP_API_BEGIN
  g_intermediates.clear();
  SBP_API_END
}

SbpStatus sbp_partition_replayed(const SbpGraph* g, const SbpOptions* opt, int32_t max_sweeps, int32_t num_calls,
                                 const SbpMoveReplay* calls, int32_t* out_assignment, int32_t* block_counts,
                                 int32_t* calls_made, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(g && opt && out_assignment && calls && num_calls > 0, "NULL argument");
  SBP_REQUIRE(opt->algorithm >= 0 && opt->algorithm <= 2, "unknown algorithm");
  SBP_REQUIRE(opt->batches >= 1, "batches must be >= 1");
  for (int k = 0; k < num_calls; ++k) SBP_REQUIRE(calls[k].proposal && calls[k].records > 0, "empty call stream");
  PartitionReplay rp;
  rp.calls = calls;
  rp.num_calls = num_calls;
  rp.max_sweeps = max_sweeps;
  SbpStats st;
  partition(const_cast<SbpGraph&>(*g), *opt, out_assignment, st, nullptr, &rp);
  if (calls_made) *calls_made = rp.calls_made;
  if (block_counts)
    for (size_t k = 0; k < rp.block_counts.size() && k < (size_t)num_calls; ++k) block_counts[k] = rp.block_counts[k];
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_partition(const SbpGraph* g, const SbpOptions* opt, int32_t* out_assignment, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(g && opt && out_assignment, "NULL argument");
  SBP_REQUIRE(opt->algorithm >= 0 && opt->algorithm <= 2, "unknown algorithm");
  SBP_REQUIRE(opt->batches >= 1, "batches must be >= 1");
  SbpStats st;
  partition(const_cast<SbpGraph&>(*g), *opt, out_assignment, st);
  if (stats) *stats = st;
  SBP_API_END
}

}  // extern "C"
