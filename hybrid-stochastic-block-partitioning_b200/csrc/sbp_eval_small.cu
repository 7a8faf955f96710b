// Asynchronous-Gibbs evaluation of the light vertices of a batch on a dense block matrix, one
// group of lanes per vertex (the same proposal, Hastings correction, delta-MDL and accept test as
// evaluate_vertex in sbp_device.cuh; src/common.cpp:131-192, src/entropy.cpp:296-401, 495-557,
// src/finetune.cpp:19-29).
//
// Layout of the work:
//  * a group of G lanes evaluates one vertex, so a warp carries 32 / G vertices at a time; every
//    loop runs to the largest trip count of the warp's groups (lanes past their own count are
//    predicated off), so the group shuffles always see the whole warp converged;
//  * the neighbour-block histogram of a vertex is a per-group structure in shared memory: for
//    B <= kSmallB a direct-indexed array of B words (out count | in count << 15 | presence << 30),
//    above it an open-addressing table of twice the light-vertex degree bound; plus the list of
//    entries present;
//  * the multinomial walk finds the chunk through the chunk sums, sixteen per lane per step, then
//    the column inside it, sixteen counts per lane;
//  * the frozen state of the batch (assignment, block matrix, degrees, log table) is read through
//    the read-only data cache;
//  * the FP64 terms of a changed cell are computed by the lane that loaded the cell.
// Summation orders differ from evaluate_vertex, so delta-MDL and the Hastings factor agree with
// it to rounding; the integer zero-snap scale T and every integer input are the same.
#include "sbp_engine.cuh"

namespace sbpb {
namespace {

constexpr unsigned kInShift = 15;
constexpr unsigned kCountMask = (1u << 15) - 1;
constexpr unsigned kPresent = 1u << 30;

template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o, G);
  return v;
}
template <int G>
__device__ __forceinline__ long long group_sum_ll(long long v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o, G);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_ull(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ int warp_max_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Neighbour-block histogram of one group: direct-indexed by block (kHash false, B <= kSmallB) or
// an open-addressing table of `mask + 1` slots (kHash true).  Slot words hold out count | in count
// << 15 | presence << 30; the list holds the slots in use.
template <bool kHash>
struct GroupTable {
  int* keys;        // kHash: block of each slot, -1 = empty
  unsigned* w;      // counts per slot (per block when direct)
  int* list;        // slots in use
  int* n;           // their number
  int mask;
  int* status;
  // slot of `key`, inserted if absent (*created set for the inserting lane)
  __device__ __forceinline__ int insert(int key, bool* created) const {
    *created = false;
    if constexpr (!kHash) {
      return key;
    } else {
      unsigned h = ((unsigned)key * 2654435761u) & (unsigned)mask;
      for (int probe = 0; probe <= mask; ++probe) {
        const int k = keys[h];
        if (k == key) return (int)h;
        if (k == -1) {
          const int prev = atomicCAS(keys + h, -1, key);
          if (prev == -1) {
            *created = true;
            return (int)h;
          }
          if (prev == key) return (int)h;
        }
        h = (h + 1) & (unsigned)mask;
      }
      atomicOr(status, kErrTableFull);
      return -1;
    }
  }
  __device__ __forceinline__ unsigned counts_of(int key) const {
    if constexpr (!kHash) {
      return w[key];
    } else {
      unsigned h = ((unsigned)key * 2654435761u) & (unsigned)mask;
      for (int probe = 0; probe <= mask; ++probe) {
        const int k = keys[h];
        if (k == key) return w[h];
        if (k == -1) return 0u;
        h = (h + 1) & (unsigned)mask;
      }
      return 0u;
    }
  }
  __device__ __forceinline__ void add(int key, unsigned delta) const {
    bool created;
    const int slot = insert(key, &created);
    if (slot < 0) return;
    const unsigned old = delta == kPresent ? atomicOr(w + slot, kPresent) : atomicAdd(w + slot, delta);
    if (kHash ? created : old == 0u) list[atomicAdd(n, 1)] = slot;
  }
  __device__ __forceinline__ int key_of(int slot) const { return kHash ? keys[slot] : slot; }
  __device__ __forceinline__ void clear(int slot) const {
    w[slot] = 0u;
    if constexpr (kHash) keys[slot] = -1;
  }
};

// Loads of the blockmodel: through the read-only data cache when no thread of the launch writes it
// (the evaluation half of a Gibbs batch), plain when commits of the same launch change it
// (Metropolis-Hastings rounds; the writers share the SM, so its L1 stays coherent).
template <bool kFrozen>
__device__ __forceinline__ int ldb(const int* p) {
  if constexpr (kFrozen) return __ldg(p);
  else return *p;
}
template <bool kFrozen>
__device__ __forceinline__ int4 ldb4(const int4* p) {
  if constexpr (kFrozen) return __ldg(p);
  else return *p;
}

// The multinomial walk of evaluate_vertex over a dense row (or column) of M: the first column
// whose running count exceeds tg.  Chunk sums (kChunk columns each) locate the chunk, sixteen per
// lane per step (one memory round trip per 16 G chunks); the chunk's counts are then scanned
// sixteen per lane.  Every lane of the warp
// takes part (loop bounds are warp-uniform); groups with walk == false get -1.
constexpr int kSumsPerLane = 16;

template <int G, bool kFrozen>
__device__ __forceinline__ int group_walk(const int* row, const int* csum, int nch, long long tg, bool walk, int gl,
                                          int gbase) {
  const unsigned gmask = (G == 32 ? kFull : ((1u << G) - 1u) << gbase);
  int chunk = 0;
  long long before = 0;   // counts of the row before the chosen chunk
  if (nch > 1) {
    bool found = !walk;
    chunk = -1;
    long long acc = 0;
    for (int c0 = 0; c0 < nch; c0 += kSumsPerLane * G) {
      int cs[kSumsPerLane];
      long long lsum = 0;
#pragma unroll
      for (int q = 0; q < kSumsPerLane; ++q) {
        const int c = c0 + gl * kSumsPerLane + q;
        cs[q] = (walk && c < nch) ? ldb<kFrozen>(csum + c) : 0;
        lsum += cs[q];
      }
      long long incl = lsum;
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const long long y = __shfl_up_sync(kFull, incl, o, G);
        if (gl >= o) incl += y;
      }
      const long long tot = __shfl_sync(kFull, incl, G - 1, G);
      const unsigned hit = __ballot_sync(kFull, !found && acc + incl > tg) & gmask;
      int pick = -1;
      long long pb = 0;
      if (hit && gl == __ffs(hit) - 1 - gbase) {
        long long run = acc + incl - lsum;
#pragma unroll
        for (int q = 0; q < kSumsPerLane; ++q) {
          if (pick < 0) {
            if (tg < run + cs[q]) {
              pick = c0 + gl * kSumsPerLane + q;
              pb = run;
            } else {
              run += cs[q];
            }
          }
        }
      }
      const int src = hit ? __ffs(hit) - 1 - gbase : 0;
      const int pk = __shfl_sync(kFull, pick, src, G);
      const long long pbb = __shfl_sync(kFull, pb, src, G);
      if (hit && !found) {
        chunk = pk;
        before = pbb;
        found = true;
      }
      acc += tot;
    }
    if (walk && chunk < 0) walk = false;
  }
  constexpr int kPer = kChunk / G;   // counts per lane
  const int* base = row + (size_t)(chunk < 0 ? 0 : chunk) * kChunk + gl * kPer;
  int vals[kPer];
  long long lsum = 0;
#pragma unroll
  for (int q = 0; q < kPer / 4; ++q) {
    const int4 c4 = ldb4<kFrozen>(reinterpret_cast<const int4*>(base) + q);
    vals[4 * q] = c4.x;
    vals[4 * q + 1] = c4.y;
    vals[4 * q + 2] = c4.z;
    vals[4 * q + 3] = c4.w;
    lsum += (long long)c4.x + c4.y + c4.z + c4.w;
  }
  long long incl = lsum;
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    const long long y = __shfl_up_sync(kFull, incl, o, G);
    if (gl >= o) incl += y;
  }
  const long long t2 = tg - before;
  const unsigned hit = __ballot_sync(kFull, walk && incl > t2) & gmask;
  int col = -1;
  if (walk && hit && gl == __ffs(hit) - 1 - gbase) {
    long long rem = t2 - (incl - lsum);
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      if (col < 0) {
        if (rem < vals[q]) col = (chunk < 0 ? 0 : chunk) * kChunk + gl * kPer + q;
        else rem -= vals[q];
      }
    }
  }
  const int found = __shfl_sync(kFull, col, hit ? __ffs(hit) - 1 - gbase : 0, G);
  return walk ? found : -1;
}

// Result of one group's evaluation of a vertex; every lane of the group holds it.
struct GroupEval {
  int v, r, s, t;        // vertex, its block, proposed block, the proposal's neighbour block (-1: none)
  int k_out, k_in, self;
  bool valid, accepted;
  double dS;
};

// Evaluate vertex v (valid lanes) against the blockmodel with record x: gather its neighbour
// blocks into the group's table (left filled for the caller), propose, delta-MDL, Hastings,
// accept.  Every lane of the warp calls it (loop bounds are warp-uniform).
template <int G, bool kHash, bool kFrozen>
__device__ __forceinline__ GroupEval group_evaluate(const GraphView& g, const BlockView& bm, const GroupTable<kHash>& T,
                                                    bool valid, int v, bool given, uint4 x, int gl, int gbase,
                                                    int* status) {
  const int B = bm.B;
  const int ld = bm.ld;
  GroupEval res;
  res.valid = valid;
  res.accepted = false;
  res.dS = 0.0;
  res.v = v;
  int r = 0, o0 = 0, i0 = 0, k_out = 0, k_in = 0, self = 0;
  if (valid) {
    r = ldb<kFrozen>(bm.b + v);
    o0 = __ldg(g.out_ptr + v);
    k_out = __ldg(g.out_ptr + v + 1) - o0;
    i0 = __ldg(g.in_ptr + v);
    k_in = __ldg(g.in_ptr + v + 1) - i0;
    self = __ldg(g.self + v);
  }
  res.r = r;
  res.k_out = k_out;
  res.k_in = k_in;
  res.self = self;
  const int k = k_out + k_in;
  const int idx = (valid && k > 0 && !given) ? (int)scale32(x.x, k) : -1;
  // 1. neighbour-block histogram and the proposal's neighbour block
  int tblk = -1;
  const int gather_iters = warp_max_int((k + G - 1) / G);
  for (int it = 0; it < gather_iters; ++it) {
    const int e = it * G + gl;
    int bu = -1;
    if (e < k) {
      const bool out = e < k_out;
      const int u = out ? __ldg(g.out_idx + o0 + e) : __ldg(g.in_idx + i0 + (e - k_out));
      bu = ldb<kFrozen>(bm.b + u);
      if (!(out && u == v)) T.add(bu, out ? 1u : (1u << kInShift));   // the self loop only marks r present
    }
    const int src = idx - it * G;
    const int pick = __shfl_sync(kFull, bu, (src >= 0 && src < G) ? src : 0, G);
    if (src >= 0 && src < G) tblk = pick;
  }
  if (valid && self && gl == 0) T.add(r, kPresent);
  __syncwarp();
  res.t = (valid && k > 0 && !given) ? tblk : -1;
  // 2. the proposal: the multinomial over row t of M then column t (ascending), as the dense
  //    walks of evaluate_vertex
  int s = r;
  {
    const bool walk = valid && !given && k > 0;
    const int t = walk ? tblk : 0;
    long long tg = -1;
    bool in_row = true;
    if (walk) {
      const int dot = ldb<kFrozen>(bm.d_out + t), dit = ldb<kFrozen>(bm.d_in + t);
      const long long target = scale32(x.y, (long long)dot + (long long)dit);
      in_row = target < dot;
      tg = in_row ? target : target - dot;
    }
    const int* row = (in_row ? bm.M : bm.MT) + (size_t)t * ld;
    const int* csum = (in_row ? bm.CS : bm.CST) + (size_t)t * bm.nch;
    const int found = group_walk<G, kFrozen>(row, csum, bm.nch, tg, walk, gl, gbase);
    if (walk) {
      s = found;
      if (s < 0 || s >= B) {
        if (gl == 0) atomicOr(status, kErrScan);
        s = r;
      }
    } else if (valid && given) {
      s = (int)x.x;
      if (s < 0 || s >= B) {   // a visit the stream has no proposal for
        if (gl == 0) atomicOr(status, kErrReplay);
        s = r;
      }
    } else if (valid) {
      s = random_block(r, B, x.y);
    }
  }
  res.s = s;
  const bool active = valid && s != r;
  // 3. delta-MDL and the Hastings correction of the move r -> s
  double fwd = 0.0, bwd = 0.0, dS = 0.0;
  long long Tz = 0;
  int co_r = 0, ci_r = 0, co_s = 0, ci_s = 0;
  int M_rr = 0, M_rs = 0, M_sr = 0, M_ss = 0, dout_r = 0, dout_s = 0, din_r = 0, din_s = 0;
  if (active) {
    const unsigned wr = T.counts_of(r), ws = T.counts_of(s);
    co_r = wr & kCountMask;
    ci_r = (wr >> kInShift) & kCountMask;
    co_s = ws & kCountMask;
    ci_s = (ws >> kInShift) & kCountMask;
    M_rr = ldb<kFrozen>(bm.M + (size_t)r * ld + r);
    M_rs = ldb<kFrozen>(bm.M + (size_t)r * ld + s);
    M_sr = ldb<kFrozen>(bm.M + (size_t)s * ld + r);
    M_ss = ldb<kFrozen>(bm.M + (size_t)s * ld + s);
    dout_r = ldb<kFrozen>(bm.d_out + r);
    dout_s = ldb<kFrozen>(bm.d_out + s);
    din_r = ldb<kFrozen>(bm.d_in + r);
    din_s = ldb<kFrozen>(bm.d_in + s);
  }
  const int d_rr = -co_r - ci_r - self;
  const int d_rs = -co_s + ci_r;
  const int d_sr = co_r - ci_s;
  const int d_ss = co_s + ci_s + self;
  const int kin_self = k_in + self;
  const int nent = active ? *T.n : 0;
  const int ent_iters = warp_max_int((nent + G - 1) / G);
  for (int it = 0; it < ent_iters; ++it) {
    const int j = it * G + gl;
    if (j < nent) {
      const int slot = T.list[j];
      const int u = T.key_of(slot);
      const unsigned wu = T.w[slot];
      const int co = wu & kCountMask, ci = (wu >> kInShift) & kCountMask;
      const int M_ru = ldb<kFrozen>(bm.M + (size_t)r * ld + u);
      const int M_ur = ldb<kFrozen>(bm.MT + (size_t)r * ld + u);
      const int M_su = ldb<kFrozen>(bm.M + (size_t)s * ld + u);
      const int M_us = ldb<kFrozen>(bm.MT + (size_t)s * ld + u);
      const int du = ldb<kFrozen>(bm.d + u);
      const bool is_r = u == r, is_s = u == s, corner = is_r || is_s;
      const double c = (double)(co + ci + (is_r ? self : 0));
      const double inv_u = 1.0 / ((double)du + (double)B);   // a non-corner block's degree is unchanged
      fwd += c * (M_su + M_us + 1.0) * inv_u;
      const double bw = is_r ? (double)(M_rr + d_rr) + (double)(M_rr + d_rr) + 1.0
                      : is_s ? (double)(M_rs + d_rs) + (double)(M_sr + d_sr) + 1.0
                             : (double)(M_ru - co) + (double)(M_ur - ci) + 1.0;
      const int nd = is_r ? (dout_r - k_out) + (din_r - k_in) - (M_rr + d_rr)
                   : is_s ? (dout_s + k_out) + (din_s + k_in) - (M_ss + d_ss) : du;
      bwd += c * bw * (corner ? 1.0 / ((double)nd + (double)B) : inv_u);
      if (!corner) {   // cells (r,u) (s,u) for out-edges to u, (u,r) (u,s) for in-edges
        if (co) {
          dS += dxlogx_int(bm.logt, M_ru, M_ru - co) + dxlogx_int(bm.logt, M_su, M_su + co);
          Tz += 2LL * (M_ru + M_su);
        }
        if (ci) {
          dS += dxlogx_int(bm.logt, M_ur, M_ur - ci) + dxlogx_int(bm.logt, M_us, M_us + ci);
          Tz += 2LL * (M_ur + M_us);
        }
      }
    }
  }
  if (active) {
    // corner cells (r,r) (r,s) (s,r) (s,s), then the out- and in-degrees of r and s
    for (int q = gl; q < 8; q += G) {
      const int a = q == 0 ? M_rr : q == 1 ? M_rs : q == 2 ? M_sr : q == 3 ? M_ss
                  : q == 4 ? dout_r : q == 5 ? dout_s : q == 6 ? din_r : din_s;
      const int d = q == 0 ? d_rr : q == 1 ? d_rs : q == 2 ? d_sr : q == 3 ? d_ss
                  : q == 4 ? -k_out : q == 5 ? k_out : q == 6 ? -kin_self : kin_self;
      if (d) dS += (q < 4 ? 1.0 : -1.0) * dxlogx_int(bm.logt, a, a + d);
      Tz += q < 4 ? (d ? 2LL * a + d : 0LL) : 2LL * a;
    }
    // the double count of a present net-zero (r,s) / (s,r) Delta cell
    if (gl == 0 && (co_s > 0 || ci_r > 0) && d_rs == 0 && M_rs > 0)
      dS += (double)M_rs * (log1p((double)kin_self / (double)din_s) + log1p(-(double)k_out / (double)dout_r));
    if (gl == (G > 1 ? 1 : 0) && (co_r > 0 || ci_s > 0) && d_sr == 0 && M_sr > 0)
      dS += (double)M_sr * (log1p(-(double)kin_self / (double)din_r) + log1p((double)k_out / (double)dout_s));
  }
  fwd = group_sum<G>(fwd);
  bwd = group_sum<G>(bwd);
  dS = group_sum<G>(dS);
  Tz = group_sum_ll<G>(Tz);
  if (active) {
    if (fabs(dS) <= 0x1p-40 * (double)Tz * g.log_E) dS = 0.0;
    const double H = (k == 0) ? 1.0 : bwd / fwd;
    double ap = exp(-3.0 * dS) * H;
    ap = ap >= 1.0 ? 1.0 : ap;
    const double u = given ? record_uniform(x) : u53(x.z, x.w);
    res.accepted = u <= ap;
    res.dS = dS;
  }
  return res;
}

// Set up the calling group's table in the dynamic shared memory after `header` ints.
template <bool kHash>
__device__ __forceinline__ GroupTable<kHash> group_table(int* smem, int header, int gid, int slots, int* status) {
  int* mine = smem + header + (size_t)gid * (kHash ? 3 : 2) * slots;
  GroupTable<kHash> T;
  T.w = reinterpret_cast<unsigned*>(mine);
  T.list = mine + slots;
  T.keys = kHash ? mine + 2 * slots : nullptr;
  T.n = smem + gid;
  T.mask = slots - 1;
  T.status = status;
  return T;
}

template <bool kHash, int G>
__device__ __forceinline__ void group_table_init(const GroupTable<kHash>& T, int slots, int gl) {
  for (int i = gl; i < slots; i += G) {
    T.w[i] = 0u;
    if constexpr (kHash) T.keys[i] = -1;
  }
  if (gl == 0) *T.n = 0;
  __syncwarp();
}

template <bool kHash, int G>
__device__ __forceinline__ void group_table_clear(const GroupTable<kHash>& T, int gl) {
  __syncwarp();
  const int nclear = *T.n;
  for (int j = gl; j < nclear; j += G) T.clear(T.list[j]);
  __syncwarp();
  if (gl == 0) *T.n = 0;
  __syncwarp();
}

// Direct-indexed tables (33 KB of shared memory per CTA): registers capped for three CTAs per SM
// (measured 17 % shorter launches than at two CTAs per SM on 71 blocks).  Hashed tables of 256
// slots take 98 KB per CTA, two CTAs per SM whatever the registers.  (Issuing the loads of four
// gather steps, or of four delta-MDL entries, together was measured 3-8 % slower.)
template <int G, bool kHash>
__global__ void __launch_bounds__(kSmallThreads, kHash ? 2 : 3)
    k_gibbs_eval_group(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep,
                       int* prop, int* moved_list, int* n_moved, unsigned long long* counters, int cap, int* status,
                       const SweepCtl* ctl, int batch) {
  constexpr int kGroups = kSmallThreads / G;
  extern __shared__ int group_smem[];
  const int slots = kHash ? cap : kSmallB;
  if (ctl) {
    sweep = ctl->sweep;
    n_moved = ctl->n_moved + ((ctl->gen0 + (unsigned)batch) & 1u);
  }
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int gid = threadIdx.x / G;
  const int gbase = lane & ~(G - 1);   // first lane of this group in the warp
  const GroupTable<kHash> T = group_table<kHash>(group_smem, kGroups, gid, slots, status);
  group_table_init<kHash, G>(T, slots, gl);
  unsigned long long c_visit = 0, c_moved = 0, c_acc = 0;
  const bool given = rng.moves != 0;
  const int groups_total = gridDim.x * kGroups;
  // warp-uniform outer loop: the warp's groups take consecutive list entries
  const int warp_first = (blockIdx.x * kSmallThreads + (threadIdx.x & ~31)) / G;
  for (int base = warp_first; base < n; base += groups_total) {
    const int item = base + (lane / G);
    const bool valid = item < n;
    int v = 0;
    uint4 x = make_uint4(0, 0, 0, 0);
    if (valid) {
      v = __ldg(verts + item);
      x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * g.V + v, status);
    }
    const GroupEval e = group_evaluate<G, kHash, true>(g, bm, T, valid, v, given, x, gl, gbase, status);
    if (e.accepted && gl == 0) {
      c_acc++;
      prop[v] = e.s;
      moved_list[atomicAdd(n_moved, 1)] = v;
    }
    if (valid && gl == 0) {
      c_visit++;
      if (e.s != e.r) c_moved++;
    }
    group_table_clear<kHash, G>(T, gl);
  }
  c_visit = warp_sum_ull(c_visit);
  c_moved = warp_sum_ull(c_moved);
  c_acc = warp_sum_ull(c_acc);
  if (lane == 0 && c_visit) {
    atomicAdd(counters + 0, c_visit);
    atomicAdd(counters + 1, c_moved);
    atomicAdd(counters + 2, c_acc);
  }
}

// Metropolis-Hastings over a vertex list with exact sequential semantics (finetune::
// metropolis_hastings, src/finetune.cpp:412-444), dense storage, one CTA of kMhGroupThreads:
// each round the groups evaluate the next kMhGroupThreads / G vertices of the list against the
// current state; the first accepted one commits, and so does every later accepted one that no
// earlier commit of the round could have influenced (the test of k_mh, on the group tables),
// scanning stops at the first dependent vertex.  Everything after that is evaluated again in the
// next round; records depend only on (vertex, sweep), so the chain is the sequential one.
// out: [0] visits [1] proposals moved [2] accepted [3] sum of accepted delta-MDL in list order.
template <int G, bool kHash>
__global__ void __launch_bounds__(kMhGroupThreads)
    k_mh_group(GraphView g, BlockView bm, const int* __restrict__ verts, int n, RngParams rng, int sweep, int cap,
               double* out, int* status) {
  constexpr int kGroups = kMhGroupThreads / G;
  extern __shared__ int group_smem[];
  __shared__ int s_acc[kGroups], s_moved[kGroups], s_r[kGroups], s_s[kGroups], s_t[kGroups], s_commit[kGroups];
  __shared__ double s_dS[kGroups];
  __shared__ int s_upto;
  const int slots = kHash ? cap : kSmallB;
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int gid = threadIdx.x / G;
  const int gbase = lane & ~(G - 1);
  const GroupTable<kHash> T = group_table<kHash>(group_smem, kGroups, gid, slots, status);
  group_table_init<kHash, G>(T, slots, gl);
  long long visits = 0, moved = 0, accepted = 0;
  double sum_dS = 0.0;
  const bool given = rng.moves != 0;
  __syncthreads();
  for (int pos = 0; pos < n;) {
    const int i = pos + gid;
    const bool valid = i < n;
    int v = 0;
    uint4 x = make_uint4(0, 0, 0, 0);
    if (valid) {
      v = __ldg(verts + i);
      x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * g.V + v, status);
    }
    const GroupEval e = group_evaluate<G, kHash, false>(g, bm, T, valid, v, given, x, gl, gbase, status);
    if (gl == 0) {
      s_acc[gid] = e.accepted ? 1 : 0;
      s_moved[gid] = (valid && e.s != e.r) ? 1 : 0;
      s_dS[gid] = e.dS;
      s_r[gid] = e.r;
      s_s[gid] = e.s;
      s_t[gid] = e.t;
      s_commit[gid] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int avail = min(kGroups, n - pos);
      int first = -1;
      for (int w = 0; w < avail; ++w)
        if (s_acc[w]) {
          first = w;
          break;
        }
      int upto = first >= 0 ? first + 1 : avail;
      if (first >= 0) {
        s_commit[first] = 1;
        int cw[kGroups];
        int ncommit = 1;
        cw[0] = first;
        for (int w = first + 1; w < avail; ++w) {
          const GroupTable<kHash> tw = group_table<kHash>(group_smem, kGroups, w, slots, status);
          bool indep = true;
          for (int q = 0; q < ncommit && indep; ++q) {
            const int c = cw[q];
            const GroupTable<kHash> tc = group_table<kHash>(group_smem, kGroups, c, slots, status);
            const int rc = s_r[c], sc = s_s[c];
            const int rw = s_r[w], sw = s_s[w], tb = s_t[w];
            if (rc == rw || rc == sw || rc == tb || sc == rw || sc == sw || sc == tb) indep = false;
            else if (tw.counts_of(rc) || tw.counts_of(sc)) indep = false;
            else if ((tb >= 0 && tc.counts_of(tb)) || tc.counts_of(rw) || tc.counts_of(sw)) indep = false;
          }
          if (!indep) break;
          upto = w + 1;
          if (s_acc[w]) {
            s_commit[w] = 1;
            cw[ncommit++] = w;
          }
        }
      }
      s_upto = upto;
      for (int w = 0; w < upto; ++w) {
        moved += s_moved[w];
        if (s_commit[w]) {   // accepted moves in list order
          accepted++;
          sum_dS += s_dS[w];
        }
      }
      visits += upto;
    }
    __syncthreads();
    if (s_commit[gid]) {
      // apply v: r -> s with the counts in this group's table; lanes own distinct non-corner
      // cells (no other commit of the round touches them), lane 0 the corners and degrees
      const int r = e.r, s = e.s;
      const unsigned wr = T.counts_of(r), ws = T.counts_of(s);
      const int co_r = wr & kCountMask, ci_r = (wr >> kInShift) & kCountMask;
      const int co_s = ws & kCountMask, ci_s = (ws >> kInShift) & kCountMask;
      const int nl = *T.n;
      for (int j = gl; j < nl; j += G) {
        const int slot = T.list[j];
        const int u = T.key_of(slot);
        if (u == r || u == s) continue;
        const unsigned wu = T.w[slot];
        const int co = wu & kCountMask, ci = (wu >> kInShift) & kCountMask;
        if (co) {
          bm.M[(size_t)r * bm.ld + u] -= co;
          bm.MT[(size_t)u * bm.ld + r] -= co;
          bm.M[(size_t)s * bm.ld + u] += co;
          bm.MT[(size_t)u * bm.ld + s] += co;
          chunk_add(bm.CS, bm.nch, r, u, -co);
          chunk_add(bm.CST, bm.nch, u, r, -co);
          chunk_add(bm.CS, bm.nch, s, u, co);
          chunk_add(bm.CST, bm.nch, u, s, co);
        }
        if (ci) {
          bm.M[(size_t)u * bm.ld + r] -= ci;
          bm.MT[(size_t)r * bm.ld + u] -= ci;
          bm.M[(size_t)u * bm.ld + s] += ci;
          bm.MT[(size_t)s * bm.ld + u] += ci;
          chunk_add(bm.CS, bm.nch, u, r, -ci);
          chunk_add(bm.CST, bm.nch, r, u, -ci);
          chunk_add(bm.CS, bm.nch, u, s, ci);
          chunk_add(bm.CST, bm.nch, s, u, ci);
        }
      }
      // only this group's lanes are here (the other groups of the warp may not commit): a
      // full-warp barrier would wait for lanes that never arrive
      __syncwarp(G == 32 ? kFull : ((1u << G) - 1u) << gbase);
      if (gl == 0) {
        const int self = e.self;
        const int d_rr = -co_r - ci_r - self, d_rs = -co_s + ci_r;
        const int d_sr = co_r - ci_s, d_ss = co_s + ci_s + self;
        const int cells[4][3] = {{r, r, d_rr}, {r, s, d_rs}, {s, r, d_sr}, {s, s, d_ss}};
        for (int q = 0; q < 4; ++q) {
          const int a = cells[q][0], b = cells[q][1], d = cells[q][2];
          if (!d) continue;
          bm.M[(size_t)a * bm.ld + b] += d;
          bm.MT[(size_t)b * bm.ld + a] += d;
          chunk_add(bm.CS, bm.nch, a, b, d);
          chunk_add(bm.CST, bm.nch, b, a, d);
        }
        bm.b[e.v] = s;
        bm.d_out[r] -= e.k_out;
        bm.d_out[s] += e.k_out;
        bm.d_in[r] -= e.k_in + self;
        bm.d_in[s] += e.k_in + self;
        // Blockmodel::move_vertex reads the already-updated diagonal and adds the delta again
        bm.d[r] = bm.d_out[r] + bm.d_in[r] - (bm.M[(size_t)r * bm.ld + r] + d_rr);
        bm.d[s] = bm.d_out[s] + bm.d_in[s] - (bm.M[(size_t)s * bm.ld + s] + d_ss);
      }
    }
    pos += s_upto;
    group_table_clear<kHash, G>(T, gl);
    __threadfence_block();
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = (double)visits;
    out[1] = (double)moved;
    out[2] = (double)accepted;
    out[3] = sum_dS;
    out[4] = 0.0;
  }
}

}  // namespace

GibbsEvalGroupKernel gibbs_eval_group_kernel(bool hashed_table) {
  return hashed_table ? k_gibbs_eval_group<kSmallGroup, true> : k_gibbs_eval_group<kSmallGroup, false>;
}

size_t gibbs_eval_group_smem(bool hashed_table, int cap) {
  const int groups = kSmallThreads / kSmallGroup;
  const int slots = hashed_table ? cap : kSmallB;
  return sizeof(int) * ((size_t)groups + (size_t)groups * (hashed_table ? 3 : 2) * slots);
}

MhGroupKernel mh_group_kernel(bool hashed_table) {
  return hashed_table ? k_mh_group<kSmallGroup, true> : k_mh_group<kSmallGroup, false>;
}

size_t mh_group_smem(bool hashed_table, int cap) {
  const int groups = kMhGroupThreads / kSmallGroup;
  const int slots = hashed_table ? cap : kSmallB;
  return sizeof(int) * ((size_t)groups + (size_t)groups * (hashed_table ? 3 : 2) * slots);
}

}  // namespace sbpb
