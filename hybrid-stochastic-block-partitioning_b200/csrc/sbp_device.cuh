// Device-side building blocks of the B200 stochastic block partitioning engine:
// counter-based random numbers, warp primitives, the per-warp neighbour-block table, and the
// warp-cooperative vertex-move evaluation (proposal, Hastings correction, delta-MDL, accept).
//
// Semantics follow the reference (vtsynergy/Hybrid-Stochastic-Block-Partitioning):
//   proposal          src/common.cpp:131-192  (canonical row-then-column multinomial order)
//   hastings          src/entropy.cpp:495-557 (new degree of r/s ignores the in-side self edge)
//   delta-MDL         src/entropy.cpp:296-401 (a present Delta cell with net change 0 and a
//                     non-zero count at (r,s) or (s,r) is counted twice, as the reference's
//                     "unchanged cell" loops do)
//   accept            src/finetune.cpp:19-29
// Log terms are FP64. delta-MDL uses the closed form
//   dS = sum_changed [g(M)-g(M')] - sum_{x in r,s} [g(d_out x)-g(d_out' x)] - [same for d_in] + Q
// with g(x) = x log x, which equals the reference's per-cell sum over rows/cols r,s.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sbpb {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Error bits written to the device status word (never trap).
enum : int {
  kErrTableFull = 1,      // neighbour-block table overflow
  kErrScan = 2,           // multinomial walk ran off the row (inconsistent counts)
  kErrReplay = 4,         // replay record index out of range
  kErrBounds = 8,         // block or vertex id out of range
};

// ------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11). Counter (a, b, call, tag), key = seed.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

struct RngParams {
  uint64_t seed;
  const uint4* replay;      // optional host-supplied stream (device copy)
  long long replay_records;
  uint32_t call;
  int moves = 0;            // 1: replay records are proposals (s, 0, u_hi, u_lo), not random words
};

// The accept uniform of a proposal record: the bits of a double in [0, 1).
__device__ __forceinline__ double record_uniform(uint4 x) {
  return __hiloint2double((int)x.z, (int)x.w);
}

// Record for (a, b, tag); replay records are indexed by `slot`.
__device__ __forceinline__ uint4 draw_record(const RngParams& p, uint32_t a, uint32_t b, uint32_t tag,
                                             long long slot, int* status) {
  if (p.replay) {
    if (slot < 0 || slot >= p.replay_records) {
      atomicOr(status, kErrReplay);
      return make_uint4(0, 0, 0, 0xffffffffu);   // u_acc ~ 1: never accepts
    }
    return p.replay[slot];
  }
  return philox4x32_10(make_uint4(a, b, p.call, tag), (uint32_t)p.seed, (uint32_t)(p.seed >> 32));
}

__device__ __forceinline__ long long scale32(uint32_t x, long long n) {
  return (long long)(((unsigned long long)x * (unsigned long long)n) >> 32);
}
__device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
  const unsigned long long m = ((unsigned long long)hi << 21) | (unsigned long long)(lo >> 11);
  return (double)m * (1.0 / 9007199254740992.0);
}
// common::propose_random_block with a scaled 32-bit draw.
__device__ __forceinline__ int random_block(int r, int B, uint32_t x) {
  int p = (int)scale32(x, (long long)B - 1);
  return p >= r ? p + 1 : p;
}

// ------------------------------------------------------------------------------------------
// FP64 helpers: g(x) = x log x and accurate differences g(a) - g(b).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double xlogx(double x) { return x > 0.0 ? x * log(x) : 0.0; }
// g(a) - g(b) = (a - b) log a + b (log a - log b) for a, b >= 0 without branches: a zero side
// is replaced by 1 inside the logs, which leaves exactly the other side's g term; a == b gives 0.
__device__ __forceinline__ double dxlogx(double a, double b) {
  const double sa = a > 0.0 ? a : 1.0, sb = b > 0.0 ? b : 1.0;
  return (a - b) * log(sa) + b * log1p((sa - sb) / sb);
}

// g(a) - g(b) for integer counts a, b >= 0 as (a - b) log a + b log(a / b), from a table of
// log(x) = hi + lo (lo carries the bits below hi's last place):
//  - a close to b (128 |a - b| <= b, b > 0): log(a / b) = 2 atanh(z), z = (a - b) / (a + b), by its
//    Taylor series 2 (z + z^3/3 + z^5/5 + z^7/7), |z| <= 1/255, which keeps the relative
//    accuracy that a difference of two table logs would lose;
//  - otherwise log(a / b) = (hi_a - hi_b) + (lo_a - lo_b).
// A zero side uses log 1 = 0, which leaves the other side's g term.  Counts beyond the table
// go through dxlogx.
constexpr int kLogTable = 1 << 20;
__device__ __forceinline__ double dxlogx_int(const double2* __restrict__ logt, int a, int b) {
  if (a < kLogTable && b < kLogTable) {
    const int d = a - b;
    const double2 la = __ldg(logt + (a > 0 ? a : 1));
    double lab;
    if (b > 0 && 128LL * (d < 0 ? -(long long)d : (long long)d) <= (long long)b) {
      const double z = (double)d / ((double)a + (double)b), w = z * z;
      lab = 2.0 * z + 2.0 * z * w * (1.0 / 3.0 + w * (1.0 / 5.0 + w * (1.0 / 7.0)));
    } else {
      const double2 lb = __ldg(logt + (b > 0 ? b : 1));
      lab = (la.x - lb.x) + (la.y - lb.y);
    }
    return (double)d * (la.x + la.y) + (double)b * lab;
  }
  return dxlogx((double)a, (double)b);
}

// Merge delta-MDLs are rounded to a multiple of 2^-20 (about 1e-6) before merges are ranked:
// values that are equal but for the rounding of different summation orders then compare equal
// on every implementation, and equal values rank by proposal order and block index, as the
// reference's loops rank exact ties.  (rint: round half to even, the same as the host's
// nearbyint in the default rounding mode.)
__host__ __device__ __forceinline__ double merge_score(double dS) { return rint(dS * 1048576.0) / 1048576.0; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ long long warp_incl_scan(long long v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long n = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

// ------------------------------------------------------------------------------------------
// Device views of the graph and the blockmodel.
// ------------------------------------------------------------------------------------------
struct GraphView {
  int V;
  long long E;
  double log_E;           // log(max(E, 2)), the zero-snap scale of a delta-MDL
  const int* out_ptr;     // [V+1]
  const int* out_idx;     // out-neighbours incl. self loop, first-occurrence order
  const int* in_ptr;      // [V+1]
  const int* in_idx;      // in-neighbours, self loop removed
  const unsigned char* self;
};

constexpr int kChunk = 128;   // columns per chunk-sum entry

struct BlockView {
  int B;
  int sparse;             // 0: dense M/MT below; 1: row-hashed regions (large B)
  // row-hashed storage: row r of M lives in rslot[rbase[r] .. rbase[r] + rmask[r]], slots
  // (col, count), col = -1 for an empty slot; MT likewise in cslot.  Keys are never removed
  // (a count can drop to 0).  An insertion that finds its row full sets overflow[0] and the
  // row's flag: overflow[1 + row] for a row of M, overflow[1 + B + row] for a row of MT.
  const long long* rbase;
  const int* rmask;
  int2* rslot;
  const long long* cbase;
  const int* cmask;
  int2* cslot;
  int* overflow;
  int ld;                 // row stride of M and MT (multiple of kChunk ints)
  int nch;                // chunks per row = ceil(B / kChunk)
  int* CS;                // [B*nch] CS[row*nch+c] = sum of M[row, c*kChunk .. c*kChunk+kChunk)
  int* CST;               // [B*nch] the same over MT (column sums of M per chunk of rows)
  int* b;                 // [V] assignment
  int* M;                 // [B*ld] row-major counts M[row*ld+col]
  int* MT;                // [B*ld] transpose: MT[col*ld+row] = M[row*ld+col]
  int* d_out;             // [B]
  int* d_in;              // [B]
  int* d;                 // [B] block degrees as the reference maintains them
  const double2* logt;    // [kLogTable] log(x) = hi + lo for integer x (entry 0 unused)
};

// Walk values row[0..n) ascending and return the first index whose running sum exceeds
// `target` (skipping index `skip`). Warp-cooperative; returns -1 if the row is exhausted.
// Plain (coherent) loads: the Metropolis-Hastings kernel updates M while it runs.
__device__ __forceinline__ int warp_select_dense(const int* row, int n, long long target, int skip,
                                                 int lane) {
  for (int base = 0; base < n; base += kWarp) {
    const int c = base + lane;
    long long v = (c < n && c != skip) ? (long long)row[c] : 0;
    const long long incl = warp_incl_scan(v, lane);
    const long long tot = __shfl_sync(kFull, incl, 31);
    if (target < tot) {
      const unsigned hit = __ballot_sync(kFull, incl > target);
      return base + __ffs(hit) - 1;
    }
    target -= tot;
  }
  return -1;
}

// ---- row-hashed storage ------------------------------------------------------------------
__device__ __forceinline__ unsigned slot_hash(int key) { return (unsigned)key * 2654435761u; }

__device__ __forceinline__ int hashed_get(const long long* base, const int* mask, const int2* slot, int row, int col) {
  const long long b0 = base[row];
  const int m = mask[row];
  unsigned h = slot_hash(col) & (unsigned)m;
  for (int probe = 0; probe <= m; ++probe) {
    const int2 e = slot[b0 + h];
    if (e.x == col) return e.y;
    if (e.x == -1) return 0;
    h = (h + 1) & (unsigned)m;
  }
  return 0;
}

__device__ __forceinline__ void hashed_add(const long long* base, const int* mask, int2* slot, int row, int col,
                                           int delta, int* overflow, int* row_full) {
  const long long b0 = base[row];
  const int m = mask[row];
  unsigned h = slot_hash(col) & (unsigned)m;
  for (int probe = 0; probe <= m; ++probe) {
    int* key = &slot[b0 + h].x;
    int k = *(volatile int*)key;
    if (k == -1) {
      const int prev = atomicCAS(key, -1, col);
      k = prev == -1 ? col : prev;
    }
    if (k == col) {
      atomicAdd(&slot[b0 + h].y, delta);
      return;
    }
    h = (h + 1) & (unsigned)m;
  }
  atomicOr(overflow, 1);
  row_full[row] = 1;
}

// M[row, col] and MT[row, col] = M[col, row] in either representation.
// Storage of the block matrix as a compile-time choice (kAny: decided by bm.sparse at run time).
// Kernels instantiated for one storage carry no code for the other.
enum class Store { kAny, kDense, kHashed, kDenseFrozen };
// kDenseFrozen: dense storage that no thread of the launch writes (the evaluation half of an
// asynchronous-Gibbs batch), read through the read-only data cache.
template <Store S>
__device__ __forceinline__ int ldi(const int* p) {
  if constexpr (S == Store::kDenseFrozen) return __ldg(p);
  else return *p;
}

template <Store S = Store::kAny>
__device__ __forceinline__ int bm_get(const BlockView& bm, int row, int col) {
  if constexpr (S == Store::kDense) return bm.M[(size_t)row * bm.ld + col];
  else if constexpr (S == Store::kDenseFrozen) return __ldg(bm.M + (size_t)row * bm.ld + col);
  else if constexpr (S == Store::kHashed) return hashed_get(bm.rbase, bm.rmask, bm.rslot, row, col);
  else return bm.sparse ? hashed_get(bm.rbase, bm.rmask, bm.rslot, row, col) : bm.M[(size_t)row * bm.ld + col];
}
template <Store S = Store::kAny>
__device__ __forceinline__ int bm_getT(const BlockView& bm, int row, int col) {
  if constexpr (S == Store::kDense) return bm.MT[(size_t)row * bm.ld + col];
  else if constexpr (S == Store::kDenseFrozen) return __ldg(bm.MT + (size_t)row * bm.ld + col);
  else if constexpr (S == Store::kHashed) return hashed_get(bm.cbase, bm.cmask, bm.cslot, row, col);
  else return bm.sparse ? hashed_get(bm.cbase, bm.cmask, bm.cslot, row, col) : bm.MT[(size_t)row * bm.ld + col];
}

// Walk of a hashed row in ascending column order: the first column whose running count
// exceeds `target`, found digit by digit (5 bits of the column at a time, most significant
// first).  Each pass sums the row's counts of the columns left in range into 32 bins (`bins`:
// 32 ints of the warp's shared memory), scans the bins and keeps the one that holds the target.
// Same result as the dense walks.
__device__ __forceinline__ int warp_select_hashed(const long long* base, const int* mask, const int2* slot, int row,
                                                  int B, long long target, int lane, int* bins) {
  const long long b0 = base[row];
  const int cap = mask[row] + 1;
  int bits = 0;
  while ((1 << bits) < B) ++bits;
  int lo = 0;
  for (int shift = ((bits + 4) / 5) * 5 - 5; shift >= 0; shift -= 5) {
    bins[lane] = 0;
    __syncwarp();
    const long long span = 32LL << shift;
    for (int i = lane; i < cap; i += kWarp) {
      const int2 e = slot[b0 + i];
      if (e.x >= lo && (long long)e.x < lo + span && e.y > 0) atomicAdd(&bins[(e.x - lo) >> shift], e.y);
    }
    __syncwarp();
    const long long v = bins[lane];
    const long long incl = warp_incl_scan(v, lane);
    const unsigned hit = __ballot_sync(kFull, incl > target);
    if (!hit) return -1;
    const int sel = __ffs(hit) - 1;
    target -= __shfl_sync(kFull, incl - v, sel);
    lo += sel << shift;
    __syncwarp();
  }
  return lo;
}

__device__ __forceinline__ int select_in_chunk(int4 q, int chunk, long long target, int lane);

// Two-level walk: find the chunk through the chunk sums, then the column inside the chunk
// with one 16-byte load per lane.  Same result as warp_select_dense on the full row.  Up to
// kWideChunks chunks, lane i loads the sums of chunks [16 i, 16 i + 16) at once (one memory
// round trip instead of one per 32 chunks), scans its lane total across the warp and walks its
// sixteen sums; longer rows take 32 chunks per step.
constexpr int kWideChunks = 16 * kWarp;
// The wide walk over chunk sums already loaded: lane i holds the sums of chunks [16 i, 16 i + 16)
// (0 beyond the row).
__device__ __forceinline__ int walk_loaded_chunk_sums(const int* row, const int (&cs)[16], long long target,
                                                      int lane) {
  long long lsum = 0;
#pragma unroll
  for (int q = 0; q < 16; ++q) lsum += cs[q];
  const long long incl = warp_incl_scan(lsum, lane);
  const unsigned hit = __ballot_sync(kFull, incl > target);
  if (!hit) return -1;
  const int src = __ffs(hit) - 1;
  int chunk = -1;
  long long before = 0;
  if (lane == src) {
    long long run = incl - lsum;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      if (chunk < 0) {
        if (target < run + cs[q]) {
          chunk = lane * 16 + q;
          before = run;
        } else {
          run += cs[q];
        }
      }
    }
  }
  chunk = __shfl_sync(kFull, chunk, src);
  before = __shfl_sync(kFull, before, src);
  const int4 q4 = *reinterpret_cast<const int4*>(row + chunk * kChunk + 4 * lane);
  return select_in_chunk(q4, chunk, target - before, lane);
}

__device__ __forceinline__ int warp_select_chunked(const int* row, const int* csum, int nch, long long target,
                                                   int lane) {
  if (nch <= kWideChunks) {
    int cs[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int c = lane * 16 + q;
      cs[q] = c < nch ? csum[c] : 0;
    }
    return walk_loaded_chunk_sums(row, cs, target, lane);
  }
  int chunk = -1;
  for (int base = 0; base < nch; base += kWarp) {
    const int c = base + lane;
    const long long v = c < nch ? (long long)csum[c] : 0;
    const long long incl = warp_incl_scan(v, lane);
    const long long tot = __shfl_sync(kFull, incl, 31);
    if (target < tot) {
      const unsigned hit = __ballot_sync(kFull, incl > target);
      const int src = __ffs(hit) - 1;
      target -= __shfl_sync(kFull, incl - v, src);
      chunk = base + src;
      break;
    }
    target -= tot;
  }
  if (chunk < 0) return -1;
  const int4 q = *reinterpret_cast<const int4*>(row + chunk * kChunk + 4 * lane);
  return select_in_chunk(q, chunk, target, lane);
}

// The column inside one chunk of kChunk counts (four per lane, q) at which the running sum
// first exceeds target; -1 if the chunk is exhausted.
__device__ __forceinline__ int select_in_chunk(int4 q, int chunk, long long target, int lane) {
  const long long lsum = (long long)q.x + q.y + q.z + q.w;
  const long long incl = warp_incl_scan(lsum, lane);
  const unsigned hit = __ballot_sync(kFull, incl > target);
  if (!hit) return -1;
  const int src = __ffs(hit) - 1;
  long long t = target - __shfl_sync(kFull, incl - lsum, src);
  const int qx = __shfl_sync(kFull, q.x, src), qy = __shfl_sync(kFull, q.y, src), qz = __shfl_sync(kFull, q.z, src);
  int k = 3;
  if (t < qx) k = 0;
  else if (t < (long long)qx + qy) k = 1;
  else if (t < (long long)qx + qy + qz) k = 2;
  return chunk * kChunk + 4 * src + k;
}

// The walk of warp_select_chunked for a row of at most 32 chunks whose chunk sums are already
// loaded (lane c holds chunk c's sum, 0 beyond the row).
__device__ __forceinline__ int select_chunk_then_column(const int* row, int csum_lane, long long target, int lane) {
  const long long v = csum_lane;
  const long long incl = warp_incl_scan(v, lane);
  const long long tot = __shfl_sync(kFull, incl, 31);
  if (target >= tot) return -1;
  const unsigned hit = __ballot_sync(kFull, incl > target);
  const int src = __ffs(hit) - 1;
  target -= __shfl_sync(kFull, incl - v, src);
  const int4 q = *reinterpret_cast<const int4*>(row + src * kChunk + 4 * lane);
  return select_in_chunk(q, src, target, lane);
}

__device__ __forceinline__ void chunk_add(int* cs, int nch, int row, int col, int delta) {
  atomicAdd(cs + (size_t)row * nch + col / kChunk, delta);
}

// Same walk over a compressed list (idx[i], val[i]), i in [0, n).
__device__ __forceinline__ int warp_select_sparse(const int* __restrict__ idx, const int* __restrict__ val, int n,
                                                  long long target, int skip, int lane) {
  for (int base = 0; base < n; base += kWarp) {
    const int i = base + lane;
    int c = -1;
    long long v = 0;
    if (i < n) {
      c = idx[i];
      v = (c != skip) ? (long long)val[i] : 0;
    }
    const long long incl = warp_incl_scan(v, lane);
    const long long tot = __shfl_sync(kFull, incl, 31);
    if (target < tot) {
      const unsigned hit = __ballot_sync(kFull, incl > target);
      return __shfl_sync(kFull, c, __ffs(hit) - 1);
    }
    target -= tot;
  }
  return -1;
}

// ------------------------------------------------------------------------------------------
// Per-warp neighbour-block table in shared memory: open addressing on block id, with a
// compact list of used slots so reset and enumeration cost O(distinct blocks).
// ------------------------------------------------------------------------------------------
struct WarpTable {
  int* keys;   // [cap], -1 = empty
  int* cout;   // [cap] out-neighbour counts (self loop excluded)
  int* cin;    // [cap] in-neighbour counts (self loop excluded)
  int* list;   // [cap] used slots
  int* nlist;  // [1]
  int mask;    // cap - 1 (cap power of two)
};

__device__ __forceinline__ int table_slot(const WarpTable& t, int key, int* status) {
  unsigned h = ((unsigned)key * 2654435761u) & (unsigned)t.mask;
  for (int probe = 0; probe <= t.mask; ++probe) {
    const int k = t.keys[h];
    if (k == key) return (int)h;
    if (k == -1) {
      const int prev = atomicCAS(&t.keys[h], -1, key);
      if (prev == -1) {
        t.list[atomicAdd(t.nlist, 1)] = (int)h;
        return (int)h;
      }
      if (prev == key) return (int)h;
    }
    h = (h + 1) & (unsigned)t.mask;
  }
  atomicOr(status, kErrTableFull);
  return -1;
}

__device__ __forceinline__ int table_find(const WarpTable& t, int key) {
  unsigned h = ((unsigned)key * 2654435761u) & (unsigned)t.mask;
  for (int probe = 0; probe <= t.mask; ++probe) {
    const int k = t.keys[h];
    if (k == key) return (int)h;
    if (k == -1) return -1;
    h = (h + 1) & (unsigned)t.mask;
  }
  return -1;
}

// Warp-aggregated insertion: lanes holding the same key add their multiplicity once.
__device__ __forceinline__ void table_add(const WarpTable& t, int key, bool valid, bool incoming, int* status) {
  const int k = valid ? key : -2;
  const unsigned peers = __match_any_sync(kFull, k);
  const int lane = threadIdx.x & 31;
  if (valid && (__ffs(peers) - 1) == lane) {
    const int slot = table_slot(t, key, status);
    if (slot >= 0) atomicAdd(incoming ? &t.cin[slot] : &t.cout[slot], __popc(peers));
  }
}

// Per-warp table of `cap` slots carved from a CTA's dynamic shared memory (table_ints(cap) ints per warp).
__device__ __forceinline__ WarpTable carve_table(int* base, int cap, int warp) {
  int* p = base + (size_t)warp * (4 * cap + 64);
  WarpTable t;
  t.keys = p;
  t.cout = p + cap;
  t.cin = p + 2 * cap;
  t.list = p + 3 * cap;
  t.nlist = p + 4 * cap;
  t.mask = cap - 1;
  return t;
}

__device__ __forceinline__ void init_table(const WarpTable& t, int lane) {
  const int cap = t.mask + 1;
  for (int i = lane; i < cap; i += kWarp) {
    t.keys[i] = -1;
    t.cout[i] = 0;
    t.cin[i] = 0;
  }
  if (lane == 0) *t.nlist = 0;
  __syncwarp();
}

__device__ __forceinline__ void table_reset(const WarpTable& t, int lane) {
  __syncwarp();
  const int n = *t.nlist;
  for (int i = lane; i < n; i += kWarp) {
    const int h = t.list[i];
    t.keys[h] = -1;
    t.cout[h] = 0;
    t.cin[h] = 0;
  }
  __syncwarp();
  if (lane == 0) *t.nlist = 0;
  __syncwarp();
}

// Build the table for vertex v from the current assignment (self loop excluded; block r is
// inserted when v has a self loop so the Hastings sum sees it).
__device__ __forceinline__ void build_table(const GraphView& g, const BlockView& bm, int v, int r, const WarpTable& t,
                                            int lane, int* status) {
  const int o0 = g.out_ptr[v], o1 = g.out_ptr[v + 1];
  for (int e0 = o0; e0 < o1; e0 += kWarp) {
    const int e = e0 + lane;
    int key = -1;
    bool valid = false;
    if (e < o1) {
      const int u = __ldg(g.out_idx + e);
      if (u != v) { key = bm.b[u]; valid = true; }
    }
    table_add(t, key, valid, false, status);
  }
  const int i0 = g.in_ptr[v], i1 = g.in_ptr[v + 1];
  for (int e0 = i0; e0 < i1; e0 += kWarp) {
    const int e = e0 + lane;
    int key = -1;
    bool valid = false;
    if (e < i1) { key = bm.b[__ldg(g.in_idx + e)]; valid = true; }
    table_add(t, key, valid, true, status);
  }
  if (lane == 0 && g.self[v]) table_slot(t, r, status);
  __syncwarp();
}

struct EvalResult {
  int t;          // block of the proposal's neighbour (-1: no neighbour, uniform proposal)
  int s;          // proposed block
  int accepted;   // 1 if accepted (s != r)
  double dS;      // delta MDL (0 when s == r)
  double H;       // Hastings correction
};

struct MoveCounts {   // self-loop-free neighbour counts by block for the four corner blocks
  int co_r, co_s, ci_r, ci_s;
};

__device__ __forceinline__ MoveCounts corner_counts(const WarpTable& t, int r, int s) {
  MoveCounts mc;
  const int hr = table_find(t, r), hs = table_find(t, s);
  mc.co_r = hr >= 0 ? t.cout[hr] : 0;
  mc.ci_r = hr >= 0 ? t.cin[hr] : 0;
  mc.co_s = hs >= 0 ? t.cout[hs] : 0;
  mc.ci_s = hs >= 0 ? t.cin[hs] : 0;
  return mc;
}

// Warp-aggregated insertion of one element per lane; lanes holding the same block add their
// out- and in-multiplicities once.
__device__ __forceinline__ void table_add_dir(const WarpTable& t, int key, bool valid, bool incoming, int* status) {
  const int k = valid ? key : -2;
  const unsigned peers = __match_any_sync(kFull, k);
  const unsigned in_mask = __ballot_sync(kFull, valid && incoming);
  const int lane = threadIdx.x & 31;
  if (valid && (__ffs(peers) - 1) == lane) {
    const int slot = table_slot(t, key, status);
    if (slot >= 0) {
      const int nin = __popc(peers & in_mask), nout = __popc(peers) - nin;
      if (nout) atomicAdd(&t.cout[slot], nout);
      if (nin) atomicAdd(&t.cin[slot], nin);
    }
  }
}

// One pass over v's virtual neighbour list (out list incl. the self loop, then in list without
// it) gathers every neighbour's block into the table (self loop excluded from the counts, its
// block r inserted with zero counts).  Returns the block of neighbour element `idx` (-1 when
// idx is out of range), the proposal's neighbour of src/common.cpp:11-26.
template <Store ST = Store::kAny>
__device__ __forceinline__ int gather_neighbour_blocks(const GraphView& g, const BlockView& bm, int v, int r, int o0,
                                                       int k_out, int i0, int k, int self, int idx,
                                                       const WarpTable& t, int lane, int* status) {
  int tblk = -1;
  for (int base = 0; base < k; base += 2 * kWarp) {   // two elements per lane in flight
    const int e0 = base + lane, e1 = base + kWarp + lane;
    int u0 = -1, u1 = -1;
    if (e0 < k) u0 = e0 < k_out ? __ldg(g.out_idx + o0 + e0) : __ldg(g.in_idx + i0 + (e0 - k_out));
    if (e1 < k) u1 = e1 < k_out ? __ldg(g.out_idx + o0 + e1) : __ldg(g.in_idx + i0 + (e1 - k_out));
    const int b0 = u0 >= 0 ? ldi<ST>(bm.b + u0) : -1;
    const int b1 = u1 >= 0 ? ldi<ST>(bm.b + u1) : -1;
    if (idx >= base && idx < base + kWarp) tblk = __shfl_sync(kFull, b0, idx - base);
    if (idx >= base + kWarp && idx < base + 2 * kWarp) tblk = __shfl_sync(kFull, b1, idx - base - kWarp);
    table_add_dir(t, b0, u0 >= 0 && u0 != v, e0 >= k_out, status);
    table_add_dir(t, b1, u1 >= 0 && u1 != v, e1 >= k_out, status);
  }
  if (lane == 0 && self) table_slot(t, r, status);
  return tblk;
}

// Loads of move_delta that do not depend on the proposed block s: issued right after the
// neighbour table is built, so that they overlap the multinomial walk that picks s.
struct NbPrefetch {
  int u, co, ci, M_ru, M_ur, du;   // this lane's first table entry (u = -1: none)
  int M_rr, dout_r, din_r;
};

template <Store ST = Store::kAny>
__device__ __forceinline__ void prefetch_nb(const BlockView& bm, int r, const WarpTable& t, int lane, NbPrefetch* p) {
  __syncwarp();
  const int n = *t.nlist;
  p->u = -1;
  p->co = p->ci = p->M_ru = p->M_ur = p->du = 0;
  if (lane < n) {
    const int h = t.list[lane];
    const int u = t.keys[h];
    p->u = u;
    p->co = t.cout[h];
    p->ci = t.cin[h];
    p->M_ru = bm_get<ST>(bm, r, u);
    p->M_ur = bm_getT<ST>(bm, r, u);
    p->du = ldi<ST>(bm.d + u);
  }
  p->M_rr = bm_get<ST>(bm, r, r);
  p->dout_r = ldi<ST>(bm.d_out + r);
  p->din_r = ldi<ST>(bm.d_in + r);
}

// Position of the n-th (0-based) set bit of m; requires n < popc(m).
__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const int c = __popc(m & ((1u << w) - 1u));
    if (n >= c) {
      n -= c;
      m >>= w;
      pos += w;
    }
  }
  return pos;
}

// Delta-MDL of moving v from r to s (s != r) against the current state, with the gathered
// table of v's neighbour blocks, and the reference's Hastings correction (*H).
//  - One load round over the distinct neighbour blocks (lane i: table entries i, i+32, ...)
//    gives the Hastings sums and the changed cells.
//  - The FP64 terms are then spread over the warp one term per lane: the eight corner-cell
//    and degree terms, and two cells per (neighbour block, direction) pair that changes:
//    (r,u) and (s,u) for v's out-edges to u, (u,r) and (u,s) for its in-edges from u.
//  - The double count of a present net-zero (r,s) / (s,r) Delta cell is added by the lanes
//    that hold it, and only then.
// Every lane returns the same values.
template <Store ST = Store::kAny>
__device__ __forceinline__ double move_delta(const GraphView& g, const BlockView& bm, int r, int s, int k_out,
                                             int k_in, int self, const WarpTable& t, int lane, double* H,
                                             const NbPrefetch* pre = nullptr) {
  __syncwarp();
  const MoveCounts mc = corner_counts(t, r, s);
  const int B = bm.B;
  const int d_rr = -mc.co_r - mc.ci_r - self;
  const int d_rs = -mc.co_s + mc.ci_r;
  const int d_sr = mc.co_r - mc.ci_s;
  const int d_ss = mc.co_s + mc.ci_s + self;
  const int M_rr = pre ? pre->M_rr : bm_get<ST>(bm, r, r), M_rs = bm_get<ST>(bm, r, s);
  const int M_sr = bm_get<ST>(bm, s, r), M_ss = bm_get<ST>(bm, s, s);
  const int dout_r = pre ? pre->dout_r : ldi<ST>(bm.d_out + r), dout_s = ldi<ST>(bm.d_out + s);
  const int din_r = pre ? pre->din_r : ldi<ST>(bm.d_in + r), din_s = ldi<ST>(bm.d_in + s);
  const int kin_self = k_in + self;

  double fwd = 0.0, bwd = 0.0, dS = 0.0;
  long long T = 0;   // integer scale of the changed cells and degrees (zero snap below)
  const int n = *t.nlist;
  for (int base = 0; base < n; base += kWarp) {
    const int i = base + lane;
    int M_su = 0, M_us = 0, M_ru = 0, M_ur = 0, co_c = 0, ci_c = 0;
    if (i < n) {
      int u, co, ci, du;
      if (pre && base == 0) {
        u = pre->u;
        co = pre->co;
        ci = pre->ci;
        M_ru = pre->M_ru;
        M_ur = pre->M_ur;
        du = pre->du;
      } else {
        const int h = t.list[i];
        u = t.keys[h];
        co = t.cout[h];
        ci = t.cin[h];
        M_ru = bm_get<ST>(bm, r, u);
        M_ur = bm_getT<ST>(bm, r, u);
        du = ldi<ST>(bm.d + u);
      }
      M_su = bm_get<ST>(bm, s, u);
      M_us = bm_getT<ST>(bm, s, u);
      const bool is_r = (u == r), is_s = (u == s), corner = is_r || is_s;
      const double c = (double)(co + ci + (is_r ? self : 0));
      const double inv_u = 1.0 / ((double)du + (double)B);   // a non-corner block's degree is unchanged
      fwd += c * (M_su + M_us + 1.0) * inv_u;
      const double bw = is_r ? (double)(M_rr + d_rr) + (double)(M_rr + d_rr) + 1.0
                      : is_s ? (double)(M_rs + d_rs) + (double)(M_sr + d_sr) + 1.0
                             : (double)(M_ru - co) + (double)(M_ur - ci) + 1.0;
      const int nd = is_r ? (dout_r - k_out) + (din_r - k_in) - (M_rr + d_rr)
                   : is_s ? (dout_s + k_out) + (din_s + k_in) - (M_ss + d_ss) : du;
      bwd += c * bw * (corner ? 1.0 / ((double)nd + (double)B) : inv_u);
      // changed non-corner cells (r,u) (s,u) (u,r) (u,s); corner cells are terms 0-3 below
      co_c = corner ? 0 : co;
      ci_c = corner ? 0 : ci;
      T += (co_c ? 2LL * (M_ru + M_su) : 0LL) + (ci_c ? 2LL * (M_ur + M_us) : 0LL);
    }
    const unsigned m_out = __ballot_sync(kFull, co_c != 0), m_in = __ballot_sync(kFull, ci_c != 0);
    const int n_out = __popc(m_out), n_terms_cells = 2 * (n_out + __popc(m_in));
    const int extra = base == 0 ? 8 : 0;   // corner-cell and degree terms, once
    const int n_terms = extra + n_terms_cells;
    for (int q0 = 0; q0 < n_terms; q0 += kWarp) {
      const int q = q0 + lane;
      const int cell = q - extra;
      const int pair = cell >> 1;
      const bool is_cell = q >= extra && q < n_terms;
      const bool out_pair = pair < n_out;
      const int owner = !is_cell ? lane : out_pair ? nth_set_bit(m_out, pair) : nth_set_bit(m_in, pair - n_out);
      const int x_ru = __shfl_sync(kFull, M_ru, owner), x_su = __shfl_sync(kFull, M_su, owner);
      const int x_ur = __shfl_sync(kFull, M_ur, owner), x_us = __shfl_sync(kFull, M_us, owner);
      const int x_co = __shfl_sync(kFull, co_c, owner), x_ci = __shfl_sync(kFull, ci_c, owner);
      int a = 0, d = 0;
      double sign = 1.0;
      if (is_cell) {
        const bool s_side = cell & 1;
        a = out_pair ? (s_side ? x_su : x_ru) : (s_side ? x_us : x_ur);
        const int m = out_pair ? x_co : x_ci;
        d = s_side ? m : -m;
      } else if (q < extra) {
        // corner cells (r,r) (r,s) (s,r) (s,s), then the out- and in-degrees of r and s
        a = q == 0 ? M_rr : q == 1 ? M_rs : q == 2 ? M_sr : q == 3 ? M_ss
          : q == 4 ? dout_r : q == 5 ? dout_s : q == 6 ? din_r : din_s;
        d = q == 0 ? d_rr : q == 1 ? d_rs : q == 2 ? d_sr : q == 3 ? d_ss
          : q == 4 ? -k_out : q == 5 ? k_out : q == 6 ? -kin_self : kin_self;
        sign = q < 4 ? 1.0 : -1.0;
      }
      if (d) dS += sign * dxlogx_int(bm.logt, a, a + d);
    }
  }
  if (lane < 8) {
    const int ca = lane == 0 ? M_rr : lane == 1 ? M_rs : lane == 2 ? M_sr : lane == 3 ? M_ss
                 : lane == 4 ? dout_r : lane == 5 ? dout_s : lane == 6 ? din_r : din_s;
    const int cd = lane == 0 ? d_rr : lane == 1 ? d_rs : lane == 2 ? d_sr : lane == 3 ? d_ss
                 : lane == 4 ? -k_out : lane == 5 ? k_out : lane == 6 ? -kin_self : kin_self;
    T += lane < 4 ? (cd ? 2LL * ca + cd : 0LL) : 2LL * ca;
  }
  {
    // the double count of a present net-zero (r,s) / (s,r) Delta cell (lanes 8 and 9)
    const bool q_rs = (mc.co_s > 0 || mc.ci_r > 0) && d_rs == 0 && M_rs > 0;
    const bool q_sr = (mc.co_r > 0 || mc.ci_s > 0) && d_sr == 0 && M_sr > 0;
    const int qm = lane == 8 ? (q_rs ? M_rs : 0) : lane == 9 ? (q_sr ? M_sr : 0) : 0;
    if (qm) {
      const double x1 = lane == 8 ? (double)kin_self / (double)din_s : -(double)kin_self / (double)din_r;
      const double x2 = lane == 8 ? -(double)k_out / (double)dout_r : (double)k_out / (double)dout_s;
      dS += (double)qm * (log1p(x1) + log1p(x2));
    }
  }
  fwd = warp_sum(fwd);
  bwd = warp_sum(bwd);
  dS = warp_sum(dS);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) T += __shfl_xor_sync(kFull, T, o);
  // A mathematically zero change reads as exactly 0 whatever the summation order: the
  // Metropolis-Hastings early stop tests `delta == 0.0` (src/finetune.cpp:147).
  if (fabs(dS) <= 0x1p-40 * (double)T * g.log_E) dS = 0.0;
  *H = bwd / fwd;
  return dS;
}

// Full evaluation of vertex v against the current state, table left filled on return
// (caller resets it). Every lane returns the same result.
//  1. gather_neighbour_blocks; the proposal's neighbour (element floor(x0 * k)) is one of the
//     gathered elements, so its block comes from the same pass;
//  2. the multinomial walk over M[t,:] + M[:,t] picks s;
//  3. move_delta gives delta-MDL and the Hastings correction.
//
// `given`: x is a proposal record (s, 0, u_hi, u_lo) of a replayed stream: the proposal is x.x
// and the accept uniform the double of (x.z, x.w); steps 1 (without the neighbour pick) and 3.
template <Store ST = Store::kAny>
__device__ __forceinline__ EvalResult evaluate_vertex(const GraphView& g, const BlockView& bm, int v, uint4 x,
                                                      const WarpTable& t, int lane, int* status, int* r_out,
                                                      int* k_out_out, int* k_in_out, bool given = false) {
  EvalResult res;
  const int r = ldi<ST>(bm.b + v);
  const int o0 = g.out_ptr[v], o1 = g.out_ptr[v + 1];
  const int i0 = g.in_ptr[v], i1 = g.in_ptr[v + 1];
  const int self = g.self[v];
  const int k_out = o1 - o0, k_in = i1 - i0, k = k_out + k_in;
  *r_out = r;
  *k_out_out = k_out;
  *k_in_out = k_in;
  res.accepted = 0;
  res.dS = 0.0;
  res.H = 1.0;
  const int idx = (k > 0 && !given) ? (int)scale32(x.x, k) : -1;
  const int tblk = gather_neighbour_blocks<ST>(g, bm, v, r, o0, k_out, i0, k, self, idx, t, lane, status);
  res.t = (k > 0 && !given) ? tblk : -1;

  NbPrefetch pre;
  prefetch_nb<ST>(bm, r, t, lane, &pre);

  int s;
  if (given) {
    s = (int)x.x;
    if (s < 0 || s >= bm.B) {   // a visit the stream has no proposal for
      if (lane == 0) atomicOr(status, kErrReplay);
      s = r;
    }
  } else if (k == 0) {
    s = random_block(r, bm.B, x.y);
  } else {
    const bool hashed = ST == Store::kHashed || (ST == Store::kAny && bm.sparse);
    if (ST != Store::kDense && hashed) {
      const int dot = bm.d_out[tblk];
      const long long target = scale32(x.y, (long long)dot + (long long)bm.d_in[tblk]);
      int* bins = t.nlist + 32;   // the 32 ints after the table's list count
      if (target < dot) s = warp_select_hashed(bm.rbase, bm.rmask, bm.rslot, tblk, bm.B, target, lane, bins);
      else s = warp_select_hashed(bm.cbase, bm.cmask, bm.cslot, tblk, bm.B, target - dot, lane, bins);
    } else if (ST != Store::kHashed) {
      // the degrees of t and, in the same round trip, row t of M and of MT (B <= kChunk: the
      // whole rows, four counts per lane) or their chunk sums (up to 32 chunks); the walk then
      // picks the row (target < d_out[t]) or the column.  (Loading the chunk sums of
      // both rows with the degrees for up to 512 chunks as well was measured 13 % slower at
      // 11,770 blocks and no faster above.)
      const int dot = ldi<ST>(bm.d_out + tblk), dit = ldi<ST>(bm.d_in + tblk);
      const size_t ro = (size_t)tblk * bm.ld, co = (size_t)tblk * bm.nch;
      int4 qa = make_int4(0, 0, 0, 0), qb = make_int4(0, 0, 0, 0);
      int ca = 0, cb = 0;
      if (bm.nch == 1) {
        if constexpr (ST == Store::kDenseFrozen) {
          qa = __ldg(reinterpret_cast<const int4*>(bm.M + ro) + lane);
          qb = __ldg(reinterpret_cast<const int4*>(bm.MT + ro) + lane);
        } else {
          qa = *reinterpret_cast<const int4*>(bm.M + ro + 4 * lane);
          qb = *reinterpret_cast<const int4*>(bm.MT + ro + 4 * lane);
        }
      } else if (lane < bm.nch) {
        ca = ldi<ST>(bm.CS + co + lane);
        cb = ldi<ST>(bm.CST + co + lane);
      }
      const long long target = scale32(x.y, (long long)dot + (long long)dit);
      const bool in_row = target < dot;
      const long long tg = in_row ? target : target - dot;
      if (bm.nch == 1) s = select_in_chunk(in_row ? qa : qb, 0, tg, lane);
      else if (bm.nch <= kWarp) s = select_chunk_then_column(in_row ? bm.M + ro : bm.MT + ro, in_row ? ca : cb, tg, lane);
      else s = warp_select_chunked(in_row ? bm.M + ro : bm.MT + ro, in_row ? bm.CS + co : bm.CST + co, bm.nch, tg, lane);
    } else {
      s = -1;
    }
    if (s < 0) {
      if (lane == 0) atomicOr(status, kErrScan);
      s = r;
    }
  }
  res.s = s;
  if (s == r) return res;
  double Hp;
  const double dS = move_delta<ST>(g, bm, r, s, k_out, k_in, self, t, lane, &Hp, &pre);
  const double H = (k == 0) ? 1.0 : Hp;
  double ap = exp(-3.0 * dS) * H;
  ap = ap >= 1.0 ? 1.0 : ap;
  res.dS = dS;
  res.H = H;
  res.accepted = ((given ? record_uniform(x) : u53(x.z, x.w)) <= ap) ? 1 : 0;
  return res;
}

}  // namespace sbpb
