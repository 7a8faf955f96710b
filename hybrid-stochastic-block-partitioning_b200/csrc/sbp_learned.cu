// Learned proposal for the vertex moves of the MCMC finetune, beside the plain proposal of
// common::propose_new_block (src/common.cpp:131-182).  It has no counterpart in the reference.
//
// Proposal.  For vertex v in block r, the candidate blocks are v's 14 neighbour blocks with
// the most edges to v (ties: lower block id).  A network (sbp_mlp.cu) maps 64 features of v
// and its candidates to 15 logits (14 slots + escape).  With eps the uniform weight,
//   q(s | v, b) = (1 - eps) pi_slot(s) + ((1 - eps) pi_escape + eps) / B,
// and a draw takes slot j with (1 - eps) pi_j, otherwise a uniformly random block.  Features
// are a function of the assignment only (neighbour-block counts, block degrees d_out + d_in,
// B, E and v's own degrees), so the features of the state after the move r -> s follow
// exactly from the current state.  The Hastings factor q(r | v, b') / q(s | v, b) therefore
// uses the same network on those reverse features, and the chain keeps the stationary
// distribution of the plain method.  Acceptance: u <= min(1, exp(-3 dS) H) with dS from the
// plain path's delta-MDL (move_delta).
//
// Feature vector (index: value), k = k_out + k_in, E the edge count, dtot(u) = d_out[u] + d_in[u]:
//   4j+0, 4j+1 (slot j < nvalid): out- / in-edges from v to the slot's block, divided by k
//   4j+2: log1p(dtot(u_j)) / log1p(2E);  4j+3: 1 if u_j is v's block
//   56: log1p(k_out)/5  57: log1p(k_in)/5  58: log(B)/10  59: nvalid/14
//   60: edges to v's block / k when that block is a slot, else 0  61: self loop
//   62: log1p(dtot(v's block)) / log1p(2E)  63: 1
//
// Training data: features and the chosen slot (escape when the accepted block is not a slot)
// of every move the plain asynchronous-Gibbs chain accepts.
#include <cuda_bf16.h>

#include <chrono>
#include <random>

#include "sbp_engine.cuh"
#include "sbp_mlp.cuh"
#include "sbp_steps.cuh"

using namespace sbpb;

struct SbpMlp {
  DevBuf<float> params, m, v, grads, bias;
  DevBuf<__nv_bfloat16> W1, W2, W3;
  DevBuf<double> loss;
  int step = 0;
  MlpWeights weights() const {
    MlpWeights w;
    w.W1 = W1.p;
    w.W2 = W2.p;
    w.W3 = W3.p;
    w.b1 = bias.p;
    w.b2 = bias.p + kMlpHid;
    w.b3 = bias.p + 2 * kMlpHid;
    return w;
  }
};

struct SbpDataset {
  DevBuf<__nv_bfloat16> X;
  DevBuf<int> target, nvalid, count;
  long long capacity = 0;
};

namespace sbpb {
namespace {

constexpr int kFeatSlots = kMlpSlots;

struct LearnedParams {
  float inv_log2E;   // 1 / log1p(2E)
  float eps;         // uniform weight of the mixture
};

__device__ __forceinline__ float feat_degree(long long dtot, float inv_log2E) {
  return log1pf((float)dtot) * inv_log2E;
}

__device__ __forceinline__ void slot_features(int co, int ci, float kf, long long dtot, bool is_cur, float inv,
                                              float* f) {
  f[0] = (float)co / kf;
  f[1] = (float)ci / kf;
  f[2] = feat_degree(dtot, inv);
  f[3] = is_cur ? 1.f : 0.f;
}

__device__ __forceinline__ void global_features(int k_out, int k_in, int B, int nvalid, int c_cur, float kf, int self,
                                                long long dtot_cur, float inv, float* f) {
  f[0] = log1pf((float)k_out) / 5.f;
  f[1] = log1pf((float)k_in) / 5.f;
  f[2] = logf((float)B) / 10.f;
  f[3] = (float)nvalid / 14.f;
  f[4] = (float)c_cur / kf;
  f[5] = self ? 1.f : 0.f;
  f[6] = feat_degree(dtot_cur, inv);
  f[7] = 1.f;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(kFull, x, o);
    x = y > x ? y : x;
  }
  return x;
}

// Features of v against the current state, written as one BF16 row; the candidate slots
// (block, edge count) and (r, k_out, k_in, self | nvalid << 1) go to slot_row / info.
// The table must hold v's gathered neighbour blocks.  Lane j < 14 ends with slot j's block
// in *my_block (-1 when invalid).
__device__ __forceinline__ void vertex_features(const BlockView& bm, const WarpTable& t, int r, int k_out, int k_in,
                                                int self, LearnedParams lp, int lane, __nv_bfloat16* frow,
                                                int2* slot_row, int4* info, int* my_block, int* nvalid_out) {
  const int n = *t.nlist;
  const int k = k_out + k_in;
  const float kf = (float)(k > 0 ? k : 1);
  // top-14 (count desc, block asc) among entries with a nonzero count (the self loop's block
  // enters the table with zero counts and never becomes a candidate)
  unsigned long long mine = 0ull, prev = ~0ull;
  int nvalid = 0;
  for (int j = 0; j < kFeatSlots; ++j) {
    unsigned long long best = 0ull;
    for (int i = lane; i < n; i += kWarp) {
      const int h = t.list[i];
      const int c = t.cout[h] + t.cin[h];
      if (c <= 0) continue;
      const unsigned long long P = ((unsigned long long)(unsigned)c << 32) | (0xFFFFFFFFu - (unsigned)t.keys[h]);
      if (P < prev && P > best) best = P;
    }
    best = warp_max_u64(best);
    if (best == 0ull) break;
    if (lane == j) mine = best;
    prev = best;
    nvalid = j + 1;
  }
  int u = -1, co = 0, ci = 0;
  if (lane < nvalid) {
    u = (int)(0xFFFFFFFFu - (unsigned)(mine & 0xFFFFFFFFull));
    const int h = table_find(t, u);
    co = t.cout[h];
    ci = t.cin[h];
  }
  const unsigned has_r = __ballot_sync(kFull, lane < nvalid && u == r);
  const int c_r = has_r ? __shfl_sync(kFull, co + ci, __ffs(has_r) - 1) : 0;
  if (lane < kFeatSlots) {
    float f[4] = {0.f, 0.f, 0.f, 0.f};
    if (lane < nvalid)
      slot_features(co, ci, kf, (long long)bm.d_out[u] + (long long)bm.d_in[u], u == r, lp.inv_log2E, f);
    const __nv_bfloat162 a = __floats2bfloat162_rn(f[0], f[1]), b = __floats2bfloat162_rn(f[2], f[3]);
    uint2 pk;
    pk.x = *reinterpret_cast<const unsigned*>(&a);
    pk.y = *reinterpret_cast<const unsigned*>(&b);
    *reinterpret_cast<uint2*>(frow + 4 * lane) = pk;
    slot_row[lane] = make_int2(u, co + ci);
  } else if (lane == kFeatSlots) {
    float f[8];
    global_features(k_out, k_in, bm.B, nvalid, c_r, kf, self, (long long)bm.d_out[r] + (long long)bm.d_in[r],
                    lp.inv_log2E, f);
    unsigned w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
      w[q] = *reinterpret_cast<const unsigned*>(&h2);
    }
    *reinterpret_cast<uint4*>(frow + 56) = make_uint4(w[0], w[1], w[2], w[3]);
    *info = make_int4(r, k_out, k_in, self | (nvalid << 1));
  }
  *my_block = u;
  *nvalid_out = nvalid;
}

struct BatchBufs {
  __nv_bfloat16* F1;
  __nv_bfloat16* F2;
  int2* slot;     // [n][14]
  int4* info;     // [n]
  int* s_prop;    // [n]
  double* qf;     // [n]
  float* L1;      // [n][16]
  float* L2;      // [n][16]
};

// Features of vertex v against the current state into row `row` of the batch buffers (one
// warp; the table is left filled, the caller resets it).
__device__ __forceinline__ void features_row(const GraphView& g, const BlockView& bm, int v, int row, BatchBufs bb,
                                             LearnedParams lp, const WarpTable& t, int lane, int* status) {
  const int r = bm.b[v];
  const int o0 = g.out_ptr[v], k_out = g.out_ptr[v + 1] - o0;
  const int i0 = g.in_ptr[v], k_in = g.in_ptr[v + 1] - i0;
  const int self = g.self[v];
  gather_neighbour_blocks(g, bm, v, r, o0, k_out, i0, k_out + k_in, self, -1, t, lane, status);
  __syncwarp();
  int blk, nv;
  vertex_features(bm, t, r, k_out, k_in, self, lp, lane, bb.F1 + (size_t)row * kMlpIn,
                  bb.slot + (size_t)row * kFeatSlots, bb.info + row, &blk, &nv);
}

// Features of the batch's vertices (rows row0 .. row0 + n - 1 of the batch buffers).
__global__ void k_learn_features(GraphView g, BlockView bm, const int* __restrict__ verts, int n, int row0,
                                 BatchBufs bb, LearnedParams lp, int cap, int* status) {
  extern __shared__ int smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  for (int i = blockIdx.x * wpb + warp; i < n; i += gridDim.x * wpb) {
    features_row(g, bm, verts[i], row0 + i, bb, lp, t, lane, status);
    table_reset(t, lane);
  }
}

// q(target | logits) of the mixture; slot = candidate slot of the target block or -1.
__device__ __forceinline__ double learned_q(const float* L, int nvalid, int slot, float eps, int B) {
  float mx = L[kMlpEscape];
  for (int j = 0; j < nvalid; ++j) mx = fmaxf(mx, L[j]);
  double S = exp((double)(L[kMlpEscape] - mx));
  for (int j = 0; j < nvalid; ++j) S += exp((double)(L[j] - mx));
  const double esc = exp((double)(L[kMlpEscape] - mx)) / S;
  const double w = 1.0 - (double)eps;
  double q = (w * esc + (double)eps) / (double)B;
  if (slot >= 0) q += w * exp((double)(L[slot] - mx)) / S;
  return q;
}

// Draw s for vertex v (row i) from the forward logits, store q(s), and build the reverse-state
// features.  One thread.
__device__ __forceinline__ void propose_row(int i, int v, const BlockView& bm, BatchBufs bb, LearnedParams lp,
                                            const RngParams& rng, int sweep, long long V, int* status) {
  const uint4 x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * V + v, status);
  const int4 inf = bb.info[i];
  const int r = inf.x, k_out = inf.y, k_in = inf.z, self = inf.w & 1, nvalid = inf.w >> 1;
  const int B = bm.B;
  const float* L = bb.L1 + (size_t)i * kMlpOut;
  const int2* sl = bb.slot + (size_t)i * kFeatSlots;
  // categorical draw over the slots and the escape
  float mx = L[kMlpEscape];
  for (int j = 0; j < nvalid; ++j) mx = fmaxf(mx, L[j]);
  double S = exp((double)(L[kMlpEscape] - mx));
  for (int j = 0; j < nvalid; ++j) S += exp((double)(L[j] - mx));
  const double w = 1.0 - (double)lp.eps;
  const double u = (double)x.x * 0x1p-32;
  double acc = 0.0;
  int pick = -1;
  for (int j = 0; j < nvalid; ++j) {
    acc += w * exp((double)(L[j] - mx)) / S;
    if (u < acc) {
      pick = j;
      break;
    }
  }
  const int s = pick >= 0 ? sl[pick].x : (int)scale32(x.y, (long long)B);
  bb.s_prop[i] = s;
  if (s == r) return;
  int slot_s = -1;
  for (int j = 0; j < nvalid; ++j)
    if (sl[j].x == s) slot_s = j;
  bb.qf[i] = learned_q(L, nvalid, slot_s, lp.eps, B);
  // reverse state: v in s; dtot of r and s change by k_out + k_in + self
  const int k = k_out + k_in;
  const float kf = (float)(k > 0 ? k : 1);
  const long long mv = (long long)k_out + k_in + self;
  const long long dt_r = (long long)bm.d_out[r] + bm.d_in[r] - mv;
  const long long dt_s = (long long)bm.d_out[s] + bm.d_in[s] + mv;
  const __nv_bfloat16* f1 = bb.F1 + (size_t)i * kMlpIn;
  __nv_bfloat16* f2 = bb.F2 + (size_t)i * kMlpIn;
  for (int q = 0; q < kMlpIn; ++q) f2[q] = f1[q];
  for (int j = 0; j < nvalid; ++j) {
    const int uj = sl[j].x;
    if (uj != r && uj != s) continue;
    f2[4 * j + 2] = __float2bfloat16_rn(feat_degree(uj == r ? dt_r : dt_s, lp.inv_log2E));
    f2[4 * j + 3] = __float2bfloat16_rn(uj == s ? 1.f : 0.f);
  }
  float g[8];
  const int c_s = slot_s >= 0 ? sl[slot_s].y : 0;
  global_features(k_out, k_in, B, nvalid, c_s, kf, self, dt_s, lp.inv_log2E, g);
  f2[56 + 4] = __float2bfloat16_rn(g[4]);
  f2[56 + 6] = __float2bfloat16_rn(g[6]);
}

// Draw s from the forward logits, store q(s), and build the reverse-state features.
__global__ void k_learn_propose(const int* __restrict__ verts, int n, BlockView bm, BatchBufs bb, LearnedParams lp,
                                RngParams rng, int sweep, long long V, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  propose_row(i, verts[i], bm, bb, lp, rng, sweep, V, status);
}

// Delta-MDL of the drawn move, the exact Hastings factor from the reverse logits, accept.
__global__ void k_learn_eval(GraphView g, BlockView bm, const int* __restrict__ verts, int n, int row0,
                             BatchBufs bb, LearnedParams lp, RngParams rng, int sweep, int* prop, int* moved_list,
                             int* n_moved, unsigned long long* counters, double* out_dS, double* out_H, int cap,
                             int* status) {
  extern __shared__ int smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  unsigned long long c_visit = 0, c_moved = 0, c_acc = 0;
  for (int i = blockIdx.x * wpb + warp; i < n; i += gridDim.x * wpb) {
    const int row = row0 + i;
    const int v = verts[i];
    c_visit++;
    const int4 inf = bb.info[row];
    const int r = inf.x, k_out = inf.y, k_in = inf.z, self = inf.w & 1, nvalid = inf.w >> 1;
    const int s = bb.s_prop[row];
    if (s == r) continue;
    c_moved++;
    const uint4 x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * g.V + v, status);
    const int o0 = g.out_ptr[v], i0 = g.in_ptr[v];
    gather_neighbour_blocks(g, bm, v, r, o0, k_out, i0, k_out + k_in, self, -1, t, lane, status);
    double Hp;
    const double dS = move_delta(g, bm, r, s, k_out, k_in, self, t, lane, &Hp);
    int slot_r = -1;
    const int2* sl = bb.slot + (size_t)row * kFeatSlots;
    for (int j = 0; j < nvalid; ++j)
      if (sl[j].x == r) slot_r = j;
    const double qr = learned_q(bb.L2 + (size_t)row * kMlpOut, nvalid, slot_r, lp.eps, bm.B);
    const double H = qr / bb.qf[row];
    double ap = exp(-3.0 * dS) * H;
    ap = ap >= 1.0 ? 1.0 : ap;
    const int accepted = (u53(x.z, x.w) <= ap) ? 1 : 0;
    if (lane == 0) {
      if (out_dS) out_dS[row] = dS;
      if (out_H) out_H[row] = H;
      if (accepted) {
        prop[v] = s;
        moved_list[atomicAdd(n_moved, 1)] = v;
      }
    }
    c_acc += accepted;
    table_reset(t, lane);
  }
  if (lane == 0 && c_visit) {
    atomicAdd(counters + 0, c_visit);
    atomicAdd(counters + 1, c_moved);
    atomicAdd(counters + 2, c_acc);
  }
}

// ------------------------------------------------------------------------------------------
// Sequential Metropolis-Hastings with the learned proposal (finetune::metropolis_hastings,
// src/finetune.cpp:412-444, with the proposal of :488-501 replaced).  A pass over a vertex list
// is a sequence of rounds over a window of list positions pos .. pos + W - 1, pos kept on the
// device so that rounds queue on the stream without the host:
//   k_learn_mh_features  features of the window's vertices against the current state (rows 0..W-1)
//   network              forward logits
//   k_learn_mh_propose   draw, q(s | v, state), reverse-state features
//   network              reverse logits
//   k_learn_mh_round     delta-MDL, exact Hastings factor and accept of every window vertex against
//                        the same state, then the commit rule of k_mh (mh_round_commits): the first
//                        accepted vertex and later ones no commit could have touched are applied,
//                        pos advances past the positions decided.
// The features read v's neighbour blocks, the degrees of those blocks and of v's own block, B and
// v's degrees; the reverse features the degrees of r and s.  A commit touches only the degrees of
// its own r and s, and a vertex whose neighbour moved holds that neighbour's old block, so the
// commit rule's independence test covers the learned draw as it covers the plain one: a vertex
// kept in a round was proposed, corrected and accepted exactly as the sequential chain would.
// out (doubles): [0] visits [1] proposals moved [2] accepted [3] sum of accepted dS, [4..9] the
// stop record of a hashed row that ran out of room (mh_apply_move).
// ------------------------------------------------------------------------------------------
constexpr int kMhRoundMaxWarps = 16;

__global__ void k_learn_mh_features(GraphView g, BlockView bm, const int* __restrict__ verts, int n,
                                    const int* __restrict__ pos_ptr, int W, BatchBufs bb, LearnedParams lp, int cap,
                                    int* status) {
  extern __shared__ int smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w = blockIdx.x * (blockDim.x >> 5) + warp;
  const int i = *pos_ptr + w;
  if (w >= W || i >= n) return;   // warp-uniform
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  features_row(g, bm, verts[i], w, bb, lp, t, lane, status);
}

__global__ void k_learn_mh_propose(const int* __restrict__ verts, int n, const int* __restrict__ pos_ptr, int W,
                                   BlockView bm, BatchBufs bb, LearnedParams lp, RngParams rng, int sweep,
                                   long long V, int* status) {
  const int w = threadIdx.x;
  const int i = *pos_ptr + w;
  if (w >= W || i >= n) return;
  propose_row(w, verts[i], bm, bb, lp, rng, sweep, V, status);
}

__global__ void __launch_bounds__(kMhRoundMaxWarps * 32)
    k_learn_mh_round(GraphView g, BlockView bm, const int* __restrict__ verts, int n, int* pos_ptr, BatchBufs bb,
                     LearnedParams lp, RngParams rng, int sweep, int cap, double* out, int* status) {
  extern __shared__ int smem[];
  __shared__ int s_acc[32], s_moved[32], s_r[32], s_s[32], s_t[32], s_commit[32];
  __shared__ double s_dS[32];
  __shared__ int s_stop, s_upto;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int W = blockDim.x >> 5;
  const int pos = *pos_ptr;
  // the list is done, or a hashed row ran out of room in an earlier round and the host has not
  // yet rebuilt the rows: nothing to do (the same for every thread)
  if (pos >= n || out[4] != 0.0) return;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  const int i = pos + warp;
  int v = -1, r = -1, s = -1, k_out = 0, k_in = 0, acc = 0;
  double dS = 0.0;
  if (i < n) {
    v = verts[i];
    const int4 inf = bb.info[warp];
    r = inf.x;
    k_out = inf.y;
    k_in = inf.z;
    const int self = inf.w & 1, nvalid = inf.w >> 1;
    s = bb.s_prop[warp];
    gather_neighbour_blocks(g, bm, v, r, g.out_ptr[v], k_out, g.in_ptr[v], k_out + k_in, self, -1, t, lane, status);
    if (s != r) {
      const uint4 x = draw_record(rng, (uint32_t)v, (uint32_t)sweep, 0u, (long long)sweep * g.V + v, status);
      double Hp;
      dS = move_delta(g, bm, r, s, k_out, k_in, self, t, lane, &Hp);
      int slot_r = -1;
      const int2* sl = bb.slot + (size_t)warp * kFeatSlots;
      for (int j = 0; j < nvalid; ++j)
        if (sl[j].x == r) slot_r = j;
      const double qr = learned_q(bb.L2 + (size_t)warp * kMlpOut, nvalid, slot_r, lp.eps, bm.B);
      const double H = qr / bb.qf[warp];
      double ap = exp(-3.0 * dS) * H;
      ap = ap >= 1.0 ? 1.0 : ap;
      acc = (u53(x.z, x.w) <= ap) ? 1 : 0;
    }
  }
  if (lane == 0) {
    s_acc[warp] = acc;
    s_moved[warp] = (i < n && s != r) ? 1 : 0;
    s_dS[warp] = dS;
    s_r[warp] = r;
    s_s[warp] = s;
    s_t[warp] = -1;   // the learned draw reads no row of a proposal block
    s_commit[warp] = 0;
  }
  if (threadIdx.x == 0) s_stop = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    int first;
    s_upto = mh_round_commits(bm, smem, cap, min(W, n - pos), s_acc, s_r, s_s, s_t, s_commit, &first);
  }
  __syncthreads();
  if (s_commit[warp]) mh_apply_move(g, bm, t, v, r, s, k_out, k_in, lane, pos + warp, out, &s_stop);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int upto = s_upto;
    double moved = out[1], accepted = out[2], sum_dS = out[3];
    for (int w = 0; w < upto; ++w) {
      moved += s_moved[w];
      if (s_commit[w]) {   // accepted moves in vertex order, summed in that order over the pass
        accepted += 1.0;
        sum_dS += s_dS[w];
      }
    }
    out[0] += (double)upto;
    out[1] = moved;
    out[2] = accepted;
    out[3] = sum_dS;
    *pos_ptr = pos + upto;
  }
}

// Training samples from the moves the plain chain just accepted (state before the apply).
__global__ void k_learn_collect(GraphView g, BlockView bm, const int* __restrict__ moved, const int* n_moved,
                                const int* __restrict__ prop, LearnedParams lp, __nv_bfloat16* X, int* target,
                                int* nvalid_out, int* count, long long capacity, int cap, int* status) {
  extern __shared__ int smem[];
  __shared__ int2 slots[kFeatSlots];
  __shared__ int4 info;
  const int lane = threadIdx.x & 31;
  WarpTable t = carve_table(smem, cap, 0);   // one warp per CTA
  init_table(t, lane);
  const int n = *n_moved;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int v = moved[i];
    const int s = prop[v];
    const int r = bm.b[v];
    const int o0 = g.out_ptr[v], k_out = g.out_ptr[v + 1] - o0;
    const int i0 = g.in_ptr[v], k_in = g.in_ptr[v + 1] - i0;
    const int self = g.self[v];
    gather_neighbour_blocks(g, bm, v, r, o0, k_out, i0, k_out + k_in, self, -1, t, lane, status);
    __syncwarp();
    int pos = 0;
    if (lane == 0) pos = atomicAdd(count, 1);
    pos = __shfl_sync(kFull, pos, 0);
    if (pos < capacity) {
      int blk, nv;
      vertex_features(bm, t, r, k_out, k_in, self, lp, lane, X + (size_t)pos * kMlpIn, slots, &info, &blk, &nv);
      const unsigned hit = __ballot_sync(kFull, lane < nv && blk == s);
      if (lane == 0) {
        target[pos] = hit ? __ffs(hit) - 1 : kMlpEscape;
        nvalid_out[pos] = nv;
      }
    }
    table_reset(t, lane);
  }
}

// q(target | v, state) of the forward path for given target blocks.
__global__ void k_learn_q(const int* __restrict__ targets, int n, BatchBufs bb, LearnedParams lp, int B, double* q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int nvalid = bb.info[i].w >> 1;
  const int2* sl = bb.slot + (size_t)i * kFeatSlots;
  int slot = -1;
  for (int j = 0; j < nvalid; ++j)
    if (sl[j].x == targets[i]) slot = j;
  q[i] = learned_q(bb.L1 + (size_t)i * kMlpOut, nvalid, slot, lp.eps, B);
}

__global__ void k_gather_rows(const __nv_bfloat16* __restrict__ X, const int* __restrict__ target,
                              const int* __restrict__ nvalid, const int* __restrict__ idx, int n, __nv_bfloat16* Xo,
                              int* to, int* no) {
  const int lane = threadIdx.x & 7;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3; i < n; i += (gridDim.x * blockDim.x) >> 3) {
    const int src = idx[i];
    reinterpret_cast<uint4*>(Xo + (size_t)i * kMlpIn)[lane] =
        reinterpret_cast<const uint4*>(X + (size_t)src * kMlpIn)[lane];
    if (lane == 0) {
      to[i] = target[src];
      no[i] = nvalid[src];
    }
  }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
struct LearnScratch {
  DevBuf<__nv_bfloat16> F1, F2;
  DevBuf<int2> slot;
  DevBuf<int4> info;
  DevBuf<int> s_prop;
  DevBuf<double> qf;
  DevBuf<float> L1, L2;
  DevBuf<int> mh_pos;   // list position of the learned Metropolis-Hastings pass
  void reserve(size_t n) {
    const size_t rows = ((n + kMlpTile - 1) / kMlpTile) * kMlpTile;
    F1.reserve(rows * kMlpIn);
    F2.reserve(rows * kMlpIn);
    slot.reserve(rows * kFeatSlots);
    info.reserve(rows);
    s_prop.reserve(rows);
    qf.reserve(rows);
    L1.reserve(rows * kMlpOut);
    L2.reserve(rows * kMlpOut);
  }
  BatchBufs view() {
    BatchBufs b;
    b.F1 = F1.p;
    b.F2 = F2.p;
    b.slot = slot.p;
    b.info = info.p;
    b.s_prop = s_prop.p;
    b.qf = qf.p;
    b.L1 = L1.p;
    b.L2 = L2.p;
    return b;
  }
};
static LearnScratch g_learn;

static LearnedParams learned_params(const SbpGraph& g, float eps) {
  LearnedParams lp;
  lp.inv_log2E = (float)(1.0 / std::log1p(2.0 * (double)std::max<long long>(g.E, 1)));
  lp.eps = eps;
  return lp;
}

// Warp-per-vertex launch over n vertices with per-warp tables of `cap` slots.
template <class K, class... A>
static void launch_warps(K kernel, int n, int cap, int warps, A... args) {
  Context& c = Context::get();
  const size_t smem = (size_t)table_ints(cap) * sizeof(int) * warps;
  set_smem_limit((const void*)kernel, smem);
  kernel<<<grid_for(n, warps, 64 * c.num_sms), warps * 32, smem, c.stream>>>(args...);
  SBP_CHECK_LAUNCH();
}

static void check_tensor_status() {
  Context& c = Context::get();
  int st = 0;
  SBP_CUDA(SBP_COPY_ASYNC(&st, c.status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  if (st & kErrTensorWait) {
    SBP_CUDA(cudaMemsetAsync(c.status, 0, sizeof(int), c.stream));
    throw Error(SBP_ERR_DEVICE, "tensor-core completion wait gave up");
  }
  c.check_status();
}

// One sequential Metropolis-Hastings pass over verts (device list of n vertices) with the
// learned proposal: rounds of k_learn_mh_* launches queued in chunks, the host reading the list
// position back between chunks (and rebuilding hashed rows that ran out of room, as mh_pass).
static MhResult learned_mh_pass(SbpBlockmodel& bm, const SbpGraph& g, const int* verts, int n, int max_k,
                                const SbpMlp& mlp, LearnedParams lp, RngParams rng, int sweep) {
  Context& c = Context::get();
  MhResult res;
  if (n == 0) return res;
  const int cap = mh_cap(max_k);
  const size_t per_warp = (size_t)table_ints(cap) * sizeof(int);
  const int W = (int)std::min<size_t>(kMhRoundMaxWarps, kSmemBudget / per_warp);
  if (W < 1) throw Error(SBP_ERR_UNSUPPORTED, "vertex degree too large for the Metropolis-Hastings kernel");
  const int fw = std::min(W, 4);   // warps per CTA of the features launch
  set_smem_limit((const void*)k_learn_mh_features, per_warp * fw);
  set_smem_limit((const void*)k_learn_mh_round, per_warp * W);
  g_learn.reserve(W);
  g_learn.mh_pos.reserve(1);
  const BatchBufs bb = g_learn.view();
  int* pos = g_learn.mh_pos.p;
  SBP_CUDA(cudaMemsetAsync(pos, 0, sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(c.mh_out, 0, 10 * sizeof(double), c.stream));
  int at = 0, rounds = 8;
  double out[10];
  while (at < n) {
    for (int k = 0; k < rounds; ++k) {
      k_learn_mh_features<<<(W + fw - 1) / fw, fw * 32, per_warp * fw, c.stream>>>(g.view(), bm.view(), verts, n,
                                                                                 pos, W, bb, lp, cap, c.status);
      SBP_CHECK_LAUNCH();
      mlp_forward(bb.F1, W, mlp.weights(), bb.L1, c.status, c.num_sms, c.stream);
      SBP_CHECK_LAUNCH();
      k_learn_mh_propose<<<1, 32, 0, c.stream>>>(verts, n, pos, W, bm.view(), bb, lp, rng, sweep, g.V, c.status);
      SBP_CHECK_LAUNCH();
      mlp_forward(bb.F2, W, mlp.weights(), bb.L2, c.status, c.num_sms, c.stream);
      SBP_CHECK_LAUNCH();
      k_learn_mh_round<<<1, W * 32, per_warp * W, c.stream>>>(g.view(), bm.view(), verts, n, pos, bb, lp, rng, sweep,
                                                              cap, c.mh_out, c.status);
      SBP_CHECK_LAUNCH();
    }
    int now = 0;
    SBP_CUDA(SBP_COPY_ASYNC(&now, pos, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    SBP_CUDA(SBP_COPY_ASYNC(out, c.mh_out, sizeof(out), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    // every round decides at least one position, so a chunk that decided none means the rounds
    // did not run as designed
    if (now <= at) throw Error(SBP_ERR_DEVICE, "learned Metropolis-Hastings rounds made no progress");
    if (out[4] != 0.0) {
      // a hashed row ran out of room: rebuild the rows with more room (keeping d), finish that
      // move's d[r], d[s]; pos is already past the move
      rebuild(bm, g, false);
      ++g_overflow_rebuilds;
      k_fix_move_degrees<<<1, 1, 0, c.stream>>>(bm.view(), (int)out[6], (int)out[7], (int)out[8], (int)out[9]);
      SBP_CHECK_LAUNCH();
      SBP_CUDA(cudaMemsetAsync(c.mh_out + 4, 0, sizeof(double), c.stream));
    }
    // queue about as many rounds as the positions left need at the rate of this chunk
    const double per_round = std::max(1.0, (double)(now - at) / rounds);
    at = now;
    rounds = (int)std::min(256.0, std::max(1.0, std::ceil((double)(n - at) / per_round)));
  }
  res.visits = (long long)out[0];
  res.moved = (long long)out[1];
  res.accepted = (long long)out[2];
  res.sum_dS = out[3];
  return res;
}

// Learned-proposal evaluation of one batch (light then heavy vertices of the plan), then apply.
static void learned_batch(SbpBlockmodel& bm, const SbpGraph& g, const BatchPlan& plan, int bt, const SbpMlp& mlp,
                          LearnedParams lp, RngParams rng, int sweep) {
  Context& c = Context::get();
  const int nl = plan.light_n[bt], nh = plan.heavy_n[bt], n = nl + nh;
  if (n == 0) return;
  g_learn.reserve(n);
  BatchBufs bb = g_learn.view();
  const int* verts = plan.order.p + plan.light_begin[bt];   // heavy vertices follow the light ones
  if (nl > 0)
    launch_warps(k_learn_features, nl, g.light_cap, kLightWarps, g.view(), bm.view(), verts, nl, 0, bb, lp,
                 g.light_cap, c.status);
  if (nh > 0)
    launch_warps(k_learn_features, nh, g.heavy_cap, 1, g.view(), bm.view(), verts + nl, nh, nl, bb, lp, g.heavy_cap,
                 c.status);
  mlp_forward(bb.F1, n, mlp.weights(), bb.L1, c.status, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  k_learn_propose<<<grid_for(n, 128, 1 << 20), 128, 0, c.stream>>>(verts, n, bm.view(), bb, lp, rng, sweep, g.V,
                                                                    c.status);
  SBP_CHECK_LAUNCH();
  mlp_forward(bb.F2, n, mlp.weights(), bb.L2, c.status, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  int* n_cur = bm.n_moved.p + (bm.gen & 1);
  double* no_out = nullptr;
  if (nl > 0)
    launch_warps(k_learn_eval, nl, g.light_cap, kLightWarps, g.view(), bm.view(), verts, nl, 0, bb, lp, rng, sweep,
                 bm.prop.p, bm.moved.p, n_cur, c.counters, no_out, no_out, g.light_cap, c.status);
  if (nh > 0)
    launch_warps(k_learn_eval, nh, g.heavy_cap, 1, g.view(), bm.view(), verts + nl, nh, nl, bb, lp, rng, sweep,
                 bm.prop.p, bm.moved.p, n_cur, c.counters, no_out, no_out, g.heavy_cap, c.status);
  gibbs_apply(bm, g, n);
}

// Finetune with the learned proposal (mlp != NULL) or the plain one (mlp == NULL), recording
// the MDL after every sweep: Metropolis-Hastings (learned_mh_pass over every vertex),
// asynchronous Gibbs, or hybrid (learned_mh_pass over the high-degree list, then the batches).
// A learned sweep whose acceptance rate falls below fallback_acceptance switches the rest of the
// call to the plain proposal.  Early stop of Metropolis-Hastings: its own rule on each sweep's
// summed accepted delta-MDL (src/finetune.cpp:144-162, 436-440).  Otherwise stop_rule 0: the
// asynchronous_gibbs early stop (changes measured from the call's first MDL,
// src/finetune.cpp:40,74); 1: per-sweep MDL changes, as metropolis_hastings.
static void finetune_learned(SbpBlockmodel& bm, SbpGraph& g, int algorithm, const SbpFinetuneOptions& opt,
                             const SbpMlp* m, float eps, float fallback, int stop_rule, SbpTrace* trace,
                             SbpStats& st) {
  Context& c = Context::get();
  std::memset(&st, 0, sizeof st);
  st.num_blocks = bm.B;
  if (trace) trace->count = 0;
  if (bm.B == 1) {
    st.mdl = bm.overall_entropy;
    return;
  }
  RngParams rng;
  rng.seed = opt.seed;
  rng.replay = nullptr;
  rng.replay_records = 0;
  rng.call = opt.call;
  const int max_sweeps = (opt.max_sweeps <= 0 || opt.max_sweeps > kMaxIterations) ? kMaxIterations : opt.max_sweeps;
  const bool bracket = opt.bracket_established != 0;
  const LearnedParams lp = learned_params(g, eps);
  const bool mh = algorithm == SBP_METROPOLIS_HASTINGS;
  const BatchPlan* plan = mh ? nullptr : &g.plan(algorithm, opt.batches);
  SBP_CUDA(cudaMemsetAsync(c.counters, 0, 8 * sizeof(unsigned long long), c.stream));
  c.sync();
  const auto t0 = std::chrono::steady_clock::now();
  bm.overall_entropy = (float)mdl(bm, g);
  const double initial_entropy = bm.overall_entropy;
  double last_entropy = initial_entropy;
  std::vector<double> deltas;
  long long mh_visits = 0, mh_moved = 0, mh_acc = 0;
  bool learned = m != nullptr;
  unsigned long long prev[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int it = 0; it < max_sweeps; ++it) {
    long long pass_visits = 0, pass_acc = 0;   // this sweep's Metropolis-Hastings pass
    double pass_dS = 0.0;
    if (mh || (algorithm == SBP_HYBRID_MCMC && !g.high.empty())) {
      const int* list = mh ? g.identity.p : g.high_dev.p;
      const int nl = mh ? g.V : (int)g.high.size();
      const int mk = mh ? g.max_k : g.max_k_of(g.high);
      const MhResult r = learned ? learned_mh_pass(bm, g, list, nl, mk, *m, lp, rng, it)
                                 : mh_pass(bm, g, list, nl, mk, rng, it);
      mh_visits += r.visits;
      mh_moved += r.moved;
      mh_acc += r.accepted;
      pass_visits = r.visits;
      pass_acc = r.accepted;
      pass_dS = r.sum_dS;
    }
    if (!mh) {
      const long long ovf_sweep = g_overflow_rebuilds;
      for (size_t bt = 0; bt < plan->light_n.size(); ++bt) {
        if (learned) learned_batch(bm, g, *plan, (int)bt, *m, lp, rng, it);
        else gibbs_batch(bm, g, *plan, (int)bt, rng, it);
      }
      tidy_hashed(bm, g, ovf_sweep);
    }
    const double entropy = mdl(bm, g);
    if (mh) deltas.push_back(pass_dS);
    else deltas.push_back(stop_rule == 1 ? entropy - last_entropy : entropy - initial_entropy);
    last_entropy = entropy;
    st.sweeps++;
    if (learned) st.learned_sweeps++;
    check_tensor_status();
    unsigned long long cnt[8];
    SBP_CUDA(SBP_COPY_ASYNC(cnt, c.counters, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (trace && trace->count < trace->capacity) {
      trace->seconds[trace->count] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      trace->mdl[trace->count] = entropy;
      trace->count++;
    }
    if (learned) {
      const double v = (double)(cnt[0] - prev[0] + pass_visits), a = (double)(cnt[2] - prev[2] + pass_acc);
      if (v > 0 && a / v < (double)fallback) learned = false;
    }
    std::memcpy(prev, cnt, sizeof cnt);
    if (early_stop(it, bracket, initial_entropy, deltas)) break;
  }
  bm.overall_entropy = (float)mdl(bm, g);
  unsigned long long cnt[8];
  SBP_CUDA(SBP_COPY_ASYNC(cnt, c.counters, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  c.check_status();
  st.visits = (long long)cnt[0] + mh_visits;
  st.proposals_moved = (long long)cnt[1] + mh_moved;
  st.accepted = (long long)cnt[2] + mh_acc;
  st.mdl = bm.overall_entropy;
  st.mcmc_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  st.num_blocks = bm.B;
}

}  // namespace sbpb

// ------------------------------------------------------------------------------------------
// Network
// ------------------------------------------------------------------------------------------
static void mlp_upload(SbpMlp& m, const float* host_params) {
  Context& c = Context::get();
  SBP_CUDA(SBP_COPY_ASYNC(m.params.p, host_params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, c.stream));
  mlp_publish(m.params.p, m.W1.p, m.W2.p, m.W3.p, m.bias.p, c.stream);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(cudaMemsetAsync(m.m.p, 0, kMlpParams * sizeof(float), c.stream));
  SBP_CUDA(cudaMemsetAsync(m.v.p, 0, kMlpParams * sizeof(float), c.stream));
  m.step = 0;
  c.sync();
}

static void mlp_alloc(SbpMlp& m) {
  m.params.reserve(kMlpParams);
  m.m.reserve(kMlpParams);
  m.v.reserve(kMlpParams);
  m.grads.reserve(kMlpParams);
  m.bias.reserve(2 * kMlpHid + kMlpOut);
  m.W1.reserve(kMlpHid * kMlpIn);
  m.W2.reserve(kMlpHid * kMlpHid);
  m.W3.reserve(kMlpOut * kMlpHid);
  m.loss.reserve(1);
}

// He-normal weights from a seeded generator, zero biases.
static std::vector<float> mlp_init(uint64_t seed) {
  std::vector<float> p(kMlpParams, 0.f);
  std::mt19937_64 gen(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  const float s1 = std::sqrt(2.f / kMlpIn), s2 = std::sqrt(2.f / kMlpHid), s3 = 0.1f * std::sqrt(1.f / kMlpHid);
  for (int i = 0; i < kMlpHid * kMlpIn; ++i) p[kOffW1 + i] = s1 * nd(gen);
  for (int i = 0; i < kMlpHid * kMlpHid; ++i) p[kOffW2 + i] = s2 * nd(gen);
  for (int i = 0; i < kMlpOut * kMlpHid; ++i) p[kOffW3 + i] = s3 * nd(gen);
  return p;
}

#define SBP_API_BEGIN try {
#define SBP_API_END                          \
  return SBP_OK;                             \
  }                                          \
  catch (const Error& e) {                   \
    set_last_error(e.what());                 \
    return e.code;                           \
  }                                          \
  catch (const std::bad_alloc&) {            \
    set_last_error("host allocation failed"); \
    return SBP_ERR_OUT_OF_MEMORY;            \
  }                                          \
  catch (const std::exception& e) {          \
    set_last_error(e.what());                 \
    return SBP_ERR_CUDA;                     \
  }

#define SBP_REQUIRE(cond, msg) \
  if (!(cond)) throw Error(SBP_ERR_INVALID_ARGUMENT, msg)

static long long dataset_size(const SbpDataset& d) {
  Context& c = Context::get();
  int n = 0;
  SBP_CUDA(SBP_COPY_ASYNC(&n, d.count.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return std::min<long long>(n, d.capacity);
}

static void check_learned_options(const SbpLearnedOptions* lopt, float* eps, float* fallback, int* stop_rule) {
  *eps = lopt ? lopt->epsilon : 0.05f;
  *fallback = lopt ? lopt->fallback_acceptance : 0.f;
  *stop_rule = lopt ? lopt->stop_rule : 0;
  SBP_REQUIRE(*eps > 0.f && *eps <= 1.f, "epsilon must be in (0, 1]");
  SBP_REQUIRE(*stop_rule == 0 || *stop_rule == 1, "stop_rule must be 0 or 1");
}

extern "C" {

SbpStatus sbp_mlp_create(uint64_t seed, SbpMlp** out) {
  SBP_API_BEGIN
  SBP_REQUIRE(out, "null output pointer");
  *out = nullptr;
  auto m = std::make_unique<SbpMlp>();
  mlp_alloc(*m);
  const std::vector<float> p = mlp_init(seed);
  mlp_upload(*m, p.data());
  *out = m.release();
  SBP_API_END
}

SbpStatus sbp_mlp_destroy(SbpMlp* m) {
  SBP_API_BEGIN
  delete m;
  SBP_API_END
}

SbpStatus sbp_mlp_get_params(const SbpMlp* m, float* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(m && out, "null argument");
  Context& c = Context::get();
  SBP_CUDA(SBP_COPY_ASYNC(out, m->params.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_mlp_set_params(SbpMlp* m, const float* params) {
  SBP_API_BEGIN
  SBP_REQUIRE(m && params, "null argument");
  mlp_upload(*m, params);
  SBP_API_END
}

SbpStatus sbp_mlp_forward(const SbpMlp* m, int64_t n, const float* features, float* logits) {
  SBP_API_BEGIN
  SBP_REQUIRE(m && n >= 0 && (n == 0 || (features && logits)), "invalid argument");
  if (n == 0) return SBP_OK;
  Context& c = Context::get();
  DevBuf<float> xf, lo;
  DevBuf<__nv_bfloat16> xb;
  xf.reserve((size_t)n * kMlpIn);
  xb.reserve((size_t)n * kMlpIn);
  lo.reserve((size_t)n * kMlpOut);
  SBP_CUDA(SBP_COPY_ASYNC(xf.p, features, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, c.stream));
  float_to_bf16(xf.p, xb.p, n * kMlpIn, c.stream);
  mlp_forward(xb.p, n, m->weights(), lo.p, c.status, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(SBP_COPY_ASYNC(logits, lo.p, (size_t)n * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  check_tensor_status();
  SBP_API_END
}

SbpStatus sbp_mlp_gradients(const SbpMlp* cm, int64_t n, const float* features, const int32_t* target,
                            const int32_t* nvalid, float* grads, double* mean_loss) {
  SBP_API_BEGIN
  SBP_REQUIRE(cm && n > 0 && features && target && nvalid && grads, "invalid argument");
  SbpMlp* m = const_cast<SbpMlp*>(cm);
  Context& c = Context::get();
  long long counted = 0;
  for (int64_t i = 0; i < n; ++i) {
    SBP_REQUIRE(target[i] >= -1 && target[i] < kMlpOut - 1, "target must be -1 or a logit index below 15");
    SBP_REQUIRE(nvalid[i] >= 0 && nvalid[i] <= kMlpSlots, "nvalid must be in [0, 14]");
    SBP_REQUIRE(target[i] < 0 || target[i] == kMlpEscape || target[i] < nvalid[i], "target slot is masked");
    counted += target[i] >= 0;
  }
  DevBuf<float> xf;
  DevBuf<__nv_bfloat16> xb;
  DevBuf<int> tg, nv;
  xf.reserve((size_t)n * kMlpIn);
  xb.reserve((size_t)n * kMlpIn);
  tg.reserve(n);
  nv.reserve(n);
  SBP_CUDA(SBP_COPY_ASYNC(xf.p, features, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(tg.p, target, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(nv.p, nvalid, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  float_to_bf16(xf.p, xb.p, n * kMlpIn, c.stream);
  SBP_CUDA(cudaMemsetAsync(m->grads.p, 0, kMlpParams * sizeof(float), c.stream));
  SBP_CUDA(cudaMemsetAsync(m->loss.p, 0, sizeof(double), c.stream));
  mlp_gradients(xb.p, tg.p, nv.p, n, 1.f / (float)std::max<long long>(counted, 1), m->weights(), m->grads.p,
                m->loss.p, c.status, c.stream);
  SBP_CHECK_LAUNCH();
  double loss = 0.0;
  SBP_CUDA(SBP_COPY_ASYNC(grads, m->grads.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(&loss, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  check_tensor_status();
  if (mean_loss) *mean_loss = loss / (double)std::max<long long>(counted, 1);
  SBP_API_END
}

SbpStatus sbp_dataset_create(int64_t capacity, SbpDataset** out) {
  SBP_API_BEGIN
  SBP_REQUIRE(out && capacity > 0 && capacity <= INT32_MAX, "capacity must be in [1, 2^31)");
  *out = nullptr;
  Context& c = Context::get();
  auto d = std::make_unique<SbpDataset>();
  d->X.reserve((size_t)capacity * kMlpIn);
  d->target.reserve(capacity);
  d->nvalid.reserve(capacity);
  d->count.reserve(1);
  d->capacity = capacity;
  SBP_CUDA(cudaMemsetAsync(d->count.p, 0, sizeof(int), c.stream));
  c.sync();
  *out = d.release();
  SBP_API_END
}

SbpStatus sbp_dataset_destroy(SbpDataset* d) {
  SBP_API_BEGIN
  delete d;
  SBP_API_END
}

SbpStatus sbp_dataset_size(const SbpDataset* d, int64_t* out) {
  SBP_API_BEGIN
  SBP_REQUIRE(d && out, "null argument");
  *out = dataset_size(*d);
  SBP_API_END
}

SbpStatus sbp_dataset_append(SbpDataset* d, int64_t n, const float* features, const int32_t* target,
                             const int32_t* nvalid) {
  SBP_API_BEGIN
  SBP_REQUIRE(d && n >= 0 && (n == 0 || (features && target && nvalid)), "invalid argument");
  const long long size = dataset_size(*d);
  SBP_REQUIRE(size + n <= d->capacity, "dataset capacity exceeded");
  if (n == 0) return SBP_OK;
  for (int64_t i = 0; i < n; ++i) {
    SBP_REQUIRE(nvalid[i] >= 0 && nvalid[i] <= kMlpSlots, "nvalid must be in [0, 14]");
    SBP_REQUIRE(target[i] == kMlpEscape || (target[i] >= 0 && target[i] < nvalid[i]),
                "target must be a valid slot or the escape (14)");
  }
  Context& c = Context::get();
  DevBuf<float> xf;
  xf.reserve((size_t)n * kMlpIn);
  SBP_CUDA(SBP_COPY_ASYNC(xf.p, features, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, c.stream));
  float_to_bf16(xf.p, d->X.p + (size_t)size * kMlpIn, n * kMlpIn, c.stream);
  SBP_CUDA(SBP_COPY_ASYNC(d->target.p + size, target, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(d->nvalid.p + size, nvalid, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  const int newsize = (int)(size + n);
  SBP_CUDA(SBP_COPY_ASYNC(d->count.p, &newsize, sizeof(int), cudaMemcpyHostToDevice, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_dataset_read(const SbpDataset* d, int64_t offset, int64_t n, uint16_t* features_bf16, int32_t* target,
                           int32_t* nvalid) {
  SBP_API_BEGIN
  SBP_REQUIRE(d && offset >= 0 && n >= 0, "invalid argument");
  SBP_REQUIRE(offset + n <= dataset_size(*d), "range beyond the dataset");
  if (n == 0) return SBP_OK;
  Context& c = Context::get();
  if (features_bf16)
    SBP_CUDA(SBP_COPY_ASYNC(features_bf16, d->X.p + (size_t)offset * kMlpIn, (size_t)n * kMlpIn * 2,
                            cudaMemcpyDeviceToHost, c.stream));
  if (target)
    SBP_CUDA(SBP_COPY_ASYNC(target, d->target.p + offset, n * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  if (nvalid)
    SBP_CUDA(SBP_COPY_ASYNC(nvalid, d->nvalid.p + offset, n * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  SBP_API_END
}

SbpStatus sbp_mlp_train(SbpMlp* m, const SbpDataset* d, const SbpTrainOptions* opt, SbpTrainStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(m && d && opt, "null argument");
  SBP_REQUIRE(opt->epochs >= 0 && opt->batch >= 1 && opt->lr > 0.f, "invalid training options");
  Context& c = Context::get();
  const long long N = dataset_size(*d);
  SbpTrainStats st;
  std::memset(&st, 0, sizeof st);
  const auto t0 = std::chrono::steady_clock::now();
  if (N > 0 && opt->epochs > 0) {
    const int batch = opt->batch;
    DevBuf<int> idx, tg, nv;
    DevBuf<__nv_bfloat16> xb;
    DevBuf<double> epoch_loss;
    idx.reserve(N);
    tg.reserve(batch);
    nv.reserve(batch);
    xb.reserve((size_t)batch * kMlpIn);
    epoch_loss.reserve(1);
    std::vector<int> perm(N);
    std::mt19937_64 gen(opt->seed);
    double first = -1.0, last = 0.0;
    for (int ep = 0; ep < opt->epochs; ++ep) {
      std::iota(perm.begin(), perm.end(), 0);
      std::shuffle(perm.begin(), perm.end(), gen);
      SBP_CUDA(SBP_COPY_ASYNC(idx.p, perm.data(), N * sizeof(int), cudaMemcpyHostToDevice, c.stream));
      SBP_CUDA(cudaMemsetAsync(epoch_loss.p, 0, sizeof(double), c.stream));
      for (long long b0 = 0; b0 < N; b0 += batch) {
        const int nb = (int)std::min<long long>(batch, N - b0);
        k_gather_rows<<<grid_for((long long)nb * 8, 256, 1 << 16), 256, 0, c.stream>>>(
            d->X.p, d->target.p, d->nvalid.p, idx.p + b0, nb, xb.p, tg.p, nv.p);
        SBP_CHECK_LAUNCH();
        SBP_CUDA(cudaMemsetAsync(m->grads.p, 0, kMlpParams * sizeof(float), c.stream));
        mlp_gradients(xb.p, tg.p, nv.p, nb, 1.f / (float)nb, m->weights(), m->grads.p, epoch_loss.p, c.status,
                      c.stream);
        SBP_CHECK_LAUNCH();
        ++m->step;
        mlp_adam(m->params.p, m->m.p, m->v.p, m->grads.p, m->step, opt->lr, 0.9f, 0.999f, 1e-8f, m->W1.p, m->W2.p,
                 m->W3.p, m->bias.p, c.stream);
        SBP_CHECK_LAUNCH();
        st.steps++;
      }
      double el = 0.0;
      SBP_CUDA(SBP_COPY_ASYNC(&el, epoch_loss.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
      check_tensor_status();
      el /= (double)N;
      if (first < 0.0) first = el;
      last = el;
    }
    st.first_loss = first;
    st.last_loss = last;
  }
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_vertex_features(const SbpBlockmodel* cbm, const SbpGraph* g, int32_t n, const int32_t* vertices,
                              float* features, int32_t* slots, int32_t* nvalid) {
  SBP_API_BEGIN
  SBP_REQUIRE(cbm && g && n >= 0 && (n == 0 || vertices), "invalid argument");
  SbpBlockmodel* bm = const_cast<SbpBlockmodel*>(cbm);
  if (n == 0) return SBP_OK;
  for (int i = 0; i < n; ++i) SBP_REQUIRE(vertices[i] >= 0 && vertices[i] < g->V, "vertex out of range");
  Context& c = Context::get();
  DevBuf<int> verts;
  verts.reserve(n);
  SBP_CUDA(SBP_COPY_ASYNC(verts.p, vertices, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  g_learn.reserve(n);
  BatchBufs bb = g_learn.view();
  const LearnedParams lp = learned_params(*g, 0.f);
  const int cap = std::max(g->heavy_cap, g->light_cap);
  launch_warps(k_learn_features, n, cap, 1, g->view(), bm->view(), verts.p, n, 0, bb, lp, cap, c.status);
  std::vector<uint16_t> fb((size_t)n * kMlpIn);
  std::vector<int2> sl((size_t)n * kFeatSlots);
  std::vector<int4> inf(n);
  SBP_CUDA(SBP_COPY_ASYNC(fb.data(), bb.F1, fb.size() * 2, cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(sl.data(), bb.slot, sl.size() * sizeof(int2), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(inf.data(), bb.info, inf.size() * sizeof(int4), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  c.check_status();
  if (features)
    for (size_t i = 0; i < fb.size(); ++i) {
      const uint32_t u = (uint32_t)fb[i] << 16;
      std::memcpy(features + i, &u, 4);
    }
  for (int i = 0; i < n; ++i) {
    const int nv = inf[i].w >> 1;
    if (nvalid) nvalid[i] = nv;
    if (slots)
      for (int j = 0; j < kFeatSlots; ++j)
        slots[(size_t)i * kFeatSlots + j] = j < nv ? sl[(size_t)i * kFeatSlots + j].x : -1;
  }
  SBP_API_END
}

SbpStatus sbp_learned_evaluate(const SbpBlockmodel* cbm, const SbpGraph* g, const SbpMlp* m, int32_t n,
                               const int32_t* vertices, const uint32_t* records, float epsilon, int32_t* proposal,
                               double* q_forward, double* delta_mdl, double* hastings, int32_t* accepted) {
  SBP_API_BEGIN
  SBP_REQUIRE(cbm && g && m && n >= 0 && (n == 0 || (vertices && records)), "invalid argument");
  SBP_REQUIRE(epsilon > 0.f && epsilon <= 1.f, "epsilon must be in (0, 1]");
  SbpBlockmodel* bm = const_cast<SbpBlockmodel*>(cbm);
  if (n == 0) return SBP_OK;
  std::vector<char> seen(g->V, 0);
  for (int i = 0; i < n; ++i) {
    SBP_REQUIRE(vertices[i] >= 0 && vertices[i] < g->V, "vertex out of range");
    SBP_REQUIRE(!seen[vertices[i]], "vertices must be distinct");
    seen[vertices[i]] = 1;
  }
  Context& c = Context::get();
  DevBuf<int> verts, moved, nm;
  DevBuf<uint4> rec;
  DevBuf<double> dS, H;
  verts.reserve(n);
  rec.reserve(g->V);
  moved.reserve(n);
  nm.reserve(1);
  dS.reserve(n);
  H.reserve(n);
  SBP_CUDA(SBP_COPY_ASYNC(verts.p, vertices, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  // records are indexed by vertex (replay of sweep 0): scatter the caller's per-row records
  std::vector<uint4> per_vertex(g->V, make_uint4(0, 0, 0, 0));
  for (int i = 0; i < n; ++i)
    per_vertex[vertices[i]] = make_uint4(records[4 * i], records[4 * i + 1], records[4 * i + 2], records[4 * i + 3]);
  SBP_CUDA(SBP_COPY_ASYNC(rec.p, per_vertex.data(), (size_t)g->V * sizeof(uint4), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(cudaMemsetAsync(nm.p, 0, sizeof(int), c.stream));
  SBP_CUDA(cudaMemsetAsync(dS.p, 0, n * sizeof(double), c.stream));
  SBP_CUDA(cudaMemsetAsync(H.p, 0, n * sizeof(double), c.stream));
  SBP_CUDA(cudaMemsetAsync(bm->prop.p, 0xff, (size_t)g->V * sizeof(int), c.stream));
  g_learn.reserve(n);
  BatchBufs bb = g_learn.view();
  const LearnedParams lp = learned_params(*g, epsilon);
  RngParams rng;
  rng.seed = 0;
  rng.replay = rec.p;
  rng.replay_records = g->V;
  rng.call = 0;
  const int cap = std::max(g->heavy_cap, g->light_cap);
  launch_warps(k_learn_features, n, cap, 1, g->view(), bm->view(), verts.p, n, 0, bb, lp, cap, c.status);
  mlp_forward(bb.F1, n, m->weights(), bb.L1, c.status, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  k_learn_propose<<<grid_for(n, 128, 1 << 20), 128, 0, c.stream>>>(verts.p, n, bm->view(), bb, lp, rng, 0, g->V,
                                                                    c.status);
  SBP_CHECK_LAUNCH();
  mlp_forward(bb.F2, n, m->weights(), bb.L2, c.status, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(cudaMemsetAsync(c.counters, 0, 8 * sizeof(unsigned long long), c.stream));
  launch_warps(k_learn_eval, n, cap, 1, g->view(), bm->view(), verts.p, n, 0, bb, lp, rng, 0, bm->prop.p, moved.p,
               nm.p, c.counters, dS.p, H.p, cap, c.status);
  std::vector<int> sp(n), pr(g->V), bh(g->V);
  std::vector<double> qf(n);
  SBP_CUDA(SBP_COPY_ASYNC(sp.data(), bb.s_prop, n * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(qf.data(), bb.qf, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(pr.data(), bm->prop.p, (size_t)g->V * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(bh.data(), bm->b.p, (size_t)g->V * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  if (delta_mdl) SBP_CUDA(SBP_COPY_ASYNC(delta_mdl, dS.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (hastings) SBP_CUDA(SBP_COPY_ASYNC(hastings, H.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  check_tensor_status();
  SBP_CUDA(cudaMemsetAsync(bm->prop.p, 0xff, (size_t)g->V * sizeof(int), c.stream));
  c.sync();
  for (int i = 0; i < n; ++i) {
    const int v = vertices[i];
    if (proposal) proposal[i] = sp[i];
    if (q_forward) q_forward[i] = sp[i] == bh[v] ? 0.0 : qf[i];
    if (accepted) accepted[i] = pr[v] >= 0 ? 1 : 0;
  }
  SBP_API_END
}

SbpStatus sbp_learned_q(const SbpBlockmodel* cbm, const SbpGraph* g, const SbpMlp* m, int32_t n,
                        const int32_t* vertices, const int32_t* blocks, float epsilon, double* q) {
  SBP_API_BEGIN
  SBP_REQUIRE(cbm && g && m && n >= 0 && (n == 0 || (vertices && blocks && q)), "invalid argument");
  SBP_REQUIRE(epsilon > 0.f && epsilon <= 1.f, "epsilon must be in (0, 1]");
  SbpBlockmodel* bm = const_cast<SbpBlockmodel*>(cbm);
  if (n == 0) return SBP_OK;
  for (int i = 0; i < n; ++i) {
    SBP_REQUIRE(vertices[i] >= 0 && vertices[i] < g->V, "vertex out of range");
    SBP_REQUIRE(blocks[i] >= 0 && blocks[i] < bm->B, "block out of range");
  }
  Context& c = Context::get();
  DevBuf<int> verts, tg;
  DevBuf<double> qd;
  verts.reserve(n);
  tg.reserve(n);
  qd.reserve(n);
  SBP_CUDA(SBP_COPY_ASYNC(verts.p, vertices, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  SBP_CUDA(SBP_COPY_ASYNC(tg.p, blocks, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  g_learn.reserve(n);
  BatchBufs bb = g_learn.view();
  const LearnedParams lp = learned_params(*g, epsilon);
  const int cap = std::max(g->heavy_cap, g->light_cap);
  launch_warps(k_learn_features, n, cap, 1, g->view(), bm->view(), verts.p, n, 0, bb, lp, cap, c.status);
  mlp_forward(bb.F1, n, m->weights(), bb.L1, c.status, c.num_sms, c.stream);
  SBP_CHECK_LAUNCH();
  k_learn_q<<<grid_for(n, 128, 1 << 20), 128, 0, c.stream>>>(tg.p, n, bb, lp, bm->B, qd.p);
  SBP_CHECK_LAUNCH();
  SBP_CUDA(SBP_COPY_ASYNC(q, qd.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  check_tensor_status();
  SBP_API_END
}

// Plain asynchronous-Gibbs sweeps that record every accepted move as a training sample.
SbpStatus sbp_collect_moves(SbpBlockmodel* bm, const SbpGraph* cg, SbpDataset* d, const SbpFinetuneOptions* opt,
                            SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && cg && d && opt, "null argument");
  SBP_REQUIRE(opt->batches >= 1, "batches must be >= 1");
  SbpGraph& g = *const_cast<SbpGraph*>(cg);
  Context& c = Context::get();
  SbpStats st;
  std::memset(&st, 0, sizeof st);
  const int sweeps = (opt->max_sweeps <= 0 || opt->max_sweeps > kMaxIterations) ? kMaxIterations : opt->max_sweeps;
  RngParams rng;
  rng.seed = opt->seed;
  rng.replay = nullptr;
  rng.replay_records = 0;
  rng.call = opt->call;
  const BatchPlan& plan = g.plan(SBP_ASYNC_GIBBS, opt->batches);
  const LearnedParams lp = learned_params(g, 0.f);
  const int cap = std::max(g.heavy_cap, g.light_cap);
  SBP_CUDA(cudaMemsetAsync(c.counters, 0, 8 * sizeof(unsigned long long), c.stream));
  const auto t0 = std::chrono::steady_clock::now();
  for (int it = 0; it < sweeps; ++it) {
    const long long ovf_sweep = g_overflow_rebuilds;
    for (size_t bt = 0; bt < plan.light_n.size(); ++bt) {
      // plain evaluation (gibbs_batch without its apply), record, then apply
      const int nl = plan.light_n[bt], nh = plan.heavy_n[bt];
      int* n_cur = bm->n_moved.p + (bm->gen & 1);
      const GibbsEvalKernel k_eval = gibbs_eval_kernel(bm->sparse, bm->B);
      if (nl > 0) {
        const size_t smem = (size_t)table_ints(g.light_cap) * sizeof(int) * kLightWarps;
        set_smem_limit((const void*)k_eval, smem);
        k_eval<<<grid_for(nl, kLightWarps, 64 * c.num_sms), kLightWarps * 32, smem, c.stream>>>(
            g.view(), bm->view(), plan.order.p + plan.light_begin[bt], nl, rng, it, bm->prop.p, bm->moved.p, n_cur,
            c.counters, g.light_cap, c.status, nullptr, 0);
        SBP_CHECK_LAUNCH();
      }
      if (nh > 0) {
        const size_t smem = (size_t)table_ints(g.heavy_cap) * sizeof(int);
        set_smem_limit((const void*)k_eval,
                       std::max(smem, (size_t)table_ints(g.light_cap) * sizeof(int) * kLightWarps));
        k_eval<<<grid_for(nh, 1, 64 * c.num_sms), 32, smem, c.stream>>>(
            g.view(), bm->view(), plan.order.p + plan.heavy_begin[bt], nh, rng, it, bm->prop.p, bm->moved.p, n_cur,
            c.counters, g.heavy_cap, c.status, nullptr, 0);
        SBP_CHECK_LAUNCH();
      }
      const int batch = nl + nh;
      launch_warps(k_learn_collect, batch, cap, 1, g.view(), bm->view(), bm->moved.p, n_cur, bm->prop.p, lp,
                   d->X.p, d->target.p, d->nvalid.p, d->count.p, d->capacity, cap, c.status);
      gibbs_apply(*bm, g, batch);
    }
    tidy_hashed(*bm, g, ovf_sweep);
    st.sweeps++;
    c.check_status();
  }
  bm->overall_entropy = (float)mdl(*bm, g);
  unsigned long long cnt[8];
  SBP_CUDA(SBP_COPY_ASYNC(cnt, c.counters, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  st.visits = (long long)cnt[0];
  st.proposals_moved = (long long)cnt[1];
  st.accepted = (long long)cnt[2];
  st.mdl = bm->overall_entropy;
  st.num_blocks = bm->B;
  st.mcmc_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (stats) *stats = st;
  SBP_API_END
}

SbpStatus sbp_finetune_learned(SbpBlockmodel* bm, const SbpGraph* cg, int32_t algorithm,
                               const SbpFinetuneOptions* opt, const SbpMlp* m, const SbpLearnedOptions* lopt,
                               SbpTrace* trace, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(bm && cg && opt, "null argument");
  SBP_REQUIRE(algorithm >= SBP_METROPOLIS_HASTINGS && algorithm <= SBP_HYBRID_MCMC, "unknown finetune algorithm");
  SBP_REQUIRE(opt->batches >= 1 || algorithm == SBP_METROPOLIS_HASTINGS, "batches must be >= 1");
  SBP_REQUIRE(!trace || (trace->capacity >= 0 && (trace->capacity == 0 || (trace->seconds && trace->mdl))),
              "invalid trace");
  float eps, fallback;
  int stop_rule;
  check_learned_options(lopt, &eps, &fallback, &stop_rule);
  SbpStats st;
  finetune_learned(*bm, *const_cast<SbpGraph*>(cg), algorithm, *opt, m, eps, fallback, stop_rule, trace, st);
  if (stats) *stats = st;
  SBP_API_END
}

// stochastic_block_partition with the learned proposal in every finetune (mlp == NULL: the plain
// proposal with the chosen stop rule).
SbpStatus sbp_partition_learned(const SbpGraph* cg, const SbpOptions* opt, const SbpMlp* m,
                                const SbpLearnedOptions* lopt, int32_t* out_assignment, SbpStats* stats) {
  SBP_API_BEGIN
  SBP_REQUIRE(cg && opt && out_assignment, "null argument");
  SBP_REQUIRE(opt->algorithm >= SBP_METROPOLIS_HASTINGS && opt->algorithm <= SBP_HYBRID_MCMC,
              "unknown finetune algorithm");
  SBP_REQUIRE(opt->batches >= 1 || opt->algorithm == SBP_METROPOLIS_HASTINGS, "batches must be >= 1");
  float eps, fallback;
  int stop_rule;
  check_learned_options(lopt, &eps, &fallback, &stop_rule);
  SbpGraph& g = *const_cast<SbpGraph*>(cg);
  long long learned_sweeps = 0;
  const FinetuneStep step = [&](SbpBlockmodel& bm, SbpGraph& gg, int algo, const SbpFinetuneOptions& fo,
                                SbpStats& fs) {
    finetune_learned(bm, gg, algo, fo, m, eps, fallback, stop_rule, nullptr, fs);
    learned_sweeps += fs.learned_sweeps;
  };
  SbpStats st;
  partition(g, *opt, out_assignment, st, &step);
  st.learned_sweeps = (int32_t)learned_sweeps;
  if (stats) *stats = st;
  SBP_API_END
}

}  // extern "C"
