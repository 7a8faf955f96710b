// Internal host-side declarations of the engine shared by its translation units
// (sbp_engine.cu: graph, blockmodel, finetune, merge, partition and the C ABI;
// sbp_learned.cu: the learned proposal).  Not part of the public C ABI.
#pragma once
#include <atomic>
#include <condition_variable>
#include <functional>
#include <map>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/sbp_b200.h"
#include "sbp_error.h"
#include "sbp_kernels.cuh"
#include "sbp_sort.cuh"

namespace sbpb {

// ------------------------------------------------------------------------------------------
// Errors
// ------------------------------------------------------------------------------------------
struct Error : std::runtime_error {
  SbpStatus code;
  Error(SbpStatus c, const std::string& m) : std::runtime_error(m), code(c) {}
};


#define SBP_CUDA(x)                                                                                     \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess) {                                                                            \
      if (e_ == cudaErrorMemoryAllocation) throw Error(SBP_ERR_OUT_OF_MEMORY, std::string(#x) + ": " + cudaGetErrorString(e_)); \
      throw Error(SBP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));                       \
    }                                                                                                   \
  } while (0)

// Counters shared by every host thread that calls the library.
inline std::atomic<long long> g_launches{0};   // kernels launched by this library (all entry points)
inline std::atomic<long long> g_h2d{0}, g_d2h{0};   // bytes copied host->device / device->host

#define SBP_CHECK_LAUNCH() \
  do {                     \
    ++g_launches;          \
    SBP_CUDA(cudaGetLastError()); \
  } while (0)

inline cudaError_t count_copy(cudaError_t e, size_t bytes, cudaMemcpyKind kind) {
  if (kind == cudaMemcpyHostToDevice) g_h2d += (long long)bytes;
  if (kind == cudaMemcpyDeviceToHost) g_d2h += (long long)bytes;
  return e;
}
#define SBP_COPY(dst, src, bytes, kind) count_copy(cudaMemcpy(dst, src, bytes, kind), bytes, kind)
#define SBP_COPY_ASYNC(dst, src, bytes, kind, stream) \
  count_copy(cudaMemcpyAsync(dst, src, bytes, kind, stream), bytes, kind)

// Total memory of the current device, asked once.
inline size_t device_memory_bytes() {
  static size_t total = [] {
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
      cudaGetLastError();
      t = 0;
    }
    return t;
  }();
  return total;
}

// Released device buffers are kept for reuse instead of being freed: cudaFree synchronizes
// the whole device, and every partition round releases and reallocates its blockmodel's
// buffers.  A released buffer carries an event recorded on the releasing thread's stream, and
// it is handed out again only after that event has completed, so no queued kernel of any
// stream still uses it.  Thread-safe.
cudaStream_t engine_stream();

struct DeviceCache {
  // at most half the device's memory (at least 32 GB) stays cached: the dense block matrix of a
  // 100,000-block finetune (two 40 GB buffers) is reused by the next partition instead of being
  // freed and allocated again
  static size_t cap_bytes() {
    static const size_t cap = std::max<size_t>(32ull << 30, device_memory_bytes() / 2);
    return cap;
  }
  struct Block {
    void* p;
    cudaEvent_t released;   // null: released while its stream was being captured (wait for the stream)
  };
  std::multimap<size_t, Block> blocks;   // bytes -> buffer
  std::vector<cudaEvent_t> spare;        // events for reuse
  size_t cached = 0;
  std::mutex mu;
  static DeviceCache& get() {
    static DeviceCache* c = new DeviceCache();   // never destroyed: buffers live until exit
    return *c;
  }
  static void wait(const Block& b) {
    SBP_CUDA(b.released ? cudaEventSynchronize(b.released) : cudaStreamSynchronize(engine_stream()));
  }
  void* take(size_t bytes, size_t* got) {
    Block b{nullptr, nullptr};
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = blocks.lower_bound(bytes);
      if (it != blocks.end() && it->first <= bytes + bytes / 4 + (1u << 20)) {
        b = it->second;
        *got = it->first;
        cached -= it->first;
        blocks.erase(it);
      }
    }
    if (b.p) {
      wait(b);
      recycle(b.released);
      return b.p;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaErrorMemoryAllocation) {   // give the cache back and retry
      cudaGetLastError();
      std::multimap<size_t, Block> all;
      {
        std::lock_guard<std::mutex> lk(mu);
        all.swap(blocks);
        cached = 0;
      }
      for (auto& kv : all) {
        wait(kv.second);
        cudaFree(kv.second.p);
        recycle(kv.second.released);
      }
      if (!all.empty()) e = cudaMalloc(&p, bytes);
    }
    if (e == cudaErrorMemoryAllocation) throw Error(SBP_ERR_OUT_OF_MEMORY, "cudaMalloc: out of device memory");
    SBP_CUDA(e);
    *got = bytes;
    return p;
  }
  // Called from destructors: never throws.
  void give(void* p, size_t bytes) noexcept {
    cudaEvent_t ev = nullptr;
    try {
      const cudaStream_t st = engine_stream();
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
        ev = event();
        if (ev && cudaEventRecord(ev, st) != cudaSuccess) {
          cudaGetLastError();
          cudaStreamSynchronize(st);
          recycle(ev);
          ev = nullptr;
        }
      }
    } catch (...) {
      ev = nullptr;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      if (cached + bytes <= cap_bytes()) {
        blocks.emplace(bytes, Block{p, ev});
        cached += bytes;
        return;
      }
    }
    cudaFree(p);   // synchronizes the device first
    recycle(ev);
  }
  size_t cached_bytes() {
    std::lock_guard<std::mutex> lk(mu);
    return cached;
  }
  // Free every cached buffer (after the work that released it).
  void release_all() {
    std::multimap<size_t, Block> all;
    {
      std::lock_guard<std::mutex> lk(mu);
      all.swap(blocks);
      cached = 0;
    }
    for (auto& kv : all) {
      wait(kv.second);
      cudaFree(kv.second.p);
      recycle(kv.second.released);
    }
  }
  cudaEvent_t event() {
    {
      std::lock_guard<std::mutex> lk(mu);
      if (!spare.empty()) {
        cudaEvent_t e = spare.back();
        spare.pop_back();
        return e;
      }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return e;
  }
  void recycle(cudaEvent_t e) {
    if (!e) return;
    std::lock_guard<std::mutex> lk(mu);
    spare.push_back(e);
  }
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t bytes = 0;   // size of the underlying allocation
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) DeviceCache::get().give(p, bytes);
    p = nullptr;
    n = 0;
    bytes = 0;
  }
  void reserve(size_t count) {   // grow-only, contents not preserved
    if (count <= n && p) return;
    release();
    const size_t want = std::max<size_t>(count, 1) * sizeof(T);
    p = static_cast<T*>(DeviceCache::get().take(want, &bytes));
    n = std::max<size_t>(count, 1);
  }
};

// ------------------------------------------------------------------------------------------
// Process-wide context: one stream, the device status word, counters and readback buffers.
// ------------------------------------------------------------------------------------------
// log(x) for the integers 1 <= x < kLogTable as a pair of doubles (hi = log x rounded, lo = the
// rest), from the host's long-double log (64-bit mantissa): the vertex-move delta-MDL takes
// g(a) - g(b), g(x) = x log x, of integer counts from it (dxlogx_int in sbp_device.cuh).
inline double2* make_log_table() {
  std::vector<double2> h(kLogTable);
  h[0] = make_double2(0.0, 0.0);
  const int nt = 8;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&h, t, nt] {
      for (int x = 1 + t; x < kLogTable; x += nt) {
        const long double l = logl((long double)x);
        const double hi = (double)l;
        h[x] = make_double2(hi, (double)(l - (long double)hi));
      }
    });
  for (auto& t : th) t.join();
  double2* d = nullptr;
  SBP_CUDA(cudaMalloc(&d, sizeof(double2) * kLogTable));
  SBP_CUDA(cudaMemcpy(d, h.data(), sizeof(double2) * kLogTable, cudaMemcpyHostToDevice));
  return d;
}

struct Context {
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int* status = nullptr;                 // device error bits
  unsigned long long* counters = nullptr;  // device counters [8]
  double* partial = nullptr;             // MDL partial sums
  double* scalar = nullptr;              // MDL result
  double* mh_out = nullptr;              // MH sweep outputs [4]
  unsigned* done = nullptr;              // CTAs finished in the current k_mdl launch (0 between launches)
  double2* logt = nullptr;               // [kLogTable] log(x) as hi + lo doubles (entry 0 unused)
  int npartial = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // A context: its own stream and scratch; the log table is shared when given.
  static Context* create(double2* logt) {
    auto* c = new Context();
    SBP_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    int dev = 0;
    SBP_CUDA(cudaGetDevice(&dev));
    SBP_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
    c->npartial = 4 * c->num_sms;
    SBP_CUDA(cudaMalloc(&c->status, 8 * sizeof(int)));
    SBP_CUDA(cudaMalloc(&c->counters, 8 * sizeof(unsigned long long)));
    SBP_CUDA(cudaMalloc(&c->partial, c->npartial * sizeof(double)));
    SBP_CUDA(cudaMalloc(&c->scalar, sizeof(double)));
    SBP_CUDA(cudaMalloc(&c->mh_out, 16 * sizeof(double)));
    SBP_CUDA(cudaMalloc(&c->done, sizeof(unsigned)));
    SBP_CUDA(cudaMemset(c->status, 0, 8 * sizeof(int)));
    SBP_CUDA(cudaMemset(c->done, 0, sizeof(unsigned)));
    SBP_CUDA(cudaEventCreate(&c->ev0));
    SBP_CUDA(cudaEventCreate(&c->ev1));
    c->logt = logt ? logt : make_log_table();
    return c;
  }
  // The process's context: every entry point runs on it.
  static Context& primary() {
    static Context* ctx = nullptr;
    if (!ctx) {
      int n = 0;
      if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw Error(SBP_ERR_CUDA, "no CUDA device available (the engine has no CPU fallback)");
      }
      ctx = create(nullptr);
    }
    return *ctx;
  }
  // A second context, for work that runs beside the primary stream's kernels (the batched
  // partitioner's merges while its sweep kernel runs).
  static Context& secondary() {
    static Context* ctx = nullptr;
    if (!ctx) ctx = create(primary().logt);
    return *ctx;
  }
  // The calling thread's current context: the primary one unless a ContextScope is open.
  static Context*& current() {
    static thread_local Context* cur = nullptr;
    return cur;
  }
  static Context& get() {
    Context* c = current();
    return c ? *c : primary();
  }
  void sync() { SBP_CUDA(cudaStreamSynchronize(stream)); }
  // Read and clear the device status word; throw on any error bit.
  void check_status() {
    int st = 0;
    SBP_CUDA(SBP_COPY_ASYNC(&st, status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    sync();
    if (st) {
      SBP_CUDA(cudaMemsetAsync(status, 0, sizeof(int), stream));
      if (st & kErrReplay)
        throw Error(SBP_ERR_REPLAY, "replay stream shorter than the run needs, or a replayed proposal out of range");
      char msg[200];
      snprintf(msg, sizeof msg,
               "device status 0x%x (table overflow=1, multinomial walk=2, bounds=8, batched sweep found no "
               "claimable work within its wait limit=16)", st);
      throw Error(SBP_ERR_DEVICE, msg);
    }
  }
};

inline cudaStream_t engine_stream() { return Context::get().stream; }

// Makes a context current on the calling thread for the scope's lifetime (null: no change).
struct ContextScope {
  Context* prev;
  explicit ContextScope(Context* c) : prev(Context::current()) {
    if (c) Context::current() = c;
  }
  ~ContextScope() { Context::current() = prev; }
  ContextScope(const ContextScope&) = delete;
  ContextScope& operator=(const ContextScope&) = delete;
};

// Optional timing of the vertex-evaluation kernel: CUDA events around every light-vertex
// evaluation launch on the launching stream, resolved when the profile is read.
struct EvalProfiler {
  bool on = false;
  std::mutex mu;   // launches may come from several host threads (the batched partitioner's merges)
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  double ms = 0.0, bytes = 0.0;
  long long launches = 0, visits = 0;
  void add(cudaEvent_t e0, cudaEvent_t e1, long long n, double b) {
    std::lock_guard<std::mutex> lk(mu);
    pending.push_back({e0, e1});
    launches++;
    visits += n;
    bytes += b;
  }
  cudaEvent_t get() {
    std::lock_guard<std::mutex> lk(mu);
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    SBP_CUDA(cudaEventCreate(&e));
    return e;
  }
  void resolve() {
    std::lock_guard<std::mutex> lk(mu);
    for (auto& pr : pending) {
      SBP_CUDA(cudaEventSynchronize(pr.second));
      float t = 0.f;
      SBP_CUDA(cudaEventElapsedTime(&t, pr.first, pr.second));
      ms += t;
      pool.push_back(pr.first);
      pool.push_back(pr.second);
    }
    pending.clear();
  }
};
inline EvalProfiler g_prof;

inline int grid_for(long long work_items, int per_block, int max_blocks) {
  long long g = (work_items + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return (int)g;
}

inline int pow2_at_least(int x) {
  int c = 1;
  while (c < x) c <<= 1;
  return c;
}

constexpr int kLightCap = 256;        // per-warp table slots for light vertices
constexpr int kLightCapMax = 512;     // largest per-warp table of the 8-warp evaluation CTA
constexpr int kLightWarps = 8;
constexpr int kMaxCap = 8192;         // largest per-warp table
constexpr size_t kSmemBudget = 200 * 1024;
constexpr int kSmemRebuildMaxB = 100;

// Blocks above which the block matrix is row-hashed instead of dense, and the largest share of the
// free device memory (percent) a dense matrix may take (sbp_set_option).
inline int g_dense_max_blocks = 131072;
inline int g_dense_max_memory_pct = 60;
// Hashed row capacity = power of two >= factor * (cells after a rebuild) + 4 * factor.
inline int g_hashed_row_factor = 4;
// 1: an asynchronous-Gibbs finetune on dense storage runs as one CUDA graph launch with the
// sweep loop decided on the GPU; 0: one host-driven launch sequence per sweep (sbp_set_option).
inline int g_graph_sweeps = 1;
inline thread_local long long g_overflow_rebuilds = 0;   // rebuilds forced by a full hashed row (calling thread)
// Light vertices of dense blockmodels (sbp_set_option "group_kernel"): 1 (default) evaluated by the
// group kernels (sbp_eval_small.cu) when B <= kSmallB (direct-indexed group tables), by the warp-
// per-vertex kernels above; 2 by the group kernels at every B (hashed group tables above kSmallB:
// half the occupancy of the warp kernel at the light-table size of the 200,000-vertex graph,
// measured slower there); 0 by the warp-per-vertex kernels always.
inline int g_group_kernel = 1;
// Batched partitioner: idle claim attempts of a persistent CTA before the launch gives up with an
// error (each attempt sleeps ~0.25 us), and the fault injection of the failure-detection test
// (index of a graph whose sweep queue never opens; -1: none).  sbp_set_option.
inline long long g_batched_wait_limit = 1LL << 22;
inline int g_batched_stall_graph = -1;
// CTA slots the batched sweep kernel leaves free while the merges of the graphs between two
// finetunes run beside it on the secondary context (0: merges run after each sweep launch).
inline int g_batched_overlap = 64;
// Host threads (each with its own context) that run the steps between finetunes of several
// graphs of a batched partition at once; 1: the calling thread alone.
inline int g_batched_threads = 8;

}  // namespace sbpb

using namespace sbpb;

// ------------------------------------------------------------------------------------------
// Graph
// ------------------------------------------------------------------------------------------
struct BatchPlan {
  DevBuf<int> order;                       // per batch: light vertices then heavy vertices
  std::vector<int> light_begin, light_n, heavy_begin, heavy_n;
  std::vector<int> group_n;                // light vertices of k <= kGroupMaxK, at the front of each light list
  std::vector<double> light_bytes;         // algorithmic bytes of each light evaluation launch
  int max_batch = 0;
};

struct SbpGraph {
  int V = 0;
  long long E = 0;
  DevBuf<int> out_ptr, out_idx, out_src, in_ptr, in_idx, identity, high_dev;
  DevBuf<unsigned char> self;
  std::vector<int> h_k;        // k_out + k_in per vertex (self loop counted once, on the out side)
  std::vector<int> high, low;  // hybrid split
  int max_k = 0;
  int heavy_cap = 512;         // table slots for heavy vertices
  int light_cap = 256;         // table slots per warp for light vertices (k <= light_cap / 2)
  std::unordered_map<long long, std::unique_ptr<BatchPlan>> plans;

  GraphView view() const {
    GraphView g;
    g.V = V;
    g.E = E;
    g.log_E = std::log(E > 2 ? (double)E : 2.0);
    g.out_ptr = out_ptr.p;
    g.out_idx = out_idx.p;
    g.in_ptr = in_ptr.p;
    g.in_idx = in_idx.p;
    g.self = self.p;
    return g;
  }

  int max_k_of(const std::vector<int>& verts) const {
    int m = 0;
    for (int v : verts) m = std::max(m, h_k[v]);
    return m;
  }

  // Batches of asynchronous Gibbs over `list` (src/finetune.cpp:43-47, 352-366): batch_size =
  // ceil(n / batches), loop bound n / batch_size (a trailing partial batch is skipped).
  BatchPlan& plan(int algo, int batches) {
    const long long key = (long long)algo * 1000003LL + batches;
    auto it = plans.find(key);
    if (it != plans.end()) return *it->second;
    std::vector<int> list;
    if (algo == SBP_ASYNC_GIBBS) {
      list.resize(V);
      std::iota(list.begin(), list.end(), 0);
    } else {
      list = low;
    }
    auto p = std::make_unique<BatchPlan>();
    const int n = (int)list.size();
    const int batch_size = (int)std::ceil(n / (double)batches);
    std::vector<int> order;
    order.reserve(n);
    if (batch_size > 0) {
      for (int bt = 0; bt < n / batch_size; ++bt) {
        const int start = bt * batch_size, end = std::min(n, (bt + 1) * batch_size);
        p->light_begin.push_back((int)order.size());
        for (int i = start; i < end; ++i)   // vertices that fit the group tables first
          if (h_k[list[i]] <= std::min(kGroupMaxK, light_cap / 2)) order.push_back(list[i]);
        p->group_n.push_back((int)order.size() - p->light_begin.back());
        for (int i = start; i < end; ++i)
          if (h_k[list[i]] > kGroupMaxK && h_k[list[i]] <= light_cap / 2) order.push_back(list[i]);
        p->light_n.push_back((int)order.size() - p->light_begin.back());
        double lb = 0.0;   // 12 B (CSR offsets + b[v]) + 8 B per neighbour (id + block gather)
        for (int i = p->light_begin.back(); i < (int)order.size(); ++i) lb += 12.0 + 8.0 * h_k[order[i]];
        p->light_bytes.push_back(lb);
        p->heavy_begin.push_back((int)order.size());
        for (int i = start; i < end; ++i)
          if (h_k[list[i]] > light_cap / 2) order.push_back(list[i]);
        p->heavy_n.push_back((int)order.size() - p->heavy_begin.back());
        p->max_batch = std::max(p->max_batch, end - start);
      }
    }
    p->order.reserve(order.size());
    if (!order.empty())
      SBP_CUDA(SBP_COPY(p->order.p, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
    auto& ref = *p;
    plans[key] = std::move(p);
    return ref;
  }
};

// ------------------------------------------------------------------------------------------
// Blockmodel
// ------------------------------------------------------------------------------------------
struct SbpBlockmodel {
  int V = 0, B = 0, ld = 0;
  const SbpGraph* graph = nullptr;   // the graph the blockmodel was created on (must outlive it)
  DevBuf<int> b, M, MT, CS, CST, d_out, d_in, d;
  DevBuf<int> prop, qr, qs, moved, n_moved;   // n_moved: two slots, alternating per batch
  DevBuf<unsigned long long> last;           // (batch generation << 32 | last mover) per block
  unsigned gen = 0;                          // batch generation
  int nch = 0;
  // row-hashed representation (B > dense_max_blocks)
  bool sparse = false;
  DevBuf<long long> rbase, cbase;
  DevBuf<int> rmask, cmask, overflow, old_block;
  DevBuf<int2> rslot, cslot;
  long long rtop = 0, ctop = 0;       // slots in use (rows are regrown after them)
  long long rlimit = 0, climit = 0;   // slots allocated
  DevBuf<int> csr_rptr, csr_ridx, csr_rval, csr_cptr, csr_cidx, csr_cval;   // sorted rows after a rebuild
  float overall_entropy = 3.40282347e+38f;
  int num_blocks_to_merge = 0;

  BlockView view() {
    BlockView v;
    v.B = B;
    v.sparse = sparse ? 1 : 0;
    v.rbase = rbase.p;
    v.rmask = rmask.p;
    v.rslot = rslot.p;
    v.cbase = cbase.p;
    v.cmask = cmask.p;
    v.cslot = cslot.p;
    v.overflow = overflow.p;
    v.ld = ld;
    v.nch = nch;
    v.CS = CS.p;
    v.CST = CST.p;
    v.b = b.p;
    v.M = M.p;
    v.MT = MT.p;
    v.d_out = d_out.p;
    v.d_in = d_in.p;
    v.d = d.p;
    v.logt = Context::get().logt;
    return v;
  }

  void init_vertex_scratch(int nv) {
    Context& c = Context::get();
    V = nv;
    b.reserve(V);
    prop.reserve(V);
    qr.reserve(V);
    qs.reserve(V);
    moved.reserve(V);
    old_block.reserve(V);
    n_moved.reserve(2);
    overflow.reserve(1);
    SBP_CUDA(cudaMemsetAsync(overflow.p, 0, sizeof(int), c.stream));
    SBP_CUDA(cudaMemsetAsync(prop.p, 0xff, sizeof(int) * V, c.stream));
    SBP_CUDA(cudaMemsetAsync(n_moved.p, 0, 2 * sizeof(int), c.stream));
  }

  void set_blocks(int nb) {
    Context& c = Context::get();
    B = nb;
    sparse = B > g_dense_max_blocks;
    const double dense_bytes = 2.0 * (double)B * (double)(((B + kChunk - 1) / kChunk) * kChunk) * sizeof(int);
    // dense only while it takes at most 60 % of the free device memory; cudaMemGetInfo can
    // stall the host for tens of milliseconds, so it is asked only for a matrix above 5 % of
    // the device's memory
    if (!sparse && dense_bytes > 0.05 * (double)device_memory_bytes()) {
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        // buffers this blockmodel already holds, and those the device cache keeps for reuse,
        // count as free
        const size_t have = M.n * sizeof(int) * 2 + DeviceCache::get().cached_bytes();
        if (dense_bytes > 0.01 * g_dense_max_memory_pct * (double)(free_b + have)) sparse = true;
      } else {
        cudaGetLastError();
      }
    }
    ld = ((B + kChunk - 1) / kChunk) * kChunk;
    nch = (B + kChunk - 1) / kChunk;
    if (sparse) {
      rbase.reserve(B);
      cbase.reserve(B);
      rmask.reserve(B);
      cmask.reserve(B);
      overflow.reserve(1 + 2 * (size_t)B);   // any-row flag, then one flag per row of M and of MT
    } else {
      const size_t cells = (size_t)B * (size_t)ld;
      M.reserve(cells);
      MT.reserve(cells);
      CS.reserve((size_t)B * nch);
      CST.reserve((size_t)B * nch);
    }
    d_out.reserve(B);
    d_in.reserve(B);
    d.reserve(B);
    last.reserve(B);
    SBP_CUDA(cudaMemsetAsync(last.p, 0, sizeof(unsigned long long) * B, c.stream));
  }
};

namespace sbpb {

inline bool use_group_kernel(const SbpBlockmodel& bm) {
  return !bm.sparse && (g_group_kernel == 2 || (g_group_kernel == 1 && bm.B <= kSmallB));
}

void set_smem_limit(const void* fn, size_t bytes);

// Launch of the group kernel over n light vertices (dense storage); with hashed group tables
// (B > kSmallB) every vertex must have k <= kGroupMaxK.
inline void launch_group_eval(const SbpGraph& g, SbpBlockmodel& bm, const int* verts, int n, const RngParams& rng,
                              int sweep, int* n_moved, const SweepCtl* ctl, int batch, cudaStream_t stream) {
  Context& c = Context::get();
  const bool hashed_table = bm.B > kSmallB;
  const int cap = std::min(g.light_cap, 2 * kGroupMaxK);
  const size_t smem = gibbs_eval_group_smem(hashed_table, cap);
  const GibbsEvalGroupKernel k = gibbs_eval_group_kernel(hashed_table);
  set_smem_limit((const void*)k, smem);
  k<<<grid_for(n, kSmallThreads / kSmallGroup, 64 * c.num_sms), kSmallThreads, smem, stream>>>(
      g.view(), bm.view(), verts, n, rng, sweep, bm.prop.p, bm.moved.p, n_moved, c.counters, cap, c.status, ctl,
      batch);
}

struct MhResult {
  long long visits = 0, moved = 0, accepted = 0;
  double sum_dS = 0.0;
};

struct ReplayDev {
  DevBuf<uint4> buf;
  long long records = 0;
  int moves = 0;   // 1: the records are proposals (sbp_*_replayed), 0: random words
  void upload(const SbpReplay* r) {
    if (!r || !r->words || r->records <= 0) return;
    buf.reserve((size_t)r->records);
    SBP_CUDA(SBP_COPY(buf.p, r->words, (size_t)r->records * sizeof(uint4), cudaMemcpyHostToDevice));
    records = r->records;
  }
  // Proposal records (s, 0, u_hi, u_lo): the proposed block and the bits of the accept uniform
  // (2.0, which never accepts, where the stream has none).
  void upload_moves(const SbpMoveReplay* r) {
    if (!r || !r->proposal || r->records <= 0) return;
    std::vector<uint4> h((size_t)r->records);
    for (long long i = 0; i < r->records; ++i) {
      const double u = r->uniform ? r->uniform[i] : 2.0;
      unsigned long long bits;
      std::memcpy(&bits, &u, sizeof bits);
      h[i] = make_uint4((unsigned)r->proposal[i], 0u, (unsigned)(bits >> 32), (unsigned)bits);
    }
    buf.reserve((size_t)r->records);
    SBP_CUDA(SBP_COPY(buf.p, h.data(), h.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    records = r->records;
    moves = 1;
  }
};

// ------------------------------------------------------------------------------------------
// Golden-section triplet over B (src/blockmodel/blockmodel_triplet.cpp:3-100) holding
// host copies of the assignment; a restored blockmodel is rebuilt on the device.
// ------------------------------------------------------------------------------------------
struct Snapshot {
  bool empty = true;
  std::vector<int> b;
  int B = 0;
  float entropy = 0.f;
};

struct Triplet {
  Snapshot s[3];
  bool optimal = false;
  void update(const Snapshot& x) {
    int index;
    if (s[1].empty) index = 1;
    else if (x.entropy <= s[1].entropy) {
      const int old_index = (s[1].B > x.B) ? 0 : 2;
      s[old_index] = s[1];
      index = 1;
    } else index = (s[1].B > x.B) ? 2 : 0;
    s[index] = x;
  }
  // returns the snapshot to continue from and its num_blocks_to_merge
  Snapshot next(const Snapshot& old, int* to_merge) {
    update(old);
    if (s[2].empty) {
      Snapshot r = s[1];
      *to_merge = (int)(r.B * 0.5);
      if (*to_merge == 0) optimal = true;
      return r;
    }
    if ((!s[0].empty && s[0].B - s[2].B == 2) || (s[0].empty && s[1].B - s[2].B == 1)) optimal = true;
    if (optimal) {
      *to_merge = 0;
      return s[1];
    }
    int index;
    if (s[0].empty && s[1].B > s[2].B) index = 1;
    else if ((s[0].B - s[1].B) >= (s[1].B - s[2].B)) index = 0;
    else index = 1;
    int next_b = s[index + 1].B;
    next_b += (int)((s[index].B - s[index + 1].B) * 0.618);
    *to_merge = s[index].B - next_b;
    return s[index];
  }
};

// One graph's partition in progress (sbp::stochastic_block_partition's loop state).
struct PartitionState {
  SbpBlockmodel bm;
  Triplet t;
  float iteration = 0;
  uint32_t call = 0;
  SbpStats st;
  bool done = false;
  // A partition driven by recorded streams (sbp_partition_replayed): the k-th merge or finetune
  // call takes replays[k]; the finetune sweep cap and the blocks after every call.
  const SbpMoveReplay* replays = nullptr;
  int nreplays = 0, next_replay = 0;
  int max_sweeps = 0;
  std::vector<int> block_counts;
  // sbp::add_intermediate records (src/sbp.cpp:36-59) of a single-graph partition
  bool record = false;
  cudaEvent_t t_start = nullptr;
  const SbpMoveReplay* take_replay() {
    if (!replays) return nullptr;
    if (next_replay >= nreplays)
      throw Error(SBP_ERR_REPLAY, "the partition makes more merge / finetune calls than the replay holds");
    return &replays[next_replay++];
  }
};

// Process-wide finetune counters (finetune::MCMC_iterations / MCMC_time, src/finetune.cpp:15-16)
// and intermediate records of partitions (sbp::intermediate_results, src/sbp.cpp:16-20).
inline thread_local long long g_mcmc_iterations = 0;   // the calling thread's finetune sweeps so far
inline thread_local double g_mcmc_time = 0.0;
inline std::vector<SbpIntermediate> g_intermediates;
// Record one intermediate of a partition in progress (modularity only when asked: the reference
// computes it for the final record alone).
void add_intermediate(PartitionState& ps, const SbpGraph& g, float iteration, double mdl, bool modularity);

// Engine steps shared by the translation units (defined in sbp_engine.cu).
void rebuild(SbpBlockmodel& bm, const SbpGraph& g, bool recompute_d = true);
double mdl(SbpBlockmodel& bm, const SbpGraph& g);
bool early_stop(int iteration, bool bracket, double initial_entropy, const std::vector<double>& deltas);
void set_smem_limit(const void* fn, size_t bytes);
// Apply half of an asynchronous-Gibbs batch: the accepted moves in bm.moved / n_moved[gen & 1].
void tidy_hashed(SbpBlockmodel& bm, const SbpGraph& g, long long overflows_before);
void gibbs_apply(SbpBlockmodel& bm, const SbpGraph& g, int batch);
// One asynchronous-Gibbs batch with the plain proposal (evaluation + apply).
void gibbs_batch(SbpBlockmodel& bm, const SbpGraph& g, const BatchPlan& plan, int bt, RngParams rng, int sweep);
// finetune::{metropolis_hastings, asynchronous_gibbs, hybrid_mcmc} on the device.
// `moves` (optional) replays proposals instead of random words.
void finetune(SbpBlockmodel& bm, SbpGraph& g, int algo, const SbpFinetuneOptions& opt, const SbpReplay* replay,
              SbpStats& st, const SbpMoveReplay* moves = nullptr);
// The finetune step of a partition, replaceable (the learned proposal's partition).
using FinetuneStep = std::function<void(SbpBlockmodel&, SbpGraph&, int, const SbpFinetuneOptions&, SbpStats&)>;
// Recorded streams of a partition's merge and finetune calls, in call order (in), and what
// the partition made of them (out).
struct PartitionReplay {
  const SbpMoveReplay* calls = nullptr;
  int num_calls = 0;
  int max_sweeps = 0;
  int calls_made = 0;
  std::vector<int> block_counts;
};
// sbp::stochastic_block_partition; `step` = nullptr runs the plain finetune; `replay` drives
// every call from recorded streams.
void partition(SbpGraph& g, const SbpOptions& opt, int* out, SbpStats& st, const FinetuneStep* step = nullptr,
               PartitionReplay* replay = nullptr);
// The partition loop's steps: start at B = V; merge step of the next round (returns the
// round's finetune algorithm and fills its options); statistics and golden-section step after
// the round's finetune (writes `out` and sets done when the search ends).
void partition_begin(PartitionState& ps, SbpGraph& g);
int partition_merge(PartitionState& ps, SbpGraph& g, const SbpOptions& opt, SbpFinetuneOptions* fo);
void partition_finish_round(PartitionState& ps, SbpGraph& g, const SbpStats& fs, int* out);
// block_merge::merge_blocks; best_out / dS_out optional.
void merge_blocks(SbpBlockmodel& bm, SbpGraph& g, const SbpMergeOptions& opt, const SbpReplay* replay,
                  int* best_out, double* dS_out, SbpStats& st, const SbpMoveReplay* moves = nullptr);
Snapshot snapshot(SbpBlockmodel& bm);
void restore(SbpBlockmodel& bm, SbpGraph& g, const Snapshot& x);
// Per-warp table slots of the Metropolis-Hastings kernels for vertices of degree up to max_k.
int mh_cap(int max_k);
// One sequential Metropolis-Hastings pass over a device list of n vertices.
MhResult mh_pass(SbpBlockmodel& bm, const SbpGraph& g, const int* verts, int n, int max_k, RngParams rng, int sweep);

}  // namespace sbpb
