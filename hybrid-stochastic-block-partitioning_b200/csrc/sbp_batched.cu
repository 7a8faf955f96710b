// Batched stochastic block partitioning: many graphs of uneven sizes partitioned together.
// Each graph runs the reference's loop (sbp::stochastic_block_partition, src/sbp.cpp:61-98:
// block merge, finetune, golden-section step) through the same per-graph state machine as
// sbp_partition, and moves on to its next merge as soon as its own finetune ends.  The
// asynchronous-Gibbs sweeps of every graph that is finetuning run in ONE persistent kernel
// launch per sweep:
//
//   * every graph has a work queue: its sweep is a fixed list of stages (per batch: evaluation
//     items - a chunk of light vertices or one heavy vertex -, apply stripes, finish stripes;
//     then the MDL's partial sums, one item per run of virtual CTAs, and its final sum);
//   * a CTA claims the next item of any graph whose current stage still has unclaimed items
//     (one 64-bit atomic: stage << 32 | next item); the CTA finishing a stage's last item opens
//     the graph's next stage.  No CTA ever waits while holding an item, so one graph's stages
//     stay in order while the other graphs keep the GPU busy;
//   * the per-element work is the single-graph kernels' own code (evaluate_vertex,
//     apply_moved_vertex, finish_moved_vertex, the MDL parts with the same virtual grid), so
//     every graph's chain and MDL are those of sbp_partition, bit for bit;
//   * each sweep's launch (parameter upload, queue reset, kernel, result read-back) is a
//     captured CUDA graph, replayed once per sweep;
//   * an autotuner times candidate item shapes (light vertices per evaluation item, CTAs per
//     SM) on the first sweeps of a workload and keeps the fastest for workloads of that shape.
//     Results do not depend on the shape, so tuning never changes an answer.
//
// A graph whose round cannot use the kernel (row-hashed storage at large B, Metropolis-
// Hastings or hybrid finetunes, degrees beyond the kernel's tables) runs that round's
// finetune on the single-graph path, between two sweep launches of the others.
//
// The steps of the graphs between two finetunes (end of the finetune, golden-section step,
// merge, set-up of the next finetune) run on a pool of host threads, each with its own context,
// while the next sweep launch of the other graphs runs; the launch leaves a few CTA slots free
// for their kernels.
#include <chrono>
#include <map>

#include "sbp_engine.cuh"
#include "sbp_steps.cuh"

namespace sbpb {
namespace {

enum StageKind : int { kEval = 0, kApply = 1, kFinish = 2, kMdlPart = 3, kMdlFinal = 4 };

// One stage of a graph's sweep: kind, batch, items, light-vertex chunks among the items.
// (int4: x kind, y batch, z items, w light chunks)

struct BGraph {   // one graph of the batch (device side)
  GraphView g;
  BlockView bm;
  const int* order;          // the batch plan's vertex order
  const int4* batches;       // per batch: light begin, light count, heavy begin, heavy count
  const int4* stages;        // the sweep's stages
  const int* out_src;
  int* prop;
  int* moved;
  int* n_moved;              // two slots, alternating per batch
  int* qr;
  int* qs;
  unsigned long long* last;
  unsigned long long* counters;   // visits, proposals moved, accepted
  double* partial;           // MDL partial sums, one per virtual CTA
  double* mdl_out;
  RngParams rng;
  int sweep;                 // the graph's sweep index within its finetune
  unsigned gen0;             // batch generation before the sweep
  int nstages;
  int chunk;                 // light vertices per evaluation item
  int mdl_cells;             // 1: cell form of the MDL, 0: edge form
};

struct Queue {                 // per graph, reset before every launch
  unsigned long long ctr;      // stage << 32 | next item
  int done;                    // items of the current stage finished
  int finished;                // 1 once the last stage is done
};

struct SweepParams {
  int ngraphs;                 // graphs in this launch (indices in glist)
  int mdl_ctas;
  int heavy_cap;
  unsigned wait_limit;         // idle claim attempts of a CTA before the launch gives up
};

constexpr int kBWarps = 8;
constexpr int kBThreads = kBWarps * 32;
constexpr int kErrBatchWait = 16;        // no claimable work for too long
constexpr int kMdlCtasPerItem = 16;
constexpr int kApplyPerStripe = 256;     // moved vertices per apply / finish stripe (bound)

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__global__ void __launch_bounds__(kBThreads, 2)
    k_batched_sweep(const BGraph* __restrict__ G, const int* __restrict__ glist, Queue* queue, int* nfinished,
                    int* abort_flag, const SweepParams* __restrict__ sp, int cap, int* status) {
  extern __shared__ int smem[];
  __shared__ int s_g, s_stage, s_idx, s_exit;
  __shared__ double red[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const SweepParams P = *sp;
  WarpTable t = carve_table(smem, cap, warp);
  init_table(t, lane);
  unsigned idle = 0;
  unsigned rot = blockIdx.x * 13u;
  for (;;) {
    // ---- claim an item of some graph (warp 0) ----
    if (warp == 0) {
      int cg = -1, cst = 0, cidx = 0;
      for (int base = 0; base < P.ngraphs && cg < 0; base += 32) {
        const int k = base + lane;
        int g = -1;
        bool avail = false;
        if (k < P.ngraphs) {
          g = glist[(k + rot) % P.ngraphs];
          const Queue& q = queue[g];
          if (!*(volatile const int*)&q.finished) {
            const unsigned long long c = ld_relaxed_u64(&q.ctr);
            const int st = (int)(c >> 32), idx = (int)(c & 0xffffffffu);
            avail = st < G[g].nstages && idx < G[g].stages[st].z;
          }
        }
        unsigned m = __ballot_sync(kFull, avail);
        while (m && cg < 0) {
          const int l = __ffs(m) - 1;
          m &= m - 1;
          int got = 0, gst = 0, gidx = 0;
          if (lane == l) {
            const unsigned long long old = atomicAdd(&queue[g].ctr, 1ull);
            gst = (int)(old >> 32);
            gidx = (int)(old & 0xffffffffu);
            got = gst < G[g].nstages && gidx < G[g].stages[gst].z;
          }
          got = __shfl_sync(kFull, got, l);
          if (got) {
            cg = __shfl_sync(kFull, g, l);
            cst = __shfl_sync(kFull, gst, l);
            cidx = __shfl_sync(kFull, gidx, l);
          }
        }
      }
      if (lane == 0) {
        s_g = cg;
        s_stage = cst;
        s_idx = cidx;
        // nothing claimable: every graph done, a failure elsewhere, or a stage still running
        int ex = 0;
        if (cg < 0) {
          if (*(volatile int*)nfinished >= P.ngraphs || *(volatile int*)abort_flag) {
            ex = 1;
          } else if (++idle > P.wait_limit) {   // bounded: no stage opened for too long
            atomicExch(abort_flag, 1);
            atomicOr(status, kErrBatchWait);
            ex = 1;
          }
        } else {
          idle = 0;
        }
        s_exit = ex;
      }
    }
    __syncthreads();
    if (s_exit) break;   // the same value for every thread of the CTA
    const int gi = s_g;
    if (gi < 0) {
      if (warp == 0) __nanosleep(256);
      rot += 1;
      __syncthreads();
      continue;
    }
    __threadfence();
    const BGraph& gr = G[gi];
    const int4 stg = gr.stages[s_stage];
    const int idx = s_idx;
    const unsigned gen = gr.gen0 + (unsigned)stg.y + 1u;   // gibbs_apply's ++bm.gen of batch stg.y
    int* n_cur = gr.n_moved + ((gen - 1u) & 1u);
    switch (stg.x) {
      case kEval: {
        const int4 bt = gr.batches[stg.y];
        if (idx < stg.w) {   // a chunk of light vertices
          const int* verts = gr.order + bt.x;
          const int a = idx * gr.chunk;
          const int end = min(a + gr.chunk, bt.y);
          unsigned long long c_visit = 0, c_moved = 0, c_acc = 0;
          for (int i = a + warp; i < end; i += kBWarps) {
            const int v = verts[i];
            const uint4 x =
                draw_record(gr.rng, (uint32_t)v, (uint32_t)gr.sweep, 0u, (long long)gr.sweep * gr.g.V + v, status);
            int r, k_out, k_in;
            const EvalResult res = evaluate_vertex<Store::kDense>(gr.g, gr.bm, v, x, t, lane, status, &r, &k_out, &k_in);
            c_visit++;
            if (res.s != r) c_moved++;
            if (res.accepted) {
              c_acc++;
              if (lane == 0) {
                gr.prop[v] = res.s;
                gr.moved[atomicAdd(n_cur, 1)] = v;
              }
            }
            table_reset(t, lane);
          }
          if (lane == 0 && c_visit) {
            atomicAdd(gr.counters + 0, c_visit);
            atomicAdd(gr.counters + 1, c_moved);
            atomicAdd(gr.counters + 2, c_acc);
          }
        } else {             // one heavy vertex on warp 0, its table over the whole shared memory
          if (warp == 0) {
            WarpTable big = carve_table(smem, P.heavy_cap, 0);
            init_table(big, lane);
            const int v = gr.order[bt.z + (idx - stg.w)];
            const uint4 x =
                draw_record(gr.rng, (uint32_t)v, (uint32_t)gr.sweep, 0u, (long long)gr.sweep * gr.g.V + v, status);
            int r, k_out, k_in;
            const EvalResult res = evaluate_vertex<Store::kDense>(gr.g, gr.bm, v, x, big, lane, status, &r, &k_out, &k_in);
            if (lane == 0) {
              atomicAdd(gr.counters + 0, 1ull);
              if (res.s != r) atomicAdd(gr.counters + 1, 1ull);
              if (res.accepted) {
                atomicAdd(gr.counters + 2, 1ull);
                gr.prop[v] = res.s;
                gr.moved[atomicAdd(n_cur, 1)] = v;
              }
            }
          }
          __syncthreads();
          init_table(t, lane);   // the per-warp tables under the big one are empty again
        }
        break;
      }
      case kApply: {
        const int n = *(volatile int*)n_cur;
        for (int i = idx * kBWarps + warp; i < n; i += stg.z * kBWarps)
          apply_moved_vertex(gr.g, gr.bm, gr.moved[i], gr.prop, gr.qr, gr.qs, gr.last, gen, lane);
        break;
      }
      case kFinish: {
        const int n = *(volatile int*)n_cur;
        if (idx == 0 && tid == 0) gr.n_moved[gen & 1u] = 0;   // the next batch's slot
        for (int i = idx * kBThreads + tid; i < n; i += stg.z * kBThreads)
          finish_moved_vertex(gr.bm, gr.moved[i], gr.prop, gr.qr, gr.qs, gr.last, gen);
        break;
      }
      case kMdlPart: {
        const int c0 = idx * kMdlCtasPerItem, c1 = min(c0 + kMdlCtasPerItem, P.mdl_ctas);
        for (int cc = c0; cc < c1; ++cc) {
          const double v = gr.mdl_cells ? mdl_cells_part(gr.bm, cc, P.mdl_ctas, red)
                                        : mdl_edges_part(gr.g, gr.bm, gr.out_src, cc, P.mdl_ctas, red);
          if (tid == 0) gr.partial[cc] = v;
        }
        break;
      }
      case kMdlFinal: {
        const double v = mdl_final_value(gr.partial, P.mdl_ctas, gr.g.V, gr.g.E, gr.bm.B, red);
        if (tid == 0) *gr.mdl_out = v;
        break;
      }
      default:
        break;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      Queue& q = queue[gi];
      const int prev = atomicAdd(&q.done, 1);
      if (prev + 1 == stg.z) {   // last item of the stage: open the next one
        atomicExch(&q.done, 0);
        __threadfence();
        if (s_stage + 1 >= gr.nstages) {
          atomicExch(&q.finished, 1);
          atomicAdd(nfinished, 1);
        } else {
          atomicExch(&q.ctr, (unsigned long long)(s_stage + 1) << 32);
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------
// Autotuner: candidate item shapes, the choice cached per workload shape.
// ------------------------------------------------------------------------------------------
struct Shape {
  int chunk;         // light vertices per evaluation item
  int ctas_per_sm;   // persistent CTAs per SM
};
const Shape kCandidates[] = {{8, 2}, {16, 2}, {32, 2}, {64, 2}, {16, 1}, {64, 1}};
constexpr int kNumCandidates = sizeof(kCandidates) / sizeof(kCandidates[0]);
std::map<unsigned long long, Shape> g_tuned;   // workload key -> shape

unsigned long long workload_key(int ngraphs, long long vertices) {
  int lv = 0;
  while ((1LL << lv) < vertices) ++lv;
  int lg = 0;
  while ((1 << lg) < ngraphs) ++lg;
  return ((unsigned long long)lg << 8) | (unsigned long long)lv;
}

bool batchable(const SbpBlockmodel& bm, const SbpGraph& g) {
  return !bm.sparse && g.light_cap <= kLightCapMax && g.heavy_cap <= 4096 && bm.B > 1;
}

// The stages of one sweep of a graph with the given plan and chunk.
std::vector<int4> sweep_stages(const BatchPlan& p, int chunk, int mdl_ctas) {
  std::vector<int4> st;
  for (size_t b = 0; b < p.light_n.size(); ++b) {
    const int lc = (p.light_n[b] + chunk - 1) / chunk;
    st.push_back(make_int4(kEval, (int)b, lc + p.heavy_n[b], lc));
    const int stripes = std::max(1, (p.light_n[b] + p.heavy_n[b] + kApplyPerStripe - 1) / kApplyPerStripe);
    st.push_back(make_int4(kApply, (int)b, stripes, 0));
    st.push_back(make_int4(kFinish, (int)b, stripes, 0));
  }
  st.push_back(make_int4(kMdlPart, 0, (mdl_ctas + kMdlCtasPerItem - 1) / kMdlCtasPerItem, 0));
  st.push_back(make_int4(kMdlFinal, 0, 1, 0));
  return st;
}

enum SlotState { kNeedMerge, kFinetuning, kEnded, kDone };   // kEnded: finetune over, not yet wrapped up

struct Slot {
  int index = 0;
  SbpGraph* g = nullptr;
  std::unique_ptr<PartitionState> ps;
  int* out = nullptr;
  SlotState state = kNeedMerge;
  // the finetune in progress (asynchronous Gibbs, as sbpb::finetune)
  SbpFinetuneOptions fo{};
  SbpStats fs{};
  const BatchPlan* plan = nullptr;
  double initial = 0.0;
  std::vector<double> deltas;
  int sweep = 0;
  int stage_chunk = -1;
  std::chrono::steady_clock::time_point t0;
  DevBuf<int4> batches, stages;
  DevBuf<unsigned long long> counters;
  DevBuf<double> partial;
};

// Host threads for the steps of several graphs between their finetunes.  Each thread has its
// own context (stream, status word, MDL scratch), so the small kernels and the host
// synchronisations of different graphs' merges overlap one another.  Created once, never
// destroyed (its threads wait for work until the process exits).
class StepPool {
 public:
  static StepPool& get() {
    static StepPool* pool = new StepPool(kMaxThreads);
    return *pool;
  }
  // fn(item) for every item, spread over `threads` of the pool's threads (each item handled by
  // one thread, its device work finished on return); rethrows the first exception.
  void run(const std::vector<Slot*>& items, int threads, const std::function<void(Slot&)>& fn) {
    threads = std::max(1, std::min({threads, kMaxThreads, (int)items.size()}));
    {
      std::lock_guard<std::mutex> lk(mu_);
      items_ = &items;
      fn_ = &fn;
      next_ = 0;
      active_ = threads;
      busy_ = threads;
      err_ = nullptr;
      ++gen_;
    }
    cv_work_.notify_all();
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return busy_ == 0; });
    if (err_) std::rethrow_exception(err_);
  }

 private:
  static constexpr int kMaxThreads = 64;
  explicit StepPool(int n) {
    int dev = 0;
    SBP_CUDA(cudaGetDevice(&dev));
    double2* logt = Context::primary().logt;
    for (int i = 0; i < n; ++i) std::thread([this, i, dev, logt] { worker(i, dev, logt); }).detach();
  }
  void worker(int i, int dev, double2* logt) {
    Context* ctx = nullptr;
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (i >= active_) continue;   // not one of this round's threads
      }
      try {
        if (!ctx) {
          SBP_CUDA(cudaSetDevice(dev));
          ctx = Context::create(logt);
          Context::current() = ctx;
        }
        for (;;) {
          const int k = next_.fetch_add(1);
          if (k >= (int)items_->size()) break;
          (*fn_)(*(*items_)[k]);
          ctx->sync();
        }
      } catch (...) {
        std::lock_guard<std::mutex> lk(mu_);
        if (!err_) err_ = std::current_exception();
      }
      std::lock_guard<std::mutex> lk(mu_);
      if (--busy_ == 0) cv_done_.notify_all();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  const std::vector<Slot*>* items_ = nullptr;
  const std::function<void(Slot&)>* fn_ = nullptr;
  std::atomic<int> next_{0};
  int active_ = 0, busy_ = 0;
  unsigned long long gen_ = 0;
  std::exception_ptr err_;
};

}  // namespace

// The batched driver: per-graph state machines, one persistent launch per sweep of the
// graphs that are finetuning.
static void partition_batched(std::vector<std::unique_ptr<Slot>>& slots, const SbpOptions& opt, SbpBatchInfo& info) {
  Context& c = Context::get();
  const int n = (int)slots.size();
  int cap = kLightCap, heavy_cap = 512;
  long long vertices = 0;
  for (auto& s : slots) {
    cap = std::max(cap, std::min(s->g->light_cap, kLightCapMax));
    if (s->g->heavy_cap <= 4096) heavy_cap = std::max(heavy_cap, s->g->heavy_cap);
    vertices += s->g->V;
  }
  const size_t smem = std::max((size_t)kBWarps * table_ints(cap), (size_t)table_ints(heavy_cap)) * sizeof(int);
  set_smem_limit((const void*)k_batched_sweep, smem);
  int max_per_sm = 0;
  SBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_per_sm, k_batched_sweep, kBThreads, smem));
  if (max_per_sm < 1) throw Error(SBP_ERR_UNSUPPORTED, "batched sweep kernel does not fit on an SM");

  DevBuf<BGraph> dG;
  DevBuf<int> dList, dSync;   // dSync: nfinished, abort
  Queue* hQ = nullptr;        // the queues' start state, copied in before every launch
  DevBuf<Queue> dQ;
  DevBuf<SweepParams> dP;
  DevBuf<double> dMdl;
  dG.reserve(n);
  dList.reserve(n);
  dSync.reserve(2);
  dQ.reserve(n);
  dP.reserve(1);
  dMdl.reserve(n);
  BGraph* hG = nullptr;
  int* hList = nullptr;
  SweepParams* hP = nullptr;
  double* hMdl = nullptr;
  int* hStatus = nullptr;
  SBP_CUDA(cudaMallocHost(&hG, n * sizeof(BGraph)));
  SBP_CUDA(cudaMallocHost(&hList, n * sizeof(int)));
  SBP_CUDA(cudaMallocHost(&hP, sizeof(SweepParams)));
  SBP_CUDA(cudaMallocHost(&hMdl, n * sizeof(double)));
  SBP_CUDA(cudaMallocHost(&hStatus, sizeof(int)));
  SBP_CUDA(cudaMallocHost(&hQ, n * sizeof(Queue)));
  std::memset(hQ, 0, n * sizeof(Queue));
  struct Cleanup {
    void* pinned[6];
    std::map<int, cudaGraphExec_t> execs;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Cleanup() {
      for (void* x : pinned)
        if (x) cudaFreeHost(x);
      for (auto& kv : execs) cudaGraphExecDestroy(kv.second);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } cl{{hG, hList, hP, hMdl, hStatus, hQ}, {}, nullptr, nullptr};
  SBP_CUDA(cudaEventCreate(&cl.e0));
  SBP_CUDA(cudaEventCreate(&cl.e1));

  const unsigned long long key = workload_key(n, vertices);
  const bool tuning = g_tuned.find(key) == g_tuned.end();
  if (tuning) info.tuned = 1;
  double cand_ms[kNumCandidates];
  int ncand = 0;
  auto current_shape = [&]() -> Shape {
    Shape sh = tuning ? (ncand < kNumCandidates ? kCandidates[ncand] : g_tuned[key]) : g_tuned[key];
    sh.ctas_per_sm = std::min(sh.ctas_per_sm, max_per_sm);
    return sh;
  };

  auto start_finetune = [&](Slot& s) {
    Context& c = Context::get();   // primary, or secondary beside a sweep launch
    SbpBlockmodel& bm = s.ps->bm;
    std::memset(&s.fs, 0, sizeof s.fs);
    s.fs.num_blocks = bm.B;
    s.plan = &s.g->plan(SBP_ASYNC_GIBBS, s.fo.batches);
    if (!s.batches.p) {   // the plan is the graph's, the same in every round
      std::vector<int4> bt(s.plan->light_n.size());
      for (size_t b = 0; b < bt.size(); ++b)
        bt[b] = make_int4(s.plan->light_begin[b], s.plan->light_n[b], s.plan->heavy_begin[b], s.plan->heavy_n[b]);
      s.batches.reserve(std::max<size_t>(bt.size(), 1));
      if (!bt.empty())
        SBP_CUDA(SBP_COPY_ASYNC(s.batches.p, bt.data(), bt.size() * sizeof(int4), cudaMemcpyHostToDevice, c.stream));
      s.stages.reserve(3 * bt.size() + 2);
      s.counters.reserve(3);
      s.partial.reserve(c.npartial);
    }
    SBP_CUDA(cudaMemsetAsync(s.counters.p, 0, 3 * sizeof(unsigned long long), c.stream));
    bm.overall_entropy = (float)mdl(bm, *s.g);
    s.initial = bm.overall_entropy;
    s.deltas.clear();
    s.sweep = 0;
    s.t0 = std::chrono::steady_clock::now();
    s.state = kFinetuning;
  };
  auto end_finetune = [&](Slot& s) {
    Context& c = Context::get();
    SbpBlockmodel& bm = s.ps->bm;
    bm.overall_entropy = (float)mdl(bm, *s.g);
    unsigned long long cnt[3];
    SBP_CUDA(SBP_COPY_ASYNC(cnt, s.counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    s.fs.visits = (long long)cnt[0];
    s.fs.proposals_moved = (long long)cnt[1];
    s.fs.accepted = (long long)cnt[2];
    s.fs.mdl = bm.overall_entropy;
    s.fs.mcmc_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - s.t0).count();
    s.fs.num_blocks = bm.B;
    partition_finish_round(*s.ps, *s.g, s.fs, s.out);
    s.state = s.ps->done ? kDone : kNeedMerge;
  };

  // The steps of one graph between two finetunes: the end of the last one, the golden-section
  // step, the merge, and the start of the next finetune (batched) or a whole single-graph one.
  // Runs on any host thread, on that thread's current context.
  std::atomic<int> n_batched{0}, n_fallback{0};
  const std::function<void(Slot&)> between = [&](Slot& s) {
    if (s.state == kEnded) end_finetune(s);
    if (s.state != kNeedMerge) return;
    const int algo = partition_merge(*s.ps, *s.g, opt, &s.fo);
    if (algo == SBP_ASYNC_GIBBS && batchable(s.ps->bm, *s.g)) {
      start_finetune(s);
      n_batched++;
    } else {
      SbpStats fs;
      finetune(s.ps->bm, *s.g, algo, s.fo, nullptr, fs);
      n_fallback++;
      partition_finish_round(*s.ps, *s.g, fs, s.out);
      s.state = s.ps->done ? kDone : kNeedMerge;
    }
  };
  // The graphs between finetunes, each once: on the step pool's threads (each with its own
  // context), or with batched_threads 1 on this thread -- beside a sweep launch on the secondary
  // context, else on the primary one.  Beside a launch they touch none of the buffers of the
  // graphs in it, and buffers released to the device cache carry their stream's event.
  const int threads = g_batched_threads;
  const bool overlap = g_batched_overlap > 0;
  Context* side = (overlap && threads == 1) ? &Context::secondary() : nullptr;
  auto run_between = [&](bool beside_launch) {
    std::vector<Slot*> v;
    for (auto& sp : slots)
      if (sp->state == kEnded || sp->state == kNeedMerge) v.push_back(sp.get());
    if (v.empty()) return;
    const auto h0 = std::chrono::steady_clock::now();
    if (threads > 1) {
      StepPool::get().run(v, threads, between);
    } else {
      ContextScope scope(beside_launch ? side : nullptr);
      for (Slot* sp : v) between(*sp);
      if (beside_launch) side->sync();
    }
    (beside_launch ? info.overlapped_seconds : info.serial_seconds) +=
        std::chrono::duration<double>(std::chrono::steady_clock::now() - h0).count();
  };

  for (;;) {
    std::vector<Slot*> act;
    bool all_done = true, waiting = false;
    for (auto& sp : slots) {
      if (sp->state == kFinetuning) act.push_back(sp.get());
      if (sp->state == kNeedMerge || sp->state == kEnded) waiting = true;
      if (sp->state != kDone) all_done = false;
    }
    if (all_done) break;
    if (act.empty() || (waiting && !overlap)) {   // no launch to run beside: the steps first
      run_between(false);
      act.clear();
      for (auto& sp : slots)
        if (sp->state == kFinetuning) act.push_back(sp.get());
      waiting = false;
      if (act.empty()) continue;
    }

    // one sweep of every finetuning graph
    const Shape shape = current_shape();
    for (Slot* s : act) {
      if (s->stage_chunk != shape.chunk) {
        const std::vector<int4> st = sweep_stages(*s->plan, shape.chunk, c.npartial);
        SBP_CUDA(SBP_COPY_ASYNC(s->stages.p, st.data(), st.size() * sizeof(int4), cudaMemcpyHostToDevice, c.stream));
        s->stage_chunk = shape.chunk;
      }
      BGraph& b = hG[s->index];
      SbpBlockmodel& bm = s->ps->bm;
      b.g = s->g->view();
      b.bm = bm.view();
      b.order = s->plan->order.p;
      b.batches = s->batches.p;
      b.stages = s->stages.p;
      b.out_src = s->g->out_src.p;
      b.prop = bm.prop.p;
      b.moved = bm.moved.p;
      b.n_moved = bm.n_moved.p;
      b.qr = bm.qr.p;
      b.qs = bm.qs.p;
      b.last = bm.last.p;
      b.counters = s->counters.p;
      b.partial = s->partial.p;
      b.mdl_out = dMdl.p + s->index;
      b.rng.seed = s->fo.seed;
      b.rng.replay = nullptr;
      b.rng.replay_records = 0;
      b.rng.call = s->fo.call;
      b.sweep = s->sweep;
      b.gen0 = bm.gen;
      b.nstages = (int)(3 * s->plan->light_n.size() + 2);
      b.chunk = shape.chunk;
      b.mdl_cells = (!bm.sparse && (long long)bm.B * bm.B <= 4LL * s->g->E) ? 1 : 0;
    }
    for (size_t k = 0; k < act.size(); ++k) hList[k] = act[k]->index;
    hP->ngraphs = (int)act.size();
    hP->mdl_ctas = c.npartial;
    hP->heavy_cap = heavy_cap;
    hP->wait_limit = (unsigned)g_batched_wait_limit;
    // fault injection for the failure-detection test: the stalled graph's first stage starts
    // with every item taken, so it never completes and no stage of that graph opens again
    for (Slot* s : act) {
      Queue& q = hQ[s->index];
      std::memset(&q, 0, sizeof q);
      if (g_batched_stall_graph == s->index) q.ctr = 1ull << 20;   // stage 0, item 2^20: beyond every stage
    }
    const int reserve = waiting ? std::min(g_batched_overlap, shape.ctas_per_sm * c.num_sms / 2) : 0;
    const int grid = shape.ctas_per_sm * c.num_sms - reserve;
    auto ex = cl.execs.find(grid);
    if (ex == cl.execs.end()) {
      cudaGraph_t graph;
      SBP_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
      cudaMemcpyAsync(dG.p, hG, n * sizeof(BGraph), cudaMemcpyHostToDevice, c.stream);
      cudaMemcpyAsync(dList.p, hList, n * sizeof(int), cudaMemcpyHostToDevice, c.stream);
      cudaMemcpyAsync(dP.p, hP, sizeof(SweepParams), cudaMemcpyHostToDevice, c.stream);
      cudaMemcpyAsync(dQ.p, hQ, n * sizeof(Queue), cudaMemcpyHostToDevice, c.stream);
      cudaMemsetAsync(dSync.p, 0, 2 * sizeof(int), c.stream);
      k_batched_sweep<<<grid, kBThreads, smem, c.stream>>>(dG.p, dList.p, dQ.p, dSync.p, dSync.p + 1, dP.p, cap,
                                                           c.status);
      cudaMemcpyAsync(hMdl, dMdl.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
      cudaMemcpyAsync(hStatus, c.status, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
      SBP_CUDA(cudaStreamEndCapture(c.stream, &graph));
      cudaGraphExec_t exec;
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      SBP_CUDA(ie);
      ex = cl.execs.emplace(grid, exec).first;
    }
    SBP_CUDA(cudaEventRecord(cl.e0, c.stream));
    SBP_CUDA(cudaGraphLaunch(ex->second, c.stream));
    SBP_CUDA(cudaEventRecord(cl.e1, c.stream));
    ++g_launches;
    g_h2d += (long long)(n * (sizeof(BGraph) + sizeof(int) + sizeof(Queue)) + sizeof(SweepParams));
    g_d2h += (long long)(n * sizeof(double) + sizeof(int));
    if (waiting) {   // beside the launch
      try {
        run_between(true);
      } catch (...) {
        cudaStreamSynchronize(c.stream);   // no launch outlives the call
        throw;
      }
    }
    c.sync();
    info.sweep_launches++;
    if (*hStatus) c.check_status();
    float ms = 0.f;
    SBP_CUDA(cudaEventElapsedTime(&ms, cl.e0, cl.e1));
    info.sweep_seconds += ms * 1e-3;
    if (tuning && ncand < kNumCandidates) {
      cand_ms[ncand] = ms / std::max<size_t>(act.size(), 1);   // per graph swept
      if (++ncand == kNumCandidates) {
        int best = 0;
        for (int q = 1; q < kNumCandidates; ++q)
          if (cand_ms[q] < cand_ms[best]) best = q;
        g_tuned[key] = kCandidates[best];
      }
    }
    for (Slot* s : act) {
      SbpBlockmodel& bm = s->ps->bm;
      bm.gen += (unsigned)s->plan->light_n.size();
      const double entropy = hMdl[s->index];
      s->deltas.push_back(entropy - s->initial);   // last_iteration_entropy is never updated
      s->fs.sweeps++;
      const int it = s->sweep++;
      if (early_stop(it, s->fo.bracket_established != 0, s->initial, s->deltas) || s->sweep >= kMaxIterations)
        s->state = kEnded;
    }
  }
  if (tuning && g_tuned.find(key) == g_tuned.end() && ncand > 0) {
    int best = 0;
    for (int q = 1; q < ncand; ++q)
      if (cand_ms[q] < cand_ms[best]) best = q;
    g_tuned[key] = kCandidates[best];
  }
  if (tuning) {
    info.candidates = ncand;
    for (int q = 0; q < ncand && q < 8; ++q) info.candidate_ms[q] = cand_ms[q];
  }
  if (g_tuned.count(key)) {
    info.chunk = g_tuned[key].chunk;
    info.ctas_per_sm = std::min(g_tuned[key].ctas_per_sm, max_per_sm);
  }
  info.batched_finetunes = n_batched;
  info.fallback_finetunes = n_fallback;
  c.check_status();
}

}  // namespace sbpb

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

extern "C" {

SbpStatus sbp_partition_batched(int32_t n, const SbpGraph* const* graphs, const SbpOptions* opt,
                                int32_t* const* out_assignments, SbpStats* stats, SbpBatchInfo* info) {
  SBP_API_BEGIN
  SBP_REQUIRE(n >= 1 && graphs && opt && out_assignments, "invalid argument");
  SBP_REQUIRE(opt->batches >= 1, "batches must be >= 1");
  SBP_REQUIRE(opt->algorithm >= 0 && opt->algorithm <= 2, "unknown finetune algorithm");
  for (int i = 0; i < n; ++i) SBP_REQUIRE(graphs[i] && out_assignments[i], "null graph or output");
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) SBP_REQUIRE(graphs[i] != graphs[j], "a graph appears twice in the batch");
  Context& c = Context::get();
  SbpBatchInfo bi;
  std::memset(&bi, 0, sizeof bi);
  cudaEvent_t t0, t1;
  SBP_CUDA(cudaEventCreate(&t0));
  SBP_CUDA(cudaEventCreate(&t1));
  SBP_CUDA(cudaEventRecord(t0, c.stream));
  std::vector<std::unique_ptr<Slot>> slots(n);
  for (int i = 0; i < n; ++i) {
    slots[i] = std::make_unique<Slot>();
    Slot& s = *slots[i];
    s.index = i;
    s.g = const_cast<SbpGraph*>(graphs[i]);
    s.out = out_assignments[i];
    s.ps = std::make_unique<PartitionState>();
    partition_begin(*s.ps, *s.g);
  }
  partition_batched(slots, *opt, bi);
  SBP_CUDA(cudaEventRecord(t1, c.stream));
  c.sync();
  float ms = 0.f;
  SBP_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  bi.seconds = ms * 1e-3;
  for (int i = 0; i < n; ++i) {
    slots[i]->ps->st.total_seconds = bi.seconds;   // the batch's device time, shared
    bi.rounds = std::max(bi.rounds, slots[i]->ps->st.outer_iterations);
    if (stats) stats[i] = slots[i]->ps->st;
  }
  if (info) *info = bi;
  SBP_API_END
}

SbpStatus sbp_batched_reset_tuning(void) {
  SBP_API_BEGIN
  g_tuned.clear();
  SBP_API_END
}

}  // extern "C"
