// Replay hooks of the patched reference build (declared in sbp_replay.h).  TEST INFRASTRUCTURE
// ONLY: compiled together with a patched copy of the reference's sources into
// oracle/_ref/replay/ref_driver by oracle/build_reference.py.
//
// Log (SBP_REPLAY_LOG=<path>; no log when unset), little-endian records, each starting with a
// one-byte tag:
//   'B' call start  int32 id, kind, bracket; state
//   'E' call end    int32 id, kind, sweeps; state
//   'P' visit       int32 id, sweep, vertex, proposed block
//   'U' uniform     int32 id, sweep, vertex; float64 u
//   'M' merge       int32 id, block, proposal index, proposed block
//   'S' scores      int32 id, B; int32 best[B]; float64 delta[B]
//   'G' split       int32 n_high; int32 high[n_high]; int32 n_low; int32 low[n_low]
// state = int32 B, V, num_blocks_to_merge; float32 overall_entropy; int32 b[V], d_out[B],
//         d_in[B], d[B]; int64 nnz; nnz x (int32 row, col, count)
#include "sbp_replay.h"

#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <numeric>

#include "blockmodel/blockmodel.hpp"
#include "block_merge.hpp"
#include "entropy.hpp"
#include "finetune.hpp"

namespace sbp_replay {

namespace {
std::mutex g_mutex;
FILE *g_log = nullptr;
bool g_opened = false;
int g_next_id = 0;
int g_cur_call = -1;
int g_sweep0 = 0;
thread_local int t_sweep = -1, t_vertex = -1, t_block = -1, t_slot = -1;

FILE *log_file() {  // call with g_mutex held
    if (!g_opened) {
        g_opened = true;
        const char *p = std::getenv("SBP_REPLAY_LOG");
        if (p && *p) {
            g_log = std::fopen(p, "wb");
            if (g_log) std::setvbuf(g_log, nullptr, _IOFBF, 1 << 22);
        }
    }
    return g_log;
}

template <class T>
void put(FILE *f, const T &x) {
    std::fwrite(&x, sizeof(T), 1, f);
}
template <class T>
void put_vec(FILE *f, const std::vector<T> &v) {
    if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
}

void put_state(FILE *f, Blockmodel &bm) {
    const int B = bm.getNum_blocks();
    const std::vector<int> &b = bm.block_assignment();
    put<int32_t>(f, B);
    put<int32_t>(f, (int32_t)b.size());
    put<int32_t>(f, bm.getNum_blocks_to_merge());
    put<float>(f, bm.getOverall_entropy());
    put_vec(f, b);
    put_vec(f, bm.degrees_out());
    put_vec(f, bm.degrees_in());
    put_vec(f, bm.degrees());
    std::vector<int32_t> cells;
    for (int row = 0; row < B; ++row) {
        std::vector<std::pair<int, int>> r;
        for (const auto &e : bm.blockmatrix()->getrow_sparse(row))
            if (e.second != 0) r.emplace_back(e.first, e.second);
        std::sort(r.begin(), r.end());
        for (const auto &e : r) {
            cells.push_back(row);
            cells.push_back(e.first);
            cells.push_back(e.second);
        }
    }
    put<int64_t>(f, (int64_t)(cells.size() / 3));
    put_vec(f, cells);
}
}  // namespace

unsigned seed() {
    const char *p = std::getenv("SBP_REF_SEED");
    return p ? (unsigned)std::strtoul(p, nullptr, 10) : 1u;
}

int max_sweeps() {
    const char *p = std::getenv("SBP_REF_MAX_SWEEPS");
    const int n = p ? std::atoi(p) : 100;
    return n > 0 ? n : 100;
}

CallScope::CallScope(int k, Blockmodel &b, int bracket) : kind(k), id(0), sweep0(finetune::MCMC_iterations), bm(b) {
    std::lock_guard<std::mutex> lock(g_mutex);
    id = g_next_id++;
    g_cur_call = id;
    g_sweep0 = sweep0;
    if (FILE *f = log_file()) {
        put<char>(f, 'B');
        put<int32_t>(f, id);
        put<int32_t>(f, kind);
        put<int32_t>(f, bracket);
        put_state(f, bm);
    }
}

CallScope::~CallScope() {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (FILE *f = log_file()) {
        put<char>(f, 'E');
        put<int32_t>(f, id);
        put<int32_t>(f, kind);
        put<int32_t>(f, finetune::MCMC_iterations - sweep0);
        put_state(f, bm);
        std::fflush(f);
    }
}

void on_split(const std::vector<int> &high, const std::vector<int> &low) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (FILE *f = log_file()) {
        put<char>(f, 'G');
        put<int32_t>(f, (int32_t)high.size());
        put_vec(f, high);
        put<int32_t>(f, (int32_t)low.size());
        put_vec(f, low);
    }
}

void on_proposal(int vertex, int s) {
    t_sweep = finetune::MCMC_iterations - g_sweep0;
    t_vertex = vertex;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (FILE *f = log_file()) {
        put<char>(f, 'P');
        const int32_t rec[4] = {g_cur_call, t_sweep, vertex, s};
        std::fwrite(rec, sizeof rec, 1, f);
    }
}

void on_uniform(double u) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (FILE *f = log_file()) {
        put<char>(f, 'U');
        const int32_t rec[3] = {g_cur_call, t_sweep, t_vertex};
        std::fwrite(rec, sizeof rec, 1, f);
        put<double>(f, u);
    }
}

void on_merge_slot(int block, int i) {
    t_block = block;
    t_slot = i;
}

void on_merge_proposal(int s) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (FILE *f = log_file()) {
        put<char>(f, 'M');
        const int32_t rec[4] = {g_cur_call, t_block, t_slot, s};
        std::fwrite(rec, sizeof rec, 1, f);
    }
}

void on_merge_scores(const std::vector<int> &best, const std::vector<double> &delta) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (FILE *f = log_file()) {
        put<char>(f, 'S');
        put<int32_t>(f, g_cur_call);
        put<int32_t>(f, (int32_t)best.size());
        put_vec(f, best);
        put_vec(f, delta);
    }
}

// The engine's ranking score of a merge: the delta-MDL rounded to a multiple of 2^-20.
static double merge_score(double dS) { return std::nearbyint(dS * 1048576.0) / 1048576.0; }

double merge_delta_canonical(int r, int s, int k_out, int k_in, const Blockmodel &bm) {
    if (r < s) {
        const utils::ProposalAndEdgeCounts p{s, k_out, k_in, k_out + k_in};
        const Delta d = block_merge::blockmodel_delta(r, s, bm);
        return merge_score(entropy::block_merge_delta_mdl(r, p, bm, d));
    }
    // the same merge seen from the higher block: s into r, with s's edge counts taken as
    // common::propose_new_block takes them for a merge (outgoing / incoming edge weights)
    const EdgeWeights out_b = bm.blockmatrix()->outgoing_edges(s);
    const EdgeWeights in_b = bm.blockmatrix()->incoming_edges(s);
    const int ko = std::accumulate(out_b.values.begin(), out_b.values.end(), 0);
    const int ki = std::accumulate(in_b.values.begin(), in_b.values.end(), 0);
    const utils::ProposalAndEdgeCounts q{r, ko, ki, ko + ki};
    const Delta d = block_merge::blockmodel_delta(s, r, bm);
    return merge_score(entropy::block_merge_delta_mdl(s, q, bm, d));
}

std::vector<int> stable_sort_indices(const std::vector<double> &values) {
    std::vector<int> idx(values.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&values](int a, int b) { return values[a] < values[b]; });
    return idx;
}

}  // namespace sbp_replay
