// Partition quality against a known (planted) partition: evaluate::evaluate_blockmodel
// (src/evaluate.cpp:98-178) with calculate_f1_score and calculate_nmi (src/evaluate.cpp:7-96).
//
// The contingency table (algorithm block x true community) is counted on the device in one pass
// over the vertices; the matching of blocks to communities (the reference solves it with the
// Hungarian method, extern/hungarian) and the metrics run on the host on the B x K table.  The
// matching only sets the accuracy (the matched counts over V); F1, precision, recall, the Rand
// index and NMI do not depend on the order of rows or columns.
//
// Arithmetic: 64-bit integer pair counts (the reference multiplies ints, which wraps for
// V > 46340 in the Rand index and for counts above 46340 in cells_squared), FP64 logs (the
// reference's marginal entropies use logf through utils::nat_log).
#include <limits>

#include "sbp_engine.cuh"

namespace sbpb {
namespace {

// One vertex per thread; labels already mapped to 0..K-1 (-1: unknown, not counted).  A
// CTA-private table in shared memory when it fits, else global atomics.
__global__ void k_contingency(const int* __restrict__ b, const int* __restrict__ truth, int V, int ncols,
                              int cells, int use_smem, unsigned long long* table) {
  extern __shared__ unsigned sm_table[];
  if (use_smem) {
    for (int i = threadIdx.x; i < cells; i += blockDim.x) sm_table[i] = 0u;
    __syncthreads();
  }
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int t = truth[v];
    if (t < 0) continue;
    const int cell = b[v] * ncols + t;
    if (use_smem) atomicAdd(sm_table + cell, 1u);
    else atomicAdd(table + cell, 1ull);
  }
  if (use_smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < cells; i += blockDim.x)
      if (sm_table[i]) atomicAdd(table + i, (unsigned long long)sm_table[i]);
  }
}

// Maximum-weight matching of the rows of an n x m table (n <= m) to distinct columns: the
// Hungarian method in its shortest-augmenting-path form with row and column potentials
// (Kuhn 1955, Munkres 1957; O(n^2 m)), on costs -w.  Returns the matched weight.
long long max_weight_matching(int n, int m, const std::vector<long long>& w) {
  const long long INF = std::numeric_limits<long long>::max() / 4;
  std::vector<long long> u(n + 1, 0), p_col(m + 1, 0), minv(m + 1);
  std::vector<int> match(m + 1, 0), way(m + 1, 0);   // match[j]: row (1-based) matched to column j
  std::vector<char> used(m + 1);
  for (int i = 1; i <= n; ++i) {
    match[0] = i;
    int j0 = 0;
    std::fill(minv.begin(), minv.end(), INF);
    std::fill(used.begin(), used.end(), 0);
    do {
      used[j0] = 1;
      const int i0 = match[j0];
      long long delta = INF;
      int j1 = 0;
      for (int j = 1; j <= m; ++j) {
        if (used[j]) continue;
        const long long cur = -w[(size_t)(i0 - 1) * m + (j - 1)] - u[i0] - p_col[j];
        if (cur < minv[j]) {
          minv[j] = cur;
          way[j] = j0;
        }
        if (minv[j] < delta) {
          delta = minv[j];
          j1 = j;
        }
      }
      for (int j = 0; j <= m; ++j) {
        if (used[j]) {
          u[match[j]] += delta;
          p_col[j] -= delta;
        } else {
          minv[j] -= delta;
        }
      }
      j0 = j1;
    } while (match[j0] != 0);
    do {
      const int j1 = way[j0];
      match[j0] = match[j1];
      j0 = j1;
    } while (j0);
  }
  long long total = 0;
  for (int j = 1; j <= m; ++j)
    if (match[j]) total += w[(size_t)(match[j] - 1) * m + (j - 1)];
  return total;
}

}  // namespace

// calculate_f1_score and calculate_nmi (src/evaluate.cpp:7-96) of a table with rows = algorithm
// blocks and columns = true communities, plus the accuracy of the best matching.
void contingency_metrics(int nrows, int ncols, const std::vector<long long>& table, long long num_vertices,
                         SbpEvaluation* out) {
  std::vector<double> rowsums(nrows, 0.0), colsums(ncols, 0.0);
  long long cell_pairs2 = 0, cells_squared = 0, total = 0;
  for (int r = 0; r < nrows; ++r)
    for (int c = 0; c < ncols; ++c) {
      const long long x = table[(size_t)r * ncols + c];
      rowsums[r] += (double)x;
      colsums[c] += (double)x;
      cell_pairs2 += x * (x - 1);
      cells_squared += x * x;
      total += x;
    }
  const double cell_pairs = (double)cell_pairs2 / 2.0;
  double row_pairs = 0.0, col_pairs = 0.0, rows_sq = 0.0, cols_sq = 0.0;
  for (double s : rowsums) {
    row_pairs += s * (s - 1.0);
    rows_sq += s * s;
  }
  for (double s : colsums) {
    col_pairs += s * (s - 1.0);
    cols_sq += s * s;
  }
  row_pairs /= 2.0;
  col_pairs /= 2.0;
  const double N = (double)num_vertices;
  const double num_pairs = N * (N - 1.0) / 2.0;
  const double agree_diff = (N * N + (double)cells_squared - (rows_sq + cols_sq)) / 2.0;
  out->rand_index = (cell_pairs + agree_diff) / num_pairs;
  out->recall = cell_pairs / row_pairs;
  out->precision = cell_pairs / col_pairs;
  out->f1_score = 2.0 * out->precision * out->recall / (out->precision + out->recall);
  // NMI with the probabilities of the table over num_vertices (src/evaluate.cpp:61-96)
  double h_rows = 0.0, h_cols = 0.0, mi = 0.0;
  for (double s : rowsums)
    if (s > 0) h_rows -= (s / N) * std::log(s / N);
  for (double s : colsums)
    if (s > 0) h_cols -= (s / N) * std::log(s / N);
  for (int r = 0; r < nrows; ++r)
    for (int c = 0; c < ncols; ++c) {
      const double pj = (double)table[(size_t)r * ncols + c] / N;
      if (pj == 0.0) continue;
      mi += pj * std::log(pj / ((rowsums[r] / N) * (colsums[c] / N)));
    }
  out->nmi = mi / std::sqrt(h_rows * h_cols);
  // accuracy: the matched counts of the best one-to-one matching over the smaller side
  long long matched = 0;
  if (nrows <= ncols) {
    matched = max_weight_matching(nrows, ncols, table);
  } else {
    std::vector<long long> tt((size_t)nrows * ncols);
    for (int r = 0; r < nrows; ++r)
      for (int c = 0; c < ncols; ++c) tt[(size_t)c * nrows + r] = table[(size_t)r * ncols + c];
    matched = max_weight_matching(ncols, nrows, tt);
  }
  out->accuracy = (double)matched / N;
  out->num_blocks = nrows;
  out->true_num_blocks = ncols;
  out->counted_vertices = total;
}

}  // namespace sbpb

extern "C" {

SbpStatus sbp_contingency_metrics(int32_t nrows, int32_t ncols, const int64_t* table, int64_t num_vertices,
                                  SbpEvaluation* out) {
  try {
    if (!table || !out || nrows < 1 || ncols < 1 || num_vertices < 2)
      throw Error(SBP_ERR_INVALID_ARGUMENT, "sbp_contingency_metrics: bad argument");
    std::vector<long long> t(table, table + (size_t)nrows * ncols);
    for (long long x : t)
      if (x < 0) throw Error(SBP_ERR_INVALID_ARGUMENT, "sbp_contingency_metrics: negative count");
    std::memset(out, 0, sizeof *out);
    out->true_mdl = std::nan("");
    contingency_metrics(nrows, ncols, t, num_vertices, out);
    return SBP_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SBP_ERR_CUDA;
  }
}

SbpStatus sbp_evaluate_blockmodel(const SbpBlockmodel* bm, const SbpGraph* g, const int32_t* true_assignment,
                                  SbpEvaluation* out, int64_t* table_out) {
  try {
    if (!bm || !g || !true_assignment || !out || bm->V != g->V)
      throw Error(SBP_ERR_INVALID_ARGUMENT, "sbp_evaluate_blockmodel: bad argument");
    Context& c = Context::get();
    const int V = g->V, B = bm->B;
    // evaluate::hungarian's translator: true communities numbered in order of first appearance
    std::vector<int> truth(V);
    std::unordered_map<int, int> tr;
    bool unknown = false;
    for (int v = 0; v < V; ++v) {
      const int t = true_assignment[v];
      if (t < 0) {
        truth[v] = -1;
        unknown = true;
        continue;
      }
      auto it = tr.find(t);
      if (it == tr.end()) it = tr.emplace(t, (int)tr.size()).first;
      truth[v] = it->second;
    }
    const int K = (int)tr.size();
    if (K == 0) throw Error(SBP_ERR_INVALID_ARGUMENT, "sbp_evaluate_blockmodel: no known true community");
    const long long cells = (long long)B * K;
    if (cells > (1LL << 31)) throw Error(SBP_ERR_UNSUPPORTED, "sbp_evaluate_blockmodel: contingency table too large");
    DevBuf<int> d_truth;
    DevBuf<unsigned long long> d_table;
    d_truth.reserve(V);
    d_table.reserve((size_t)cells);
    SBP_CUDA(SBP_COPY_ASYNC(d_truth.p, truth.data(), V * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    SBP_CUDA(cudaMemsetAsync(d_table.p, 0, cells * sizeof(unsigned long long), c.stream));
    const int use_smem = cells <= 12288 ? 1 : 0;   // 48 KB of 32-bit counters
    const int grid = grid_for(V, 256, use_smem ? 2 * c.num_sms : 8 * c.num_sms);
    k_contingency<<<grid, 256, use_smem ? cells * sizeof(unsigned) : 0, c.stream>>>(bm->b.p, d_truth.p, V, K,
                                                                                    (int)cells, use_smem, d_table.p);
    SBP_CHECK_LAUNCH();
    std::vector<long long> table((size_t)cells);
    SBP_CUDA(SBP_COPY_ASYNC(table.data(), d_table.p, cells * sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    std::memset(out, 0, sizeof *out);
    contingency_metrics(B, K, table, V, out);   // probabilities over all V vertices, as the reference
    if (table_out) std::memcpy(table_out, table.data(), table.size() * sizeof(long long));
    // entropy::mdl of the true partition (evaluate_blockmodel, src/evaluate.cpp:103-110)
    out->true_mdl = std::nan("");
    if (!unknown) {
      SbpBlockmodel tb;
      tb.graph = g;
      tb.init_vertex_scratch(V);
      SBP_CUDA(SBP_COPY_ASYNC(tb.b.p, truth.data(), V * sizeof(int), cudaMemcpyHostToDevice, c.stream));
      tb.set_blocks(K);
      rebuild(tb, *g);
      out->true_mdl = mdl(tb, *g);
    }
    return SBP_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SBP_ERR_CUDA;
  }
}

}  // extern "C"
