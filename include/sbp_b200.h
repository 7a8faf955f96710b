/*
 * sbp_b200.h -- C ABI of the B200 stochastic block partitioning engine (libsbp_b200.so).
 *
 * Plain pointers and sizes only; no exceptions cross this boundary.  Every function returns
 * an SbpStatus; sbp_last_error() gives a message for the last failure on the calling thread.
 * Device memory is owned by the handles; the caller owns every host buffer.  Calls on the
 * same handle are not thread-safe.  There is no CPU fallback: without a usable CUDA device
 * every compute call fails with SBP_ERR_CUDA.
 *
 * Each entry point names the reference interface it replaces
 * (vtsynergy/Hybrid-Stochastic-Block-Partitioning, file:line).
 */
#ifndef SBP_B200_H
#define SBP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SBP_OK = 0,
    SBP_ERR_INVALID_ARGUMENT = 1,  /* bad pointer, size, vertex or block id */
    SBP_ERR_CUDA = 2,              /* CUDA runtime failure or no device */
    SBP_ERR_UNSUPPORTED = 3,       /* input outside what the kernels support (e.g. degree) */
    SBP_ERR_REPLAY = 4,            /* replay stream shorter than the run needs */
    SBP_ERR_DEVICE = 5,            /* a kernel reported an inconsistency (status word) */
    SBP_ERR_OUT_OF_MEMORY = 6
} SbpStatus;

/* Finetune algorithms (include/args.hpp:45-48, `-a`). */
typedef enum {
    SBP_METROPOLIS_HASTINGS = 0,
    SBP_ASYNC_GIBBS = 1,
    SBP_HYBRID_MCMC = 2
} SbpAlgorithm;

typedef struct SbpGraph SbpGraph;
typedef struct SbpBlockmodel SbpBlockmodel;

/* Host-supplied random stream: `records` 4-word records (x_neighbour, x_multinomial,
 * u_hi, u_lo).  A finetune call reads record sweep*V + v for the visit of vertex v in that
 * sweep; a merge call reads record block*10 + proposal. */
typedef struct {
    const uint32_t *words;   /* 4 * records words */
    int64_t records;
} SbpReplay;

/* Counters of one finetune, merge or partition call. */
typedef struct {
    int64_t visits;            /* vertex evaluations (proposals drawn) */
    int64_t proposals_moved;   /* proposals with s != r */
    int64_t accepted;          /* accepted vertex moves */
    int32_t sweeps;            /* MCMC iterations */
    int32_t outer_iterations;  /* partition only: merge+finetune rounds */
    int32_t num_blocks;        /* blocks after the call */
    int32_t overflow_rebuilds; /* row-hashed storage rebuilt because a row ran out of room */
    double mdl;                /* overall entropy after the call (the reference stores it as float) */
    double mcmc_seconds;       /* device time spent in finetune */
    double merge_seconds;      /* device time spent in block merge */
    int64_t merge_proposals;   /* block-merge proposals drawn */
    int64_t merge_avoided;     /* proposals skipped as duplicates */
    double total_seconds;      /* partition only: device-clock time of the whole call */
    int32_t learned_sweeps;    /* sweeps that used the learned proposal (sbp_finetune_learned) */
    int32_t _reserved;
} SbpStats;

/* Launch and timing counters of this library (process-wide). */
typedef struct {
    int64_t launches;          /* kernels launched by the library since load */
    int64_t eval_launches;     /* profiled vertex-evaluation launches */
    int64_t eval_visits;       /* vertices they evaluated */
    double eval_ms;            /* summed CUDA-event duration of those launches */
    double eval_bytes;         /* algorithmic bytes: sum over vertices of 12 + 8 (k_out + k_in) */
    int64_t h2d_bytes;         /* bytes the library copied host -> device since load */
    int64_t d2h_bytes;         /* bytes the library copied device -> host since load */
} SbpProfile;

/* Options of sbp_partition (src/sbp.cpp:61-98; include/args.hpp flags). */
typedef struct {
    int32_t algorithm;         /* SbpAlgorithm */
    int32_t batches;           /* --batches (default 10) */
    int32_t approximate;       /* --approximate: simple merge carry-out */
    int32_t asynciterations;   /* --asynciterations (async Gibbs rounds before MH) */
    uint64_t seed;             /* Philox key */
} SbpOptions;

/* Finetune call options. */
typedef struct {
    int32_t batches;               /* --batches */
    int32_t bracket_established;   /* BlockmodelTriplet::get(2) non-empty: early-stop threshold 1e-4 */
    int32_t max_sweeps;            /* <= 0: MAX_NUM_ITERATIONS (100) */
    uint32_t call;                 /* Philox counter word 2 */
    uint64_t seed;
} SbpFinetuneOptions;

/* Merge call options. */
typedef struct {
    int32_t approximate;       /* 1: Blockmodel::carry_out_best_merges, 0: advanced */
    uint32_t call;
    uint64_t seed;
} SbpMergeOptions;

/* Last error message of the calling thread (static storage). */
const char *sbp_last_error(void);

/* Number of usable CUDA devices (0 if none). */
int32_t sbp_device_count(void);

/* Engine options (no reference counterpart).  "dense_max_blocks": blockmodels with more blocks
 * than this keep their block matrix as row-hashed regions (a sparse device-resident matrix with
 * integer counts updated by atomics) instead of dense B x B arrays; default 131072 (dense storage
 * is faster wherever it fits).  "dense_max_memory_pct" (default 60, range 1-90): a dense matrix
 * that would take more than this percentage of the free device memory is row-hashed instead.
 * Both apply to blockmodels whose block count is set after the call.  "group_kernel" (default
 * 1): asynchronous-Gibbs and Metropolis-Hastings evaluation with a group of 8 lanes per vertex
 * on dense blockmodels of at most 128 blocks; 2: at every block count (vertices of degree up to
 * 128); 0: one warp per vertex everywhere (same results).  "hashed_row_factor" (default 4, range 2-64): a rebuilt hashed row gets room
 * for factor x its cells, at most 2 x for rows of more than 128 cells (larger: rows fill up and
 * are regrown less often; smaller: less memory and a cheaper walk of the row).  "graph_sweeps" (default 1): an
 * asynchronous-Gibbs finetune on dense storage runs as one CUDA graph launch whose sweep loop and
 * early stop are decided on the GPU; 0 drives every sweep from the host (same results).
 * "batched_wait_limit" (default 2^22, range 16-2^30): idle claim attempts (about 0.25 us each) of a
 * persistent CTA of sbp_partition_batched before its launch gives up and the call fails with
 * SBP_ERR_DEVICE.  "batched_stall_graph" (default -1): fault injection for failure-detection
 * tests -- the sweep queue of that graph of a batched launch starts with its first stage taken,
 * so no stage of it ever opens and the launch must end by its wait limit.  "batched_overlap"
 * (default 64, range 0-1024): while a sweep launch of sbp_partition_batched runs, the graphs
 * between two finetunes (merge, golden-section step, the next finetune's set-up) are processed
 * on a second stream, and the launch leaves this many CTA slots free for their kernels; 0 runs
 * them before the next launch instead (same results either way).  "batched_threads" (default 8,
 * range 1-64): host threads, each with its own stream and scratch, that run those steps for
 * several graphs at once; 1: the calling thread alone. */
SbpStatus sbp_set_option(const char *name, int64_t value);

/* The CUDA stream every call of this library runs on (cudaStream_t), for interop and timing.
 * No reference counterpart (the reference is CPU-only). */
SbpStatus sbp_get_stream(void **out);

/* Released device buffers stay cached for reuse (up to half the device's memory, at least 32 GB;
 * a new allocation that does not fit frees them first).  This frees them now, once the work that
 * used them has finished.  No reference counterpart. */
SbpStatus sbp_release_cached_memory(void);
/* Enable CUDA-event timing of the vertex-evaluation kernel launches (off by default), and read
 * the counters.  No reference counterpart. */
SbpStatus sbp_profile_enable(int32_t on);
SbpStatus sbp_profile_read(SbpProfile *out, int32_t reset);

/* Graph(out_neighbors, in_neighbors, ...) built from an edge list: duplicates are dropped
 * keeping the first occurrence (utils::insert_nodup, src/utils.cpp:52-60), self loops kept,
 * vertices split high/low by degree for the hybrid schedule (Graph::sort_vertices,
 * src/graph.cpp:215-228; ties by vertex id).  Replaces Graph::load_text (src/graph.cpp:123-140). */
SbpStatus sbp_graph_create(int32_t num_vertices, int64_t num_edges, const int32_t *src, const int32_t *dst,
                           SbpGraph **out);
SbpStatus sbp_graph_destroy(SbpGraph *graph);
/* Graph::num_edges (include/graph.hpp:106): unique directed edges. */
SbpStatus sbp_graph_num_edges(const SbpGraph *graph, int64_t *out);
/* Graph::high_degree_vertices / low_degree_vertices (include/graph.hpp:100-102). */
SbpStatus sbp_graph_get_split(const SbpGraph *graph, int32_t *num_high, int32_t *high, int32_t *low);
SbpStatus sbp_graph_set_split(SbpGraph *graph, int32_t num_high, const int32_t *high, int32_t num_low,
                              const int32_t *low);

/* Blockmodel(num_blocks, graph, 0.5, assignment) (include/blockmodel/blockmodel.hpp:70-76):
 * counts rebuilt on the device (Blockmodel::initialize_edge_counts, blockmodel.cpp:187-255). */
SbpStatus sbp_blockmodel_create(const SbpGraph *graph, int32_t num_blocks, const int32_t *assignment,
                                SbpBlockmodel **out);
/* Blockmodel::copy (src/blockmodel/blockmodel.cpp:95-105).  A blockmodel keeps a reference to
 * the graph it was created on; the graph must outlive it and its copies. */
SbpStatus sbp_blockmodel_copy(const SbpBlockmodel *src, SbpBlockmodel **out);
SbpStatus sbp_blockmodel_destroy(SbpBlockmodel *bm);
SbpStatus sbp_blockmodel_num_blocks(const SbpBlockmodel *bm, int32_t *out);
/* Blockmodel::setNum_blocks_to_merge (include/blockmodel/blockmodel.hpp:167). */
SbpStatus sbp_blockmodel_set_num_blocks_to_merge(SbpBlockmodel *bm, int32_t n);
/* Blockmodel::getOverall_entropy (float, include/blockmodel/blockmodel.hpp:164). */
SbpStatus sbp_blockmodel_overall_entropy(const SbpBlockmodel *bm, float *out);
/* Blockmodel::block_assignment (include/blockmodel/blockmodel.hpp:126). out: V ints. */
SbpStatus sbp_get_assignment(const SbpBlockmodel *bm, int32_t *out);
/* Dense dump of the block matrix (ISparseMatrix::get). out: B*B ints, row-major. */
SbpStatus sbp_get_block_matrix(const SbpBlockmodel *bm, int32_t *out);
/* Blockmodel::degrees_out / degrees_in / degrees. Each out: B ints. */
SbpStatus sbp_get_degrees(const SbpBlockmodel *bm, int32_t *d_out, int32_t *d_in, int32_t *d);

/* Blockmodel::degrees(std::vector<int>) (include/blockmodel/blockmodel.hpp:148): overwrite the
 * block degrees d (B ints), e.g. with the drifted values of a reference Blockmodel being mirrored. */
SbpStatus sbp_set_degrees(SbpBlockmodel *bm, const int32_t *d);

/* entropy::mdl(blockmodel, num_vertices, num_edges) (src/entropy.cpp:584-589) of block counts
 * given on the host as nonzero cells (rows[i], cols[i], counts[i]; ISparseMatrix::nonzero() and
 * values()) and block degrees (num_blocks ints each), with each term count * log(count /
 * (d_out[row] * d_in[col])) in FP64 (Blockmodel::log_posterior_probability,
 * src/blockmodel/blockmodel.cpp:267-285).  Needs no graph or blockmodel handle. */
SbpStatus sbp_mdl_of_cells(int32_t num_blocks, int64_t nnz, const int32_t *rows, const int32_t *cols,
                           const int32_t *counts, const int32_t *d_out, const int32_t *d_in, int32_t num_vertices,
                           int64_t num_edges, double *out);

/* entropy::mdl (src/entropy.cpp:584-589), FP64 logs. */
SbpStatus sbp_mdl(const SbpBlockmodel *bm, const SbpGraph *graph, double *out);

/* Evaluate vertices against the current (frozen) state without moving them: proposal,
 * Hastings correction, delta-MDL and the accept test for each vertex with the given records
 * (finetune::propose_gibbs_move_v2, src/finetune.cpp:531-545).  records: 4*n words.
 * Outputs (n each): proposed block, delta-MDL, Hastings, accepted flag. */
SbpStatus sbp_evaluate_vertices(const SbpBlockmodel *bm, const SbpGraph *graph, int32_t n, const int32_t *vertices,
                                const uint32_t *records, int32_t *proposal, double *delta_mdl, double *hastings,
                                int32_t *accepted);

/* Blockmodel::move_vertex(vertex, delta, proposal) (src/blockmodel/blockmodel.cpp:344-360):
 * move one vertex to `block`, updating counts and degrees as the reference does (d[r], d[s]
 * are set from the already-updated diagonal plus the diagonal delta). */
SbpStatus sbp_move_vertex(SbpBlockmodel *bm, const SbpGraph *graph, int32_t vertex, int32_t block);

/* finetune::metropolis_hastings / asynchronous_gibbs / hybrid_mcmc
 * (src/finetune.cpp:412-444, 31-89, 342-410).  `replay` may be NULL (Philox stream). */
SbpStatus sbp_finetune(SbpBlockmodel *bm, const SbpGraph *graph, int32_t algorithm, const SbpFinetuneOptions *opt,
                       const SbpReplay *replay, SbpStats *stats);

/* block_merge::merge_blocks (src/block_merge.cpp:278-311).  `replay` may be NULL.
 * best_merge / delta_mdl (B entries each, may be NULL) receive the per-block best proposal
 * and its delta-MDL before the merges are carried out. */
SbpStatus sbp_merge_blocks(SbpBlockmodel *bm, const SbpGraph *graph, const SbpMergeOptions *opt,
                           const SbpReplay *replay, int32_t *best_merge, double *delta_mdl, SbpStats *stats);

/* A recorded proposal stream: the proposed block and the accept uniform of every draw, as the
 * reference's own proposal and accept steps made them (common::propose_new_block,
 * src/common.cpp:131-182, and finetune::accept, src/finetune.cpp:19-29).  A finetune call reads
 * record t*V + v for the visit of vertex v in its sweep t; a merge call reads record block*10 + i
 * for proposal i of a block (NUM_AGG_PROPOSALS_PER_BLOCK = 10) and no uniforms.  A visit that
 * keeps its block has the current block as proposal; its uniform is not read. */
typedef struct {
    const int32_t *proposal;   /* records proposed blocks */
    const double *uniform;     /* records accept uniforms in [0, 1); NULL for a merge call */
    int64_t records;
} SbpMoveReplay;

/* finetune::metropolis_hastings / asynchronous_gibbs / hybrid_mcmc (src/finetune.cpp:412-444,
 * 31-89, 342-410) with the proposals and accept uniforms taken from `replay` instead of drawn:
 * the Hastings correction, delta-MDL, accept test and move are the engine's.  Fails with
 * SBP_ERR_REPLAY when a visit has no record or a proposal is out of range. */
SbpStatus sbp_finetune_replayed(SbpBlockmodel *bm, const SbpGraph *graph, int32_t algorithm,
                                const SbpFinetuneOptions *opt, const SbpMoveReplay *replay, SbpStats *stats);
/* block_merge::merge_blocks (src/block_merge.cpp:278-311) with every merge proposal taken from
 * `replay` (a proposal equal to its own block, or out of range, fails with SBP_ERR_REPLAY). */
SbpStatus sbp_merge_blocks_replayed(SbpBlockmodel *bm, const SbpGraph *graph, const SbpMergeOptions *opt,
                                    const SbpMoveReplay *replay, int32_t *best_merge, double *delta_mdl,
                                    SbpStats *stats);

/* One intermediate record of a partition (sbp::Intermediate, include/sbp.hpp:18-28, recorded by
 * sbp::add_intermediate, src/sbp.cpp:36-59): at the start (iteration 0, B = V), after the first
 * merge (0.5), after the k-th finetune (k) and for the result (-1). */
typedef struct {
    float iteration;
    int32_t num_blocks;
    double mdl;                  /* entropy::mdl; after a finetune the float overall entropy */
    double normalized_mdl_v1;    /* entropy::normalize_mdl_v1 / v2 (src/entropy.cpp:559-583) */
    double normalized_mdl_v2;
    double modularity;           /* Graph::modularity of the result (src/graph.cpp:142-163); -1 before */
    double interblock_edges;     /* Blockmodel::interblock_edges (src/blockmodel/blockmodel.cpp:257-261) */
    double block_size_variation; /* Blockmodel::block_size_variation (src/blockmodel/blockmodel.cpp:9-27) */
    int32_t mcmc_iterations;     /* finetune sweeps so far in this process (finetune::MCMC_iterations) */
    int32_t _pad;
    double mcmc_time;            /* device seconds of finetune so far in this process (finetune::MCMC_time) */
    int64_t visits;              /* vertex visits of this partition so far (no reference counterpart) */
    double seconds;              /* device seconds since this partition started (no reference counterpart) */
} SbpIntermediate;

/* sbp::get_intermediates (src/sbp.cpp:18-20): the records of every sbp_partition call of this
 * process so far (count receives their number; at most capacity are copied).  The batched,
 * learned and replayed partitions record none. */
SbpStatus sbp_get_intermediates(SbpIntermediate *out, int32_t capacity, int32_t *count);
SbpStatus sbp_clear_intermediates(void);

/* Quality of a partition against a known one (evaluate::Eval and the printed figures of
 * evaluate::calculate_f1_score / calculate_nmi, src/evaluate.cpp:7-96). */
typedef struct {
    double f1_score;          /* pair-counting F1 */
    double nmi;               /* normalised mutual information */
    double accuracy;          /* matched vertices of the best block <-> community matching, over V */
    double rand_index;
    double precision;         /* pairs together in both / pairs together in the true partition */
    double recall;            /* pairs together in both / pairs together in the algorithm's */
    double true_mdl;          /* entropy::mdl of the true partition (NaN when some labels are unknown) */
    int64_t counted_vertices; /* vertices with a known true community */
    int32_t num_blocks;       /* rows of the table: algorithm blocks */
    int32_t true_num_blocks;  /* columns: true communities */
} SbpEvaluation;

/* calculate_f1_score and calculate_nmi (src/evaluate.cpp:7-96) of a contingency table given on the
 * host (nrows x ncols, row-major; rows = algorithm blocks, columns = true communities) over
 * num_vertices vertices, plus the accuracy of the best one-to-one matching (the reference's
 * Hungarian step, src/evaluate.cpp:114-178).  Host arithmetic only; needs no device.  Pair
 * counts are 64-bit (the reference's int products wrap above 46340 in the Rand index). */
SbpStatus sbp_contingency_metrics(int32_t nrows, int32_t ncols, const int64_t *table, int64_t num_vertices,
                                  SbpEvaluation *out);
/* evaluate::evaluate_blockmodel (src/evaluate.cpp:98-112): the contingency table of the
 * blockmodel's assignment against true_assignment (V ints; community ids numbered in order of
 * first appearance as evaluate::hungarian does; -1 = unknown, not counted) is counted on the
 * device, then the metrics above and the true partition's MDL.  table_out (optional,
 * B x K int64, columns in first-appearance order) receives the table. */
SbpStatus sbp_evaluate_blockmodel(const SbpBlockmodel *bm, const SbpGraph *graph, const int32_t *true_assignment,
                                  SbpEvaluation *out, int64_t *table_out);

/* sbp::stochastic_block_partition (src/sbp.cpp:61-98) driven by recorded streams: calls[k] is
 * the stream of the partition's k-th merge or finetune call (merge, finetune, merge, ... in the
 * order the loop makes them), read as by sbp_merge_blocks_replayed / sbp_finetune_replayed.
 * max_sweeps caps every finetune call (<= 0: 100, MAX_NUM_ITERATIONS).  block_counts (num_calls
 * ints, may be NULL) receives the number of blocks after each call and calls_made (may be NULL)
 * the number of calls made; SBP_ERR_REPLAY if the partition needs more calls than given. */
SbpStatus sbp_partition_replayed(const SbpGraph *graph, const SbpOptions *opt, int32_t max_sweeps, int32_t num_calls,
                                 const SbpMoveReplay *calls, int32_t *out_assignment, int32_t *block_counts,
                                 int32_t *calls_made, SbpStats *stats);

/* sbp::stochastic_block_partition (src/sbp.cpp:61-98): golden-section search over B with
 * merge + finetune rounds.  out_assignment: V ints. */
SbpStatus sbp_partition(const SbpGraph *graph, const SbpOptions *opt, int32_t *out_assignment, SbpStats *stats);

/* MDL of block counts that are already on the device, E h(B^2/E) + V log B - sum_cells M log M
 * + sum_blocks (d_out log d_out + d_in log d_in) with h(x) = (1+x) log(1+x) - x log x and FP64
 * log terms, for callers that cannot allocate GPU memory: code running under a device-memory budget fixed
 * at start-up, or code that must not call cudaMalloc/cudaFree because those synchronize the
 * whole device while it has work in flight.  No counterpart in the reference (a CPU-only code
 * base).  It allocates nothing: the caller passes the inputs and the output, and the only
 * scratch is a static device array of one double per block row, held by every GPU that loads
 * this library until the process exits.
 *   d_matrix: num_blocks rows of counts, row stride `ld` ints (ld >= num_blocks), on the device;
 *   d_degrees_out / d_degrees_in: num_blocks ints each, on the device;
 *   d_result: one double on the device; `stream`: a cudaStream_t (NULL = legacy default stream).
 * Limit: num_blocks <= 32768 (SBP_ERR_UNSUPPORTED above it).  The work is queued on `stream`;
 * the result is ready when the stream reaches it.  Calls share the scratch array, so calls
 * that overlap on the GPU race and must be serialised.  The first call on a device looks up
 * the scratch array's address on that device; make it before any stream capture. */
SbpStatus sbp_mdl_device_noalloc(const int32_t *d_matrix, int32_t num_blocks, int64_t ld, const int32_t *d_degrees_out,
                                 const int32_t *d_degrees_in, int32_t num_vertices, int64_t num_edges,
                                 double *d_result, void *stream);

/* ------------------------------------------------------------------------------------------
 * Learned proposal (no counterpart in the reference).  A network maps 64 features of a vertex
 * and its 14 candidate neighbour blocks to 15 logits (14 candidates + "uniformly random
 * block"); the draw mixes them with weight (1 - epsilon) with a uniform block (epsilon), and the
 * Hastings factor q(r | state after the move) / q(s | state) is computed exactly from the same
 * network, so the MCMC keeps the plain method's stationary distribution.  Network: 64 -> 128
 * -> 128 -> 16 with ReLU, BF16 weights and activations, FP32 accumulation on the tensor cores.
 * ------------------------------------------------------------------------------------------ */
typedef struct SbpMlp SbpMlp;           /* network weights and optimiser state (device) */
typedef struct SbpDataset SbpDataset;   /* training samples (device) */

#define SBP_MLP_FEATURES 64
#define SBP_MLP_OUTPUTS 16
#define SBP_MLP_SLOTS 14
#define SBP_MLP_ESCAPE 14
/* parameter vector: W1[128][64], b1[128], W2[128][128], b2[128], W3[16][128], b3[16] */
#define SBP_MLP_PARAMS 26896

typedef struct {
    int32_t epochs;
    int32_t batch;             /* rows per Adam step */
    float lr;
    int32_t _pad;
    uint64_t seed;             /* shuffling */
} SbpTrainOptions;

typedef struct {
    int64_t steps;
    double first_loss;         /* mean cross-entropy of the first epoch */
    double last_loss;          /* of the last epoch */
    double seconds;
} SbpTrainStats;

typedef struct {
    float epsilon;             /* uniform weight of the proposal mixture, (0, 1] */
    float fallback_acceptance; /* a learned sweep accepting less than this fraction of its visits
                                  switches the rest of the call to the plain proposal */
    int32_t stop_rule;         /* 0: early stop of sbp_finetune for the algorithm; 1: per-sweep MDL
                                  changes (the metropolis_hastings rule) */
    int32_t _pad;
} SbpLearnedOptions;

typedef struct {               /* MDL after every sweep (caller-owned arrays of `capacity`) */
    int32_t capacity;
    int32_t count;
    double *seconds;           /* host wall time since the call started, stream synchronised */
    double *mdl;
} SbpTrace;

SbpStatus sbp_mlp_create(uint64_t seed, SbpMlp **out);
SbpStatus sbp_mlp_destroy(SbpMlp *mlp);
SbpStatus sbp_mlp_get_params(const SbpMlp *mlp, float *params);
SbpStatus sbp_mlp_set_params(SbpMlp *mlp, const float *params);   /* also resets the optimiser */
/* logits[n][16] of features[n][64] (host buffers; features are rounded to BF16). */
SbpStatus sbp_mlp_forward(const SbpMlp *mlp, int64_t n, const float *features, float *logits);
/* Gradient of the mean masked cross-entropy over the rows with target >= 0 (targets: a
 * candidate slot < nvalid, or 14 = escape; -1 = row ignored).  Slots >= nvalid and logit 15
 * are masked.  grads[SBP_MLP_PARAMS] in parameter-vector order. */
SbpStatus sbp_mlp_gradients(const SbpMlp *mlp, int64_t n, const float *features, const int32_t *target,
                            const int32_t *nvalid, float *grads, double *mean_loss);
/* Adam on the samples of `data` (shuffled each epoch). */
SbpStatus sbp_mlp_train(SbpMlp *mlp, const SbpDataset *data, const SbpTrainOptions *opt, SbpTrainStats *stats);

SbpStatus sbp_dataset_create(int64_t capacity, SbpDataset **out);
SbpStatus sbp_dataset_destroy(SbpDataset *data);
SbpStatus sbp_dataset_size(const SbpDataset *data, int64_t *out);
SbpStatus sbp_dataset_append(SbpDataset *data, int64_t n, const float *features, const int32_t *target,
                             const int32_t *nvalid);
SbpStatus sbp_dataset_read(const SbpDataset *data, int64_t offset, int64_t n, uint16_t *features_bf16,
                           int32_t *target, int32_t *nvalid);

/* Features of vertices against the blockmodel: features[n][64] (BF16 values), the candidate
 * blocks slots[n][14] (-1 past nvalid) and nvalid[n]. */
SbpStatus sbp_vertex_features(const SbpBlockmodel *bm, const SbpGraph *g, int32_t n, const int32_t *vertices,
                              float *features, int32_t *slots, int32_t *nvalid);
/* One learned-proposal evaluation of distinct vertices against the frozen blockmodel with
 * caller records (4 words per vertex: x_choice, x_uniform_block, u_hi, u_lo): proposal[n],
 * q_forward[n] (0 when the proposal is the current block), delta_mdl[n], hastings[n],
 * accepted[n].  The blockmodel is not changed. */
SbpStatus sbp_learned_evaluate(const SbpBlockmodel *bm, const SbpGraph *g, const SbpMlp *mlp, int32_t n,
                               const int32_t *vertices, const uint32_t *records, float epsilon, int32_t *proposal,
                               double *q_forward, double *delta_mdl, double *hastings, int32_t *accepted);
/* q(block | vertex, blockmodel) of the learned proposal for given (vertex, block) pairs. */
SbpStatus sbp_learned_q(const SbpBlockmodel *bm, const SbpGraph *g, const SbpMlp *mlp, int32_t n, const int32_t *vertices,
                        const int32_t *blocks, float epsilon, double *q);
/* Plain asynchronous-Gibbs sweeps (opt->max_sweeps of them) that append the features and chosen
 * candidate slot of every accepted move to `data` (samples past its capacity are dropped). */
SbpStatus sbp_collect_moves(SbpBlockmodel *bm, const SbpGraph *g, SbpDataset *data, const SbpFinetuneOptions *opt,
                            SbpStats *stats);
/* finetune::{metropolis_hastings, asynchronous_gibbs, hybrid_mcmc} (src/finetune.cpp:412-444,
 * 31-89, 342-410) with the learned proposal (mlp != NULL) in place of common::propose_new_block
 * (src/common.cpp:131-182) or with the plain one (mlp == NULL), same sweeps as sbp_finetune.
 * Metropolis-Hastings (and the hybrid's high-degree pass) keeps the sequential chain exactly: each
 * visit is proposed, corrected and accepted against the state left by every earlier visit.
 * Early stop: Metropolis-Hastings its own rule (each sweep's summed accepted delta-MDL); the
 * others per lopt->stop_rule.  Optional per-sweep MDL trace. */
SbpStatus sbp_finetune_learned(SbpBlockmodel *bm, const SbpGraph *g, int32_t algorithm, const SbpFinetuneOptions *opt,
                               const SbpMlp *mlp, const SbpLearnedOptions *lopt, SbpTrace *trace, SbpStats *stats);
/* sbp_partition with the learned proposal in every finetune, Metropolis-Hastings included
 * (mlp == NULL: the plain proposal, with lopt->stop_rule). */
SbpStatus sbp_partition_learned(const SbpGraph *g, const SbpOptions *opt, const SbpMlp *mlp,
                                const SbpLearnedOptions *lopt, int32_t *out_assignment, SbpStats *stats);

/* ------------------------------------------------------------------------------------------
 * Batched partitioning (no counterpart in the reference, which partitions one graph per run):
 * n graphs of uneven sizes, each partitioned exactly as by sbp_partition (same options, same
 * result), with the asynchronous-Gibbs finetune of all graphs in one persistent kernel launch
 * per sweep (per-graph work queues, replayed as a CUDA graph) and work-item shapes chosen by
 * an autotuner that times candidates on the first sweeps of a workload.
 * ------------------------------------------------------------------------------------------ */
typedef struct {
    int32_t rounds;             /* lockstep rounds (merge + finetune of every unfinished graph) */
    int32_t batched_finetunes;  /* finetune calls run by the persistent kernel */
    int32_t fallback_finetunes; /* finetune calls run by the single-graph path (row-hashed storage,
                                   Metropolis-Hastings or hybrid rounds, very large degrees) */
    int32_t sweep_launches;     /* persistent-kernel launches (one per sweep of a round) */
    int32_t chunk;              /* light vertices per evaluation work item (autotuned) */
    int32_t ctas_per_sm;        /* persistent CTAs per SM (autotuned) */
    int32_t tuned;              /* 1: this call ran the autotuner; 0: it used an earlier choice */
    int32_t candidates;         /* candidates timed */
    double candidate_ms[8];     /* their sweep times, per graph swept */
    double sweep_seconds;       /* device time of the persistent sweep launches */
    double seconds;             /* device-clock time of the whole call */
    double overlapped_seconds;  /* host time of the steps between finetunes (merges and the rest)
                                   that ran beside a sweep launch */
    double serial_seconds;      /* host time of those steps while no sweep launch ran */
} SbpBatchInfo;

/* graphs[n] -> out_assignments[i][V_i]; stats[i] per graph (optional; total_seconds is the
 * batch's time); info optional.  The graphs must not be used by another call meanwhile. */
SbpStatus sbp_partition_batched(int32_t n, const SbpGraph *const *graphs, const SbpOptions *opt,
                                int32_t *const *out_assignments, SbpStats *stats, SbpBatchInfo *info);
/* Forget the autotuner's choices (the next batched call tunes again). */
SbpStatus sbp_batched_reset_tuning(void);

#ifdef __cplusplus
}
#endif

#endif /* SBP_B200_H */
