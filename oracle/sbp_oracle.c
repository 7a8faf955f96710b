/*
 * sbp_oracle.c -- CPU restatement of the reference's stochastic block partitioning hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA engine.  Only the
 * test-suite, the smoke check and the CPU-baseline leg of the benchmark may load it; the
 * product library never links or calls it.
 *
 * It restates, function by function, the reference (vtsynergy/Hybrid-Stochastic-Block-
 * Partitioning) in plain C with every log term in FP64 (the reference uses FP32 logf in
 * common::cell_entropy and utils::nat_log; the product contract is FP64).  Every quirk of the
 * reference that changes integer state or accept decisions is kept on purpose:
 *
 *   Q1  delta_mdl double-counts a cell that is present in the Delta with a net change of 0
 *       and non-zero in the matrix (src/entropy.cpp:344-371, the `delta.get(row,col) != 0`
 *       test); only cells (r,s) and (s,r) can be in that state.
 *   Q2  Blockmodel::move_vertex sets d[r], d[s] from the *updated* matrix plus the delta
 *       again (src/blockmodel/blockmodel.cpp:348-351), so d drifts from d_out+d_in-M[x,x].
 *   Q3  hastings_correction's new degree of r/s ignores the self edge on the in side
 *       (src/entropy.cpp:539-546).
 *   Q4  asynchronous_gibbs / hybrid_mcmc never update last_iteration_entropy, so the early
 *       stop compares cumulative entropy change (src/finetune.cpp:40,74,351,395).
 *   Q5  the Gibbs batch loop bound V/batch_size skips a tail (src/finetune.cpp:44-47).
 *
 * Two deliberate, documented departures from the reference (shared with the CUDA engine):
 *   D1  random numbers come from Philox4x32-10 keyed by (seed) with counter
 *       (vertex, sweep, call, 0) for a finetune visit and (block, proposal, call, 1) for a
 *       merge proposal, or from a host-supplied replay buffer of the same 4-word records,
 *       instead of per-translation-unit std::default_random_engine objects.  A replay buffer
 *       may instead hold a recorded proposal stream (moves mode): records (s, 0, u_hi, u_lo)
 *       with the proposed block of every visit or merge proposal and the bits of its accept
 *       uniform, as the patched reference logs them;
 *   D2  the multinomial over M[t,:]+M[:,t] (src/common.cpp:159-180) walks row t ascending
 *       and then column t ascending (a canonical order; the reference walks robin_map
 *       buckets), and the dead `std::rand() <= B/(d_t+B)` branch (src/common.cpp:154, true
 *       only when rand() returns 0) is not taken.
 *   D3  a vertex-move delta-MDL whose magnitude is at most 2^-40 * T * log(max(E,2)) is set to
 *       exactly 0, T being the integer sum of old + new counts of the changed cells and of the
 *       old + new out/in degrees of r and s.  A mathematically zero change (a symmetric move)
 *       then reads as 0.0 whatever the summation order, which keeps the Metropolis-Hastings
 *       early stop (`delta == 0.0`, src/finetune.cpp:147) identical across implementations.
 *   Sorts that the reference does with std::sort (unstable) break ties by index.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define SBPO_MAX_ITERATIONS 100          /* include/finetune.hpp:56 */
#define SBPO_PROPOSALS_PER_BLOCK 10      /* include/block_merge.hpp:24 */
#define SBPO_REDUCTION_RATE 0.5          /* include/blockmodel/blockmodel.hpp:26 */

/* ------------------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).                                      */
/* ------------------------------------------------------------------------------------- */
void sbpo_philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct {
    uint64_t seed;
    const uint32_t *replay;   /* optional: 4 words per record */
    int64_t replay_records;
    int moves;                /* 1: replay records are recorded proposals (s, 0, u_hi, u_lo) */
} SbpoRng;

/* Draw the 4-word record for (a, b, call, tag). Replay records are indexed by `slot`. */
static int sbpo_draw(const SbpoRng *rng, uint32_t a, uint32_t b, uint32_t call, uint32_t tag,
                     int64_t slot, uint32_t out[4]) {
    if (rng->replay) {
        if (slot < 0 || slot >= rng->replay_records) return -1;
        memcpy(out, rng->replay + 4 * slot, 4 * sizeof(uint32_t));
        return 0;
    }
    uint32_t ctr[4] = {a, b, call, tag};
    uint32_t key[2] = {(uint32_t)rng->seed, (uint32_t)(rng->seed >> 32)};
    sbpo_philox(ctr, key, out);
    return 0;
}

double sbpo_u53(uint32_t hi, uint32_t lo) {
    uint64_t m = ((uint64_t)hi << 21) | (uint64_t)(lo >> 11);
    return (double)m * (1.0 / 9007199254740992.0);
}

static inline int64_t sbpo_scale(uint32_t x, int64_t n) { return (int64_t)(((uint64_t)x * (uint64_t)n) >> 32); }

/* The accept uniform of a recorded proposal: the double whose bits are (u_hi, u_lo). */
static double record_uniform(const uint32_t x[4]) {
    uint64_t bits = ((uint64_t)x[2] << 32) | (uint64_t)x[3];
    double u;
    memcpy(&u, &bits, sizeof u);
    return u;
}

/* ------------------------------------------------------------------------------------- */
/* Graph (include/graph.hpp:15-113, src/graph.cpp:165-228, src/utils.cpp:52-60)            */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    int V, E;
    int *out_ptr, *out_idx;   /* out-neighbours incl. self loops, first-occurrence order */
    int *in_ptr, *in_idx;     /* in-neighbours incl. self loops (Graph::in_neighbors) */
    unsigned char *self;
    int nhigh, nlow;
    int *high, *low;          /* hybrid split (Graph::sort_vertices) */
} SbpoGraph;

typedef struct { int v, deg; } VD;
static int vd_cmp(const void *a, const void *b) {
    const VD *x = (const VD *)a, *y = (const VD *)b;
    if (x->deg != y->deg) return (x->deg > y->deg) ? -1 : 1;
    return (x->v < y->v) ? -1 : (x->v > y->v);
}

/* Graph::sort_vertices with ties broken by vertex id (std::sort's tie order is unspecified). */
static void sbpo_graph_split(SbpoGraph *g) {
    VD *vd = (VD *)malloc(sizeof(VD) * (size_t)(g->V > 0 ? g->V : 1));
    for (int v = 0; v < g->V; ++v) {
        int deg = (g->out_ptr[v + 1] - g->out_ptr[v]) + (g->in_ptr[v + 1] - g->in_ptr[v]) - g->self[v];
        vd[v].v = v; vd[v].deg = deg;
    }
    qsort(vd, (size_t)g->V, sizeof(VD), vd_cmp);
    free(g->high); free(g->low);
    g->high = (int *)malloc(sizeof(int) * (size_t)(g->V + 1));
    g->low = (int *)malloc(sizeof(int) * (size_t)(g->V + 1));
    g->nhigh = g->nlow = 0;
    for (int i = 0; i < g->V; ++i) {
        if ((double)i < 0.15 * (double)g->V) g->high[g->nhigh++] = vd[i].v;
        else g->low[g->nlow++] = vd[i].v;
    }
    free(vd);
}

SbpoGraph *sbpo_graph_create(int V, int64_t n, const int *src, const int *dst) {
    for (int64_t i = 0; i < n; ++i)
        if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V) return NULL;
    /* de-duplicate keeping the first occurrence (utils::insert_nodup) */
    uint64_t cap = 16;
    while (cap < (uint64_t)(2 * n + 16)) cap <<= 1;
    uint64_t *table = (uint64_t *)malloc(sizeof(uint64_t) * cap);
    memset(table, 0xff, sizeof(uint64_t) * cap);
    int *keep_s = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    int *keep_d = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        uint64_t key = (uint64_t)(uint32_t)src[i] * (uint64_t)V + (uint64_t)(uint32_t)dst[i];
        uint64_t h = (key * 0x9E3779B97F4A7C15ull) & (cap - 1);
        int dup = 0;
        while (table[h] != ~0ull) {
            if (table[h] == key) { dup = 1; break; }
            h = (h + 1) & (cap - 1);
        }
        if (dup) continue;
        table[h] = key;
        keep_s[m] = src[i]; keep_d[m] = dst[i]; ++m;
    }
    free(table);
    SbpoGraph *g = (SbpoGraph *)calloc(1, sizeof(SbpoGraph));
    g->V = V; g->E = (int)m;
    g->out_ptr = (int *)calloc((size_t)V + 1, sizeof(int));
    g->in_ptr = (int *)calloc((size_t)V + 1, sizeof(int));
    g->out_idx = (int *)malloc(sizeof(int) * (size_t)(m + 1));
    g->in_idx = (int *)malloc(sizeof(int) * (size_t)(m + 1));
    g->self = (unsigned char *)calloc((size_t)V + 1, 1);
    for (int64_t i = 0; i < m; ++i) { g->out_ptr[keep_s[i] + 1]++; g->in_ptr[keep_d[i] + 1]++; }
    for (int v = 0; v < V; ++v) { g->out_ptr[v + 1] += g->out_ptr[v]; g->in_ptr[v + 1] += g->in_ptr[v]; }
    int *fo = (int *)malloc(sizeof(int) * (size_t)(V + 1));
    int *fi = (int *)malloc(sizeof(int) * (size_t)(V + 1));
    memcpy(fo, g->out_ptr, sizeof(int) * (size_t)V);
    memcpy(fi, g->in_ptr, sizeof(int) * (size_t)V);
    for (int64_t i = 0; i < m; ++i) {
        g->out_idx[fo[keep_s[i]]++] = keep_d[i];
        g->in_idx[fi[keep_d[i]]++] = keep_s[i];
        if (keep_s[i] == keep_d[i]) g->self[keep_s[i]] = 1;
    }
    free(fo); free(fi); free(keep_s); free(keep_d);
    sbpo_graph_split(g);
    return g;
}

void sbpo_graph_destroy(SbpoGraph *g) {
    if (!g) return;
    free(g->out_ptr); free(g->out_idx); free(g->in_ptr); free(g->in_idx); free(g->self);
    free(g->high); free(g->low); free(g);
}

int sbpo_graph_num_edges(const SbpoGraph *g) { return g->E; }
int sbpo_graph_num_high(const SbpoGraph *g) { return g->nhigh; }
void sbpo_graph_get_split(const SbpoGraph *g, int *high, int *low) {
    memcpy(high, g->high, sizeof(int) * (size_t)g->nhigh);
    memcpy(low, g->low, sizeof(int) * (size_t)g->nlow);
}
/* Replace the hybrid split (e.g. with the order the reference's std::sort produced). */
int sbpo_graph_set_split(SbpoGraph *g, int nhigh, const int *high, int nlow, const int *low) {
    if (nhigh + nlow != g->V) return -1;
    memcpy(g->high, high, sizeof(int) * (size_t)nhigh);
    memcpy(g->low, low, sizeof(int) * (size_t)nlow);
    g->nhigh = nhigh; g->nlow = nlow;
    return 0;
}

/* ------------------------------------------------------------------------------------- */
/* Blockmodel (include/blockmodel/blockmodel.hpp:45-184), dense B x B counts                */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    int B, V;
    int *b;
    int *M;              /* row-major B*B */
    int *d_out, *d_in, *d;
    float overall_entropy;
    int num_blocks_to_merge;
    int empty;
} SbpoBM;

#define MAT(bm, i, j) ((bm)->M[(size_t)(i) * (size_t)(bm)->B + (size_t)(j)])

/* Blockmodel::initialize_edge_counts (src/blockmodel/blockmodel.cpp:187-255). */
void sbpo_bm_rebuild(SbpoBM *bm, const SbpoGraph *g) {
    size_t BB = (size_t)bm->B * (size_t)bm->B;
    free(bm->M); free(bm->d_out); free(bm->d_in); free(bm->d);
    bm->M = (int *)calloc(BB ? BB : 1, sizeof(int));
    bm->d_out = (int *)calloc((size_t)bm->B + 1, sizeof(int));
    bm->d_in = (int *)calloc((size_t)bm->B + 1, sizeof(int));
    bm->d = (int *)calloc((size_t)bm->B + 1, sizeof(int));
    for (int v = 0; v < g->V; ++v) {
        int blk = bm->b[v];
        for (int e = g->out_ptr[v]; e < g->out_ptr[v + 1]; ++e) {
            int nb = bm->b[g->out_idx[e]];
            MAT(bm, blk, nb) += 1;
            bm->d_out[blk] += 1;
            bm->d[blk] += 1;
        }
        for (int e = g->in_ptr[v]; e < g->in_ptr[v + 1]; ++e) {
            int nb = bm->b[g->in_idx[e]];
            bm->d_in[blk] += 1;
            if (blk != nb) bm->d[blk] += 1;
        }
    }
}

SbpoBM *sbpo_bm_create(const SbpoGraph *g, int B, const int *assignment) {
    SbpoBM *bm = (SbpoBM *)calloc(1, sizeof(SbpoBM));
    bm->B = B; bm->V = g->V;
    bm->b = (int *)malloc(sizeof(int) * (size_t)(g->V + 1));
    for (int v = 0; v < g->V; ++v) {
        if (assignment[v] < 0 || assignment[v] >= B) { free(bm->b); free(bm); return NULL; }
        bm->b[v] = assignment[v];
    }
    bm->overall_entropy = 3.40282347e+38f;   /* std::numeric_limits<float>::max() */
    bm->num_blocks_to_merge = (int)(B * (float)SBPO_REDUCTION_RATE);
    sbpo_bm_rebuild(bm, g);
    return bm;
}

SbpoBM *sbpo_bm_copy(const SbpoBM *src) {   /* Blockmodel::copy (blockmodel.cpp:95-105) */
    SbpoBM *bm = (SbpoBM *)calloc(1, sizeof(SbpoBM));
    *bm = *src;
    size_t BB = (size_t)src->B * (size_t)src->B;
    bm->b = (int *)malloc(sizeof(int) * (size_t)(src->V + 1));
    memcpy(bm->b, src->b, sizeof(int) * (size_t)src->V);
    bm->M = (int *)malloc(sizeof(int) * (BB ? BB : 1));
    memcpy(bm->M, src->M, sizeof(int) * BB);
    bm->d_out = (int *)malloc(sizeof(int) * (size_t)(src->B + 1));
    bm->d_in = (int *)malloc(sizeof(int) * (size_t)(src->B + 1));
    bm->d = (int *)malloc(sizeof(int) * (size_t)(src->B + 1));
    memcpy(bm->d_out, src->d_out, sizeof(int) * (size_t)src->B);
    memcpy(bm->d_in, src->d_in, sizeof(int) * (size_t)src->B);
    memcpy(bm->d, src->d, sizeof(int) * (size_t)src->B);
    bm->num_blocks_to_merge = 0;
    return bm;
}

void sbpo_bm_destroy(SbpoBM *bm) {
    if (!bm) return;
    free(bm->b); free(bm->M); free(bm->d_out); free(bm->d_in); free(bm->d); free(bm);
}

int sbpo_bm_num_blocks(const SbpoBM *bm) { return bm->B; }
void sbpo_bm_get_assignment(const SbpoBM *bm, int *out) { memcpy(out, bm->b, sizeof(int) * (size_t)bm->V); }
void sbpo_bm_get_matrix(const SbpoBM *bm, int *out) { memcpy(out, bm->M, sizeof(int) * (size_t)bm->B * (size_t)bm->B); }
void sbpo_bm_get_degrees(const SbpoBM *bm, int *d_out, int *d_in, int *d) {
    memcpy(d_out, bm->d_out, sizeof(int) * (size_t)bm->B);
    memcpy(d_in, bm->d_in, sizeof(int) * (size_t)bm->B);
    memcpy(d, bm->d, sizeof(int) * (size_t)bm->B);
}
float sbpo_bm_overall_entropy(const SbpoBM *bm) { return bm->overall_entropy; }

/* ------------------------------------------------------------------------------------- */
/* Entropy                                                                                */
/* ------------------------------------------------------------------------------------- */
/* common::cell_entropy (include/common.hpp:35-44), FP64. */
static inline double cell_entropy(double value, double d_in, double d_out) {
    if (value == 0.0) return 0.0;
    return value * log(value / (d_in * d_out));
}

/* entropy::mdl (src/entropy.cpp:584-589) + Blockmodel::log_posterior_probability (blockmodel.cpp:267-285). */
double sbpo_mdl(const SbpoBM *bm, int V, int E) {
    double lp = 0.0;
    for (int i = 0; i < bm->B; ++i)
        for (int j = 0; j < bm->B; ++j) {
            int m = MAT(bm, i, j);
            if (m == 0) continue;
            double val = (double)m;
            lp += val * log(val / ((double)bm->d_out[i] * (double)bm->d_in[j]));
        }
    double x = pow((double)bm->B, 2) / (double)E;
    double h = ((1 + x) * log(1 + x)) - (x * log(x));
    return ((double)E * h) + ((double)V * log((double)bm->B)) - lp;
}

double sbpo_null_mdl_v1(long E) {     /* src/entropy.cpp:567-573 */
    double lp = E * log(1.0 / E);
    double x = 1.0 / E;
    double h = ((1 + x) * log(1 + x)) - (x * log(x));
    return (E * h) - lp;
}

double sbpo_null_mdl_v2(long V, long E) {   /* src/entropy.cpp:575-582 */
    double lp = E * log(1.0 / E);
    double x = pow((double)V, 2) / E;
    double h = ((1 + x) * log(1 + x)) - (x * log(x));
    return (E * h) + (V * log((double)V)) - lp;
}

/* ------------------------------------------------------------------------------------- */
/* Delta (include/blockmodel/sparse/delta.hpp:22-149), dense maps with presence flags      */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    int r, s, B, self_w;
    int *val[4];                  /* 0 current row, 1 proposed row, 2 current col, 3 proposed col */
    unsigned char *has[4];
    int *keys[4]; int nkeys[4];   /* insertion order of keys (for entries()) */
} Delta;

static void delta_init(Delta *dl, int r, int s, int B) {
    dl->r = r; dl->s = s; dl->B = B; dl->self_w = 0;
    for (int k = 0; k < 4; ++k) {
        dl->val[k] = (int *)calloc((size_t)B + 1, sizeof(int));
        dl->has[k] = (unsigned char *)calloc((size_t)B + 1, 1);
        dl->keys[k] = (int *)malloc(sizeof(int) * ((size_t)B + 1));
        dl->nkeys[k] = 0;
    }
}
static void delta_free(Delta *dl) {
    for (int k = 0; k < 4; ++k) { free(dl->val[k]); free(dl->has[k]); free(dl->keys[k]); }
}
static int delta_route(const Delta *dl, int row, int col, int *key) {
    if (row == dl->r) { *key = col; return 0; }
    if (row == dl->s) { *key = col; return 1; }
    if (col == dl->r) { *key = row; return 2; }
    if (col == dl->s) { *key = row; return 3; }
    return -1;
}
static void delta_add(Delta *dl, int row, int col, int value) {
    int key, m = delta_route(dl, row, col, &key);
    if (m < 0) { fprintf(stderr, "oracle: delta cell outside rows/cols r,s\n"); abort(); }
    if (!dl->has[m][key]) { dl->has[m][key] = 1; dl->keys[m][dl->nkeys[m]++] = key; }
    dl->val[m][key] += value;
}
static int delta_get(const Delta *dl, int row, int col) {
    int key, m = delta_route(dl, row, col, &key);
    if (m < 0) { fprintf(stderr, "oracle: delta get outside rows/cols r,s\n"); abort(); }
    return dl->has[m][key] ? dl->val[m][key] : 0;
}
static void delta_entry(const Delta *dl, int m, int i, int *row, int *col, int *change) {
    int key = dl->keys[m][i];
    *change = dl->val[m][key];
    switch (m) {
        case 0: *row = dl->r; *col = key; break;
        case 1: *row = dl->s; *col = key; break;
        case 2: *row = key; *col = dl->r; break;
        default: *row = key; *col = dl->s; break;
    }
}

/* finetune::blockmodel_delta (src/finetune.cpp:108-142); in-edges exclude the self loop. */
static void vertex_delta(Delta *dl, const SbpoBM *bm, const SbpoGraph *g, int v, int r, int s) {
    delta_init(dl, r, s, bm->B);
    for (int e = g->out_ptr[v]; e < g->out_ptr[v + 1]; ++e) {
        int u = g->out_idx[e], bu = bm->b[u];
        if (u == v) { delta_add(dl, s, s, 1); dl->self_w = 1; }
        else delta_add(dl, s, bu, 1);
        delta_add(dl, r, bu, -1);
    }
    for (int e = g->in_ptr[v]; e < g->in_ptr[v + 1]; ++e) {
        int u = g->in_idx[e];
        if (u == v) continue;
        int bu = bm->b[u];
        delta_add(dl, bu, s, 1);
        delta_add(dl, bu, r, -1);
    }
}

typedef struct { int s, k_out, k_in, k; } Proposal;   /* utils::ProposalAndEdgeCounts */

/* entropy::delta_mdl(Blockmodel, Delta, Proposal) (src/entropy.cpp:296-401), FP64, with Q1. */
static double delta_mdl_move(const SbpoBM *bm, const Delta *dl, const Proposal *p, int E) {
    int r = dl->r, s = dl->s, B = bm->B;
    int64_t T = 0;   /* D3 scale */
    int din_shift = p->k_in + dl->self_w, dout_shift = p->k_out;
#define DIN_NEW(i) ((double)(bm->d_in[i] + ((i) == r ? -din_shift : ((i) == s ? din_shift : 0))))
#define DOUT_NEW(i) ((double)(bm->d_out[i] + ((i) == r ? -dout_shift : ((i) == s ? dout_shift : 0))))
    double dS = 0.0;
    for (int m = 0; m < 4; ++m)
        for (int i = 0; i < dl->nkeys[m]; ++i) {
            int row, col, change;
            delta_entry(dl, m, i, &row, &col, &change);
            double val = (double)MAT(bm, row, col);
            dS += cell_entropy(val, (double)bm->d_in[col], (double)bm->d_out[row]);
            dS -= cell_entropy(val + change, DIN_NEW(col), DOUT_NEW(row));
            if (change != 0) T += 2 * (int64_t)MAT(bm, row, col) + change;
        }
    T += 2 * ((int64_t)bm->d_out[r] + bm->d_out[s] + bm->d_in[r] + bm->d_in[s]);
    for (int pass = 0; pass < 2; ++pass) {           /* rows r and s */
        int row = pass == 0 ? r : s;
        for (int col = 0; col < B; ++col) {
            int val = MAT(bm, row, col);
            if (val == 0 || delta_get(dl, row, col) != 0) continue;
            dS += cell_entropy(val, (double)bm->d_in[col], (double)bm->d_out[row]);
            dS -= cell_entropy(val, DIN_NEW(col), DOUT_NEW(row));
        }
    }
    for (int pass = 0; pass < 2; ++pass) {           /* columns r and s */
        int col = pass == 0 ? r : s;
        for (int row = 0; row < B; ++row) {
            int val = MAT(bm, row, col);
            if (val == 0 || delta_get(dl, row, col) != 0 || row == r || row == s) continue;
            dS += cell_entropy(val, (double)bm->d_in[col], (double)bm->d_out[row]);
            dS -= cell_entropy(val, DIN_NEW(col), DOUT_NEW(row));
        }
    }
#undef DIN_NEW
#undef DOUT_NEW
    if (fabs(dS) <= 0x1p-40 * (double)T * log(E > 2 ? (double)E : 2.0)) dS = 0.0;   /* D3 */
    return dS;
}

/* entropy::hastings_correction(vertex, ...) (src/entropy.cpp:495-557), with Q3. */
static double hastings_move(const SbpoBM *bm, const SbpoGraph *g, const Delta *dl, int v, const Proposal *p) {
    if (p->k == 0) return 1.0;
    int B = bm->B, r = dl->r, s = p->s;
    int *cnt = (int *)calloc((size_t)B + 1, sizeof(int));
    int *order = (int *)malloc(sizeof(int) * ((size_t)B + 1));
    int n = 0;
    for (int e = g->out_ptr[v]; e < g->out_ptr[v + 1]; ++e) {
        int bu = bm->b[g->out_idx[e]];
        if (cnt[bu]++ == 0) order[n++] = bu;
    }
    for (int e = g->in_ptr[v]; e < g->in_ptr[v + 1]; ++e) {
        int u = g->in_idx[e];
        if (u == v) continue;
        int bu = bm->b[u];
        if (cnt[bu]++ == 0) order[n++] = bu;
    }
    double p_fwd = 0.0, p_bwd = 0.0;
    for (int i = 0; i < n; ++i) {
        int u = order[i];
        double c = cnt[u];
        double pw = MAT(bm, s, u) + MAT(bm, u, s) + 1.0;
        double bd = bm->d[u] + (double)B;
        double bw = MAT(bm, r, u) + delta_get(dl, r, u) + MAT(bm, u, r) + delta_get(dl, u, r) + 1.0;
        int nd = bm->d[u];
        if (u == r) {
            int self_edges = MAT(bm, r, r) + delta_get(dl, r, r);
            nd = (bm->d_out[r] - p->k_out) + (bm->d_in[r] - p->k_in) - self_edges;
        } else if (u == s) {
            int self_edges = MAT(bm, s, s) + delta_get(dl, s, s);
            nd = (bm->d_out[s] + p->k_out) + (bm->d_in[s] + p->k_in) - self_edges;
        }
        double pd = nd + (double)B;
        p_fwd += c * pw / bd;
        p_bwd += c * bw / pd;
    }
    free(cnt); free(order);
    return p_bwd / p_fwd;
}

/* Blockmodel::move_vertex(vertex, Delta, Proposal) (src/blockmodel/blockmodel.cpp:344-360), with Q2. */
static void apply_move(SbpoBM *bm, const Delta *dl, int v, const Proposal *p) {
    int r = dl->r, s = p->s;
    bm->b[v] = s;
    for (int m = 0; m < 4; ++m)
        for (int i = 0; i < dl->nkeys[m]; ++i) {
            int row, col, change;
            delta_entry(dl, m, i, &row, &col, &change);
            MAT(bm, row, col) += change;
        }
    int cur_self = MAT(bm, r, r) + delta_get(dl, r, r);
    int prop_self = MAT(bm, s, s) + delta_get(dl, s, s);
    bm->d_out[r] -= p->k_out; bm->d_out[s] += p->k_out;
    bm->d_in[r] -= (p->k_in + dl->self_w); bm->d_in[s] += (p->k_in + dl->self_w);
    bm->d[r] = bm->d_out[r] + bm->d_in[r] - cur_self;
    bm->d[s] = bm->d_out[s] + bm->d_in[s] - prop_self;
}

/* ------------------------------------------------------------------------------------- */
/* Proposals (src/common.cpp:131-192), canonical order D2                                  */
/* ------------------------------------------------------------------------------------- */
static int random_block(int r, int B, uint32_t x) {   /* common::propose_random_block */
    int proposed = (int)sbpo_scale(x, (int64_t)B - 1);
    if (proposed >= r) proposed++;
    return proposed;
}

/* Sample s from M[t,:]+M[:,t] (row then column, ascending), excluding block `skip` if >= 0. */
static int multinomial_block(const SbpoBM *bm, int t, int skip, int64_t target) {
    for (int c = 0; c < bm->B; ++c) {
        if (c == skip) continue;
        target -= MAT(bm, t, c);
        if (target < 0) return c;
    }
    for (int c = 0; c < bm->B; ++c) {
        if (c == skip) continue;
        target -= MAT(bm, c, t);
        if (target < 0) return c;
    }
    return -1;
}

static int64_t row_sum(const SbpoBM *bm, int t, int skip) {
    int64_t s = 0;
    for (int c = 0; c < bm->B; ++c) if (c != skip) s += MAT(bm, t, c);
    return s;
}
static int64_t col_sum(const SbpoBM *bm, int t, int skip) {
    int64_t s = 0;
    for (int c = 0; c < bm->B; ++c) if (c != skip) s += MAT(bm, c, t);
    return s;
}

/* finetune::propose_move's proposal half (src/finetune.cpp:488-501 -> src/common.cpp:131-182). */
static Proposal propose_vertex(const SbpoBM *bm, const SbpoGraph *g, int v, const uint32_t x[4]) {
    Proposal p;
    int r = bm->b[v];
    int k_out = g->out_ptr[v + 1] - g->out_ptr[v];
    int k_in = (g->in_ptr[v + 1] - g->in_ptr[v]) - g->self[v];
    p.k_out = k_out; p.k_in = k_in; p.k = k_out + k_in;
    if (p.k == 0) { p.s = random_block(r, bm->B, x[1]); return p; }
    int idx = (int)sbpo_scale(x[0], p.k);
    int nbr;
    if (idx < k_out) nbr = g->out_idx[g->out_ptr[v] + idx];
    else {
        int j = idx - k_out, e = g->in_ptr[v];
        for (;; ++e) { if (g->in_idx[e] == v) continue; if (j-- == 0) break; }
        nbr = g->in_idx[e];
    }
    int t = bm->b[nbr];
    int64_t total = row_sum(bm, t, -1) + col_sum(bm, t, -1);
    p.s = multinomial_block(bm, t, -1, sbpo_scale(x[1], total));
    return p;
}

/* One vertex evaluation: proposal, Hastings, delta-MDL and the accept test
 * (finetune::propose_move/move_vertex/accept, src/finetune.cpp:19-29,446-501). */
typedef struct { int s; int moved_proposal; int accepted; double dS, H; } Eval;

/* The proposal of a visit: drawn from the record x, or (moves) the recorded block x[0].
 * Returns 0 when a recorded block is out of range. */
static int visit_proposal(const SbpoBM *bm, const SbpoGraph *g, int v, const uint32_t x[4], int moves,
                          Proposal *p) {
    if (!moves) { *p = propose_vertex(bm, g, v, x); return 1; }
    p->k_out = g->out_ptr[v + 1] - g->out_ptr[v];
    p->k_in = (g->in_ptr[v + 1] - g->in_ptr[v]) - g->self[v];
    p->k = p->k_out + p->k_in;
    p->s = (int)x[0];
    if (p->s < 0 || p->s >= bm->B) { p->s = bm->b[v]; return 0; }
    return 1;
}

static double visit_uniform(const uint32_t x[4], int moves) {
    return moves ? record_uniform(x) : sbpo_u53(x[2], x[3]);
}

static Eval eval_vertex(const SbpoBM *bm, const SbpoGraph *g, int v, const uint32_t x[4], int moves, int *bad) {
    Eval ev = {0};
    int r = bm->b[v];
    Proposal p;
    if (!visit_proposal(bm, g, v, x, moves, &p)) *bad = 1;
    ev.s = p.s;
    if (p.s == r) return ev;   /* no move, no uniform consumed */
    ev.moved_proposal = 1;
    Delta dl;
    vertex_delta(&dl, bm, g, v, r, p.s);
    ev.H = hastings_move(bm, g, &dl, v, &p);
    ev.dS = delta_mdl_move(bm, &dl, &p, g->E);
    delta_free(&dl);
    double u = visit_uniform(x, moves);
    double ap = exp(-3.0 * ev.dS) * ev.H;
    ap = (ap >= 1.0) ? 1.0 : ap;
    ev.accepted = (u <= ap);
    return ev;
}

/* Public single-step helpers for unit tests. */
int sbpo_eval_vertex(const SbpoBM *bm, const SbpoGraph *g, int v, const uint32_t x[4],
                     int *s, double *dS, double *H, int *accepted) {
    int bad = 0;
    Eval ev = eval_vertex(bm, g, v, x, 0, &bad);
    *s = ev.s; *dS = ev.dS; *H = ev.H; *accepted = ev.accepted;
    return ev.moved_proposal;
}

double sbpo_delta_mdl_move(const SbpoBM *bm, const SbpoGraph *g, int v, int s, double *hastings) {
    int r = bm->b[v];
    Proposal p;
    p.s = s; p.k_out = g->out_ptr[v + 1] - g->out_ptr[v];
    p.k_in = (g->in_ptr[v + 1] - g->in_ptr[v]) - g->self[v]; p.k = p.k_out + p.k_in;
    Delta dl;
    vertex_delta(&dl, bm, g, v, r, s);
    double dS = delta_mdl_move(bm, &dl, &p, g->E);
    if (hastings) *hastings = hastings_move(bm, g, &dl, v, &p);
    delta_free(&dl);
    return dS;
}

void sbpo_move_vertex(SbpoBM *bm, const SbpoGraph *g, int v, int s) {
    int r = bm->b[v];
    Proposal p;
    p.s = s; p.k_out = g->out_ptr[v + 1] - g->out_ptr[v];
    p.k_in = (g->in_ptr[v + 1] - g->in_ptr[v]) - g->self[v]; p.k = p.k_out + p.k_in;
    Delta dl;
    vertex_delta(&dl, bm, g, v, r, s);
    apply_move(bm, &dl, v, &p);
    delta_free(&dl);
}

/* ------------------------------------------------------------------------------------- */
/* Finetune (src/finetune.cpp)                                                            */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    int64_t visits;          /* vertex evaluations (proposals drawn) */
    int64_t proposals_moved; /* proposals with s != r */
    int64_t accepted;        /* accepted moves */
    int sweeps;              /* MCMC iterations done by this call */
    double mdl;              /* overall entropy after the call */
    int rng_error;
} SbpoStats;

/* finetune::early_stop (src/finetune.cpp:144-162). */
static int early_stop(int iteration, int bracket_established, double initial_entropy,
                      const double *deltas, int n) {
    int last = n - 1;
    if (deltas[last] == 0.0) return 1;
    if (iteration < 3) return 0;
    double average = deltas[last] + deltas[last - 1] + deltas[last - 2];
    average /= -3.0;
    double threshold = bracket_established ? 1e-4 * initial_entropy : 5e-4 * initial_entropy;
    return average < threshold;
}

static int64_t visit_slot(int sweep, int V, int v) { return (int64_t)sweep * V + v; }

/* Serial MH visit of v (finetune::propose_move); returns 1 on accept and adds dS. */
static int mh_visit(SbpoBM *bm, const SbpoGraph *g, const SbpoRng *rng, int v, int sweep,
                    uint32_t call, SbpoStats *st, double *sum_dS) {
    uint32_t x[4];
    if (sbpo_draw(rng, (uint32_t)v, (uint32_t)sweep, call, 0, visit_slot(sweep, g->V, v), x)) { st->rng_error = 1; return 0; }
    st->visits++;
    int r = bm->b[v];
    Proposal p;
    if (!visit_proposal(bm, g, v, x, rng->moves, &p)) { st->rng_error = 1; return 0; }
    if (p.s == r) return 0;
    st->proposals_moved++;
    Delta dl;
    vertex_delta(&dl, bm, g, v, r, p.s);
    double H = hastings_move(bm, g, &dl, v, &p);
    double dS = delta_mdl_move(bm, &dl, &p, g->E);
    double u = visit_uniform(x, rng->moves);
    double ap = exp(-3.0 * dS) * H;
    ap = (ap >= 1.0) ? 1.0 : ap;
    int acc = (u <= ap);
    if (acc) { apply_move(bm, &dl, v, &p); *sum_dS += dS; st->accepted++; }
    delta_free(&dl);
    return acc;
}

/* One asynchronous-Gibbs batch over `verts[0..n)`: evaluate on the frozen state, then apply
 * accepted moves one by one in ascending vertex order (src/finetune.cpp:45-71, 364-392). */
static void gibbs_batch(SbpoBM *bm, const SbpoGraph *g, const SbpoRng *rng, const int *verts, int n,
                        int sweep, uint32_t call, SbpoStats *st, int *prop_of, unsigned char *moved) {
    for (int i = 0; i < n; ++i) {
        int v = verts[i];
        uint32_t x[4];
        if (sbpo_draw(rng, (uint32_t)v, (uint32_t)sweep, call, 0, visit_slot(sweep, g->V, v), x)) { st->rng_error = 1; return; }
        st->visits++;
        int bad = 0;
        Eval ev = eval_vertex(bm, g, v, x, rng->moves, &bad);
        if (bad) { st->rng_error = 1; return; }
        if (ev.moved_proposal) st->proposals_moved++;
        if (ev.accepted) { moved[v] = 1; prop_of[v] = ev.s; }
    }
    /* apply in vertex-id order (the reference's moves vector is indexed by vertex) */
    int lo = g->V, hi = -1;
    for (int i = 0; i < n; ++i) { if (verts[i] < lo) lo = verts[i]; if (verts[i] > hi) hi = verts[i]; }
    for (int v = lo; v <= hi; ++v) {
        if (!moved[v]) continue;
        moved[v] = 0;
        st->accepted++;
        int r = bm->b[v];
        Proposal p;
        p.s = prop_of[v]; p.k_out = g->out_ptr[v + 1] - g->out_ptr[v];
        p.k_in = (g->in_ptr[v + 1] - g->in_ptr[v]) - g->self[v]; p.k = p.k_out + p.k_in;
        Delta dl;
        vertex_delta(&dl, bm, g, v, r, p.s);
        apply_move(bm, &dl, v, &p);
        delta_free(&dl);
    }
}

enum { SBPO_MH = 0, SBPO_GIBBS = 1, SBPO_HYBRID = 2 };

/* finetune::{metropolis_hastings, asynchronous_gibbs, hybrid_mcmc}. */
static int finetune_run(SbpoBM *bm, const SbpoGraph *g, int algo, int batches, int bracket_established,
                        SbpoRng rng, uint32_t call, int max_sweeps, SbpoStats *st) {
    memset(st, 0, sizeof(*st));
    if (max_sweeps <= 0 || max_sweeps > SBPO_MAX_ITERATIONS) max_sweeps = SBPO_MAX_ITERATIONS;
    if (bm->B == 1) { st->mdl = bm->overall_entropy; return 0; }
    int V = g->V, E = g->E;
    double deltas[SBPO_MAX_ITERATIONS];
    bm->overall_entropy = (float)sbpo_mdl(bm, V, E);
    double initial_entropy = bm->overall_entropy;
    int *prop_of = (int *)malloc(sizeof(int) * (size_t)(V + 1));
    unsigned char *moved = (unsigned char *)calloc((size_t)V + 1, 1);
    int *ident = NULL;
    for (int it = 0; it < max_sweeps; ++it) {
        if (algo == SBPO_MH) {
            double sum = 0.0;
            for (int v = 0; v < V; ++v) mh_visit(bm, g, &rng, v, it, call, st, &sum);
            deltas[it] = sum;
            st->sweeps++;
            if (early_stop(it, bracket_established, (double)bm->overall_entropy, deltas, it + 1)) break;
        } else {
            if (algo == SBPO_HYBRID) {
                double dummy = 0.0;
                for (int i = 0; i < g->nhigh; ++i) mh_visit(bm, g, &rng, g->high[i], it, call, st, &dummy);
            }
            const int *list; int nlist;
            if (algo == SBPO_GIBBS) {
                if (!ident) { ident = (int *)malloc(sizeof(int) * (size_t)(V + 1)); for (int v = 0; v < V; ++v) ident[v] = v; }
                list = ident; nlist = V;
            } else { list = g->low; nlist = g->nlow; }
            double num_batches = batches;
            int batch_size = (int)ceil(nlist / num_batches);
            if (batch_size > 0) {
                for (int batch = 0; batch < nlist / batch_size; ++batch) {
                    int start = batch * batch_size;
                    int end = (batch + 1) * batch_size < nlist ? (batch + 1) * batch_size : nlist;
                    gibbs_batch(bm, g, &rng, list + start, end - start, it, call, st, prop_of, moved);
                }
            }
            double entropy = sbpo_mdl(bm, V, E);
            deltas[it] = entropy - initial_entropy;   /* Q4 */
            st->sweeps++;
            if (early_stop(it, bracket_established, initial_entropy, deltas, it + 1)) break;
        }
        if (st->rng_error) break;
    }
    free(prop_of); free(moved); free(ident);
    bm->overall_entropy = (float)sbpo_mdl(bm, V, E);
    st->mdl = bm->overall_entropy;
    return st->rng_error ? -1 : 0;
}

int sbpo_finetune(SbpoBM *bm, const SbpoGraph *g, int algo, int batches, int bracket_established,
                  uint64_t seed, uint32_t call, const uint32_t *replay, int64_t replay_records,
                  int max_sweeps, SbpoStats *st) {
    SbpoRng rng = {seed, replay, replay_records, 0};
    return finetune_run(bm, g, algo, batches, bracket_established, rng, call, max_sweeps, st);
}

/* The finetune driven by a recorded proposal stream: record t*V + v holds the proposed block
 * of vertex v's visit in sweep t and the bits of its accept uniform. */
int sbpo_finetune_moves(SbpoBM *bm, const SbpoGraph *g, int algo, int batches, int bracket_established,
                        const uint32_t *records, int64_t num_records, int max_sweeps, SbpoStats *st) {
    SbpoRng rng = {0, records, num_records, 1};
    return finetune_run(bm, g, algo, batches, bracket_established, rng, 0, max_sweeps, st);
}

/* ------------------------------------------------------------------------------------- */
/* Block merge (src/block_merge.cpp)                                                       */
/* ------------------------------------------------------------------------------------- */
/* block_merge::blockmodel_delta (src/block_merge.cpp:13-37). */
static void merge_delta(Delta *dl, const SbpoBM *bm, int r, int s) {
    delta_init(dl, r, s, bm->B);
    for (int col = 0; col < bm->B; ++col) {
        int value = MAT(bm, r, col);
        if (value == 0) continue;
        if (col == r || col == s) delta_add(dl, s, s, value);
        else delta_add(dl, s, col, value);
        delta_add(dl, r, col, -value);
    }
    for (int row = 0; row < bm->B; ++row) {
        int value = MAT(bm, row, r);
        if (value == 0 || row == r) continue;
        if (row == s) delta_add(dl, s, s, value);
        else delta_add(dl, row, s, value);
        delta_add(dl, row, r, -value);
    }
}

/* entropy::block_merge_delta_mdl(current_block, proposal, blockmodel, delta) (src/entropy.cpp:127-180). */
static double merge_delta_mdl(const SbpoBM *bm, const Delta *dl, int k_out, int k_in) {
    int r = dl->r, s = dl->s;
#define DIN_NEW(i) ((double)(bm->d_in[i] + ((i) == r ? -k_in : ((i) == s ? k_in : 0))))
#define DOUT_NEW(i) ((double)(bm->d_out[i] + ((i) == r ? -k_out : ((i) == s ? k_out : 0))))
    double dS = 0.0;
    for (int m = 0; m < 4; ++m)
        for (int i = 0; i < dl->nkeys[m]; ++i) {
            int row, col, change;
            delta_entry(dl, m, i, &row, &col, &change);
            double val = (double)MAT(bm, row, col);
            dS += cell_entropy(val, (double)bm->d_in[col], (double)bm->d_out[row]);
            if (row == r || col == r) continue;
            dS -= cell_entropy(val + change, DIN_NEW(col), DOUT_NEW(row));
        }
    for (int col = 0; col < bm->B; ++col) {
        int val = MAT(bm, s, col);
        if (val == 0 || delta_get(dl, s, col) != 0) continue;
        dS += cell_entropy(val, (double)bm->d_in[col], (double)bm->d_out[s]);
        dS -= cell_entropy(val, DIN_NEW(col), DOUT_NEW(s));
    }
    for (int row = 0; row < bm->B; ++row) {
        int val = MAT(bm, row, s);
        if (val == 0 || delta_get(dl, row, s) != 0 || row == r || row == s) continue;
        dS += cell_entropy(val, (double)bm->d_in[s], (double)bm->d_out[row]);
        dS -= cell_entropy(val, DIN_NEW(s), DOUT_NEW(row));
    }
#undef DIN_NEW
#undef DOUT_NEW
    return dS;
}

/* Merge delta-MDL of r and s.  It is the same for r -> s and s -> r (the merged block is the
 * same); it is evaluated in one fixed orientation (lower id into higher id) so that a mutual
 * best pair ties exactly and the carry-out order of a tie is decided by index, on every
 * implementation alike. */
double sbpo_merge_delta_mdl(const SbpoBM *bm, int r, int s) {
    if (r > s) { int t = r; r = s; s = t; }
    Delta dl;
    merge_delta(&dl, bm, r, s);
    double dS = merge_delta_mdl(bm, &dl, (int)row_sum(bm, r, -1), (int)col_sum(bm, r, -1));
    delta_free(&dl);
    return dS;
}

/* The ranking score of a merge: its delta-MDL rounded to a multiple of 2^-20 (D4), so that values
 * equal but for the rounding of their summation order compare equal on every implementation. */
static double merge_score(double dS) { return nearbyint(dS * 1048576.0) / 1048576.0; }

/* common::propose_new_block(block_merge = true) for block r with record x (D2 order). */
static int propose_merge(const SbpoBM *bm, int r, const uint32_t x[4], int moves) {
    int B = bm->B;
    if (moves) {   /* a recorded proposal: any block but r */
        int s = (int)x[0];
        return (s < 0 || s >= B || s == r) ? -1 : s;
    }
    int64_t k_out = row_sum(bm, r, -1), k_in = col_sum(bm, r, -1), k = k_out + k_in;
    if (k == 0) return random_block(r, B, x[1]);
    int64_t target = sbpo_scale(x[0], k);
    int t = -1;
    for (int c = 0; c < B && t < 0; ++c) { target -= MAT(bm, r, c); if (target < 0) t = c; }
    for (int c = 0; c < B && t < 0; ++c) { target -= MAT(bm, c, r); if (target < 0) t = c; }
    int64_t total = row_sum(bm, t, r) + col_sum(bm, t, r);
    if (total == 0) return random_block(r, B, x[1]);
    return multinomial_block(bm, t, r, sbpo_scale(x[1], total));
}

typedef struct { double dS; int block; } DI;
static int di_cmp(const void *a, const void *b) {
    const DI *x = (const DI *)a, *y = (const DI *)b;
    if (x->dS < y->dS) return -1;
    if (x->dS > y->dS) return 1;
    return (x->block > y->block) - (x->block < y->block);
}

/* Blockmodel::build_mapping + relabel (src/blockmodel/blockmodel.cpp:29-41, 71-76). */
static void relabel_dense(SbpoBM *bm) {
    int *seen = (int *)calloc((size_t)bm->B + 1, sizeof(int));
    for (int v = 0; v < bm->V; ++v) seen[bm->b[v]] = 1;
    int counter = 0;
    for (int i = 0; i < bm->B; ++i) seen[i] = seen[i] ? counter++ : -1;
    for (int v = 0; v < bm->V; ++v) bm->b[v] = seen[bm->b[v]];
    free(seen);
}

/* Blockmodel::carry_out_best_merges (src/blockmodel/blockmodel.cpp:50-78): the `--approximate` path. */
static int carry_out_simple(SbpoBM *bm, const double *dS, const int *best) {
    int B = bm->B;
    DI *order = (DI *)malloc(sizeof(DI) * (size_t)(B + 1));
    for (int i = 0; i < B; ++i) { order[i].dS = dS[i]; order[i].block = i; }
    qsort(order, (size_t)B, sizeof(DI), di_cmp);
    int *block_map = (int *)malloc(sizeof(int) * (size_t)(B + 1));
    for (int i = 0; i < B; ++i) block_map[i] = i;
    int num_merged = 0, counter = 0;
    while (num_merged < bm->num_blocks_to_merge) {
        if (counter >= B) { free(order); free(block_map); return -1; }
        int merge_from = order[counter].block;
        int merge_to = block_map[best[merge_from]];
        counter++;
        if (merge_to != merge_from) {
            for (int i = 0; i < B; ++i) if (block_map[i] == merge_from) block_map[i] = merge_to;
            for (int v = 0; v < bm->V; ++v) if (bm->b[v] == merge_from) bm->b[v] = merge_to;
            num_merged++;
        }
    }
    relabel_dense(bm);
    bm->B -= bm->num_blocks_to_merge;
    free(order); free(block_map);
    return 0;
}

/* block_merge::carry_out_best_merges_advanced (src/block_merge.cpp:123-217): min-heap with
 * lazy re-evaluation. Heap order is (dS, block) so ties are deterministic. */
typedef struct { int from, to; double dS; } HItem;
static int h_less(const HItem *a, const HItem *b) {
    if (a->dS != b->dS) return a->dS < b->dS;
    return a->from < b->from;
}
static void h_push(HItem *h, int *n, HItem it) {
    int i = (*n)++;
    h[i] = it;
    while (i > 0) { int p = (i - 1) / 2; if (!h_less(&h[i], &h[p])) break; HItem t = h[i]; h[i] = h[p]; h[p] = t; i = p; }
}
static HItem h_pop(HItem *h, int *n) {
    HItem top = h[0];
    h[0] = h[--(*n)];
    int i = 0;
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < *n && h_less(&h[l], &h[m])) m = l;
        if (r < *n && h_less(&h[r], &h[m])) m = r;
        if (m == i) break;
        HItem t = h[i]; h[i] = h[m]; h[m] = t; i = m;
    }
    return top;
}

static int carry_out_advanced(SbpoBM *bm, const double *dS, const int *best) {
    int B = bm->B;
    HItem *heap = (HItem *)malloc(sizeof(HItem) * (size_t)(2 * B + 2));
    int n = 0;
    for (int i = 0; i < B; ++i) { HItem it = {i, best[i], dS[i]}; h_push(heap, &n, it); }
    int *block_map = (int *)malloc(sizeof(int) * (size_t)(B + 1));
    for (int i = 0; i < B; ++i) block_map[i] = i;
    int num_merged = 0;
    while (num_merged < bm->num_blocks_to_merge && n > 0) {
        HItem merge = h_pop(heap, &n);
        int from = merge.from, to = block_map[merge.to];
        if (from == to) continue;
        int k_out = (int)row_sum(bm, from, -1), k_in = (int)col_sum(bm, from, -1);
        Delta dl;
        merge_delta(&dl, bm, from, to);
        int prop_self = MAT(bm, to, to) + delta_get(&dl, to, to);
        double actual = merge_score(sbpo_merge_delta_mdl(bm, from, to));
        if (n > 0 && actual > heap[0].dS) {
            merge.dS = actual;
            h_push(heap, &n, merge);
            delta_free(&dl);
            continue;
        }
        for (int i = 0; i < B; ++i) if (block_map[i] == from) block_map[i] = to;
        for (int v = 0; v < bm->V; ++v) if (bm->b[v] == from) bm->b[v] = to;
        for (int m = 0; m < 4; ++m)
            for (int i = 0; i < dl.nkeys[m]; ++i) {
                int row, col, change;
                delta_entry(&dl, m, i, &row, &col, &change);
                MAT(bm, row, col) += change;
            }
        bm->d_out[from] = 0; bm->d_out[to] += k_out;
        bm->d_in[from] = 0; bm->d_in[to] += k_in;
        bm->d[from] = 0; bm->d[to] = bm->d_out[to] + bm->d_in[to] - prop_self;
        delta_free(&dl);
        num_merged++;
    }
    relabel_dense(bm);
    bm->B -= bm->num_blocks_to_merge;
    free(heap); free(block_map);
    return 0;
}

typedef struct { int64_t proposals, avoided; } SbpoMergeStats;

/* block_merge::merge_blocks (src/block_merge.cpp:278-311). best/dS may be NULL. */
static int merge_run(SbpoBM *bm, const SbpoGraph *g, int approximate, SbpoRng rng, uint32_t call, int *best_out,
                     double *dS_out, SbpoMergeStats *ms) {
    int B = bm->B;
    int *best = (int *)malloc(sizeof(int) * (size_t)(B + 1));
    double *dS = (double *)malloc(sizeof(double) * (size_t)(B + 1));
    unsigned char *past = (unsigned char *)calloc((size_t)B + 1, 1);
    int *pl = (int *)malloc(sizeof(int) * SBPO_PROPOSALS_PER_BLOCK);
    if (ms) { ms->proposals = 0; ms->avoided = 0; }
    for (int r = 0; r < B; ++r) {
        best[r] = -1; dS[r] = 1.79769313486231570815e+308;
        int npl = 0;
        for (int i = 0; i < SBPO_PROPOSALS_PER_BLOCK; ++i) {
            uint32_t x[4];
            if (sbpo_draw(&rng, (uint32_t)r, (uint32_t)i, call, 1, (int64_t)r * SBPO_PROPOSALS_PER_BLOCK + i, x)) {
                free(best); free(dS); free(past); free(pl); return -1;
            }
            int s = propose_merge(bm, r, x, rng.moves);
            if (s < 0) { free(best); free(dS); free(past); free(pl); return -1; }
            if (ms) ms->proposals++;
            if (past[s]) { if (ms) ms->avoided++; continue; }
            double d = merge_score(sbpo_merge_delta_mdl(bm, r, s));
            past[s] = 1; pl[npl++] = s;
            if (d < dS[r]) { best[r] = s; dS[r] = d; }
        }
        for (int i = 0; i < npl; ++i) past[pl[i]] = 0;
    }
    if (best_out) memcpy(best_out, best, sizeof(int) * (size_t)B);
    if (dS_out) memcpy(dS_out, dS, sizeof(double) * (size_t)B);
    int rc = approximate ? carry_out_simple(bm, dS, best) : carry_out_advanced(bm, dS, best);
    free(best); free(dS); free(past); free(pl);
    if (rc) return rc;
    sbpo_bm_rebuild(bm, g);
    return 0;
}

int sbpo_merge_blocks(SbpoBM *bm, const SbpoGraph *g, int approximate, uint64_t seed, uint32_t call,
                      const uint32_t *replay, int64_t replay_records, int *best_out, double *dS_out,
                      SbpoMergeStats *ms) {
    SbpoRng rng = {seed, replay, replay_records, 0};
    return merge_run(bm, g, approximate, rng, call, best_out, dS_out, ms);
}

/* The merge step driven by a recorded proposal stream: record r*10 + i holds proposal i of
 * block r. */
int sbpo_merge_blocks_moves(SbpoBM *bm, const SbpoGraph *g, int approximate, const uint32_t *records,
                            int64_t num_records, int *best_out, double *dS_out, SbpoMergeStats *ms) {
    SbpoRng rng = {0, records, num_records, 1};
    return merge_run(bm, g, approximate, rng, 0, best_out, dS_out, ms);
}

void sbpo_bm_set_num_blocks_to_merge(SbpoBM *bm, int n) { bm->num_blocks_to_merge = n; }

/* ------------------------------------------------------------------------------------- */
/* SBP driver + golden-section triplet (src/sbp.cpp:61-112, blockmodel_triplet.cpp:3-100)  */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    SbpoBM *bm[3];     /* NULL = empty */
    int optimal_found;
} Triplet;

static int tri_B(const Triplet *t, int i) { return t->bm[i] ? t->bm[i]->B : 0; }

static void tri_update(Triplet *t, const SbpoBM *bm) {
    int index;
    if (!t->bm[1]) index = 1;
    else if (bm->overall_entropy <= t->bm[1]->overall_entropy) {
        int old_index = (t->bm[1]->B > bm->B) ? 0 : 2;
        sbpo_bm_destroy(t->bm[old_index]);
        t->bm[old_index] = sbpo_bm_copy(t->bm[1]);
        index = 1;
    } else index = (t->bm[1]->B > bm->B) ? 2 : 0;
    sbpo_bm_destroy(t->bm[index]);
    t->bm[index] = sbpo_bm_copy(bm);
}

static SbpoBM *tri_next(Triplet *t, SbpoBM *old) {
    old->num_blocks_to_merge = 0;
    tri_update(t, old);
    if (!t->bm[2]) {   /* golden ratio not reached */
        SbpoBM *bm = sbpo_bm_copy(t->bm[1]);
        bm->num_blocks_to_merge = (int)(bm->B * SBPO_REDUCTION_RATE);
        if (bm->num_blocks_to_merge == 0) t->optimal_found = 1;
        return bm;
    }
    if ((t->bm[0] && tri_B(t, 0) - tri_B(t, 2) == 2) || (!t->bm[0] && tri_B(t, 1) - tri_B(t, 2) == 1))
        t->optimal_found = 1;
    if (t->optimal_found) return sbpo_bm_copy(t->bm[1]);
    int index;
    if (!t->bm[0] && tri_B(t, 1) > tri_B(t, 2)) index = 1;
    else if (tri_B(t, 0) - tri_B(t, 1) >= tri_B(t, 1) - tri_B(t, 2)) index = 0;
    else index = 1;
    int next = tri_B(t, index + 1);
    next += (int)((tri_B(t, index) - tri_B(t, index + 1)) * 0.618);
    SbpoBM *bm = sbpo_bm_copy(t->bm[index]);
    bm->num_blocks_to_merge = bm->B - next;
    return bm;
}

typedef struct {
    int algo, batches, approximate, asynciterations;
    uint64_t seed;
} SbpoOptions;

typedef struct {
    double mdl;
    int num_blocks;
    int outer_iterations;
    int mcmc_sweeps;
    int64_t visits, accepted;
} SbpoRunStats;

/* Recorded streams of a partition's calls, in call order (merges and finetunes alternate as
 * the loop makes them); block_counts receives the block count after every call. */
typedef struct {
    int num_calls;
    const uint32_t *const *records;
    const int64_t *num_records;
    int max_sweeps;
    int calls_made;
    int *block_counts;
} SbpoPartitionReplay;

static int sbp_run(const SbpoGraph *g, const SbpoOptions *opt, int *assignment_out, SbpoRunStats *rs,
                   SbpoPartitionReplay *rp);

/* sbp::stochastic_block_partition (src/sbp.cpp:61-98). */
int sbpo_sbp(const SbpoGraph *g, const SbpoOptions *opt, int *assignment_out, SbpoRunStats *rs) {
    return sbp_run(g, opt, assignment_out, rs, NULL);
}

/* The same loop driven by recorded streams: call k reads records[k] (num_records[k] records),
 * every finetune capped at max_sweeps sweeps (0: no cap, as the reference's patched
 * MAX_NUM_ITERATIONS).  Returns the number of calls made, or -1 when a stream runs out. */
int sbpo_sbp_moves(const SbpoGraph *g, const SbpoOptions *opt, int num_calls, const uint32_t *const *records,
                   const int64_t *num_records, int max_sweeps, int *assignment_out, int *block_counts,
                   SbpoRunStats *rs) {
    SbpoPartitionReplay rp = {num_calls, records, num_records, max_sweeps, 0, block_counts};
    int rc = sbp_run(g, opt, assignment_out, rs, &rp);
    return rc ? -1 : rp.calls_made;
}

static int sbp_run(const SbpoGraph *g, const SbpoOptions *opt, int *assignment_out, SbpoRunStats *rs,
                   SbpoPartitionReplay *rp) {
    memset(rs, 0, sizeof(*rs));
    int V = g->V;
    int *ident = (int *)malloc(sizeof(int) * (size_t)(V + 1));
    for (int v = 0; v < V; ++v) ident[v] = v;
    SbpoBM *bm = sbpo_bm_create(g, V, ident);
    free(ident);
    Triplet t = {{NULL, NULL, NULL}, 0};
    float iteration = 0;
    uint32_t call = 0;
    int rc = 0;
    while (!t.optimal_found) {
        SbpoRng rng = {opt->seed, NULL, 0, 0};
        if (rp) {
            if (rp->calls_made >= rp->num_calls) { rc = -1; break; }
            rng = (SbpoRng){0, rp->records[rp->calls_made], rp->num_records[rp->calls_made], 1};
        }
        if (merge_run(bm, g, opt->approximate, rng, call, NULL, NULL, NULL)) { rc = -1; break; }
        if (rp) rp->block_counts[rp->calls_made++] = bm->B;
        int algo = opt->algo;
        if (algo == SBPO_GIBBS && !(iteration < (float)opt->asynciterations)) algo = SBPO_MH;
        SbpoStats st;
        rng = (SbpoRng){opt->seed, NULL, 0, 0};
        if (rp) {
            if (rp->calls_made >= rp->num_calls) { rc = -1; break; }
            rng = (SbpoRng){0, rp->records[rp->calls_made], rp->num_records[rp->calls_made], 1};
        }
        if (finetune_run(bm, g, algo, opt->batches, t.bm[2] != NULL, rng, call, rp ? rp->max_sweeps : 0, &st) &&
            rp) { rc = -1; break; }
        if (rp) rp->block_counts[rp->calls_made++] = bm->B;
        rs->mcmc_sweeps += st.sweeps; rs->visits += st.visits; rs->accepted += st.accepted;
        ++iteration; ++call;
        SbpoBM *next = tri_next(&t, bm);
        sbpo_bm_destroy(bm);
        bm = next;
        rs->outer_iterations++;
    }
    rs->mdl = bm->overall_entropy;
    rs->num_blocks = bm->B;
    if (rc == 0) memcpy(assignment_out, bm->b, sizeof(int) * (size_t)V);
    sbpo_bm_destroy(bm);
    for (int i = 0; i < 3; ++i) sbpo_bm_destroy(t.bm[i]);
    return rc;
}

/* Normalised mutual information of two labelings (src/evaluate.cpp:61-96), FP64 logs. */
double sbpo_nmi(int V, const int *a, const int *b) {
    int na = 0, nb = 0;
    for (int v = 0; v < V; ++v) { if (a[v] + 1 > na) na = a[v] + 1; if (b[v] + 1 > nb) nb = b[v] + 1; }
    double *joint = (double *)calloc((size_t)na * (size_t)nb, sizeof(double));
    double *pa = (double *)calloc((size_t)na, sizeof(double)), *pb = (double *)calloc((size_t)nb, sizeof(double));
    for (int v = 0; v < V; ++v) joint[(size_t)a[v] * nb + b[v]] += 1.0;
    for (int i = 0; i < na; ++i) for (int j = 0; j < nb; ++j) {
        double p = joint[(size_t)i * nb + j] / V;
        joint[(size_t)i * nb + j] = p; pa[i] += p; pb[j] += p;
    }
    double ha = 0, hb = 0, mi = 0;
    for (int i = 0; i < na; ++i) if (pa[i] > 0) ha -= pa[i] * log(pa[i]);
    for (int j = 0; j < nb; ++j) if (pb[j] > 0) hb -= pb[j] * log(pb[j]);
    for (int i = 0; i < na; ++i) for (int j = 0; j < nb; ++j) {
        double p = joint[(size_t)i * nb + j];
        if (p == 0.0) continue;
        mi += p * log(p / (pa[i] * pb[j]));
    }
    free(joint); free(pa); free(pb);
    if (ha * hb == 0.0) return 0.0;
    return mi / sqrt(ha * hb);
}
