/*
 * louvain_oracle.c -- CPU oracle (test infrastructure only, never shipped).
 *
 * Restates the update rule of olearczuk/gpu-louvain in exact integer
 * arithmetic so that the CUDA engine can be checked decision-for-decision.
 * Reference files cited per function.  OpenMP parallelises the per-vertex
 * decisions of one sub-round (they are independent by construction: every
 * decision reads only the state committed before the sub-round), so the
 * result does not depend on the thread count.
 */
#define _GNU_SOURCE
#include "louvain_oracle.h"

#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef __int128 i128;
typedef unsigned __int128 u128;

/* Degree buckets of the update order, modularity_optimisation.cuh:7-8.
 * A vertex of degree d belongs to bucket b when BOUNDS[b] < d <= BOUNDS[b+1];
 * degree-0 vertices belong to no bucket and never move
 * (modularity_optimisation.cu:259-275 isInBucket). */
#define NBUCKETS 7
static const int64_t BOUNDS[NBUCKETS + 1] = {0, 4, 8, 16, 32, 84, 319, INT64_MAX};

struct orc_state {
    int32_t V0, V;
    int64_t E;
    int64_t *rowptr;
    int32_t *col;
    int64_t *w;
    int scale;
    uint64_t T;
    int32_t *comm, *size, *newc, *orig2comm;
    uint64_t *k, *S;
    int32_t *bucket_list;            /* vertices grouped by bucket, id order */
    int64_t bucket_off[NBUCKETS + 1];
    int nthreads;
    int level;
};

/* ------------------------------------------------------------------ */
/* fixed-point scale                                                   */
/* ------------------------------------------------------------------ */

static int ceil_log2_u64(uint64_t x) {
    int r = 0;
    while (r < 64 && ((uint64_t)1 << r) < x) r++;
    return r;
}

/* Per-weight analysis: returns 0 for a valid weight, sets need (fractional
 * bits of its exact binary value) and top (floor(log2 w)); zero weights
 * report top = INT_MIN. */
static int weight_bits(float wf, int *need, int *top) {
    uint32_t bits;
    memcpy(&bits, &wf, 4);
    uint32_t ex = (bits >> 23) & 0xFF, man = bits & 0x7FFFFF;
    if (ex == 0xFF) return ORC_EWEIGHT;                  /* NaN / Inf */
    if ((bits & 0x7FFFFFFFu) == 0) { *need = 0; *top = INT_MIN; return 0; }
    if (bits >> 31) return ORC_EWEIGHT;                  /* negative */
    uint32_t m;
    int e;
    if (ex == 0) { m = man; e = -149; *top = (31 - __builtin_clz(man)) - 149; }
    else { m = man | 0x800000u; e = (int)ex - 150; *top = (int)ex - 127; }
    e += __builtin_ctz(m);
    *need = e < 0 ? -e : 0;
    return 0;
}

int orc_choose_scale(const float *w, int64_t E, int *scale, int *exact) {
    int need = 0, top = INT_MIN;
    for (int64_t i = 0; i < E; i++) {
        int n, t;
        int rc = weight_bits(w[i], &n, &t);
        if (rc) return rc;
        if (n > need) need = n;
        if (t > top) top = t;
    }
    if (top == INT_MIN) top = 0;
    int cap = 61 - top - ceil_log2_u64((uint64_t)(E > 0 ? E : 1));
    int s = need < cap ? need : cap;
    if (s < 0) return ORC_ETOOLARGE;
    *scale = s;
    if (exact) *exact = (s == need);
    return ORC_OK;
}

static inline int64_t to_fixed(float wf, int s) {
    return llrint(ldexp((double)wf, s));
}

/* ------------------------------------------------------------------ */
/* per-thread open-addressing map community -> uint64 sum              */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t *keys;
    uint64_t *vals;
    int32_t *used;      /* slots touched, for clearing */
    int64_t nused;
    int64_t cap;        /* power of two */
    int lg;
} cmap;

static int cmap_reserve(cmap *m, int64_t n) {
    int64_t need = 16;
    int lg = 4;
    while (need < 2 * n) { need <<= 1; lg++; }
    if (need <= m->cap) return 0;
    free(m->keys); free(m->vals); free(m->used);
    m->keys = (int32_t *)malloc(sizeof(int32_t) * need);
    m->vals = (uint64_t *)malloc(sizeof(uint64_t) * need);
    m->used = (int32_t *)malloc(sizeof(int32_t) * need);
    if (!m->keys || !m->vals || !m->used) return ORC_ENOMEM;
    for (int64_t i = 0; i < need; i++) m->keys[i] = -1;
    m->cap = need;
    m->lg = lg;
    m->nused = 0;
    return 0;
}

static inline void cmap_add(cmap *m, int32_t key, uint64_t v) {
    uint64_t mask = (uint64_t)m->cap - 1;
    uint64_t h = ((uint64_t)(uint32_t)key * 0x9E3779B97F4A7C15ull) >> (64 - m->lg);
    for (;;) {
        int32_t k = m->keys[h];
        if (k == key) { m->vals[h] += v; return; }
        if (k == -1) {
            m->keys[h] = key;
            m->vals[h] = v;
            m->used[m->nused++] = (int32_t)h;
            return;
        }
        h = (h + 1) & mask;
    }
}

static inline void cmap_clear(cmap *m) {
    for (int64_t i = 0; i < m->nused; i++) m->keys[m->used[i]] = -1;
    m->nused = 0;
}

static void cmap_free(cmap *m) {
    free(m->keys); free(m->vals); free(m->used);
    memset(m, 0, sizeof(*m));
}

/* ------------------------------------------------------------------ */
/* state                                                               */
/* ------------------------------------------------------------------ */

static int nthreads_of(const orc_state *s) { return s->nthreads > 0 ? s->nthreads : 1; }

static void free_level(orc_state *s) {
    free(s->rowptr); free(s->col); free(s->w);
    s->rowptr = NULL; s->col = NULL; s->w = NULL;
}

void orc_destroy(orc_state *s) {
    if (!s) return;
    free_level(s);
    free(s->comm); free(s->size); free(s->newc); free(s->orig2comm);
    free(s->k); free(s->S); free(s->bucket_list);
    free(s);
}

/* Level set-up: k_i = row sums (computeEdgesSum, modularity_optimisation.cu:23-40),
 * identity communities, Sigma_tot = k (utils.cu:84-87, community_aggregation.cu:337-344),
 * and the vertex list grouped by degree bucket. */
static void level_setup(orc_state *s) {
    int32_t V = s->V;
#pragma omp parallel for num_threads(nthreads_of(s)) schedule(static)
    for (int32_t v = 0; v < V; v++) {
        uint64_t acc = 0;
        for (int64_t e = s->rowptr[v]; e < s->rowptr[v + 1]; e++) acc += (uint64_t)s->w[e];
        s->k[v] = acc;
        s->S[v] = acc;
        s->comm[v] = v;
        s->newc[v] = v;
        s->size[v] = 1;
    }
    int64_t cnt[NBUCKETS] = {0};
    for (int32_t v = 0; v < V; v++) {
        int64_t d = s->rowptr[v + 1] - s->rowptr[v];
        for (int b = 0; b < NBUCKETS; b++)
            if (d > BOUNDS[b] && d <= BOUNDS[b + 1]) { cnt[b]++; break; }
    }
    s->bucket_off[0] = 0;
    for (int b = 0; b < NBUCKETS; b++) s->bucket_off[b + 1] = s->bucket_off[b] + cnt[b];
    int64_t pos[NBUCKETS];
    for (int b = 0; b < NBUCKETS; b++) pos[b] = s->bucket_off[b];
    for (int32_t v = 0; v < V; v++) {
        int64_t d = s->rowptr[v + 1] - s->rowptr[v];
        for (int b = 0; b < NBUCKETS; b++)
            if (d > BOUNDS[b] && d <= BOUNDS[b + 1]) { s->bucket_list[pos[b]++] = v; break; }
    }
}

orc_state *orc_create(int32_t V, int64_t E, const int32_t *rowptr,
                      const int32_t *col, const float *w, int nthreads, int *err) {
    int rc = ORC_OK;
    orc_state *s = NULL;
    if (V < 0 || E < 0 || (V > 0 && !rowptr) || (E > 0 && (!col || !w))) { rc = ORC_EINVAL; goto fail; }
    if (V > 0 && (rowptr[0] != 0 || rowptr[V] != E)) { rc = ORC_EINVAL; goto fail; }
    for (int32_t v = 0; v < V; v++)
        if (rowptr[v + 1] < rowptr[v]) { rc = ORC_EINVAL; goto fail; }
    for (int64_t e = 0; e < E; e++)
        if (col[e] < 0 || col[e] >= V) { rc = ORC_EINVAL; goto fail; }
    int scale;
    rc = orc_choose_scale(w, E, &scale, NULL);
    if (rc) goto fail;
    s = (orc_state *)calloc(1, sizeof(orc_state));
    if (!s) { rc = ORC_ENOMEM; goto fail; }
    s->V0 = V; s->V = V; s->E = E; s->scale = scale;
    s->nthreads = nthreads;
    size_t nv = (size_t)(V > 0 ? V : 1);
    s->rowptr = (int64_t *)malloc(sizeof(int64_t) * (nv + 1));
    s->col = (int32_t *)malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
    s->w = (int64_t *)malloc(sizeof(int64_t) * (size_t)(E > 0 ? E : 1));
    s->comm = (int32_t *)malloc(sizeof(int32_t) * nv);
    s->size = (int32_t *)malloc(sizeof(int32_t) * nv);
    s->newc = (int32_t *)malloc(sizeof(int32_t) * nv);
    s->orig2comm = (int32_t *)malloc(sizeof(int32_t) * nv);
    s->k = (uint64_t *)malloc(sizeof(uint64_t) * nv);
    s->S = (uint64_t *)malloc(sizeof(uint64_t) * nv);
    s->bucket_list = (int32_t *)malloc(sizeof(int32_t) * nv);
    if (!s->rowptr || !s->col || !s->w || !s->comm || !s->size || !s->newc ||
        !s->orig2comm || !s->k || !s->S || !s->bucket_list) { rc = ORC_ENOMEM; goto fail; }
    s->rowptr[0] = 0;
    for (int32_t v = 0; v < V; v++) s->rowptr[v + 1] = rowptr[v + 1];
    if (V == 0) s->rowptr[0] = 0;
    uint64_t T = 0;
    for (int64_t e = 0; e < E; e++) {
        s->col[e] = col[e];
        s->w[e] = to_fixed(w[e], scale);
        T += (uint64_t)s->w[e];
    }
    s->T = T;
    for (int32_t v = 0; v < V; v++) s->orig2comm[v] = v;
    level_setup(s);
    if (err) *err = ORC_OK;
    return s;
fail:
    orc_destroy(s);
    if (err) *err = rc;
    return NULL;
}

int32_t orc_num_vertices(const orc_state *s) { return s->V; }
int64_t orc_num_edges(const orc_state *s) { return s->E; }
int orc_scale(const orc_state *s) { return s->scale; }
uint64_t orc_total_weight(const orc_state *s) { return s->T; }
int orc_level(const orc_state *s) { return s->level; }

/* ------------------------------------------------------------------ */
/* move phase                                                          */
/* ------------------------------------------------------------------ */

/* computeMove (modularity_optimisation.cu:111-198) with full sums:
 *   e_{v,C} = sum of w(v,j) over j != v with C(j) = C      (:148-153)
 *   candidates C != C(v), except singleton -> larger singleton (:154-155)
 *   gain g(C) = e_C/M + k(S_own - k - S_C)/(2M^2)         (:96-102)
 * compared exactly as G(C) = T*e_C + k*(S_own - k - S_C) = g(C)*T^2/2.
 * best starts at (C(v), 0), ties go to the lower community id (:137-138,157),
 * and v moves iff G_best - T*e_own > 0 (:192). */
static int32_t decide(const orc_state *s, int32_t v, cmap *m) {
    int32_t own = s->comm[v];
    for (int64_t e = s->rowptr[v]; e < s->rowptr[v + 1]; e++) {
        int32_t j = s->col[e];
        if (j == v) continue;
        cmap_add(m, s->comm[j], (uint64_t)s->w[e]);
    }
    i128 T = (i128)s->T;
    i128 kv = (i128)s->k[v];
    i128 sown = (i128)s->S[own];
    uint64_t e_own = 0;
    int32_t best_c = own;
    i128 best_g = 0;
    int own_single = s->size[own] == 1;
    for (int64_t u = 0; u < m->nused; u++) {
        int32_t slot = m->used[u];
        int32_t c = m->keys[slot];
        uint64_t ec = m->vals[slot];
        if (c == own) { e_own = ec; continue; }
        if (own_single && c > own && s->size[c] == 1) continue;
        i128 g = T * (i128)ec + kv * (sown - kv - (i128)s->S[c]);
        if (g > best_g || (g == best_g && c < best_c)) { best_g = g; best_c = c; }
    }
    cmap_clear(m);
    if (best_g - T * (i128)e_own > 0) return best_c;
    return own;
}

/* One sweep: sub-rounds over buckets 0..6 (modularity_optimisation.cu:310-349),
 * decisions against the state committed before the sub-round, then the
 * commit of updateVertexCommunity (:237-249) and the Sigma_tot rebuild
 * (:328-330), here as exact incremental updates. */
int64_t orc_sweep(orc_state *s) {
    int64_t moves = 0;
    for (int b = 0; b < NBUCKETS; b++) {
        int64_t lo = s->bucket_off[b], hi = s->bucket_off[b + 1];
        if (lo == hi) continue;
        int rc = 0;
#pragma omp parallel num_threads(nthreads_of(s))
        {
            cmap m;
            memset(&m, 0, sizeof(m));
            int64_t maxdeg = BOUNDS[b + 1] == INT64_MAX ? 0 : BOUNDS[b + 1];
            if (maxdeg == 0) {
                for (int64_t i = lo; i < hi; i++) {
                    int32_t v = s->bucket_list[i];
                    int64_t d = s->rowptr[v + 1] - s->rowptr[v];
                    if (d > maxdeg) maxdeg = d;
                }
            }
            if (cmap_reserve(&m, maxdeg)) {
#pragma omp atomic write
                rc = 1;
            }
#pragma omp for schedule(dynamic, 64)
            for (int64_t i = lo; i < hi; i++) {
                if (rc) continue;
                int32_t v = s->bucket_list[i];
                s->newc[v] = decide(s, v, &m);
            }
            cmap_free(&m);
        }
        if (rc) return -1;
        for (int64_t i = lo; i < hi; i++) {
            int32_t v = s->bucket_list[i];
            int32_t o = s->comm[v], n = s->newc[v];
            if (o != n) {
                s->comm[v] = n;
                s->size[o] -= 1;
                s->size[n] += 1;
                s->S[o] -= s->k[v];
                s->S[n] += s->k[v];
                moves++;
            }
        }
    }
    return moves;
}

/* calculateModularity (modularity_optimisation.cu:365-401):
 *   Q = sum_i e_{i->C(i)} / (2M) - sum_C Sigma_tot^2 / (4M^2)
 * with e_{i->C(i)} over the whole row, self-loop included (:370-381). */
void orc_modularity_parts(const orc_state *s, uint64_t *e_own, uint64_t *s2_hi, uint64_t *s2_lo) {
    int nt = nthreads_of(s);
    uint64_t *pe = (uint64_t *)calloc((size_t)nt, sizeof(uint64_t));
    u128 *ps = (u128 *)calloc((size_t)nt, sizeof(u128));
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        uint64_t le = 0;
        u128 ls = 0;
#pragma omp for schedule(static)
        for (int32_t v = 0; v < s->V; v++) {
            int32_t c = s->comm[v];
            for (int64_t e = s->rowptr[v]; e < s->rowptr[v + 1]; e++)
                if (s->comm[s->col[e]] == c) le += (uint64_t)s->w[e];
            ls += (u128)s->S[v] * (u128)s->S[v];
        }
        pe[t] = le;
        ps[t] = ls;
    }
    uint64_t te = 0;
    u128 ts = 0;
    for (int t = 0; t < nt; t++) { te += pe[t]; ts += ps[t]; }
    free(pe); free(ps);
    *e_own = te;
    *s2_hi = (uint64_t)(ts >> 64);
    *s2_lo = (uint64_t)ts;
}

double orc_q_from_parts(uint64_t T, uint64_t e_own, uint64_t s2_hi, uint64_t s2_lo) {
    u128 s2 = ((u128)s2_hi << 64) | (u128)s2_lo;
    double t = (double)T;
    double a = (double)e_own / t;
    double b = (double)s2 / (t * t);
    return a - b;
}

double orc_modularity(const orc_state *s) {
    uint64_t e, hi, lo;
    orc_modularity_parts(s, &e, &hi, &lo);
    return orc_q_from_parts(s->T, e, hi, lo);
}

/* optimiseModularity (modularity_optimisation.cu:284-363).  The first sweep
 * always runs (totalGain starts at minGain, :341); sweeps repeat while the
 * sweep's gain >= min_gain; the level counts as changed when any sweep had a
 * positive gain (:352-353).  A sweep that moved nothing leaves the state as it
 * was, so the loop also stops there (the reference would repeat it forever
 * when min_gain <= 0).  Finally originalToCommunity <- C(originalToCommunity)
 * (:251-257, :361). */
int orc_optimise_level(orc_state *s, float min_gain, int max_sweeps, int *sweeps_out) {
    double gain = (double)min_gain;
    int changed = 0, sweeps = 0;
    double q_before = orc_modularity(s);
    while (gain >= (double)min_gain) {
        if (max_sweeps > 0 && sweeps >= max_sweeps) break;
        int64_t moves = orc_sweep(s);
        if (moves < 0) return -1;
        sweeps++;
        double q_after = orc_modularity(s);
        gain = q_after - q_before;
        if (gain > 0) changed = 1;
        q_before = q_after;
        if (moves == 0) break;
    }
    for (int32_t v = 0; v < s->V0; v++) s->orig2comm[v] = s->comm[s->orig2comm[v]];
    if (sweeps_out) *sweeps_out = sweeps;
    return changed;
}

static int cmp_pair(const void *a, const void *b) {
    const int32_t ka = *(const int32_t *)a, kb = *(const int32_t *)b;
    return (ka > kb) - (ka < kb);
}

typedef struct { int32_t key; int32_t pad; int64_t val; } pair_t;

/* aggregateCommunities (community_aggregation.cu:248-347): non-empty
 * communities are renumbered by an exclusive scan in ascending old id
 * (:272-273); each new vertex's row is the sum of its members' rows keyed by
 * the neighbours' new community, intra-community edges becoming one self-loop
 * that counts both directions (:76-163, :196-220); new Sigma_tot = row sum,
 * new communities are the identity, originalToCommunity <- newID[...]
 * (:222-228). */
int orc_aggregate(orc_state *s) {
    int32_t V = s->V;
    int32_t *newid = (int32_t *)malloc(sizeof(int32_t) * (size_t)(V > 0 ? V : 1));
    int32_t *start = (int32_t *)calloc((size_t)V + 2, sizeof(int32_t));
    int32_t *members = (int32_t *)malloc(sizeof(int32_t) * (size_t)(V > 0 ? V : 1));
    if (!newid || !start || !members) { free(newid); free(start); free(members); return ORC_ENOMEM; }
    int32_t nv = 0;
    for (int32_t c = 0; c < V; c++) newid[c] = s->size[c] > 0 ? nv++ : -1;
    /* members grouped by new id (stable in vertex id) */
    for (int32_t v = 0; v < V; v++) start[newid[s->comm[v]] + 1]++;
    for (int32_t c = 0; c < nv; c++) start[c + 1] += start[c];
    {
        int32_t *pos = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nv > 0 ? nv : 1));
        for (int32_t c = 0; c < nv; c++) pos[c] = start[c];
        for (int32_t v = 0; v < V; v++) members[pos[newid[s->comm[v]]]++] = v;
        free(pos);
    }
    int64_t *rowcnt = (int64_t *)calloc((size_t)nv + 1, sizeof(int64_t));
    pair_t **rows = (pair_t **)calloc((size_t)(nv > 0 ? nv : 1), sizeof(pair_t *));
    int rc = 0;
#pragma omp parallel num_threads(nthreads_of(s))
    {
        cmap m;
        memset(&m, 0, sizeof(m));
#pragma omp for schedule(dynamic, 16)
        for (int32_t c = 0; c < nv; c++) {
            int64_t bound = 0;
            for (int32_t i = start[c]; i < start[c + 1]; i++) {
                int32_t v = members[i];
                bound += s->rowptr[v + 1] - s->rowptr[v];
            }
            if (cmap_reserve(&m, bound)) { rc = 1; continue; }
            for (int32_t i = start[c]; i < start[c + 1]; i++) {
                int32_t v = members[i];
                for (int64_t e = s->rowptr[v]; e < s->rowptr[v + 1]; e++)
                    cmap_add(&m, newid[s->comm[s->col[e]]], (uint64_t)s->w[e]);
            }
            pair_t *r = (pair_t *)malloc(sizeof(pair_t) * (size_t)(m.nused > 0 ? m.nused : 1));
            for (int64_t u = 0; u < m.nused; u++) {
                r[u].key = m.keys[m.used[u]];
                r[u].pad = 0;
                r[u].val = (int64_t)m.vals[m.used[u]];
            }
            qsort(r, (size_t)m.nused, sizeof(pair_t), cmp_pair);
            rows[c] = r;
            rowcnt[c] = m.nused;
            cmap_clear(&m);
        }
        cmap_free(&m);
    }
    if (rc) {
        for (int32_t c = 0; c < nv; c++) free(rows[c]);
        free(rows); free(rowcnt); free(newid); free(start); free(members);
        return ORC_ENOMEM;
    }
    int64_t E2 = 0;
    for (int32_t c = 0; c < nv; c++) E2 += rowcnt[c];
    int64_t *rp = (int64_t *)malloc(sizeof(int64_t) * ((size_t)nv + 1));
    int32_t *cl = (int32_t *)malloc(sizeof(int32_t) * (size_t)(E2 > 0 ? E2 : 1));
    int64_t *wt = (int64_t *)malloc(sizeof(int64_t) * (size_t)(E2 > 0 ? E2 : 1));
    rp[0] = 0;
    for (int32_t c = 0; c < nv; c++) {
        for (int64_t u = 0; u < rowcnt[c]; u++) {
            cl[rp[c] + u] = rows[c][u].key;
            wt[rp[c] + u] = rows[c][u].val;
        }
        rp[c + 1] = rp[c] + rowcnt[c];
        free(rows[c]);
    }
    free(rows); free(rowcnt); free(start); free(members);
    for (int32_t v = 0; v < s->V0; v++) s->orig2comm[v] = newid[s->orig2comm[v]];
    free(newid);
    free_level(s);
    s->rowptr = rp; s->col = cl; s->w = wt;
    s->V = nv; s->E = E2;
    s->level++;
    level_setup(s);
    return ORC_OK;
}

/* Level loop of gpulouvain.cu:30-37. */
int orc_run(orc_state *s, float min_gain, int max_sweeps, double *q,
            int *levels_out, int64_t *sweeps_out, int64_t *edge_sweeps_out) {
    int levels = 0;
    int64_t sweeps = 0, edge_sweeps = 0;
    for (;;) {
        int sw = 0;
        int64_t e = s->E;
        int changed = orc_optimise_level(s, min_gain, max_sweeps, &sw);
        if (changed < 0) return ORC_ENOMEM;
        levels++;
        sweeps += sw;
        edge_sweeps += (int64_t)sw * e;
        if (!changed) break;
        int rc = orc_aggregate(s);
        if (rc) return rc;
    }
    if (q) *q = orc_modularity(s);
    if (levels_out) *levels_out = levels;
    if (sweeps_out) *sweeps_out = sweeps;
    if (edge_sweeps_out) *edge_sweeps_out = edge_sweeps;
    return ORC_OK;
}

void orc_get_communities(const orc_state *s, int32_t *out) {
    memcpy(out, s->comm, sizeof(int32_t) * (size_t)s->V);
}

int orc_set_communities(orc_state *s, const int32_t *comm) {
    for (int32_t v = 0; v < s->V; v++)
        if (comm[v] < 0 || comm[v] >= s->V) return ORC_EINVAL;
    for (int32_t v = 0; v < s->V; v++) { s->size[v] = 0; s->S[v] = 0; }
    for (int32_t v = 0; v < s->V; v++) {
        s->comm[v] = comm[v];
        s->newc[v] = comm[v];
        s->size[comm[v]] += 1;
        s->S[comm[v]] += s->k[v];
    }
    return ORC_OK;
}

void orc_get_original_to_community(const orc_state *s, int32_t *out) {
    memcpy(out, s->orig2comm, sizeof(int32_t) * (size_t)s->V0);
}

void orc_get_csr(const orc_state *s, int64_t *rowptr, int32_t *col, int64_t *wfix) {
    if (rowptr) memcpy(rowptr, s->rowptr, sizeof(int64_t) * ((size_t)s->V + 1));
    if (col) memcpy(col, s->col, sizeof(int32_t) * (size_t)s->E);
    if (wfix) memcpy(wfix, s->w, sizeof(int64_t) * (size_t)s->E);
}

void orc_get_vertex_weights(const orc_state *s, uint64_t *k) {
    memcpy(k, s->k, sizeof(uint64_t) * (size_t)s->V);
}

void orc_get_community_weights(const orc_state *s, uint64_t *S) {
    memcpy(S, s->S, sizeof(uint64_t) * (size_t)s->V);
}

/* ------------------------------------------------------------------ */
/* MTX reader: utils.cu:9-62                                           */
/* ------------------------------------------------------------------ */

typedef struct { int32_t j; float w; } nb_t;
typedef struct { nb_t *a; int32_t n, cap; } nbvec;

static int nb_push(nbvec *v, int32_t j, float w) {
    if (v->n == v->cap) {
        int32_t nc = v->cap ? v->cap * 2 : 4;
        nb_t *na = (nb_t *)realloc(v->a, sizeof(nb_t) * (size_t)nc);
        if (!na) return ORC_ENOMEM;
        v->a = na; v->cap = nc;
    }
    v->a[v->n].j = j; v->a[v->n].w = w; v->n++;
    return 0;
}

/* Header: lines starting with '%' are skipped (utils.cu:14-16); the size line
 * is "rows cols nnz" and the vertex count is the SECOND number (utils.cu:18).
 * Each entry "i j w" is 1-based; v1's list gets (v2,w) and, unless it is a
 * self-loop, v2's list gets (v1,w) (utils.cu:32-46).  CSR rows keep that
 * insertion order (utils.cu:50-59).  m_ref reproduces the FP32 sequential
 * accumulation of M (utils.cu:36-46). */
int orc_read_mtx(const char *path, int32_t *Vout, int64_t *Eout, int32_t **rowptr,
                 int32_t **col, float **w, float *m_ref) {
    FILE *f = fopen(path, "r");
    if (!f) return ORC_EIO;
    char *line = NULL;
    size_t cap = 0;
    ssize_t n;
    int pattern = 0;
    long long rows = 0, cols = 0, nnz = 0;
    int have_size = 0;
    while ((n = getline(&line, &cap, f)) >= 0) {
        if (line[0] == '%') {
            if (strncmp(line, "%%MatrixMarket", 14) == 0 && strstr(line, "pattern")) pattern = 1;
            continue;
        }
        char *p = line;
        while (*p == ' ' || *p == '\t') p++;
        if (*p == '\n' || *p == '\r' || *p == 0) continue;
        if (sscanf(line, "%lld %lld %lld", &rows, &cols, &nnz) == 3) have_size = 1;
        break;
    }
    free(line);
    if (!have_size || cols < 0 || cols > INT32_MAX || nnz < 0) { fclose(f); return ORC_EIO; }
    (void)rows;
    int32_t V = (int32_t)cols;
    nbvec *nb = (nbvec *)calloc((size_t)(V > 0 ? V : 1), sizeof(nbvec));
    float M = 0;
    int64_t E = 0;
    int rc = 0;
    for (long long i = 0; i < nnz; i++) {
        long long a, b;
        float wv = 1.0f;
        int got = pattern ? fscanf(f, "%lld %lld", &a, &b) : fscanf(f, "%lld %lld %f", &a, &b, &wv);
        if (got != (pattern ? 2 : 3)) { rc = ORC_EIO; break; }
        a--; b--;
        if (a < 0 || b < 0 || a >= V || b >= V) { rc = ORC_EINVAL; break; }
        if (nb_push(&nb[a], (int32_t)b, wv)) { rc = ORC_ENOMEM; break; }
        E++;
        if (a != b) {
            if (nb_push(&nb[b], (int32_t)a, wv)) { rc = ORC_ENOMEM; break; }
            E++;
            M += wv;
        }
        M += wv;
    }
    fclose(f);
    if (rc == 0 && E > INT32_MAX) rc = ORC_ETOOLARGE;
    if (rc) {
        for (int32_t v = 0; v < V; v++) free(nb[v].a);
        free(nb);
        return rc;
    }
    M /= 2;
    int32_t *rp = (int32_t *)malloc(sizeof(int32_t) * ((size_t)V + 1));
    int32_t *cl = (int32_t *)malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
    float *wt = (float *)malloc(sizeof(float) * (size_t)(E > 0 ? E : 1));
    int64_t idx = 0;
    for (int32_t v = 0; v < V; v++) {
        rp[v] = (int32_t)idx;
        for (int32_t t = 0; t < nb[v].n; t++) {
            cl[idx] = nb[v].a[t].j;
            wt[idx] = nb[v].a[t].w;
            idx++;
        }
        free(nb[v].a);
    }
    rp[V] = (int32_t)idx;
    free(nb);
    *Vout = V; *Eout = E; *rowptr = rp; *col = cl; *w = wt;
    if (m_ref) *m_ref = M;
    return ORC_OK;
}

void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------ */
/* seeded R-MAT input (the benchmark graph, generated without the      */
/* product library)                                                    */
/* ------------------------------------------------------------------ */

/* Counter-based draws: splitmix64's finaliser (Steele, Lea, Flood 2014)
 * applied to key + i * golden ratio, key = mix(seed ^ (stream << 32)).  The
 * R-MAT recursion (Chakrabarti, Zhan, Faloutsos 2004) takes, for bit level l
 * (most significant first), 32 bits of draw(key_{l/2}, i): quadrant
 * q = [x >= a] + [x >= a+b] + [x >= a+b+c] gives the row bit q >> 1 and the
 * column bit q & 1.  Self-loops and repeated pairs are dropped and the
 * graph is symmetrised with ascending rows.  Weight of pair (lo, hi):
 * (m + 2^23) * 2^-24 from 24 bits of draw(key_w, lo << 32 | hi), uniform on
 * [0.5, 1.5) and exact in float32.  The same seed gives the same graph as
 * the engine's generators. */
static uint64_t rng_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t rng_key(uint64_t seed, uint64_t stream) { return rng_mix(seed ^ (stream << 32)); }
static uint64_t rng_draw(uint64_t key, uint64_t i) { return rng_mix(key + i * 0x9E3779B97F4A7C15ull); }

/* LSD radix sort of n keys on their low nbits bits (tmp holds n keys). */
static void radix_sort_keys(uint64_t *a, uint64_t *tmp, int64_t n, int nbits, int nt) {
    int64_t *hist = (int64_t *)malloc(sizeof(int64_t) * (size_t)nt * 256);
    for (int shift = 0; shift < nbits; shift += 8) {
        memset(hist, 0, sizeof(int64_t) * (size_t)nt * 256);
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
            int64_t *h = hist + (size_t)t * 256;
            for (int64_t i = lo; i < hi; i++) h[(a[i] >> shift) & 255]++;
        }
        int64_t run = 0;
        for (int d = 0; d < 256; d++)
            for (int t = 0; t < nt; t++) {
                int64_t c = hist[(size_t)t * 256 + d];
                hist[(size_t)t * 256 + d] = run;
                run += c;
            }
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
            int64_t *h = hist + (size_t)t * 256;
            for (int64_t i = lo; i < hi; i++) tmp[h[(a[i] >> shift) & 255]++] = a[i];
        }
        memcpy(a, tmp, sizeof(uint64_t) * (size_t)n);
    }
    free(hist);
}

int orc_gen_rmat(int scale, int edge_factor, uint64_t seed, double a, double b, double c,
                 int unit_weights, int nthreads, int32_t *Vout, int64_t *Eout, int32_t **rowptr,
                 int32_t **col, float **w) {
    if (scale < 1 || scale > 30 || edge_factor < 1 || !Vout || !Eout || !rowptr || !col || !w)
        return ORC_EINVAL;
    int nt = nthreads > 0 ? nthreads : 1;
    const int64_t n = (int64_t)edge_factor << scale;
    const uint32_t ta = (uint32_t)(a * 4294967296.0), tb = (uint32_t)((a + b) * 4294967296.0),
                   tc = (uint32_t)((a + b + c) * 4294967296.0);
    uint64_t keys_l[16];
    for (int i = 0; i < 16; i++) keys_l[i] = rng_key(seed, (uint64_t)(1 + i));
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    int64_t *cnt = (int64_t *)calloc((size_t)nt + 1, sizeof(int64_t));
    if (!keys || !tmp || !cnt) { free(keys); free(tmp); free(cnt); return ORC_ENOMEM; }
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        int64_t lo = n * t / nt, hi = n * (t + 1) / nt, k = lo;
        for (int64_t i = lo; i < hi; i++) {
            uint32_t u = 0, v = 0;
            for (int pr = 0; 2 * pr < scale; pr++) {
                uint64_t r = rng_draw(keys_l[pr], (uint64_t)i);
                for (int half = 0; half < 2 && 2 * pr + half < scale; half++) {
                    uint32_t x = (uint32_t)(r >> (32 * half));
                    uint32_t q = (uint32_t)(x >= ta) + (uint32_t)(x >= tb) + (uint32_t)(x >= tc);
                    u = (u << 1) | (q >> 1);
                    v = (v << 1) | (q & 1u);
                }
            }
            if (u == v) continue;
            uint32_t lo32 = u < v ? u : v, hi32 = u < v ? v : u;
            keys[k++] = ((uint64_t)lo32 << scale) | hi32;
        }
        cnt[t + 1] = k - lo;
    }
    int64_t m = 0;
    for (int t = 0; t < nt; t++) {
        int64_t lo = n * t / nt;
        if (m != lo) memmove(keys + m, keys + lo, sizeof(uint64_t) * (size_t)cnt[t + 1]);
        m += cnt[t + 1];
    }
    free(cnt);
    radix_sort_keys(keys, tmp, m, 2 * scale, nt);
    free(tmp);
    int64_t nk = 0;
    for (int64_t i = 0; i < m; i++)
        if (nk == 0 || keys[i] != keys[nk - 1]) keys[nk++] = keys[i];
    const int32_t V = (int32_t)(1u << scale);
    const int64_t E = 2 * nk;
    if (E > INT32_MAX) { free(keys); return ORC_ETOOLARGE; }
    const uint64_t mask = ((uint64_t)1 << scale) - 1;
    int64_t *dlo = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    int64_t *dhi = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    int32_t *rp = (int32_t *)malloc(sizeof(int32_t) * ((size_t)V + 1));
    int32_t *cl = (int32_t *)malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
    float *wt = (float *)malloc(sizeof(float) * (size_t)(E > 0 ? E : 1));
    if (!dlo || !dhi || !rp || !cl || !wt) {
        free(keys); free(dlo); free(dhi); free(rp); free(cl); free(wt);
        return ORC_ENOMEM;
    }
    for (int64_t i = 0; i < nk; i++) {
        dhi[keys[i] >> scale]++;   /* a row's larger neighbours */
        dlo[keys[i] & mask]++;     /* ... and its smaller ones */
    }
    /* row v: smaller neighbours (ascending), then larger ones (ascending) */
    int64_t acc = 0;
    for (int32_t v = 0; v < V; v++) {
        rp[v] = (int32_t)acc;
        int64_t d_lo = dlo[v], d_hi = dhi[v];
        dlo[v] = acc;           /* cursor of the smaller neighbours */
        dhi[v] = acc + d_lo;    /* cursor of the larger neighbours */
        acc += d_lo + d_hi;
    }
    rp[V] = (int32_t)acc;
    const uint64_t wkey = rng_key(seed, 0xFFFF);
    for (int64_t i = 0; i < nk; i++) {
        int32_t x = (int32_t)(keys[i] >> scale), y = (int32_t)(keys[i] & mask);
        float wv = 1.0f;
        if (!unit_weights) {
            uint64_t h = rng_draw(wkey, ((uint64_t)(uint32_t)x << 32) | (uint32_t)y);
            wv = (float)((uint32_t)(h >> 40) + 8388608u) * 5.9604644775390625e-08f;
        }
        int64_t px = dhi[x]++, py = dlo[y]++;
        cl[px] = y; wt[px] = wv;
        cl[py] = x; wt[py] = wv;
    }
    free(keys); free(dlo); free(dhi);
    *Vout = V; *Eout = E; *rowptr = rp; *col = cl; *w = wt;
    return ORC_OK;
}

double orc_modularity_f64(int32_t V, const int32_t *rowptr, const int32_t *col,
                          const float *w, const int32_t *comm) {
    double T = 0, eown = 0;
    double *S = (double *)calloc((size_t)(V > 0 ? V : 1), sizeof(double));
    for (int32_t v = 0; v < V; v++) {
        for (int32_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
            T += w[e];
            S[comm[v]] += w[e];
            if (comm[col[e]] == comm[v]) eown += w[e];
        }
    }
    double s2 = 0;
    for (int32_t c = 0; c < V; c++) s2 += S[c] * S[c];
    free(S);
    return eown / T - s2 / (T * T);
}
