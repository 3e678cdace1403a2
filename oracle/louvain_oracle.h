/*
 * louvain_oracle.h -- CPU oracle for the Louvain level loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA engine is
 * compared against; it is never linked into, called by or shipped with the
 * product library.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference leg may load it.
 *
 * It restates the update rule of olearczuk/gpu-louvain in exact arithmetic:
 *   - modularity_optimisation.cu:96-102   computeGain (gain formula)
 *   - modularity_optimisation.cu:111-198  computeMove (candidates, tie-break,
 *                                          singleton-swap guard, move rule)
 *   - modularity_optimisation.cu:237-249  updateVertexCommunity (commit)
 *   - modularity_optimisation.cu:284-363  optimiseModularity (bucket
 *                                          sub-rounds, sweep loop)
 *   - modularity_optimisation.cu:365-401  calculateModularity
 *   - community_aggregation.cu:47-347     aggregateCommunities
 *   - gpulouvain.cu:30-37                 level loop + final modularity
 *   - utils.cu:9-62                       readInputData (MTX conventions)
 *
 * Arithmetic: every weight is mapped to an integer on a 2^-scale grid
 * (exact for float32 weights whose grid fits), all sums (k_i, Sigma_tot,
 * e_{i,C}) are exact uint64, and gains are compared exactly in 128-bit
 * integers after multiplying the reference's gain by T^2/2 (T = 2M = sum of
 * all CSR weights).  Modularity is formed in FP64 from exact integer totals.
 */
#ifndef LOUVAIN_ORACLE_H
#define LOUVAIN_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_OK = 0,
    ORC_EINVAL = 1,      /* malformed CSR / arguments */
    ORC_EWEIGHT = 2,     /* negative, NaN or infinite weight */
    ORC_ETOOLARGE = 3,   /* total weight does not fit the fixed-point grid */
    ORC_ENOMEM = 4,
    ORC_EIO = 5
};

typedef struct orc_state orc_state;

/* Fixed-point scale selection shared by oracle and engine (same rule):
 * need = max fractional bits of any weight, top = max floor(log2 w),
 * scale = min(need, 61 - top - ceil_log2(E)), scale >= 0 required.
 * *exact = 1 when scale == need (no weight was rounded). */
int orc_choose_scale(const float *w, int64_t E, int *scale, int *exact);

orc_state *orc_create(int32_t V, int64_t E, const int32_t *rowptr,
                      const int32_t *col, const float *w, int nthreads,
                      int *err);
void orc_destroy(orc_state *s);

int32_t orc_num_vertices(const orc_state *s);
int64_t orc_num_edges(const orc_state *s);
int orc_scale(const orc_state *s);
uint64_t orc_total_weight(const orc_state *s);
int orc_level(const orc_state *s);

/* One sweep = the 7 degree-bucket sub-rounds; returns number of moves. */
int64_t orc_sweep(orc_state *s);
/* Exact modularity parts: e_own total (uint64) and sum of Sigma_tot^2 as
 * two uint64 halves; orc_modularity forms the FP64 value from them. */
void orc_modularity_parts(const orc_state *s, uint64_t *e_own,
                          uint64_t *s2_hi, uint64_t *s2_lo);
double orc_modularity(const orc_state *s);
double orc_q_from_parts(uint64_t T, uint64_t e_own, uint64_t s2_hi,
                        uint64_t s2_lo);

/* optimiseModularity: sweeps until gain < min_gain; returns changed flag. */
int orc_optimise_level(orc_state *s, float min_gain, int max_sweeps,
                       int *sweeps_out);
/* aggregateCommunities: rows of the new CSR sorted by neighbour id. */
int orc_aggregate(orc_state *s);
/* Whole level loop (gpulouvain.cu:30-37); returns final modularity. */
int orc_run(orc_state *s, float min_gain, int max_sweeps, double *q,
            int *levels_out, int64_t *sweeps_out, int64_t *edge_sweeps_out);

/* State access (current level). */
void orc_get_communities(const orc_state *s, int32_t *out);
int orc_set_communities(orc_state *s, const int32_t *comm);
void orc_get_original_to_community(const orc_state *s, int32_t *out);
/* CSR of the current level; rowptr has V+1 entries (int64), weights are the
 * fixed-point integers (divide by 2^scale for the real value). */
void orc_get_csr(const orc_state *s, int64_t *rowptr, int32_t *col,
                 int64_t *wfix);
void orc_get_vertex_weights(const orc_state *s, uint64_t *k);
void orc_get_community_weights(const orc_state *s, uint64_t *S);

/* utils.cu:9-62 readInputData restated: CSR in file order, both directions
 * for off-diagonal entries, self-loops once.  Arrays are malloc'd; free with
 * orc_free.  m_ref is the reference's FP32 sequential M for comparison. */
int orc_read_mtx(const char *path, int32_t *V, int64_t *E, int32_t **rowptr,
                 int32_t **col, float **w, float *m_ref);
void orc_free(void *p);

/* Seeded R-MAT graph (scale, edge factor, a, b, c), symmetrised without
 * self-loops or repeated pairs, ascending rows; unit weights or weights
 * uniform on [0.5, 1.5) exact in float32.  The same seed gives the same CSR
 * as the engine's generators, so baselines can build the benchmark input
 * without loading the product library.  Arrays are malloc'd (orc_free). */
int orc_gen_rmat(int scale, int edge_factor, uint64_t seed, double a, double b, double c,
                 int unit_weights, int nthreads, int32_t *V, int64_t *E, int32_t **rowptr,
                 int32_t **col, float **w);

/* Modularity in FP64 of an arbitrary partition of the level-0 graph given as
 * float weights (a plain recomputation, used to check printed maps). */
double orc_modularity_f64(int32_t V, const int32_t *rowptr, const int32_t *col,
                          const float *w, const int32_t *comm);

#ifdef __cplusplus
}
#endif
#endif
