/*
 * louvain_b200.h -- C ABI of the B200 Louvain engine (liblouvain_b200.so).
 *
 * Drop-in boundary for the level loop of olearczuk/gpu-louvain.  The
 * reference has no library API: its boundary is the `gpulouvain` CLI and the
 * three C++ functions that the CLI calls over `device_structures`.  Each entry
 * point below names the reference interface it replaces (file:line in the
 * reference tree).  All functions return an lv_status (0 = LV_OK) instead of
 * calling exit() (the reference's HANDLE_ERROR, utils.cuh:92-98); the text of
 * the last error of a handle is available from lv_last_error().
 *
 * Arithmetic: weights are mapped onto an integer grid of 2^-scale (exact for
 * float32 weights whose binary expansions fit, see lv_get_scale); all sums
 * are exact and gains are compared exactly, so results do not depend on the
 * order of parallel additions and are bit-identical run to run.
 *
 * Threading: a handle owns one CUDA stream and its device memory; calls on
 * one handle must not overlap.  Different handles are independent.
 */
#ifndef LOUVAIN_B200_H
#define LOUVAIN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum lv_status {
    LV_OK = 0,
    LV_ERR_INVALID = 1,    /* bad argument or malformed CSR                 */
    LV_ERR_WEIGHT = 2,     /* negative, NaN or infinite edge weight         */
    LV_ERR_TOO_LARGE = 3,  /* beyond int32 ids/offsets or the fixed grid    */
    LV_ERR_NOMEM = 4,      /* device or host allocation failed              */
    LV_ERR_CUDA = 5,       /* CUDA runtime error                            */
    LV_ERR_DEVICE = 6,     /* a device-side check failed (see lv_last_error) */
    LV_ERR_IO = 7,         /* file could not be read or parsed              */
    LV_ERR_NO_DEVICE = 8   /* no usable CUDA device                         */
} lv_status;

typedef struct lv_handle lv_handle;

typedef struct lv_opts {
    uint32_t struct_size;  /* sizeof(lv_opts), for forward compatibility   */
    int32_t device;        /* CUDA device ordinal (default 0)              */
    int32_t max_sweeps;    /* per-level sweep cap, 0 = unlimited (default) */
    int32_t profile;       /* 1: time every kernel class with CUDA events  */
    int32_t verify;        /* 1: after every sweep, check the incrementally
                              maintained modularity against a full pass    */
    int32_t trace;         /* 1: per-level and per-sweep lines on stderr
                              (class sizes, moves, modularity, device ms)  */
    int32_t sweep_graph;   /* 1 (default): a level's sweep loop runs as one
                              CUDA graph whose while-node condition is set
                              on the device after each sweep (no host round
                              trip per sweep); used when profile, verify and
                              trace are 0.  0: one host round trip per sweep.
                              Results are identical.                      */
    int32_t active_set;    /* 1: learned active-set sweeps on levels of at
                              least 65536 vertices (needs a model,
                              lv_set_active_model); results then differ from
                              the plain method (final modularity close to it).
                              0 (default): plain sweeps                    */
    int32_t active_full_every; /* learned mode: every this many sweeps a full
                              sweep measures the predictor's recall
                              (default 0 = 4)                              */
    float active_min_recall;   /* learned mode: below this recall the plain
                              sweep takes over for the rest of the level
                              (default 0 = 0.9)                            */
    float trace_sample;    /* > 0: record move traces (features before each
                              sweep and whether the vertex then moved) for
                              this fraction of vertices per sweep           */
    float active_start;    /* learned mode: proposals start after a full
                              sweep moved less than this fraction of the
                              level's vertices (default 0 = 0.05)          */
    int32_t wide_weights;  /* 1: the move phase reads aggregated levels as
                              uint64 sums and sums every table in 64 bits;
                              0 (default): when every weight it reads is
                              below 2^32 (level 0 whose fixed-point weights
                              fit, aggregated levels whose merged sums other
                              than the self-loops, which the move phase
                              skips, fit) it reads 32-bit values and sums in
                              16-bit-piece counters.  Same results.       */
    int32_t giant_degree;  /* work mapping (results never depend on it): a
                              vertex of degree above this is decided by the
                              staged-chunk path instead of a warp; 0 =
                              default 8192, else 1024..65536              */
    int32_t warp_limit;    /* work mapping: distinct neighbour communities
                              after which a warp hands its vertex to a
                              fallback CTA; 0 = default 352, else 32..384  */
    int32_t reserved[1];
} lv_opts;

/* Per-run counters; times in milliseconds (device time, CUDA events). */
typedef struct lv_stats {
    int32_t levels;            /* levels run by lv_run / lv_optimise_level   */
    int32_t final_vertices;    /* vertices of the last level                 */
    int64_t sweeps;            /* sweeps over all levels                     */
    int64_t edge_sweeps;       /* sum over sweeps of that level's CSR size   */
    int64_t moves;             /* committed vertex moves                     */
    double move_ms;            /* move kernels + commits                     */
    double modularity_ms;      /* modularity reductions                      */
    double aggregate_ms;       /* aggregation                                */
    double setup_ms;           /* level set-up (k_i, classes, hub tables)    */
    double move_bytes;         /* algorithmic bytes of the move sweeps       */
    int64_t kernel_launches;   /* engine kernels launched since the handle's
                                  creation or last lv_clear_stats (counted
                                  process-wide)                              */
} lv_stats;

/* Per work-class kernel timing (filled when opts.profile = 1). */
#define LV_NUM_CLASSES 9
typedef struct lv_class_stats {
    int64_t launches[LV_NUM_CLASSES];
    int64_t vertices[LV_NUM_CLASSES];
    int64_t edges[LV_NUM_CLASSES];
    double ms[LV_NUM_CLASSES];
    double bytes[LV_NUM_CLASSES];   /* algorithmic bytes: 12 per edge, 20 per vertex
                                       (col, weight and community gather as 4 bytes
                                       each; row offset, own community, k_i,
                                       Sigma_tot[own] and new community)           */
    double stored_bytes[LV_NUM_CLASSES]; /* the same with the stored weight width:
                                            8 + 4 or 8 bytes per edge            */
} lv_class_stats;

void lv_default_opts(lv_opts *opts);
const char *lv_status_string(int status);
const char *lv_version(void);

/* Create an engine from a HOST CSR (symmetric, as produced by the MTX reader).
 * Replaces copyStructures (utils.cu:64-106) + initM
 * (modularity_optimisation.cu:420-422): device allocation, host->device copy
 * and M.  rowptr has V+1 entries, col/w have E entries, E < 2^31. */
int lv_create(const int32_t *rowptr, const int32_t *col, const float *w, int32_t V, int64_t E,
              const lv_opts *opts, lv_handle **out);
/* Same, for a CSR already resident in device memory.  The arrays are
 * borrowed (not copied) and must stay valid and unchanged until
 * lv_destroy. */
int lv_create_device(const int32_t *d_rowptr, const int32_t *d_col, const float *d_w, int32_t V,
                     int64_t E, const lv_opts *opts, lv_handle **out);
/* Return to level 0 with singleton communities (no reallocation). */
int lv_reset(lv_handle *h);
/* deleteStructures (utils.cu:108-141).  The handle's device memory goes back
 * to the library's per-device memory pool, which keeps it mapped so that the
 * next handle on that device reuses it instead of allocating again; call
 * lv_trim_device_memory to return it to the system. */
int lv_destroy(lv_handle *h);
/* Release the device memory that destroyed handles left in the library's pool
 * for `device` (memory of live handles is untouched).  No counterpart in the
 * reference, which allocates and frees per call. */
int lv_trim_device_memory(int32_t device);
const char *lv_last_error(const lv_handle *h);

/* optimiseModularity (modularity_optimisation.cuh:28): sweeps of the current
 * level until a sweep gains less than min_gain; *changed = 1 when any sweep
 * gained (> 0), which is when the reference aggregates. */
int lv_optimise_level(lv_handle *h, float min_gain, int32_t *changed);
/* aggregateCommunities (community_aggregation.cuh:11): contract communities
 * into the next level's vertices. */
int lv_aggregate(lv_handle *h);
/* calculateModularity (modularity_optimisation.cuh:30) of the current state,
 * computed exactly and returned in FP64. */
int lv_modularity(lv_handle *h, double *q);
/* The level loop + final modularity of main() (gpulouvain.cu:30-37). */
int lv_run(lv_handle *h, float min_gain, double *q);

/* One sweep (the 7 degree-bucket sub-rounds) at the current level. */
int lv_sweep(lv_handle *h, int64_t *moves);

/* Original vertex -> final community (the data printed by
 * printOriginalToCommunity, modularity_optimisation.cu:403-418); out has
 * V0 entries; *num_communities = vertex count of the current level. */
int lv_get_original_to_community(lv_handle *h, int32_t *out, int32_t *num_communities);
/* Current level: vertex -> community (out has V entries). */
int lv_get_communities(lv_handle *h, int32_t *out);
/* Test hook: set the current level's communities (Sigma_tot and sizes are
 * recomputed), e.g. to drive lv_aggregate from a given community vector. */
int lv_set_communities(lv_handle *h, const int32_t *comm);
int lv_get_level_info(lv_handle *h, int32_t *V, int64_t *E, int32_t *level);
/* The current level's work classes (LV_NUM_CLASSES entries each): vertices
 * and CSR entries per class (degree (0,4], (4,8], (8,16], (16,32], (32,84],
 * (84,319], (319,1024], (1024,giant_degree], above giant_degree). */
int lv_get_level_classes(lv_handle *h, int32_t *vertices, int64_t *entries);
/* "name (sm_XY, N SMs)" of a CUDA device (the autotuner's cache key). */
int lv_get_device_name(int32_t device, char *name, int32_t len);
/* Test hook: current level CSR; weights as fixed-point integers
 * (value = wfix / 2^scale).  Any pointer may be NULL. */
int lv_get_csr(lv_handle *h, int32_t *rowptr, int32_t *col, int64_t *wfix);
int lv_get_scale(lv_handle *h, int32_t *scale, uint64_t *total_weight, int32_t *exact);
int lv_get_stats(lv_handle *h, lv_stats *stats);
int lv_get_class_stats(lv_handle *h, lv_class_stats *stats);
int lv_clear_stats(lv_handle *h);

/* ---- host-side I/O (no GPU needed) ---- */

/* readInputData (utils.cu:9-62): symmetric Matrix Market -> CSR in file
 * order (both directions for off-diagonal entries, self-loops once).  The
 * file is memory-mapped; large files with one entry per line are parsed by
 * all host threads, other layouts by the reference's token-stream reading
 * (same result either way).
 * Arrays are malloc'd; release with lv_free_host.  m_ref receives M as the
 * reference accumulates it (FP32, sequential). */
int lv_read_mtx(const char *path, int32_t *V, int64_t *E, int32_t **rowptr, int32_t **col,
                float **w, float *m_ref);
/* lv_read_mtx with the CSR built on the device (no counterpart in the
 * reference, whose CSR is built on the host, utils.cu:32-59): the file is
 * parsed on the host as lv_read_mtx parses it, and lv_csr_from_entries_device
 * builds the same CSR (same rows, same order) in device memory allocated by
 * the library on `device` (free with lv_free_device).  m_ref (may be NULL)
 * as for lv_read_mtx. */
int lv_read_mtx_device(const char *path, int32_t device, int32_t *V, int64_t *E, int32_t **d_rowptr,
                       int32_t **d_col, float **d_w, float *m_ref);
/* The parsed entries of a Matrix Market file in file order (0-based
 * v1[i], v2[i], w[i]; unit weights for pattern files) and the vertex count:
 * what lv_read_mtx reads before building its CSR.  Arrays are malloc'd
 * (lv_free_host). */
int lv_read_mtx_entries(const char *path, int32_t *V, int64_t *nnz, int32_t **v1, int32_t **v2, float **w);
/* CSR on the device from nnz Matrix Market entries (host arrays, 0-based,
 * file order) with the reference's conventions: entry (v1, v2, w) appends
 * (v2, w) to row v1 and, unless v1 == v2, (v1, w) to row v2; rows keep file
 * order.  Directed entries are numbered by a scan and stably radix-sorted by
 * row on the device.  Entries outside [0, V) give LV_ERR_INVALID. */
int lv_csr_from_entries_device(int32_t device, int32_t V, int64_t nnz, const int32_t *v1, const int32_t *v2,
                               const float *w, int64_t *E, int32_t **d_rowptr, int32_t **d_col, float **d_w);
/* Binary CSR file, a cache for lv_read_mtx's output (no counterpart in the
 * reference, which parses the text file on every run): header "LVCSR002",
 * V and E (int64), m_ref (float), 4 pad bytes, the size and the modification
 * time in nanoseconds of the file the CSR came from (int64; 0 = unknown),
 * then rowptr[V+1], col[E] (int32) and w[E] (float32), little-endian.
 * lv_read_csr checks the header, the file size, the offsets and the column
 * range (LV_ERR_IO otherwise); arrays are malloc'd (lv_free_host).
 * lv_write_csr writes a zero source stamp; lv_write_csr_stamped records
 * one, and lv_read_csr_stamp reads it back (header only), so a cache can be
 * trusted only when its source's size and modification time still match. */
int lv_write_csr(const char *path, int32_t V, int64_t E, const int32_t *rowptr, const int32_t *col,
                 const float *w, float m_ref);
int lv_write_csr_stamped(const char *path, int32_t V, int64_t E, const int32_t *rowptr, const int32_t *col,
                         const float *w, float m_ref, int64_t src_size, int64_t src_mtime_ns);
int lv_read_csr(const char *path, int32_t *V, int64_t *E, int32_t **rowptr, int32_t **col, float **w,
                float *m_ref);
int lv_read_csr_stamp(const char *path, int64_t *src_size, int64_t *src_mtime_ns);
/* Write an undirected edge list as symmetric Matrix Market (i > j, 1-based). */
int lv_write_mtx(const char *path, int32_t V, int64_t n_edges, const int32_t *u, const int32_t *v,
                 const float *w);
void lv_free_host(void *p);

/* Print the verbose map exactly as printOriginalToCommunity
 * (modularity_optimisation.cu:403-418): first line = num_communities, then
 * one line per community c: "c+1 m1+1 m2+1 ...".  path NULL = stdout. */
int lv_print_communities(const char *path, const int32_t *orig2comm, int32_t V0,
                         int32_t num_communities);

/* ---- seeded synthetic graphs (host, OpenMP) ----
 * Output CSR rows are sorted by neighbour id; arrays malloc'd.
 * R-MAT: ef * 2^scale draws with quadrant probabilities a, b, c,
 * self-loops and duplicates removed, symmetrised; weight_mode 0 = unit,
 * 1 = uniform [0.5, 1.5) on the 2^-24 grid. */
int lv_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b, double c,
                int32_t weight_mode, int32_t *V, int64_t *E, int32_t **rowptr, int32_t **col,
                float **w);
/* Planted partition: V vertices in `blocks` equal blocks, round(V*d_in/2)
 * intra-block and round(V*d_out/2) inter-block uniform draws. */
int lv_gen_planted(int32_t V, int32_t blocks, double d_in, double d_out, uint64_t seed,
                   int32_t weight_mode, int64_t *E, int32_t **rowptr, int32_t **col, float **w);
/* G planted-partition graphs (graph i as lv_gen_planted(V[i], blocks[i],
 * d_in[i], d_out[i], seeds[i], weight_mode)) generated by all host threads
 * into one block-diagonal CSR: graph i's vertices are
 * [graph_ptr[i], graph_ptr[i+1]) and its columns are offset by graph_ptr[i]
 * (the layout lv_batch_create takes).  Arrays are malloc'd (lv_free_host). */
int lv_gen_planted_batch(int32_t G, const int32_t *V, const int32_t *blocks, const double *d_in,
                         const double *d_out, const uint64_t *seeds, int32_t weight_mode, int32_t *Vtot,
                         int64_t *Etot, int32_t **rowptr, int32_t **col, float **w, int32_t **graph_ptr);
/* LFR-like benchmark graph (Lancichinetti-Fortunato-Radicchi construction,
 * simplified): power-law degrees (exponent tau1, mean mean_degree, at most
 * kmax), power-law community sizes (exponent tau2, in [cmin, cmax]), mixing
 * parameter mu (fraction of each vertex's stubs outside its community),
 * random stub pairing, unit weights, vertex ids permuted.  comm (may be NULL)
 * receives the planted community of each vertex (malloc'd). */
int lv_gen_lfr(int32_t V, double tau1, double mean_degree, int32_t kmax, double tau2, int32_t cmin,
               int32_t cmax, double mu, uint64_t seed, int64_t *E, int32_t **rowptr, int32_t **col,
               float **w, int32_t **comm);
/* R-MAT drawn on the device into device buffers allocated by the library
 * (free with lv_free_device); same graph as lv_gen_rmat. */
int lv_gen_rmat_device(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b,
                       double c, int32_t weight_mode, int32_t device, int32_t *V, int64_t *E,
                       int32_t **d_rowptr, int32_t **d_col, float **d_w);
void lv_free_device(void *p);

/* ---- allocation-free modularity of a given partition ----
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they need the value: a process whose device memory is all
 * owned by another allocator (a framework's caching allocator, or a pool
 * sized to the whole GPU), or a latency-critical loop that cannot take the
 * device-wide synchronisation of cudaMalloc / cudaFree.  Returns the same
 * modularity as lv_create_device + lv_set_communities + lv_modularity for a
 * level-0 device CSR (as lv_create_device takes it) and a device array
 * d_comm of V community ids in [0, V).  V = 0 with E > 0 is a malformed CSR
 * (LV_ERR_INVALID), as for lv_create_device.
 *
 * Working memory is a fixed array inside the library (about 8 MiB per
 * device, held by every GPU that loads the library until exit), so V may be
 * at most LV_NOALLOC_MAX_VERTICES; larger V returns LV_ERR_TOO_LARGE.  No
 * device memory is allocated.  Runs on the calling thread's current device
 * and on `stream` (a cudaStream_t; NULL = the default stream), and
 * synchronises that stream before returning.  Every call looks up the
 * array's device address on the current device (nothing is kept between
 * calls, so a device reset between calls is harmless).  All calls on one
 * device share the array, which keeps the last call's contents (each call
 * clears what it sums into), so calls that overlap on the GPU (other threads
 * or streams) race and must be serialised by the caller.  On failure a message is written to err (may be
 * NULL) of err_len bytes. */
#define LV_NOALLOC_MAX_VERTICES (1 << 20)
int lv_modularity_noalloc(const int32_t *d_rowptr, const int32_t *d_col, const float *d_w, int32_t V,
                          int64_t E, const int32_t *d_comm, void *stream, double *q, char *err,
                          int32_t err_len);

/* ---- learned active-set proposal ----
 * No counterpart in the reference.  A per-vertex move predictor (MLP with
 * LV_ACTIVE_FEATURES inputs, LV_ACTIVE_HIDDEN ReLU units and one logit;
 * bf16 weights, fp32 accumulation) proposes which vertices to evaluate in a
 * sweep.  Parameters, as bf16 bit patterns, in the order W1[HIDDEN][FEATURES],
 * b1[HIDDEN], W2[HIDDEN], b2.  Features of a vertex: log2(1 + degree) / 16,
 * the fraction of its weight into its own community and its best move's gain
 * relative to T k (both from its last evaluation), whether it moved in the
 * previous sweep, and the fraction of its row entries whose vertex moved in
 * the previous sweep. */
#define LV_ACTIVE_FEATURES 5
#define LV_ACTIVE_HIDDEN 16
#define LV_ACTIVE_MODEL_SIZE (LV_ACTIVE_HIDDEN * LV_ACTIVE_FEATURES + 2 * LV_ACTIVE_HIDDEN + 1)
/* Model for lv_opts.active_set = 1; a vertex is proposed when its logit
 * exceeds logit_threshold. */
int lv_set_active_model(lv_handle *h, const uint16_t *model, int32_t n_params, float logit_threshold);
/* Read a predictor file as train_active_set.py writes it (JSON with
 * "model_bf16": [LV_ACTIVE_MODEL_SIZE bit patterns], "logit_threshold" and
 * the settings it was measured with, "full_every", "active_start",
 * "min_recall").  model receives the parameters (cap >= LV_ACTIVE_MODEL_SIZE),
 * *n_params their count, *logit_threshold the threshold; when opts is not
 * NULL, active_set is set to 1 and the three settings present in the file
 * are copied into it.  Host only (no device is touched).  LV_ERR_IO for a
 * missing or malformed file, LV_ERR_INVALID for a parameter count other than
 * LV_ACTIVE_MODEL_SIZE. */
int lv_read_active_model(const char *path, uint16_t *model, int32_t cap, int32_t *n_params,
                         float *logit_threshold, lv_opts *opts);
/* Move traces recorded with lv_opts.trace_sample > 0: features[n][FEATURES]
 * and labels[n] (1 = moved in the sweep after sampling); up to cap rows are
 * copied, *n receives the number of complete rows available. */
int lv_get_traces(lv_handle *h, float *features, uint8_t *labels, int64_t cap, int64_t *n);
/* Learned-mode counters since the handle's creation or lv_clear_stats: vertices evaluated,
 * full and active sweeps, the last measured recall, and whether the plain
 * sweep took over in some level. */
int lv_get_active_stats(lv_handle *h, int64_t *evaluated, int64_t *full_sweeps, int64_t *active_sweeps,
                        double *last_recall, int32_t *fell_back);
/* Train the predictor on traces (features[n][FEATURES], labels[n]) with
 * mini-batch Adam on the weighted binary cross-entropy (positives weighted
 * by pos_weight) on `device`; hand-written CUDA kernels, reproducible for a
 * seed.  model_out receives LV_ACTIVE_MODEL_SIZE bf16 parameters,
 * epoch_loss (may be NULL) the mean loss of each epoch. */
int lv_active_train(const float *features, const uint8_t *labels, int64_t n, int32_t epochs, int32_t batch,
                    float lr, float pos_weight, uint64_t seed, int32_t device, uint16_t *model_out,
                    float *epoch_loss);
/* Logits of the predictor for features[n][FEATURES] (the engine's inference
 * arithmetic). */
int lv_active_predict(const uint16_t *model, const float *features, int64_t n, int32_t device, float *logits);
/* ---- batches of independent graphs ----
 * No counterpart in the reference, whose CLI runs one graph per process.  A
 * batch is one block-diagonal CSR of num_graphs graphs: graph g owns vertices
 * graph_ptr[g] .. graph_ptr[g+1]-1 (graph_ptr is a HOST array of num_graphs+1
 * nondecreasing offsets, graph_ptr[0] = 0, graph_ptr[num_graphs] = V) and its
 * rows reference only its own vertices.  lv_batch_run runs the level loop of
 * lv_run on every graph in one persistent launch (one CTA per graph at a time,
 * largest graphs first); each graph's communities, modularity, level and sweep
 * counts equal those of lv_create + lv_run on that graph alone.  Each graph
 * gets its own fixed-point scale, as lv_create would choose it.  Whole-CSR
 * errors (offsets, column range, weights, a graph of more than
 * LV_BATCH_MAX_GRAPH_VERTICES vertices) fail lv_batch_create; per-graph
 * errors (a row that leaves its graph, a total weight beyond the fixed grid,
 * a failed device check) are reported per graph, and lv_batch_run then
 * returns LV_ERR_DEVICE with the other graphs' results still valid.  opts:
 * device and max_sweeps are used. */
#define LV_BATCH_MAX_GRAPH_VERTICES (1 << 29)   /* per graph of a batch */
typedef struct lv_batch lv_batch;
int lv_batch_create(const int32_t *rowptr, const int32_t *col, const float *w, int32_t V, int64_t E,
                    const int32_t *graph_ptr, int32_t num_graphs, const lv_opts *opts, lv_batch **out);
/* Same for a CSR resident in device memory (borrowed until lv_batch_destroy);
 * graph_ptr is still a host array. */
int lv_batch_create_device(const int32_t *d_rowptr, const int32_t *d_col, const float *d_w, int32_t V,
                           int64_t E, const int32_t *graph_ptr, int32_t num_graphs, const lv_opts *opts,
                           lv_batch **out);
/* Run every graph from singleton communities (each run starts afresh). */
int lv_batch_run(lv_batch *b, float min_gain);
/* communities[V]: final community of each vertex, numbered 0 .. n_g - 1 within
 * its graph (-1 for a failed graph); modularity[G], num_communities[G] (n_g),
 * status[G] (lv_status per graph).  Any pointer may be NULL. */
int lv_batch_get_results(lv_batch *b, int32_t *communities, double *modularity, int32_t *num_communities,
                         int32_t *status);
/* Per graph: levels, sweeps, edge-sweeps (sum over sweeps of the level's CSR
 * size) and device latency from the graph's start to its end inside the
 * launch (ms).  Any pointer may be NULL. */
int lv_batch_get_graph_stats(lv_batch *b, int32_t *levels, int64_t *sweeps, int64_t *edge_sweeps,
                             double *latency_ms);
/* Last run: device time of the launch (ms, CUDA events), total edge-sweeps
 * and vertex-sweeps (sums over sweeps of the level's entries / vertices), and
 * the number of CTAs launched.  Any pointer may be NULL. */
int lv_batch_get_stats(lv_batch *b, double *device_ms, int64_t *edge_sweeps, int64_t *vertex_sweeps,
                       int32_t *ctas);
const char *lv_batch_last_error(const lv_batch *b);
int lv_batch_destroy(lv_batch *b);
#ifdef __cplusplus
}
#endif
#endif
