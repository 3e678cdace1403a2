// lv_internal.h -- launchers shared between the engine's translation units.
#pragma once
#include "lv_common.cuh"

namespace lv {

// Layout of the global-memory hash tables of class CLS_HG (degree > 4096)
// for the current level.  Hubs are split into edge chunks (insert kernel)
// and chunks of their occupied-slot list (evaluate kernel) so that one hub
// spreads over many CTAs; a hub of degree d has at most d occupied slots.
#ifndef LV_HG_EDGE_CHUNK
#define LV_HG_EDGE_CHUNK 2048
#endif
constexpr int HG_EDGE_CHUNK = LV_HG_EDGE_CHUNK;   // aggregation: entries per insert CTA
constexpr int HG_SLOT_CHUNK = 4096;   // table slots per evaluation CTA
constexpr int HG_INSERT_THREADS = 512;
constexpr int HG_INSERT_SMEM = 2 * HG_EDGE_CHUNK * 12;   // chunk-local table
// move phase, giant vertices: chunks of STAGE_CHUNK edges reduced by
// STAGE_THREADS-thread CTAs in a 2*STAGE_CHUNK-slot table
// entries per staging chunk: 1024 (the persistent staging kernels then hold
// twice as many CTAs per SM; the giants of an R-MAT-24 run took 50.4 against
// 51.8 ms with 2048)
#ifndef LV_STAGE_CHUNK
#define LV_STAGE_CHUNK 1024
#endif
constexpr int STAGE_CHUNK = LV_STAGE_CHUNK;
constexpr int STAGE_THREADS = 256;
constexpr int STAGE_SMEM = 2 * STAGE_CHUNK * 14;
constexpr int HG_MERGE_THREADS = 1024;
constexpr int HG_MERGE_CAP = 16384;                      // shared slots of the per-hub merge
constexpr int HG_MERGE_SMEM = HG_MERGE_CAP * 14;
// giants with at most MERGE_S_CAP / 2 staged pairs are merged by smaller CTAs
constexpr int MERGE_S_THREADS = 256, MERGE_S_CAP = 2048;
#ifndef LV_MERGE_SMALL
#define LV_MERGE_SMALL 1
#endif


// Slot of the aggregation's global hash tables: the key (stored plus one, so
// that an all-zero slot is empty) and its sum share one 16-byte slot, so an
// insert's compare-and-swap and add touch one 32-byte DRAM sector instead of
// one in a key array and one in a value array.
struct GSlot {
    uint32_t key1;   // key + 1; 0 = empty
    uint32_t pad;
    u64 val;
};

struct HubGlobal {
    int32_t nhubs = 0;
    int32_t n_echunks = 0;
    int32_t n_schunks = 0;
    const int32_t *hubs = nullptr;        // [nhubs] vertex ids
    const int64_t *tbl_off = nullptr;     // [nhubs] first slot of each hub's table
    const int32_t *tbl_lg = nullptr;      // [nhubs] log2 capacity
    const int32_t *echunk_hub = nullptr;  // [n_echunks]
    const int32_t *echunk_e0 = nullptr;   // [n_echunks] edge offset within the row
    const int32_t *schunk_hub = nullptr;  // [n_schunks]
    const int32_t *schunk_s0 = nullptr;   // [n_schunks] first slot
    const int32_t *hub_schunk0 = nullptr; // [nhubs + 1]
    GSlot *slots = nullptr;               // global tables (all-zero between uses)
    u64 *res_g = nullptr;                 // [2 * n_schunks] best gain (lo, hi)
    int32_t *res_c = nullptr;             // [n_schunks] best community
    u64 *res_e = nullptr;                 // [n_schunks] e_own contribution
    u64 *res_b = nullptr;                 // [n_schunks] weight to the best community
    const int64_t *occ_off = nullptr;     // [nhubs] first entry of each hub's list / staging area
    int32_t *occ = nullptr;               // occupied slots, listed per hub
    int32_t *nocc = nullptr;              // [nhubs] list / staging lengths (kept zero between uses)
    // staged two-level reduction of the move phase (room for deg entries per hub)
    int32_t *stage_key = nullptr;
    u64 *stage_val = nullptr;
    u64 *eown = nullptr;                  // [nhubs] weight to the own community (zero between uses)
    int32_t *ovf_list = nullptr;          // hubs whose staged pairs overflow shared memory
    int32_t *ovf_count = nullptr;         // length of ovf_list (reset by the host per use)
    // staged pairs regrouped by large-queue key partition (move phase): hub h
    // owns poff[pbase[h] .. pbase[h + 1]) = its Pmax + 2 words, Pmax =
    // ceil(hub_cap[h] / FB_KEYS): poff[pbase[h] + p] is the first regrouped
    // pair of partition p (p = 0 .. P), poff[pbase[h + 1] - 1] the P used, and
    // poff[pbase[h]] = -1 when the hub's pairs were not regrouped
    const int32_t *hub_cap = nullptr;     // [nhubs] staging room (the hub's degree)
    const int32_t *pbase = nullptr;       // [nhubs + 1]
    int32_t *poff = nullptr;
    int32_t *stage2_key = nullptr;        // regrouped pairs, same layout as stage_key
    u64 *stage2_val = nullptr;
};

// Device memory from the library's per-device stream-ordered pool (freed
// memory stays mapped for the next handle).
cudaError_t pool_alloc(int dev, void **p, size_t bytes, cudaStream_t s);
void pool_free(int dev, void *p, cudaStream_t s);

// ---- learned active set (lv_active.cu) ----
struct ActiveClassOffsets {
    int32_t off[NCLS + 1];
};
void launch_active_select(const int32_t *list, int32_t n, const ActiveClassOffsets &co, const int32_t *rowptr,
                          const int32_t *rowend, const float *feat, const uint8_t *moved, const int32_t *nmoved,
                          const uint16_t *model, float logit_thr, int keep_cls, int32_t *alist, int32_t *acnt,
                          uint8_t *pred, uint8_t *fresh, cudaStream_t s);
// nmoved[x] = number of row entries of x whose vertex moved (recomputed)
void launch_nbr_moved(const int32_t *rowptr, const int32_t *rowend, const int32_t *col, int32_t V,
                      const uint8_t *moved, int32_t *nmoved, cudaStream_t s);
void launch_active_moved(const int32_t *comm, const int32_t *prev, int32_t V, uint8_t *moved, const uint8_t *pred,
                         uint8_t *fresh, u64 *counts, cudaStream_t s);
void launch_trace_sample(int32_t V, const int32_t *rowptr, const int32_t *rowend, const float *feat,
                         const uint8_t *moved, const int32_t *nmoved, u64 thr, u64 key, float *tx, int32_t *tv,
                         int64_t cap, u64 *tcount, cudaStream_t s);
void launch_trace_label(const int32_t *tv, const uint8_t *moved, int64_t r0, const u64 *tcount, int64_t cap,
                        uint8_t *ty, cudaStream_t s);

// Count of engine kernel launches (all handles, all devices of the process).
void note_launches(int n);
long long launches_total();

// Move phase for degree > 32: warp tables of WARP_CAP slots (a vertex with
// more than WARP_LIMIT distinct neighbour communities falls back).  Fallback
// items go to one of NFBQ row queues by degree (bin b takes degrees up to
// FBQ_MAXDEG(b), with CTAs of FBQ_THREADS(b) threads and shared tables of
// 2 * FBQ_MAXDEG(b) slots), or to the large queue (FB_THREADS threads,
// FB_CAP slots, key-space partitions of FB_KEYS edges).
constexpr int WARP_CAP = 512;
constexpr int WARP_LIMIT = 352;
constexpr int NFBQ = 4;
__host__ __device__ constexpr int FBQ_MAXDEG(int b) { return 512 << b; }                 // 512 .. 4096
// threads per CTA of each row queue: the two large bins hold one or two CTAs
// per SM (their tables take 57 and 114 KB), so they get 512 and 1024 threads
// to keep 32 warps per SM
__host__ __device__ constexpr int FBQ_THREADS(int b) { return b == 0 ? 128 : (b == 1 ? 256 : (b == 2 ? 512 : 1024)); }
// large queue: CTA threads, table slots and keys per partition (the
// partition bound stays below the occupied list's CAP / 2 with room for the
// hash's imbalance).  8192 slots (114 KB, leaving 124 KB of L1) measured
// slower than 16384 (229 KB): 123.6 against 119.7 ms for the degree > 319
// class, 56.1 against 55.0 ms for the giants of an R-MAT-24 run.
#ifndef LV_FB_CAP
#define LV_FB_CAP 16384
#endif
constexpr int FB_THREADS = 1024, FB_CAP = LV_FB_CAP;
constexpr int FB_KEYS = FB_CAP / 16 * 7;
constexpr int FB_SMEM = FB_CAP * 14;   // table + occupied list
// LV_WARP_PAD: extra shared bytes per CTA of the 64-bit warp kernel (0; a
// measurement knob for the shared-memory / L1 split)
#ifndef LV_WARP_PAD
#define LV_WARP_PAD 0
#endif
constexpr int WARP_SMEM = 8 * WARP_CAP * 12 + LV_WARP_PAD;   // 8 warp tables per CTA

// A fallback work list (device memory; count and next are adjacent).
struct Fallback {
    int32_t *count = nullptr;   // items queued
    int32_t *next = nullptr;    // next item to take (= count + 1)
    int32_t cap = 0;
    int32_t *v = nullptr, *p = nullptr, *P = nullptr, *first = nullptr;
    int32_t *src = nullptr;     // -1: the vertex's row; h >= 0: staged pairs of giant h
    int32_t *done = nullptr;    // per first item, zero between uses
    double *gd = nullptr;
    u64 *e = nullptr, *S = nullptr, *eo = nullptr;
    int32_t *c = nullptr;
    int32_t *cnt = nullptr;     // distinct communities seen by the item
};

// The fallback queues and the per-vertex hint "had more than 3/4 of
// warp_limit distinct neighbour communities at its last evaluation" (such a
// vertex of degree > warp_limit skips the warp attempt; the hint only routes
// work, results do not depend on it).  warp_limit: distinct communities after
// which the warp kernel hands a vertex to a fallback CTA (a tuning knob,
// lv_opts.warp_limit, at most WARP_LIMIT_MAX so that every claim fits the
// warp table).
constexpr int WARP_LIMIT_MIN = 32, WARP_LIMIT_MAX = 384;
struct FallbackSet {
    Fallback q[NFBQ + 1];   // row queues by degree, then the large queue
    uint8_t *hint = nullptr;
    int32_t *warp_next = nullptr;   // the warp kernels' vertex cursor (follows the queues' counters)
    int32_t warp_limit = 352;
    int32_t hint_set = 264;   // hint = distinct count above this
};

// Launch geometry helpers (filled once per device).
struct DeviceInfo {
    int sms = 148;
    int occ_warp = 4;   // resident CTAs per SM of the warp kernel
    int occ_warp_narrow = 4;   // ... of its narrow-weight form
    int occ_fbq[NFBQ] = {1, 1, 1, 1};   // ... of the row fallback kernels
    int occ_fbq_narrow[NFBQ] = {1, 1, 1, 1};   // ... and of their narrow-weight form
    int occ_fbq_staged[NFBQ] = {1, 1, 1, 1};   // ... and of its bulk-copy row-staging form
    int occ_merge_s = 1;                 // ... of the small giant-merge kernel
    int occ_stage_narrow = 1;            // ... of the persistent narrow staging kernel
    int occ_stage = 1;                   // ... and of the persistent 64-bit one
};
void init_kernel_attributes(DeviceInfo &di);

// ---- move phase (lv_move.cu) ----
// dE accumulates (wrapping uint64) each mover's 2 (e_best - e_own).
// Classes B0..B3 (degree <= 32): group kernels.
template <typename WT>
void launch_move_class(int cls, const GraphView<WT> &g, const StateView &st, const int32_t *list,
                       int32_t n, const DeviceInfo &di, u64 *dE, cudaStream_t s, bool narrow,
                       const FallbackSet &fb);
// 32 < degree <= 8192 (the vertices of one update bucket): warp kernel +
// fallback.  Degree > 8192: staged chunks + merge (hg describes the giants).
// narrow: every weight the kernels read is below 2^32 (piece-counter tables).
template <typename WT>
void launch_move_wide(const GraphView<WT> &g, const StateView &st, const int32_t *list, int32_t n,
                      const FallbackSet &fb, const DeviceInfo &di, u64 *dE, cudaStream_t s,
                      int32_t max_degree, bool narrow);
template <typename WT>
void launch_move_giants(const GraphView<WT> &g, const StateView &st, const HubGlobal &hg,
                        const FallbackSet &fb, const DeviceInfo &di, u64 *dE, cudaStream_t s, bool narrow);
// Exact correction of dE for neighbours that moved in the same sub-round.
template <typename WT>
void launch_correction(int cls, const GraphView<WT> &g, const StateView &st, const int32_t *list,
                       int32_t n, const DeviceInfo &di, u64 *dE, cudaStream_t s);
void launch_commit(const StateView &st, const int32_t *list, int32_t n, u64 *moves,
                   cudaStream_t s);

// k_i = row sums (mode 0) or e_own total (mode 1) over the vertices of one class.
template <typename WT>
void launch_row_reduce(int cls, int mode, const GraphView<WT> &g, const int32_t *comm, u64 *k,
                       u64 *total, const int32_t *list, int32_t n, const DeviceInfo &di,
                       cudaStream_t s);
void launch_s2(const u64 *S, int32_t V, u64 *total_hi_lo, cudaStream_t s);

// ---- primitives (lv_prims.cu) ----
// Exclusive scan of n int32 values (out may alias in); writes the total to
// *total_dev.  tmp must hold scan_tmp_elems(n) int32.
int64_t scan_tmp_elems(int64_t n);
void scan_exclusive_i32(const int32_t *in, int32_t *out, int64_t n, int32_t *total_dev,
                        int32_t *tmp, cudaStream_t s);
// Degree classification of vertices: counts[NCLS] then scatter into list.
// The count buffer holds CLASS_COUNT_WORDS int32: NCLS vertex counts, then
// (8-byte aligned) NCLS uint64 edge totals.
constexpr int CLASS_COUNT_WORDS = NCLS + (NCLS & 1) + 2 * NCLS;
void launch_class_count(const int32_t *rowptr, const int32_t *rowend, int32_t V, int32_t giant_degree,
                        int32_t *counts, cudaStream_t s);
void launch_class_scatter(const int32_t *rowptr, const int32_t *rowend, int32_t V, int32_t giant_degree,
                          int32_t warp_limit, const int32_t *offsets, int32_t *cursors, int32_t *list,
                          uint8_t *hint, cudaStream_t s);
// Reorder list[0, n) by decreasing row length (the warp kernels take their
// vertices from a shared cursor, so the longest rows start first): keys,
// keys_alt and vals_alt hold n int32 each, temp sort_by_degree_temp_bytes.
size_t sort_by_degree_temp_bytes(int32_t n, int32_t maxdeg);
void sort_by_degree_desc(const int32_t *rowptr, const int32_t *rowend, int32_t *list, int32_t n, int32_t maxdeg,
                         int32_t *keys, int32_t *keys_alt, int32_t *vals_alt, void *temp, size_t temp_bytes,
                         cudaStream_t s);
void launch_fill_i32(int32_t *p, int64_t n, int32_t v, cudaStream_t s);
void launch_iota_i32(int32_t *p, int64_t n, cudaStream_t s);
void launch_level_init(int32_t *comm, int32_t *newc, int32_t *size, const u64 *k, u64 *S,
                       int32_t V, cudaStream_t s);
void launch_set_communities(const int32_t *comm_in, int32_t *comm, int32_t *newc, int32_t *size,
                            const u64 *k, u64 *S, int32_t V, int *err, cudaStream_t s);
void launch_compose_map(int32_t *orig2comm, const int32_t *map, int32_t V0, cudaStream_t s);
template <typename WT>
void launch_weights_to_fixed(const WT *w, int64_t E, double scale, int64_t *out, cudaStream_t s);

// Fixed-point scale analysis of float weights: out[0] = max fractional bits,
// out[1] = max floor(log2 w) + 1024 (0 if no positive weight), out[2] = error flags.
void launch_weight_scan(const float *w, int64_t E, int32_t *out, cudaStream_t s);
void launch_total_weight(const float *w, int64_t E, double scale, u64 *total, cudaStream_t s);
// CSR validation: error bit 1 bad offsets, 2 bad column.
void launch_validate_csr(const int32_t *rowptr, const int32_t *col, int32_t V, int64_t E,
                         int *err, cudaStream_t s);

// ---- aggregation (lv_agg.cu) ----
struct AggBuffers {
    int32_t *flag;      // [V]   nonempty flag, then new id (exclusive scan)
    int32_t *cdeg;      // [V]   community degree bound, then merged row start (scan)
    int32_t *mstart;    // [V+1] member start per old community (scan of size)
    int32_t *cursor;    // [V]   member cursor / row counter
    int32_t *members;   // [V]   vertices grouped by community
    int32_t *lab;       // [V]   new id of each vertex's community
    int32_t *clist;     // [V]   nonempty communities grouped by merge class
    int32_t *newdeg;    // [V]   distinct neighbours per new vertex
    int32_t *epos_new;  // [V]   merged-row start per new vertex
    int32_t *scan_tmp;
    int32_t *scalars;   // [16]  device scalars (totals, counts)
};

}  // namespace lv
