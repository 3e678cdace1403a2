// lv_engine.cu -- the engine handle, the level loop and the C ABI.
//
// Host orchestration of one Louvain run on one GPU (replaces main()'s level
// loop, gpulouvain.cu:30-37, optimiseModularity,
// modularity_optimisation.cu:284-363, and aggregateCommunities,
// community_aggregation.cu:248-347).  All state lives in device memory; the
// host reads back one small totals record per sweep (the sweep's modularity
// parts, its move count and the device error word) and a few counts per
// level.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/louvain_b200.h"
#include "lv_internal.h"

namespace lv {
void init_agg_attributes();
void agg_prepare(const int32_t *rowptr, const int32_t *rowend, const int32_t *comm,
                 const int32_t *size, int32_t V, AggBuffers &ab, int32_t *mslot, int32_t *degm,
                 int32_t *P, cudaStream_t s);
void agg_classify(const int32_t *size, int32_t V, AggBuffers &ab, const int32_t *P,
                  const int32_t *offsets, cudaStream_t s);
template <typename WT>
void agg_permute(int cls, const GraphView<WT> &g, const AggBuffers &ab, const int32_t *mslot,
                 const int32_t *P, const int32_t *list, int32_t n, int32_t *vkey, u64 *vw, int sms,
                 cudaStream_t s);
void agg_new_vertices(const int32_t *size, const u64 *S, int32_t V, const AggBuffers &ab,
                      const int32_t *P, u64 *knew, cudaStream_t s);
void agg_merge_class(int acls, const AggBuffers &ab, const int32_t *P, const int32_t *list,
                     int32_t n, int32_t *vkey, u64 *vw, uint32_t *vw32, int *err, int *hiflag, uint8_t *wrow,
                     int sms, cudaStream_t s, bool narrow);
void agg_merge_global(const HubGlobal &hg, const AggBuffers &ab, const int32_t *P, int32_t *vkey,
                      u64 *vw, uint32_t *vw32, int *err, int *hiflag, uint8_t *wrow, cudaStream_t s,
                      bool narrow);
void agg_row_bounds(const AggBuffers &ab, int32_t Vn, int32_t *start, int32_t *end, cudaStream_t s);
void launch_gather_degrees(const int32_t *rowptr, const int32_t *rowend, const int32_t *list,
                           int32_t n, int32_t *out, cudaStream_t s);
void launch_gather_cdeg(const int32_t *mstart, const int32_t *P, const int32_t *list, int32_t n,
                        int32_t *out, cudaStream_t s);
}  // namespace lv

using namespace lv;

// Aggregated levels holding a sum of 2^32 or more: swept with the 64-bit
// kernels on the uint64 sums (0), through the 32-bit view with the narrow
// (piece-table) kernels and those rows sent to the large queue (1), or
// through the 32-bit view with the 64-bit-table kernels, escaped sums read
// from the uint64 copy (2).  0 is the default: on R-MAT-24 the move phase of
// a run took 241 ms in mode 0, 262 ms in mode 1 (the piece tables' two
// atomics per add serialise where many lanes add to one community) and
// 256 ms in mode 2 (the escape test per entry costs more than the 4 bytes
// per entry it saves).
#ifndef LV_NARROW_ESCAPES
#define LV_NARROW_ESCAPES 0
#endif

namespace {

constexpr int NAC = 5;   // aggregation merge classes (lv_agg.cu)
// cls_scratch layout: class counts, class cursors, then V0 int32 of scratch.
constexpr int SCRATCH_OFF = CLASS_COUNT_WORDS + NCLS + 8;

struct Totals {
    u64 e_own;   // full pass: sum_i e_{i->C(i)}
    u64 s2[2];   // hi, lo of sum_C Sigma_tot^2
    u64 moves;
    u64 dE;      // exact change of e_own over the sweep (wrapping)
    int err;
    int pad;
};

struct Pending {
    int kind;   // 0..NCLS-1 class, 100 move phase, 101 modularity, 102 aggregate, 103 setup
    cudaEvent_t a, b;
    double bytes;    // algorithmic: 12 per edge + 20 per vertex
    double sbytes;   // as stored: 8 + weight width per edge + 20 per vertex
    int64_t verts, edges;
};

struct HubLayout {
    HubGlobal view;
    void *dev = nullptr;   // packed index arrays
    size_t dev_bytes = 0;
    std::vector<int32_t> ids;
};

}  // namespace

struct lv_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    lv_opts opts{};
    std::string err;
    DeviceInfo di;

    int32_t V0 = 0;
    int64_t E0 = 0;
    bool owns_input = false;
    int32_t *in_rowptr = nullptr, *in_col = nullptr;
    float *in_w = nullptr;
    int scale = 0;
    double scale_d = 1.0;
    u64 T = 0;
    int exact = 1;
    bool w0_narrow = false;   // level-0 fixed-point weights are all below 2^32
    int32_t giant_degree = HG_MIN_DEG;   // work-mapping knobs (lv_opts.giant_degree, warp_limit)

    int level = 0;
    int32_t V = 0;
    int64_t E = 0;
    // current level: row v = cur_col/cur_w[cur_rowptr[v] .. cur_rowend[v])
    int32_t *cur_rowptr = nullptr, *cur_rowend = nullptr, *cur_col = nullptr;
    u64 *cur_w = nullptr;   // nullptr at level 0 (float input weights)
    uint32_t *cur_w32 = nullptr;   // 32-bit copy of cur_w (sums of 2^32 or more escaped to
                                   // cur_w); the move kernels read it, the modularity
                                   // pass and the aggregation read cur_w
    uint8_t *wrow = nullptr;       // [V0] current level: row holds a non-self-loop sum >= 2^32
    bool wrows_any = false;

    // aggregated levels, ping-pong: rows stay where the merge wrote them
    int32_t *lvl_start[2] = {nullptr, nullptr};
    int32_t *lvl_end[2] = {nullptr, nullptr};
    int32_t *lvl_col[2] = {nullptr, nullptr};
    u64 *lvl_w[2] = {nullptr, nullptr};
    uint32_t *lvl_w32[2] = {nullptr, nullptr};
    int cur_buf = -1;

    int32_t *comm = nullptr, *newc = nullptr, *size = nullptr, *orig2comm = nullptr;
    u64 *k = nullptr, *S = nullptr;
    int32_t *list = nullptr;
    int32_t *cls_scratch = nullptr;   // class counts, cursors, then V0 entries of scratch
    int32_t *sort_buf = nullptr;      // 3 V0 int32: keys, keys and values of the degree sort
    void *sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    int32_t cls_off[NCLS + 1] = {0};
    int64_t cls_edges[NCLS] = {0};

    HubLayout hub_move, hub_agg;
    GSlot *tbl_buf = nullptr;
    size_t tbl_slots = 0;
    int32_t *occ_buf = nullptr;    // occupied-slot lists of the global tables
    size_t occ_cap = 0;
    int32_t *nocc_buf = nullptr;   // per-hub list lengths, zero between uses
    size_t nocc_cap = 0;
    int32_t *stage_key = nullptr;  // staging area of the hub path (entries = occ_cap)
    u64 *stage_val = nullptr;
    int32_t *stage2_key = nullptr; // the staged pairs regrouped by key partition (occ_cap)
    u64 *stage2_val = nullptr;
    int32_t *poff_buf = nullptr;   // partition offsets of the regrouped pairs
    size_t poff_cap = 0;
    u64 *eown_buf = nullptr;       // per hub, zero between uses (nocc_cap entries)
    int32_t *ovf_buf = nullptr;    // overflow list (nocc_cap entries) then its count
    bool capturing = false;        // a sweep is being captured into a graph (timers off)
    bool destroying = false;       // lv_destroy: large buffers go to the per-device cache
    std::vector<std::pair<void *, size_t>> big;   // live allocations of at least BIG_BYTES
    void *loop_d = nullptr;        // device state of the graph sweep loop

    bool agg_ready = false;
    AggBuffers ab{};
    int32_t *mslot = nullptr, *degm = nullptr, *P = nullptr;

    FallbackSet fb;

    Totals *tot_d = nullptr;
    Totals *tot_h = nullptr;
    int32_t *small_h = nullptr;   // pinned scratch for counts

    lv_stats st{};
    lv_class_stats cst{};
    long long launch_base = 0;
    // sum_i e_{i->C(i)} of the current state, maintained exactly across sweeps
    u64 e_own_cur = 0;
    bool e_own_valid = false;
    std::vector<cudaEvent_t> ev_free;
    std::vector<Pending> pend;

    // learned active set and move traces
    float *feat = nullptr;          // [2 V0] features recorded by the move kernels
    uint8_t *moved = nullptr;       // [V0] moved in the previous sweep
    int32_t *nmoved = nullptr;      // [V0] row entries whose vertex moved in the previous sweep
    uint8_t *pred = nullptr;        // [V0] proposed by the predictor
    uint8_t *fresh = nullptr;       // [V0] evaluated in an active sweep since the last full sweep
    int32_t *comm_prev = nullptr;   // [V0] communities before the sweep
    int32_t *alist = nullptr;       // [V0] proposed vertices, at their class's offset
    int32_t *acnt = nullptr;        // [NCLS] proposed vertices per class
    u64 *actr = nullptr;            // [4] movers, proposed movers, trace rows
    uint16_t *model = nullptr;      // [LV_ACTIVE_MODEL_SIZE] bf16 parameters
    bool has_model = false;
    float logit_thr = 0.0f;
    float *tr_x = nullptr;          // trace rows: features, vertex, label
    int32_t *tr_v = nullptr;
    uint8_t *tr_y = nullptr;
    int64_t tr_cap = 0, tr_rows = 0;
    uint64_t tr_sweep = 0;
    int64_t act_evaluated = 0, act_full = 0, act_active = 0;
    double act_recall = -1.0;
    int32_t act_fell_back = 0;
};

namespace {

int fail(lv_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

#define LV_CUDA(h, call)                                                                   \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess)                                                            \
            return fail((h), e__ == cudaErrorMemoryAllocation ? LV_ERR_NOMEM : LV_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e__));             \
    } while (0)

#define LV_TRY(expr)            \
    do {                        \
        int rc__ = (expr);      \
        if (rc__) return rc__;  \
    } while (0)

// Device memory of every handle comes from one stream-ordered pool per
// device whose release threshold keeps freed memory mapped, so creating a
// handle after another was destroyed reuses the mapping instead of paying
// cudaMalloc/cudaFree for the ~20 GB working set of an R-MAT-24 run again.
// lv_trim_device_memory returns the unused part to the system.
constexpr int LV_MAX_DEVICES = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[LV_MAX_DEVICES] = {};

cudaMemPool_t device_pool(int dev) {
    if (dev < 0 || dev >= LV_MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool[dev]) {
        // an error left pending by an earlier asynchronous call would be
        // reported by the calls below; set-up is retried by the next
        // allocation if it fails
        cudaGetLastError();
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;
        if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
            cudaGetLastError();
            cudaMemPoolDestroy(pool);
            return nullptr;
        }
        g_pool[dev] = pool;
    }
    return g_pool[dev];
}

// Large buffers (at least BIG_BYTES) of destroyed handles are kept per device
// and handed to the next allocation of exactly the same size: handles of the
// same graph ask for the same sizes, so a handle created again reuses its
// predecessor's memory as it is, without the pool having to find or map room
// for it (which, when its free blocks are fragmented, maps new memory and
// costs hundreds of milliseconds for the ~20 GB of an R-MAT-24 handle).
// lv_trim_device_memory releases them.
constexpr size_t BIG_BYTES = size_t(16) << 20;
std::mutex g_cache_mu;
std::vector<std::pair<size_t, void *>> g_cache[LV_MAX_DEVICES];

void *cache_take(int dev, size_t bytes) {
    if (dev < 0 || dev >= LV_MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lock(g_cache_mu);
    auto &c = g_cache[dev];
    for (size_t i = 0; i < c.size(); ++i)
        if (c[i].first == bytes) {
            void *p = c[i].second;
            c[i] = c.back();
            c.pop_back();
            return p;
        }
    return nullptr;
}

// hands every cached buffer of the device back (to the pool, or to the driver
// when the device has no pool); called by lv_trim_device_memory, by each
// lv_destroy before it caches its own buffers (so the cache holds one
// handle's worth at most), and by an allocation that failed
void cache_release(int dev, cudaMemPool_t pool, cudaStream_t stream) {
    if (dev < 0 || dev >= LV_MAX_DEVICES) return;
    std::vector<std::pair<size_t, void *>> cached;
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        cached.swap(g_cache[dev]);
    }
    for (auto &c : cached) {
        if (pool) cudaFreeAsync(c.second, stream);
        else cudaFree(c.second);
    }
}

bool cache_put(int dev, size_t bytes, void *p) {
    if (dev < 0 || dev >= LV_MAX_DEVICES) return false;
    std::lock_guard<std::mutex> lock(g_cache_mu);
    g_cache[dev].emplace_back(bytes, p);
    return true;
}

template <typename T>
int dalloc(lv_handle *h, T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    const size_t bytes = n * sizeof(T);
    if (bytes >= BIG_BYTES) {
        void *c = cache_take(h->device, bytes);
        if (c) {
            *p = (T *)c;
            h->big.emplace_back(c, bytes);
            return LV_OK;
        }
    }
    cudaMemPool_t pool = device_pool(h->device);
    cudaError_t e = pool ? cudaMallocFromPoolAsync((void **)p, bytes, pool, h->stream)
                         : cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cache_release(h->device, pool, h->stream);
        e = pool ? cudaMallocFromPoolAsync((void **)p, bytes, pool, h->stream)
                 : cudaMalloc((void **)p, bytes);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(h, LV_ERR_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    if (bytes >= BIG_BYTES) h->big.emplace_back((void *)*p, bytes);
    return LV_OK;
}

}  // namespace

// The pool for other handle types of the library (lv_batch).
cudaError_t lv::pool_alloc(int dev, void **p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    cudaMemPool_t pool = device_pool(dev);
    const cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s)
                               : cudaMalloc(p, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
    }
    return e;
}

void lv::pool_free(int dev, void *p, cudaStream_t s) {
    if (!p) return;
    if (device_pool(dev)) cudaFreeAsync(p, s);
    else cudaFree(p);
}

namespace {

// Stream-ordered free (after the handle's queued work); the memory returns
// to the device pool.
template <typename T>
void dfree(lv_handle *h, T *&p) {
    if (p) {
        // a large buffer goes to the per-device cache when the handle is
        // being destroyed (its stream has drained); otherwise to the pool
        size_t big = 0;
        for (size_t i = 0; i < h->big.size(); ++i)
            if (h->big[i].first == (void *)p) {
                big = h->big[i].second;
                h->big[i] = h->big.back();
                h->big.pop_back();
                break;
            }
        if (!(big && h->destroying && cache_put(h->device, big, (void *)p))) {
            if (device_pool(h->device)) cudaFreeAsync((void *)p, h->stream);
            else cudaFree((void *)p);
        }
    }
    p = nullptr;
}

cudaEvent_t ev_get(lv_handle *h) {
    if (!h->ev_free.empty()) {
        cudaEvent_t e = h->ev_free.back();
        h->ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Begin / end a timed region on the handle's stream.
struct Timer {
    lv_handle *h;
    int kind;
    cudaEvent_t a = nullptr;
    double bytes = 0, sbytes = 0;
    int64_t verts = 0, edges = 0;
    Timer(lv_handle *hh, int k) : h(hh), kind(k) {
        if (h->capturing) return;   // graph bodies hold no event nodes
        a = ev_get(h);
        cudaEventRecord(a, h->stream);
    }
    void stop() {
        if (!a) return;
        cudaEvent_t b = ev_get(h);
        cudaEventRecord(b, h->stream);
        h->pend.push_back(Pending{kind, a, b, bytes, sbytes, verts, edges});
    }
};

void resolve_events(lv_handle *h) {
    for (const Pending &p : h->pend) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        if (p.kind < NCLS) {
            h->cst.launches[p.kind] += 1;
            h->cst.ms[p.kind] += ms;
            h->cst.bytes[p.kind] += p.bytes;
            h->cst.stored_bytes[p.kind] += p.sbytes;
            h->cst.vertices[p.kind] += p.verts;
            h->cst.edges[p.kind] += p.edges;
        } else if (p.kind == 100) {
            h->st.move_ms += ms;
        } else if (p.kind == 101) {
            h->st.modularity_ms += ms;
        } else if (p.kind == 102) {
            h->st.aggregate_ms += ms;
        } else if (p.kind == 103) {
            h->st.setup_ms += ms;
        }
        h->ev_free.push_back(p.a);
        h->ev_free.push_back(p.b);
    }
    h->pend.clear();
}

int sync(lv_handle *h) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(h, LV_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, LV_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    resolve_events(h);
    return LV_OK;
}

int check_device_error(lv_handle *h, int errword) {
    if (errword == 0) return LV_OK;
    std::string m = "device check failed:";
    if (errword & DEVERR_HASH_FULL) m += " hash table full";
    if (errword & DEVERR_BAD_STATE) m += " invalid community id";
    if (errword & DEVERR_FALLBACK_FULL) m += " fallback list full";
    return fail(h, LV_ERR_DEVICE, m);
}

template <typename WT>
GraphView<WT> view_of(lv_handle *h);
template <>
GraphView<float> view_of<float>(lv_handle *h) {
    return GraphView<float>{h->cur_rowptr, h->cur_rowend, h->cur_col, h->in_w, h->scale_d, nullptr, h->E0};
}
template <>
GraphView<u64> view_of<u64>(lv_handle *h) {
    return GraphView<u64>{h->cur_rowptr, h->cur_rowend, h->cur_col, h->cur_w, h->scale_d, nullptr, h->E0};
}
template <>
GraphView<uint32_t> view_of<uint32_t>(lv_handle *h) {
    return GraphView<uint32_t>{h->cur_rowptr, h->cur_rowend, h->cur_col, h->cur_w32, h->scale_d, h->cur_w,
                               h->E0};
}

// Calls F<WT>(args...) with the weight type the move phase reads at the
// current level: float32 input at level 0, the 32-bit copy of the sums when
// every sum other than the self-loops is below 2^32 (the move kernels skip
// self-loops), the uint64 sums otherwise.
#define LV_BY_WEIGHT(h, F, ...)                                  \
    do {                                                         \
        if ((h)->cur_w32) F<uint32_t>(__VA_ARGS__);              \
        else if ((h)->cur_w) F<u64>(__VA_ARGS__);                \
        else F<float>(__VA_ARGS__);                              \
    } while (0)

// Every weight the move phase reads is below 2^32: the 32-bit view of an
// aggregated level, or level 0 when its fixed-point weights fit 32 bits
// (the move kernels then keep their table sums in 16-bit-piece counters).
// opts.wide_weights keeps 64-bit sums everywhere.
template <typename WT>
bool narrow_weights(const lv_handle *h) {
    if (h->opts.wide_weights) return false;
    // the 32-bit view of a level holding escaped sums: narrow kernels (with
    // the marked rows sent to the large queue) only in mode 1
    if (std::is_same<WT, uint32_t>::value) return LV_NARROW_ESCAPES == 1 || !h->wrows_any;
    if (std::is_same<WT, float>::value) return h->w0_narrow;
    return false;
}

StateView state_of(lv_handle *h) {
    return StateView{h->comm, h->newc, h->size, h->k, h->S, h->T, &h->tot_d->err, h->feat,
                     (LV_NARROW_ESCAPES == 1 && h->cur_w32 && h->wrows_any) ? h->wrow : nullptr,
                     (LV_DEDUP == 2 || (LV_DEDUP == 1 && h->level > 0)) ? 1 : 0};
}

// ---------------------------------------------------------------------------
// global hash-table layouts (hub vertices in the move phase, very large
// communities in aggregation)
// ---------------------------------------------------------------------------
// Pinned host scratch (the totals block and the class counts a handle reads
// back) comes from a process-wide free list: page-locking memory is a slow
// driver call, and a handle created per run should not pay it.
struct PinnedBlock {
    Totals tot;
    int32_t small[128];
};
std::mutex g_pinned_mu;
std::vector<PinnedBlock *> g_pinned_free;

int pinned_take(lv_handle *h) {
    PinnedBlock *b = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        if (!g_pinned_free.empty()) {
            b = g_pinned_free.back();
            g_pinned_free.pop_back();
        }
    }
    if (!b) LV_CUDA(h, cudaMallocHost((void **)&b, sizeof(PinnedBlock)));
    h->tot_h = &b->tot;
    h->small_h = b->small;
    return LV_OK;
}

void pinned_give(lv_handle *h) {
    if (!h->tot_h) return;
    PinnedBlock *b = reinterpret_cast<PinnedBlock *>(h->tot_h);
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(b);
    h->tot_h = nullptr;
    h->small_h = nullptr;
}

int ensure_tables(lv_handle *h, size_t slots) {
    if (slots <= h->tbl_slots) return LV_OK;
    size_t want = slots + slots / 4;
    dfree(h, h->tbl_buf);
    h->tbl_slots = 0;
    LV_TRY(dalloc(h, &h->tbl_buf, want));
    LV_CUDA(h, cudaMemsetAsync(h->tbl_buf, 0, want * sizeof(GSlot), h->stream));
    h->tbl_slots = want;
    return LV_OK;
}

int ensure_occ(lv_handle *h, size_t entries, size_t hubs) {
    if (entries > h->occ_cap) {
        dfree(h, h->occ_buf);
        dfree(h, h->stage_key);
        dfree(h, h->stage_val);
        dfree(h, h->stage2_key);
        dfree(h, h->stage2_val);
        h->occ_cap = 0;
        size_t want = entries + entries / 4 + 1;
        LV_TRY(dalloc(h, &h->occ_buf, want));
        LV_TRY(dalloc(h, &h->stage_key, want));
        LV_TRY(dalloc(h, &h->stage_val, want));
        LV_TRY(dalloc(h, &h->stage2_key, want));
        LV_TRY(dalloc(h, &h->stage2_val, want));
        h->occ_cap = want;
    }
    if (hubs > h->nocc_cap) {
        dfree(h, h->nocc_buf);
        dfree(h, h->eown_buf);
        dfree(h, h->ovf_buf);
        h->nocc_cap = 0;
        size_t want = hubs + hubs / 4 + 1;
        LV_TRY(dalloc(h, &h->nocc_buf, want));
        LV_TRY(dalloc(h, &h->eown_buf, want));
        LV_TRY(dalloc(h, &h->ovf_buf, want + 1));   // overflow list + its count
        LV_CUDA(h, cudaMemsetAsync(h->nocc_buf, 0, want * sizeof(int32_t), h->stream));
        LV_CUDA(h, cudaMemsetAsync(h->eown_buf, 0, want * sizeof(u64), h->stream));
        LV_CUDA(h, cudaMemsetAsync(h->ovf_buf, 0, (want + 1) * sizeof(int32_t), h->stream));
        h->nocc_cap = want;
    }
    return LV_OK;
}

// ids: hub vertices / communities; deg: their degree bound; cap_limit caps
// the distinct-key count (newV for aggregation, unlimited for moves).
int build_layout(lv_handle *h, HubLayout &L, const std::vector<int32_t> &ids,
                 const std::vector<int32_t> &deg, int64_t cap_limit, bool occ_lists, int echunk,
                 bool tables) {
    const int32_t n = (int32_t)ids.size();
    std::vector<int64_t> off(n), occ_off(n);
    int64_t occ_total = 0;
    std::vector<int32_t> lg(n), ech_hub, ech_e0, sch_hub, sch_s0, hub_s0(n + 1), hub_cap(n), pbase(n + 1, 0);
    int64_t total = 0;
    for (int32_t i = 0; i < n; ++i) {
        int64_t distinct = deg[i];
        if (cap_limit > 0 && distinct > cap_limit) distinct = cap_limit;
        int l = ceil_log2_i(2 * distinct);
        if (l < 3) l = 3;
        lg[i] = l;
        off[i] = total;
        total += int64_t(1) << l;
        for (int32_t e0 = 0; e0 < deg[i]; e0 += echunk) {
            ech_hub.push_back(i);
            ech_e0.push_back(e0);
        }
        // evaluation chunks: over the occupied list (room for deg entries)
        // when occ_lists is set, else over the contiguous table
        hub_s0[i] = (int32_t)sch_hub.size();
        occ_off[i] = occ_total;
        occ_total += deg[i];
        hub_cap[i] = deg[i];
        pbase[i + 1] = pbase[i] + (deg[i] + FB_KEYS - 1) / FB_KEYS + 2;
        const int64_t span = occ_lists ? (int64_t)deg[i] : (int64_t(1) << l);
        for (int64_t s0 = 0; s0 < span; s0 += HG_SLOT_CHUNK) {
            sch_hub.push_back(i);
            sch_s0.push_back((int32_t)s0);
        }
        if (span == 0) {
            sch_hub.push_back(i);
            sch_s0.push_back(0);
        }
    }
    hub_s0[n] = (int32_t)sch_hub.size();
    if (tables) LV_TRY(ensure_tables(h, (size_t)total));
    LV_TRY(ensure_occ(h, (size_t)occ_total, (size_t)n));
    const size_t ne = ech_hub.size(), ns = sch_hub.size();
    // packed: ids | lg | ech_hub | ech_e0 | sch_hub | sch_s0 | hub_s0 | res_c | (8-aligned) off |
    // res_g | res_e | res_b | occ_off
    size_t i32_count = (size_t)n + n + ne + ne + ns + ns + (n + 1) + ns + n + (n + 1);
    size_t i32_bytes = ((i32_count * 4 + 15) / 16) * 16;
    size_t bytes = i32_bytes + (size_t)n * 8 + ns * 16 + ns * 8 + ns * 8 + (size_t)n * 8 + 64;
    if (bytes > L.dev_bytes) {
        unsigned char *old_dev = (unsigned char *)L.dev;
        dfree(h, old_dev);
        L.dev = nullptr;
        L.dev_bytes = 0;
        unsigned char *nd = nullptr;
        LV_TRY(dalloc(h, &nd, bytes));
        L.dev = nd;
        L.dev_bytes = bytes;
    }
    std::vector<unsigned char> host(bytes, 0);
    int32_t *p32 = (int32_t *)host.data();
    size_t at = 0;
    auto put = [&](const int32_t *src, size_t cnt) {
        size_t start = at;
        if (cnt) std::memcpy(p32 + at, src, cnt * 4);
        at += cnt;
        return start;
    };
    size_t o_ids = put(ids.data(), n), o_lg = put(lg.data(), n);
    size_t o_eh = put(ech_hub.data(), ne), o_e0 = put(ech_e0.data(), ne);
    size_t o_sh = put(sch_hub.data(), ns), o_s0 = put(sch_s0.data(), ns);
    size_t o_hs = put(hub_s0.data(), n + 1);
    size_t o_rc = at;
    at += ns;
    size_t o_cap = put(hub_cap.data(), n), o_pb = put(pbase.data(), n + 1);
    unsigned char *base8 = host.data() + i32_bytes;
    if (n) std::memcpy(base8, off.data(), (size_t)n * 8);
    if (n) std::memcpy(base8 + (size_t)n * 8 + ns * 32, occ_off.data(), (size_t)n * 8);
    LV_CUDA(h, cudaMemcpyAsync(L.dev, host.data(), bytes, cudaMemcpyHostToDevice, h->stream));
    // the host vector must outlive the async copy
    LV_CUDA(h, cudaStreamSynchronize(h->stream));
    int32_t *d32 = (int32_t *)L.dev;
    unsigned char *d8 = (unsigned char *)L.dev + i32_bytes;
    HubGlobal &v = L.view;
    v.nhubs = n;
    v.n_echunks = (int32_t)ne;
    v.n_schunks = (int32_t)ns;
    v.hubs = d32 + o_ids;
    v.tbl_lg = d32 + o_lg;
    v.echunk_hub = d32 + o_eh;
    v.echunk_e0 = d32 + o_e0;
    v.schunk_hub = d32 + o_sh;
    v.schunk_s0 = d32 + o_s0;
    v.hub_schunk0 = d32 + o_hs;
    v.res_c = d32 + o_rc;
    v.hub_cap = d32 + o_cap;
    v.pbase = d32 + o_pb;
    v.tbl_off = (const int64_t *)d8;
    v.res_g = (u64 *)(d8 + (size_t)n * 8);
    v.res_e = (u64 *)(d8 + (size_t)n * 8 + ns * 16);
    v.res_b = (u64 *)(d8 + (size_t)n * 8 + ns * 24);
    v.occ_off = (const int64_t *)(d8 + (size_t)n * 8 + ns * 32);
    v.occ = h->occ_buf;
    v.nocc = h->nocc_buf;
    v.stage_key = h->stage_key;
    v.stage_val = h->stage_val;
    v.stage2_key = h->stage2_key;
    v.stage2_val = h->stage2_val;
    if ((size_t)pbase[n] > h->poff_cap) {
        dfree(h, h->poff_buf);
        h->poff_cap = 0;
        LV_TRY(dalloc(h, &h->poff_buf, (size_t)pbase[n] + 1));
        h->poff_cap = (size_t)pbase[n];
    }
    v.poff = h->poff_buf;
    v.eown = h->eown_buf;
    v.ovf_list = h->ovf_buf;
    v.ovf_count = h->ovf_buf + h->nocc_cap;
    v.slots = h->tbl_buf;
    L.ids = ids;
    return LV_OK;
}

// ---------------------------------------------------------------------------
// level set-up: degree classes, k_i (level 0), singleton state, hub layout
// ---------------------------------------------------------------------------
template <typename WT>
int compute_k(lv_handle *h) {
    GraphView<WT> g = view_of<WT>(h);
    LV_CUDA(h, cudaMemsetAsync(h->k, 0, sizeof(u64) * (size_t)h->V, h->stream));
    for (int c = 0; c < NCLS; ++c)
        launch_row_reduce<WT>(c, 0, g, h->comm, h->k, nullptr, h->list + h->cls_off[c],
                              h->cls_off[c + 1] - h->cls_off[c], h->di, h->stream);
    return LV_OK;
}

int level_setup(lv_handle *h) {
    Timer t(h, 103);
    int32_t *counts = h->cls_scratch, *cursors = h->cls_scratch + CLASS_COUNT_WORDS;
    launch_class_count(h->cur_rowptr, h->cur_rowend, h->V, h->giant_degree, counts, h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->small_h, counts, sizeof(int32_t) * CLASS_COUNT_WORDS,
                               cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    h->cls_off[0] = 0;
    const u64 *esum = reinterpret_cast<const u64 *>(h->small_h + NCLS + (NCLS & 1));
    for (int c = 0; c < NCLS; ++c) {
        h->cls_off[c + 1] = h->cls_off[c] + h->small_h[c];
        h->cls_edges[c] = (int64_t)esum[c];
    }
    launch_class_scatter(h->cur_rowptr, h->cur_rowend, h->V, h->giant_degree, h->fb.warp_limit, h->cls_off,
                         cursors, h->list, h->fb.hint,
                         h->stream);
    // the warp kernels' vertices by decreasing degree within each update
    // bucket (bucket 6's warp part spans classes H1 and H2)
    {
        const int32_t V0 = h->V0;
        int32_t *kb = h->sort_buf, *ka = h->sort_buf + V0, *va = h->sort_buf + 2 * (size_t)V0;
        const int32_t seg[3][3] = {{CLS_B4, CLS_B5, 84}, {CLS_B5, CLS_H1, 319}, {CLS_H1, CLS_HG, h->giant_degree}};
        for (const auto &sg : seg) {
            const int32_t lo = h->cls_off[sg[0]], n = h->cls_off[sg[1]] - lo;
            sort_by_degree_desc(h->cur_rowptr, h->cur_rowend, h->list + lo, n, sg[2], kb, ka, va, h->sort_temp,
                                h->sort_temp_bytes, h->stream);
        }
    }
    if (h->level == 0) {
        LV_TRY(compute_k<float>(h));
    }
    launch_level_init(h->comm, h->newc, h->size, h->k, h->S, h->V, h->stream);
    // giants (degree > giant_degree): staging areas and global tables
    const int32_t nh = h->cls_off[CLS_HG + 1] - h->cls_off[CLS_HG];
    std::vector<int32_t> ids(nh), deg(nh);
    if (nh > 0) {
        int32_t *dd = h->cls_scratch + SCRATCH_OFF;   // room reserved at create: V0 entries
        launch_gather_degrees(h->cur_rowptr, h->cur_rowend, h->list + h->cls_off[CLS_HG], nh, dd,
                              h->stream);
        LV_CUDA(h, cudaMemcpyAsync(ids.data(), h->list + h->cls_off[CLS_HG], sizeof(int32_t) * nh,
                                   cudaMemcpyDeviceToHost, h->stream));
        LV_CUDA(h, cudaMemcpyAsync(deg.data(), dd, sizeof(int32_t) * nh, cudaMemcpyDeviceToHost,
                                   h->stream));
        LV_TRY(sync(h));
    }
    LV_TRY(build_layout(h, h->hub_move, ids, deg, 0, false, STAGE_CHUNK, false));
    t.stop();
    if (h->opts.trace) {
        std::fprintf(stderr, "[lv] level %d: V=%d E=%lld classes:", h->level, h->V, (long long)h->E);
        for (int c = 0; c < NCLS; ++c)
            std::fprintf(stderr, " %d/%lld", h->cls_off[c + 1] - h->cls_off[c], (long long)h->cls_edges[c]);
        std::fprintf(stderr, "\n");
    }
    return LV_OK;
}

// ---------------------------------------------------------------------------
// sweep and modularity
// ---------------------------------------------------------------------------
// Profile slots of the move phase: 0..3 the group kernels of buckets 0..3,
// 4, 5, 6 the warp + fallback kernels of buckets 4, 5 and 6.
template <typename WT>
void enqueue_sweep(lv_handle *h) {
    GraphView<WT> g = view_of<WT>(h);
    StateView st = state_of(h);
    const double wbytes = sizeof(WT) == 4 ? 4.0 : 8.0;
    u64 *dE = &h->tot_d->dE;
    Timer tm(h, 100);
    int64_t sweep_verts = 0;
    for (int b = 0; b < NBUCKETS; ++b) {
        const int c0 = b, c1 = (b < 6) ? b + 1 : NCLS;
        const int32_t lo = h->cls_off[c0], hi = h->cls_off[c1];
        if (hi == lo) continue;
        const int32_t hg0 = (b == 6) ? h->cls_off[CLS_HG] : hi;   // bucket 6: giants after
        int64_t edges = 0;
        for (int c = c0; c < c1; ++c)
            if (c != CLS_HG) edges += h->cls_edges[c];
        Timer *tc = nullptr;
        if (h->opts.profile) {
            tc = new Timer(h, b);
            tc->verts = hg0 - lo;
            tc->edges = edges;
            tc->bytes = 12.0 * (double)edges + 20.0 * (double)(hg0 - lo);
            tc->sbytes = (8.0 + wbytes) * (double)edges + 20.0 * (double)(hg0 - lo);
        }
        if (b < 4)
            launch_move_class<WT>(b, g, st, h->list + lo, hi - lo, h->di, dE, h->stream, narrow_weights<WT>(h),
                                  h->fb);
        else if (hg0 > lo)
            launch_move_wide<WT>(g, st, h->list + lo, hg0 - lo, h->fb, h->di, dE, h->stream,
                                 b == 6 ? h->giant_degree : (b == 4 ? 84 : 319), narrow_weights<WT>(h));
        if (tc) {
            tc->stop();
            delete tc;
            tc = nullptr;
        }
        if (hi > hg0) {
            if (h->opts.profile) {
                tc = new Timer(h, 7);
                tc->verts = hi - hg0;
                tc->edges = h->cls_edges[CLS_HG];
                tc->bytes = 12.0 * (double)tc->edges + 20.0 * (double)tc->verts;
                tc->sbytes = (8.0 + wbytes) * (double)tc->edges + 20.0 * (double)tc->verts;
            }
            launch_move_giants<WT>(g, st, h->hub_move.view, h->fb, h->di, dE, h->stream, narrow_weights<WT>(h));
            if (tc) {
                tc->stop();
                delete tc;
            }
        }
        // exact modularity bookkeeping for neighbours that moved together
        for (int c = c0; c < c1; ++c)
            launch_correction<WT>(c, g, st, h->list + h->cls_off[c], h->cls_off[c + 1] - h->cls_off[c],
                                  h->di, dE, h->stream);
        launch_commit(st, h->list + lo, hi - lo, &h->tot_d->moves, h->stream);
        sweep_verts += hi - lo;
    }
    tm.bytes = 12.0 * (double)h->E + 20.0 * (double)sweep_verts;
    tm.sbytes = (8.0 + wbytes) * (double)h->E + 20.0 * (double)sweep_verts;
    tm.stop();
    h->st.move_bytes += tm.bytes;
}

template <typename WT>
void enqueue_modularity(lv_handle *h) {
    GraphView<WT> g = view_of<WT>(h);
    Timer tm(h, 101);
    for (int c = 0; c < NCLS; ++c)
        launch_row_reduce<WT>(c, 1, g, h->comm, nullptr, &h->tot_d->e_own, h->list + h->cls_off[c],
                              h->cls_off[c + 1] - h->cls_off[c], h->di, h->stream);
    launch_s2(h->S, h->V, h->tot_d->s2, h->stream);
    tm.stop();
}

double q_from_totals(u64 T, const Totals &t) {
    // Same FP64 formula as the oracle: e_own/T - sum(S^2)/T^2, i.e.
    // toOwn/(2M) - sum(S^2)/(4M^2) of calculateModularity.
    const u128 s2 = ((u128)t.s2[0] << 64) | (u128)t.s2[1];
    const double td = (double)T;
    const double a = (double)t.e_own / td;
    const double b = (double)s2 / (td * td);
    return a - b;
}

int reset_totals(lv_handle *h) {
    LV_CUDA(h, cudaMemsetAsync(h->tot_d, 0, offsetof(Totals, err), h->stream));
    return LV_OK;
}

int read_totals(lv_handle *h) {
    LV_CUDA(h, cudaMemcpyAsync(h->tot_h, h->tot_d, sizeof(Totals), cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    return check_device_error(h, h->tot_h->err);
}

int modularity(lv_handle *h, double *q) {
    LV_TRY(reset_totals(h));
    if (h->cur_w) enqueue_modularity<u64>(h); else enqueue_modularity<float>(h);
    LV_TRY(read_totals(h));
    h->e_own_cur = h->tot_h->e_own;
    h->e_own_valid = true;
    *q = q_from_totals(h->T, *h->tot_h);
    return LV_OK;
}

// One sweep followed by the modularity of the resulting state.  The edge
// pass of calculateModularity is replaced by the exact update of
// sum_i e_{i->C(i)} accumulated by the move and correction kernels; only the
// sum of Sigma_tot^2 is recomputed (a pass over V).
int sweep_and_q(lv_handle *h, int64_t *moves, double *q) {
    if (!h->e_own_valid) {
        double q0;
        LV_TRY(modularity(h, &q0));
    }
    LV_TRY(reset_totals(h));
    LV_BY_WEIGHT(h, enqueue_sweep, h);
    {
        Timer tm(h, 101);
        launch_s2(h->S, h->V, h->tot_d->s2, h->stream);
        tm.stop();
    }
    LV_TRY(read_totals(h));
    h->e_own_cur += h->tot_h->dE;
    Totals t = *h->tot_h;
    t.e_own = h->e_own_cur;
    *moves = (int64_t)t.moves;
    const double q_inc = q_from_totals(h->T, t);
    if (h->opts.verify) {
        double q_full = 0;
        LV_TRY(modularity(h, &q_full));
        if (h->e_own_cur != t.e_own || q_full != q_inc)
            return fail(h, LV_ERR_DEVICE, "incremental modularity differs from the full pass");
    }
    if (q) *q = q_inc;
    if (h->opts.trace) {
        // per-class device time of this sweep (profile mode) and move phase
        std::fprintf(stderr, "[lv]   sweep: moves=%lld q=%.9f move_ms_total=%.3f", (long long)t.moves,
                     q_inc, h->st.move_ms);
        if (h->opts.profile) {
            std::fprintf(stderr, " class_ms_total:");
            for (int c = 0; c < NCLS; ++c) std::fprintf(stderr, " %.2f", h->cst.ms[c]);
        }
        std::fprintf(stderr, "\n");
    }
    h->st.sweeps += 1;
    h->st.edge_sweeps += h->E;
    h->st.moves += *moves;
    return LV_OK;
}

// ---------------------------------------------------------------------------
// device-side sweep control: a level's sweep loop as one CUDA graph
// ---------------------------------------------------------------------------
// The graph is a while-conditional node whose body is one sweep (totals reset,
// the seven sub-rounds with corrections and commits, the sum of Sigma_tot^2)
// followed by sweep_end_kernel, which updates sum_i e_{i->C(i)} by the sweep's
// exact change, forms Q with the host's FP64 operations (each correctly
// rounded, so the value is the same bit for bit), and sets the loop condition
// exactly as the host loop decides: continue while the sweep gained at least
// min_gain, moved something, the sweep cap is not reached and no device
// check failed.
struct LoopState {
    double q_before;
    double min_gain;
    u64 e_own;          // sum_i e_{i->C(i)} of the current state
    u64 T;
    u64 moves_total;
    double q_last;
    int32_t max_sweeps;
    int32_t sweeps;
    int32_t changed;
    int32_t pad;
};

__global__ void sweep_end_kernel(cudaGraphConditionalHandle cond, const Totals *t, LoopState *ls) {
    if (threadIdx.x != 0) return;
    ls->e_own += t->dE;
    const double q = q_from_parts_dev(ls->T, ls->e_own, t->s2[0], t->s2[1]);
    ls->sweeps += 1;
    ls->moves_total += t->moves;
    const double gain = __dsub_rn(q, ls->q_before);
    if (gain > 0) ls->changed = 1;
    ls->q_before = q;
    ls->q_last = q;
    const bool more = gain >= ls->min_gain && t->moves != 0 &&
                      !(ls->max_sweeps > 0 && ls->sweeps >= ls->max_sweeps) && t->err == 0;
    cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// Returns LV_OK with *done = 1 when the loop ran as a graph; *done = 0 when
// the graph could not be built (the caller then runs the host loop).
int sweep_loop_graph(lv_handle *h, float min_gain, double q_start, int *ch, int *done) {
    *done = 0;
    if (!h->loop_d) {
        LoopState *p = nullptr;
        LV_TRY(dalloc(h, &p, 1));
        h->loop_d = p;
    }
    LoopState *ld = (LoopState *)h->loop_d;
    LoopState ls{};
    ls.q_before = q_start;
    ls.min_gain = (double)min_gain;
    ls.e_own = h->e_own_cur;
    ls.T = h->T;
    ls.q_last = q_start;
    ls.max_sweeps = h->opts.max_sweeps;
    LV_CUDA(h, cudaMemcpyAsync(ld, &ls, sizeof(ls), cudaMemcpyHostToDevice, h->stream));
    LV_TRY(sync(h));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    cudaGraphNode_t node = nullptr;
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNodeParams np = {};
    if (ok) {
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = cond;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        ok = cudaGraphAddNode(&node, graph, nullptr, 0, &np) == cudaSuccess;
    }
    const long long launches0 = launches_total();
    const double bytes0 = h->st.move_bytes;
    if (ok) {
        cudaGraph_t body = np.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeRelaxed) == cudaSuccess;
        if (ok) {
            h->capturing = true;
            cudaMemsetAsync(h->tot_d, 0, offsetof(Totals, err), h->stream);
            LV_BY_WEIGHT(h, enqueue_sweep, h);
            launch_s2(h->S, h->V, h->tot_d->s2, h->stream);
            sweep_end_kernel<<<1, 32, 0, h->stream>>>(cond, h->tot_d, ld);
            note_launches(1);
            h->capturing = false;
            cudaGraph_t captured = nullptr;
            ok = cudaStreamEndCapture(h->stream, &captured) == cudaSuccess;
        }
    }
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    const long long per_sweep = launches_total() - launches0;
    const double bytes_per_sweep = h->st.move_bytes - bytes0;
    if (!ok) {
        cudaGetLastError();
        h->capturing = false;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        note_launches((int)-per_sweep);   // nothing ran
        h->st.move_bytes = bytes0;
        return LV_OK;
    }
    {
        Timer tm(h, 100);
        LV_CUDA(h, cudaGraphLaunch(exec, h->stream));
        tm.stop();
    }
    LV_CUDA(h, cudaMemcpyAsync(&ls, ld, sizeof(ls), cudaMemcpyDeviceToHost, h->stream));
    LV_CUDA(h, cudaMemcpyAsync(h->tot_h, h->tot_d, sizeof(Totals), cudaMemcpyDeviceToHost, h->stream));
    const int rc = sync(h);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    LV_TRY(rc);
    LV_TRY(check_device_error(h, h->tot_h->err));
    // the captured sweep was counted once; it ran ls.sweeps times
    note_launches((int)(per_sweep * (ls.sweeps - 1)));
    h->st.move_bytes = bytes0 + bytes_per_sweep * ls.sweeps;
    h->e_own_cur = ls.e_own;
    h->st.sweeps += ls.sweeps;
    h->st.edge_sweeps += h->E * (int64_t)ls.sweeps;
    h->st.moves += (int64_t)ls.moves_total;
    *ch = ls.changed;
    *done = 1;
    return LV_OK;
}

// ---------------------------------------------------------------------------
// learned active set (lv_opts.active_set) and move traces (trace_sample)
// ---------------------------------------------------------------------------
// Levels with fewer vertices than this run plain sweeps in learned mode: their
// sweeps are short and the device-side sweep loop (no host round trip per
// sweep) is cheaper than proposing.
constexpr int32_t ACTIVE_MIN_VERTICES = 1 << 16;

bool learned_mode(const lv_handle *h) {
    return h->opts.trace_sample > 0.0f || (h->opts.active_set != 0 && h->V >= ACTIVE_MIN_VERTICES);
}

int ensure_active(lv_handle *h) {
    if (h->feat) return LV_OK;
    const size_t V = (size_t)h->V0 + 1;
    LV_TRY(dalloc(h, &h->feat, 2 * V));
    LV_TRY(dalloc(h, &h->moved, V));
    LV_TRY(dalloc(h, &h->nmoved, V));
    LV_TRY(dalloc(h, &h->pred, V));
    LV_TRY(dalloc(h, &h->fresh, V));
    LV_CUDA(h, cudaMemsetAsync(h->fresh, 0, V, h->stream));
    LV_TRY(dalloc(h, &h->comm_prev, V));
    LV_TRY(dalloc(h, &h->alist, V));
    LV_TRY(dalloc(h, &h->acnt, (size_t)NCLS));
    LV_TRY(dalloc(h, &h->actr, 4));
    LV_CUDA(h, cudaMemsetAsync(h->actr, 0, 4 * sizeof(u64), h->stream));
    if (h->opts.trace_sample > 0.0f) {
        const double r = h->opts.trace_sample < 1.0f ? h->opts.trace_sample : 1.0;
        h->tr_cap = (int64_t)std::ceil(r * (double)h->V0 * 48.0) + 1024;
        LV_TRY(dalloc(h, &h->tr_x, (size_t)h->tr_cap * LV_ACTIVE_FEATURES));
        LV_TRY(dalloc(h, &h->tr_v, (size_t)h->tr_cap));
        LV_TRY(dalloc(h, &h->tr_y, (size_t)h->tr_cap));
    }
    return LV_OK;
}

// One sweep over the proposed vertices only (per-class counts cnt, lists at
// the classes' offsets in alist); giants are always in the list.
template <typename WT>
void enqueue_sweep_active(lv_handle *h, const int32_t *cnt) {
    GraphView<WT> g = view_of<WT>(h);
    StateView st = state_of(h);
    u64 *dE = &h->tot_d->dE;
    Timer tm(h, 100);
    int64_t verts = 0;
    for (int b = 0; b < NBUCKETS; ++b) {
        const int c0 = b, c1 = (b < 6) ? b + 1 : NCLS;
        int64_t any = 0;
        for (int c = c0; c < c1; ++c) any += cnt[c];
        if (!any) continue;
        if (b < 4) {
            launch_move_class<WT>(b, g, st, h->alist + h->cls_off[b], cnt[b], h->di, dE, h->stream,
                                  narrow_weights<WT>(h), h->fb);
        } else {
            for (int c = c0; c < c1; ++c) {
                if (c == CLS_HG || !cnt[c]) continue;
                const int32_t maxdeg = c == CLS_B4 ? 84 : (c == CLS_B5 ? 319 : (c == CLS_H1 ? 1024 : h->giant_degree));
                launch_move_wide<WT>(g, st, h->alist + h->cls_off[c], cnt[c], h->fb, h->di, dE, h->stream, maxdeg,
                                     narrow_weights<WT>(h));
            }
            if (b == 6 && cnt[CLS_HG]) launch_move_giants<WT>(g, st, h->hub_move.view, h->fb, h->di, dE, h->stream, narrow_weights<WT>(h));
        }
        for (int c = c0; c < c1; ++c)
            launch_correction<WT>(c, g, st, h->alist + h->cls_off[c], cnt[c], h->di, dE, h->stream);
        for (int c = c0; c < c1; ++c) launch_commit(st, h->alist + h->cls_off[c], cnt[c], &h->tot_d->moves, h->stream);
        verts += any;
    }
    tm.bytes = 20.0 * (double)verts;
    tm.stop();
}

// One sweep of the learned / traced loop: full (every vertex) or over the
// proposed vertices; predict = run the predictor first (the proposal of an
// active sweep, or the flags whose recall a full sweep measures).
int sweep_learned(lv_handle *h, bool full, bool predict, int64_t *moves, double *q, int64_t *movers,
                  int64_t *hits, int64_t *fresh_movers) {
    LV_TRY(reset_totals(h));
    LV_CUDA(h, cudaMemsetAsync(h->actr, 0, 2 * sizeof(u64), h->stream));
    LV_CUDA(h, cudaMemsetAsync(h->actr + 3, 0, sizeof(u64), h->stream));
    const int32_t n = h->cls_off[NCLS];
    ActiveClassOffsets co;
    for (int c = 0; c <= NCLS; ++c) co.off[c] = h->cls_off[c];
    const int32_t *rowend = h->cur_rowend ? h->cur_rowend : h->cur_rowptr + 1;
    int32_t cnt[NCLS];
    if (predict) {
        if (!full) LV_CUDA(h, cudaMemsetAsync(h->acnt, 0, NCLS * sizeof(int32_t), h->stream));
        launch_active_select(h->list, n, co, h->cur_rowptr, rowend, h->feat, h->moved, h->nmoved, h->model, h->logit_thr,
                             CLS_HG, full ? nullptr : h->alist, h->acnt, h->pred, h->fresh, h->stream);
        if (!full) {
            LV_CUDA(h, cudaMemcpyAsync(h->small_h, h->acnt, NCLS * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                       h->stream));
            LV_TRY(sync(h));
            for (int c = 0; c < NCLS; ++c) cnt[c] = h->small_h[c];
        }
    }
    const bool tracing = h->opts.trace_sample > 0.0f && h->tr_x;
    if (tracing && h->tr_sweep > 0) {
        const double r = h->opts.trace_sample < 1.0f ? h->opts.trace_sample : 1.0;
        const u64 thr = r >= 1.0 ? ~0ull : (u64)(r * 18446744073709551616.0);
        launch_trace_sample(h->V, h->cur_rowptr, rowend, h->feat, h->moved, h->nmoved, thr,
                            0x7A11ull * (h->tr_sweep + 1) ^ ((u64)h->level << 40), h->tr_x, h->tr_v, h->tr_cap,
                            h->actr + 2, h->stream);
    }
    LV_CUDA(h, cudaMemcpyAsync(h->comm_prev, h->comm, sizeof(int32_t) * (size_t)h->V, cudaMemcpyDeviceToDevice,
                               h->stream));
    if (full) {
        LV_BY_WEIGHT(h, enqueue_sweep, h);
        h->act_evaluated += n;
        h->act_full += 1;
    } else {
        LV_BY_WEIGHT(h, enqueue_sweep_active, h, cnt);
        for (int c = 0; c < NCLS; ++c) h->act_evaluated += cnt[c];
        h->act_active += 1;
    }
    {
        Timer tm(h, 101);
        launch_s2(h->S, h->V, h->tot_d->s2, h->stream);
        tm.stop();
    }
    launch_active_moved(h->comm, h->comm_prev, h->V, h->moved, predict && full ? h->pred : nullptr, h->fresh,
                        h->actr, h->stream);
    launch_nbr_moved(h->cur_rowptr, rowend, h->cur_col, h->V, h->moved, h->nmoved, h->stream);
    if (tracing && h->tr_sweep > 0)
        launch_trace_label(h->tr_v, h->moved, h->tr_rows, h->actr + 2, h->tr_cap, h->tr_y, h->stream);
    u64 ctr[4];
    LV_CUDA(h, cudaMemcpyAsync(ctr, h->actr, 4 * sizeof(u64), cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(read_totals(h));
    if (tracing) {
        if (h->tr_sweep > 0) h->tr_rows = (int64_t)ctr[2] < h->tr_cap ? (int64_t)ctr[2] : h->tr_cap;
        h->tr_sweep += 1;
    }
    h->e_own_cur += h->tot_h->dE;
    Totals t = *h->tot_h;
    t.e_own = h->e_own_cur;
    *moves = (int64_t)t.moves;
    *movers = (int64_t)ctr[0];
    *hits = (int64_t)ctr[1];
    *fresh_movers = (int64_t)ctr[3];
    *q = q_from_totals(h->T, t);
    h->st.sweeps += 1;
    h->st.edge_sweeps += h->E;
    h->st.moves += *moves;
    return LV_OK;
}

// optimiseModularity with the learned proposal: sweeps are full until one
// moves fewer than active_start of the level's vertices (the early sweeps,
// where most vertices move, stay exactly the plain method's); after that
// every active_full_every-th sweep evaluates every vertex and the others only
// the proposed ones.  A full sweep after a proposal measures its recall over
// the vertices evaluated since the previous full sweep (movers the predictor
// proposes now / movers among them); below active_min_recall the plain sweep
// takes over for the rest of the level.  An active sweep that gains less than
// min_gain (or moves nothing) is followed by a full sweep, and the level ends
// as the plain loop does, on a full sweep.  Without a model (trace recording
// only) every sweep is full and the result equals the plain loop's.
int optimise_level_learned(lv_handle *h, float min_gain, int32_t *changed) {
    LV_TRY(ensure_active(h));
    LV_CUDA(h, cudaMemsetAsync(h->feat, 0, sizeof(float) * 2 * (size_t)h->V, h->stream));
    LV_CUDA(h, cudaMemsetAsync(h->moved, 0, (size_t)h->V, h->stream));
    LV_CUDA(h, cudaMemsetAsync(h->nmoved, 0, sizeof(int32_t) * (size_t)h->V, h->stream));
    LV_CUDA(h, cudaMemsetAsync(h->fresh, 0, (size_t)h->V, h->stream));
    h->tr_sweep = 0;
    double q_before = 0, q_after = 0;
    LV_TRY(modularity(h, &q_before));
    const bool learned = h->opts.active_set != 0 && h->has_model;
    const int K = h->opts.active_full_every > 0 ? h->opts.active_full_every : 4;
    const double rmin = h->opts.active_min_recall > 0.0f ? (double)h->opts.active_min_recall : 0.9;
    const double start = h->opts.active_start > 0.0f ? (double)h->opts.active_start : 0.05;
    bool plain_rest = !learned, force_full = true, proposing = false;
    int since_full = 0, sweeps = 0, ch = 0;
    for (;;) {
        if (h->opts.max_sweeps > 0 && sweeps >= h->opts.max_sweeps) break;
        const bool full = force_full || plain_rest || !proposing || since_full + 1 >= K;
        const bool predict = learned && !plain_rest && proposing;
        int64_t moves = 0, movers = 0, hits = 0, fresh_movers = 0;
        LV_TRY(sweep_learned(h, full, predict, &moves, &q_after, &movers, &hits, &fresh_movers));
        sweeps++;
        const double gain = q_after - q_before;
        if (gain > 0) ch = 1;
        q_before = q_after;
        const bool stall = !(gain >= (double)min_gain) || moves == 0;
        if (full) {
            since_full = 0;
            force_full = false;
            if ((double)movers < start * (double)h->V) proposing = true;
            if (predict) {
                // recall over the movers whose features are current (evaluated
                // since the last full sweep): what the predictor caught, not
                // the moves it postponed
                // (no fresh mover while others moved: the proposals caught
                // nothing, recall 0; nothing moved at all: recall 1)
                h->act_recall = fresh_movers > 0 ? (double)hits / (double)fresh_movers : (movers > 0 ? 0.0 : 1.0);
                if (h->act_recall < rmin) {
                    plain_rest = true;
                    h->act_fell_back = 1;
                }
            }
            if (stall) break;
        } else {
            since_full++;
            if (stall) force_full = true;
        }
    }
    launch_compose_map(h->orig2comm, h->comm, h->V0, h->stream);
    h->st.levels += 1;
    h->st.final_vertices = h->V;
    if (changed) *changed = ch;
    return sync(h);
}

int optimise_level(lv_handle *h, float min_gain, int32_t *changed) {
    if (learned_mode(h)) return optimise_level_learned(h, min_gain, changed);
    double q_before = 0, q_after = 0;
    LV_TRY(modularity(h, &q_before));
    if (h->opts.sweep_graph && !h->opts.profile && !h->opts.verify && !h->opts.trace) {
        int ch = 0, done = 0;
        LV_TRY(sweep_loop_graph(h, min_gain, q_before, &ch, &done));
        if (done) {
            launch_compose_map(h->orig2comm, h->comm, h->V0, h->stream);
            h->st.levels += 1;
            h->st.final_vertices = h->V;
            if (changed) *changed = ch;
            return sync(h);
        }
    }
    double gain = (double)min_gain;
    int ch = 0, sweeps = 0;
    while (gain >= (double)min_gain) {
        if (h->opts.max_sweeps > 0 && sweeps >= h->opts.max_sweeps) break;
        int64_t moves = 0;
        LV_TRY(sweep_and_q(h, &moves, &q_after));
        sweeps++;
        gain = q_after - q_before;
        if (gain > 0) ch = 1;
        q_before = q_after;
        if (moves == 0) break;
    }
    launch_compose_map(h->orig2comm, h->comm, h->V0, h->stream);
    h->st.levels += 1;
    h->st.final_vertices = h->V;
    if (changed) *changed = ch;
    return sync(h);
}

// ---------------------------------------------------------------------------
// aggregation
// ---------------------------------------------------------------------------
int ensure_agg(lv_handle *h) {
    if (h->agg_ready) return LV_OK;
    const size_t V = (size_t)h->V0, E = (size_t)(h->E0 > 0 ? h->E0 : 1);
    AggBuffers &a = h->ab;
    LV_TRY(dalloc(h, &a.flag, V + 1));
    LV_TRY(dalloc(h, &a.cdeg, V + 1));
    LV_TRY(dalloc(h, &a.mstart, V + 1));
    LV_TRY(dalloc(h, &a.cursor, V + 16));
    LV_TRY(dalloc(h, &a.members, V + 1));
    LV_TRY(dalloc(h, &a.lab, V + 1));
    LV_TRY(dalloc(h, &a.clist, V + 1));
    LV_TRY(dalloc(h, &a.newdeg, V + 1));
    LV_TRY(dalloc(h, &a.epos_new, V + 1));
    LV_TRY(dalloc(h, &a.scan_tmp, (size_t)scan_tmp_elems((int64_t)V + 1) + 16));
    LV_TRY(dalloc(h, &a.scalars, 64));
    LV_TRY(dalloc(h, &h->mslot, V + 1));
    LV_TRY(dalloc(h, &h->degm, V + 1));
    LV_TRY(dalloc(h, &h->P, V + 1));
    for (int b = 0; b < 2; ++b) {
        LV_TRY(dalloc(h, &h->lvl_start[b], V + 1));
        LV_TRY(dalloc(h, &h->lvl_end[b], V + 1));
        LV_TRY(dalloc(h, &h->lvl_col[b], E));
        LV_TRY(dalloc(h, &h->lvl_w[b], E));
        LV_TRY(dalloc(h, &h->lvl_w32[b], E));
    }
    LV_TRY(dalloc(h, &h->wrow, V + 1));
    h->agg_ready = true;
    return LV_OK;
}

template <typename WT>
int aggregate_t(lv_handle *h) {
    Timer tm(h, 102);
    AggBuffers &ab = h->ab;
    const int32_t V = h->V;
    // the next level's rows are built in the other ping-pong buffer
    const int nb = (h->cur_buf == 0) ? 1 : 0;
    int32_t *vkey = h->lvl_col[nb];
    u64 *vw = h->lvl_w[nb];
    uint32_t *vw32 = h->lvl_w32[nb];
    int32_t *hiflag = ab.scalars + 12;   // set when a merged sum is 2^32 or more
    // the permuted inter-community weights are the current level's
    // non-self-loop weights: below 2^32 when the move phase reads them narrow
    const bool narrow = h->cur_w32 ? !h->wrows_any : narrow_weights<WT>(h);
    agg_prepare(h->cur_rowptr, h->cur_rowend, h->comm, h->size, V, ab, h->mslot, h->degm, h->P,
                h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->small_h, ab.scalars, sizeof(int32_t) * (2 + NAC),
                               cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    const int32_t newV = h->small_h[0];
    int32_t aoff[NAC + 1];
    aoff[0] = 0;
    for (int c = 0; c < NAC; ++c) aoff[c + 1] = aoff[c] + h->small_h[2 + c];
    agg_classify(h->size, V, ab, h->P, aoff, h->stream);
    const int32_t nbig = aoff[NAC] - aoff[NAC - 1];
    std::vector<int32_t> ids(nbig), deg(nbig);
    if (nbig > 0) {
        launch_gather_cdeg(ab.mstart, h->P, ab.clist + aoff[NAC - 1], nbig, ab.cdeg, h->stream);
        LV_CUDA(h, cudaMemcpyAsync(ids.data(), ab.clist + aoff[NAC - 1], sizeof(int32_t) * nbig,
                                   cudaMemcpyDeviceToHost, h->stream));
        LV_CUDA(h, cudaMemcpyAsync(deg.data(), ab.cdeg, sizeof(int32_t) * nbig,
                                   cudaMemcpyDeviceToHost, h->stream));
        LV_TRY(sync(h));
    }
    LV_TRY(build_layout(h, h->hub_agg, ids, deg, newV, true, HG_EDGE_CHUNK, true));
    GraphView<WT> g = view_of<WT>(h);
    for (int c = 0; c < NCLS; ++c)
        agg_permute<WT>(c, g, ab, h->mslot, h->P, h->list + h->cls_off[c],
                        h->cls_off[c + 1] - h->cls_off[c], vkey, vw, h->di.sms, h->stream);
    agg_new_vertices(h->size, h->S, V, ab, h->P, h->k, h->stream);
    LV_CUDA(h, cudaMemsetAsync(hiflag, 0, sizeof(int32_t), h->stream));
    LV_CUDA(h, cudaMemsetAsync(h->wrow, 0, (size_t)newV + 1, h->stream));
    for (int c = 0; c < NAC - 1; ++c)
        agg_merge_class(c, ab, h->P, ab.clist + aoff[c], aoff[c + 1] - aoff[c], vkey, vw, vw32,
                        &h->tot_d->err, hiflag, h->wrow, h->di.sms, h->stream, narrow);
    agg_merge_global(h->hub_agg.view, ab, h->P, vkey, vw, vw32, &h->tot_d->err, hiflag, h->wrow, h->stream,
                     narrow);
    agg_row_bounds(ab, newV, h->lvl_start[nb], h->lvl_end[nb], h->stream);
    // E' = number of stored entries (P is free again after the merges)
    scan_exclusive_i32(ab.newdeg, h->P, newV, h->P + newV, ab.scan_tmp, h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->small_h, h->P + newV, sizeof(int32_t), cudaMemcpyDeviceToHost,
                               h->stream));
    LV_CUDA(h, cudaMemcpyAsync(h->small_h + 1, hiflag, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    launch_compose_map(h->orig2comm, ab.flag, h->V0, h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->tot_h, h->tot_d, sizeof(Totals), cudaMemcpyDeviceToHost, h->stream));
    tm.stop();
    LV_TRY(sync(h));
    if (h->opts.trace)
        std::fprintf(stderr, "[lv] aggregate: newV=%d big_communities=%d agg_ms_total=%.3f\n", newV, nbig,
                     h->st.aggregate_ms);
    LV_TRY(check_device_error(h, h->tot_h->err));
    const int64_t newE = h->small_h[0];
    h->wrows_any = h->small_h[1] != 0;
    h->cur_buf = nb;
    h->cur_rowptr = h->lvl_start[nb];
    h->cur_rowend = h->lvl_end[nb];
    h->cur_col = h->lvl_col[nb];
    h->cur_w = h->lvl_w[nb];
    // mode 0: a level with escaped sums is swept on its uint64 sums
    h->cur_w32 = (h->opts.wide_weights || (LV_NARROW_ESCAPES == 0 && h->wrows_any)) ? nullptr : h->lvl_w32[nb];
    h->V = newV;
    h->E = newE;
    h->level += 1;
    h->e_own_valid = false;
    return level_setup(h);
}

int aggregate(lv_handle *h) {
    LV_TRY(ensure_agg(h));
    return h->cur_w ? aggregate_t<u64>(h) : aggregate_t<float>(h);
}

// ---------------------------------------------------------------------------
// creation
// ---------------------------------------------------------------------------
int to_level0(lv_handle *h) {
    h->level = 0;
    h->V = h->V0;
    h->E = h->E0;
    h->cur_rowptr = h->in_rowptr;
    h->cur_rowend = h->in_rowptr + 1;
    h->cur_col = h->in_col;
    h->cur_w = nullptr;
    h->cur_w32 = nullptr;
    h->wrows_any = false;
    h->cur_buf = -1;
    h->e_own_valid = false;
    launch_iota_i32(h->orig2comm, h->V0, h->stream);
    return level_setup(h);
}

int finish_create(lv_handle *h) {
    const size_t V = (size_t)h->V0;
    if (h->opts.trace)
        std::fprintf(stderr, "[lv] device %d memory pool: %s\n", h->device,
                     device_pool(h->device) ? "on" : "off (cudaMalloc per buffer)");
    LV_TRY(dalloc(h, &h->comm, V + 1));
    LV_TRY(dalloc(h, &h->newc, V + 1));
    LV_TRY(dalloc(h, &h->size, V + 1));
    LV_TRY(dalloc(h, &h->orig2comm, V + 1));
    LV_TRY(dalloc(h, &h->k, V + 1));
    LV_TRY(dalloc(h, &h->S, V + 1));
    LV_TRY(dalloc(h, &h->list, V + 1));
    LV_TRY(dalloc(h, &h->cls_scratch, V + SCRATCH_OFF + 16));
    LV_TRY(dalloc(h, &h->sort_buf, 3 * V + 16));
    h->sort_temp_bytes = sort_by_degree_temp_bytes((int32_t)V, HG_MIN_DEG_HI) + 256;
    {
        unsigned char *t = nullptr;
        LV_TRY(dalloc(h, &t, h->sort_temp_bytes));
        h->sort_temp = t;
    }
    {
        // fallback work lists of the move phase.  Only vertices of degree
        // > warp_limit are queued (at most E / warp_limit of them at any
        // level); a large item covers FB_KEYS edges of a vertex of degree
        // > FBQ_MAXDEG(NFBQ - 1), or as many staged pairs of a giant.
        FallbackSet &fs = h->fb;
        int32_t *counters = nullptr;
        LV_TRY(dalloc(h, &counters, 2 * (NFBQ + 1) + 2));
        fs.warp_next = counters + 2 * (NFBQ + 1);
        LV_TRY(dalloc(h, &fs.hint, V + 1));
        LV_CUDA(h, cudaMemsetAsync(fs.hint, 0, V + 1, h->stream));
        const size_t cap_row = (size_t)(h->E0 / fs.warp_limit) + 64;
        const size_t cap_large = (size_t)(2 * (h->E0 / FBQ_MAXDEG(NFBQ - 1) + h->E0 / FB_KEYS)) + 64;
        for (int q = 0; q <= NFBQ; ++q) {
            Fallback &f = fs.q[q];
            f.count = counters + 2 * q;
            f.next = f.count + 1;
            const size_t cap = q < NFBQ ? cap_row : cap_large;
            f.cap = (int32_t)cap;
            LV_TRY(dalloc(h, &f.v, cap));
            if (q < NFBQ) continue;
            LV_TRY(dalloc(h, &f.p, cap));
            LV_TRY(dalloc(h, &f.P, cap));
            LV_TRY(dalloc(h, &f.first, cap));
            LV_TRY(dalloc(h, &f.src, cap));
            LV_TRY(dalloc(h, &f.done, cap));
            LV_TRY(dalloc(h, &f.gd, cap));
            LV_TRY(dalloc(h, &f.e, cap));
            LV_TRY(dalloc(h, &f.S, cap));
            LV_TRY(dalloc(h, &f.eo, cap));
            LV_TRY(dalloc(h, &f.c, cap));
            LV_TRY(dalloc(h, &f.cnt, cap));
            LV_CUDA(h, cudaMemsetAsync(f.done, 0, cap * sizeof(int32_t), h->stream));
        }
    }
    LV_TRY(dalloc(h, &h->tot_d, 1));
    LV_CUDA(h, cudaMemsetAsync(h->tot_d, 0, sizeof(Totals), h->stream));
    LV_TRY(pinned_take(h));
    // CSR validation
    launch_validate_csr(h->in_rowptr, h->in_col, h->V0, h->E0, &h->tot_d->err, h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->tot_h, h->tot_d, sizeof(Totals), cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    if (h->tot_h->err) return fail(h, LV_ERR_INVALID, "malformed CSR (offsets or column ids)");
    // fixed-point scale (same rule as the oracle's orc_choose_scale)
    int32_t *ws = h->cls_scratch;
    launch_weight_scan(h->in_w, h->E0, ws, h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->small_h, ws, sizeof(int32_t) * 3, cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    if (h->small_h[2]) return fail(h, LV_ERR_WEIGHT, "negative, NaN or infinite edge weight");
    const int need = h->small_h[0];
    const int top = h->small_h[1] ? h->small_h[1] - 1024 : 0;
    const int cap = 61 - top - ceil_log2_i(h->E0 > 0 ? h->E0 : 1);
    const int s = need < cap ? need : cap;
    if (s < 0) return fail(h, LV_ERR_TOO_LARGE, "total edge weight exceeds the fixed-point range");
    h->scale = s;
    h->exact = (s == need);
    // every fixed-point weight is at most 2^(top + 1 + scale) (rounding included)
    h->w0_narrow = !h->small_h[1] || top + 1 + s <= 31;
    h->scale_d = std::ldexp(1.0, s);
    u64 *tw = (u64 *)(h->tot_d);   // reuse e_own slot
    launch_total_weight(h->in_w, h->E0, h->scale_d, tw, h->stream);
    LV_CUDA(h, cudaMemcpyAsync(h->tot_h, h->tot_d, sizeof(Totals), cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    h->T = h->tot_h->e_own;
    LV_CUDA(h, cudaMemsetAsync(h->tot_d, 0, sizeof(Totals), h->stream));
    return to_level0(h);
}

int begin_create(const lv_opts *opts, int32_t V, int64_t E, lv_handle **out, lv_handle **hp) {
    if (!out) return LV_ERR_INVALID;
    *out = nullptr;
    if (V < 0 || E < 0) return LV_ERR_INVALID;
    if (E > 0x7fffffffLL || V >= 0x7fffffff) return LV_ERR_TOO_LARGE;
    lv_handle *h = new lv_handle();
    lv_default_opts(&h->opts);
    if (opts) {
        size_t n = opts->struct_size && opts->struct_size < sizeof(lv_opts) ? opts->struct_size : sizeof(lv_opts);
        std::memcpy(&h->opts, opts, n);
        h->opts.struct_size = sizeof(lv_opts);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        delete h;
        return LV_ERR_NO_DEVICE;
    }
    if (h->opts.device < 0 || h->opts.device >= ndev) {
        delete h;
        return LV_ERR_INVALID;
    }
    // work-mapping knobs (0 = default); results never depend on them
    if (h->opts.giant_degree != 0 &&
        (h->opts.giant_degree < HG_MIN_DEG_LO || h->opts.giant_degree > HG_MIN_DEG_HI)) {
        delete h;
        return LV_ERR_INVALID;
    }
    if (h->opts.warp_limit != 0 && (h->opts.warp_limit < WARP_LIMIT_MIN || h->opts.warp_limit > WARP_LIMIT_MAX)) {
        delete h;
        return LV_ERR_INVALID;
    }
    h->giant_degree = h->opts.giant_degree ? h->opts.giant_degree : HG_MIN_DEG;
    h->fb.warp_limit = h->opts.warp_limit ? h->opts.warp_limit : WARP_LIMIT;
    h->fb.hint_set = (h->fb.warp_limit * 3) / 4;
    h->device = h->opts.device;
    cudaSetDevice(h->device);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return LV_ERR_CUDA;
    }
    static bool attrs_done[64] = {false};
    init_kernel_attributes(h->di);
    if (h->device < 64 && !attrs_done[h->device]) {
        init_agg_attributes();
        attrs_done[h->device] = true;
    }
    h->V0 = V;
    h->E0 = E;
    h->launch_base = launches_total();
    *hp = h;
    return LV_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

void lv_default_opts(lv_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(lv_opts);
    o->device = 0;
    o->max_sweeps = 0;
    o->sweep_graph = 1;
    o->profile = 0;
}

const char *lv_status_string(int s) {
    switch (s) {
    case LV_OK: return "ok";
    case LV_ERR_INVALID: return "invalid argument or malformed CSR";
    case LV_ERR_WEIGHT: return "negative, NaN or infinite weight";
    case LV_ERR_TOO_LARGE: return "graph too large for int32 ids or the fixed-point grid";
    case LV_ERR_NOMEM: return "out of memory";
    case LV_ERR_CUDA: return "CUDA error";
    case LV_ERR_DEVICE: return "device-side check failed";
    case LV_ERR_IO: return "I/O or parse error";
    case LV_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
    }
}

int lv_trim_device_memory(int32_t device) {
    if (device < 0 || device >= LV_MAX_DEVICES) return LV_ERR_INVALID;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        pool = g_pool[device];
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cache_release(device, pool, 0);
    cudaDeviceSynchronize();
    cudaSetDevice(prev);
    if (!pool) return LV_OK;
    return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? LV_OK : LV_ERR_CUDA;
}

const char *lv_version(void) { return "louvain_b200 0.1 (sm_100a)"; }

int lv_destroy(lv_handle *h) {
    if (!h) return LV_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cache_release(h->device, device_pool(h->device), h->stream);
    h->destroying = true;
    if (h->owns_input) {
        dfree(h, h->in_rowptr);
        dfree(h, h->in_col);
        dfree(h, h->in_w);
    }
    {
        FallbackSet &fs = h->fb;
        dfree(h, fs.q[0].count); dfree(h, fs.hint);
        for (int q = 0; q <= NFBQ; ++q) {
            Fallback &f = fs.q[q];
            dfree(h, f.v); dfree(h, f.p); dfree(h, f.P); dfree(h, f.first); dfree(h, f.done); dfree(h, f.src);
            dfree(h, f.gd); dfree(h, f.e); dfree(h, f.S); dfree(h, f.eo); dfree(h, f.c); dfree(h, f.cnt);
        }
    }
    dfree(h, h->comm); dfree(h, h->newc); dfree(h, h->size); dfree(h, h->orig2comm);
    dfree(h, h->k); dfree(h, h->S); dfree(h, h->list); dfree(h, h->cls_scratch); dfree(h, h->sort_buf);
    {
        unsigned char *t = (unsigned char *)h->sort_temp;
        dfree(h, t);
        h->sort_temp = nullptr;
    }
    dfree(h, h->tbl_buf); dfree(h, h->occ_buf); dfree(h, h->nocc_buf);
    dfree(h, h->stage_key); dfree(h, h->stage_val); dfree(h, h->eown_buf); dfree(h, h->ovf_buf);
    dfree(h, h->stage2_key); dfree(h, h->stage2_val); dfree(h, h->poff_buf);
    for (HubLayout *L : {&h->hub_move, &h->hub_agg}) {
        unsigned char *d = (unsigned char *)L->dev;
        dfree(h, d);
        L->dev = nullptr;
    }
    AggBuffers &a = h->ab;
    dfree(h, a.flag); dfree(h, a.cdeg); dfree(h, a.mstart); dfree(h, a.cursor); dfree(h, a.members);
    dfree(h, a.lab); dfree(h, a.clist); dfree(h, a.newdeg); dfree(h, a.epos_new); dfree(h, a.scan_tmp);
    dfree(h, a.scalars);
    dfree(h, h->mslot); dfree(h, h->degm); dfree(h, h->P);
    for (int b = 0; b < 2; ++b) {
        dfree(h, h->lvl_start[b]); dfree(h, h->lvl_end[b]); dfree(h, h->lvl_col[b]); dfree(h, h->lvl_w[b]);
        dfree(h, h->lvl_w32[b]);
    }
    dfree(h, h->wrow);
    dfree(h, h->tot_d);
    dfree(h, h->feat); dfree(h, h->moved); dfree(h, h->nmoved); dfree(h, h->pred); dfree(h, h->fresh);
    dfree(h, h->comm_prev); dfree(h, h->alist);
    dfree(h, h->acnt); dfree(h, h->actr); dfree(h, h->model); dfree(h, h->tr_x); dfree(h, h->tr_v);
    dfree(h, h->tr_y);
    {
        LoopState *ld = (LoopState *)h->loop_d;
        dfree(h, ld);
        h->loop_d = nullptr;
    }
    pinned_give(h);
    for (const Pending &p : h->pend) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (cudaEvent_t e : h->ev_free) cudaEventDestroy(e);
    if (h->stream) {
        cudaStreamSynchronize(h->stream);   // the stream-ordered frees above
        cudaStreamDestroy(h->stream);
    }
    delete h;
    return LV_OK;
}

int lv_create(const int32_t *rowptr, const int32_t *col, const float *w, int32_t V, int64_t E,
              const lv_opts *opts, lv_handle **out) {
    if (!rowptr || (E > 0 && (!col || !w))) return LV_ERR_INVALID;
    lv_handle *h = nullptr;
    int rc = begin_create(opts, V, E, out, &h);
    if (rc) return rc;
    h->owns_input = true;
    rc = dalloc(h, &h->in_rowptr, (size_t)V + 1);
    if (!rc) rc = dalloc(h, &h->in_col, (size_t)E);
    if (!rc) rc = dalloc(h, &h->in_w, (size_t)E);
    if (!rc && cudaMemcpyAsync(h->in_rowptr, rowptr, sizeof(int32_t) * ((size_t)V + 1),
                               cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        rc = LV_ERR_CUDA;
    if (!rc && E > 0 &&
        cudaMemcpyAsync(h->in_col, col, sizeof(int32_t) * (size_t)E, cudaMemcpyHostToDevice,
                        h->stream) != cudaSuccess)
        rc = LV_ERR_CUDA;
    if (!rc && E > 0 &&
        cudaMemcpyAsync(h->in_w, w, sizeof(float) * (size_t)E, cudaMemcpyHostToDevice,
                        h->stream) != cudaSuccess)
        rc = LV_ERR_CUDA;
    if (!rc) rc = finish_create(h);
    if (rc) {
        lv_destroy(h);
        return rc;
    }
    *out = h;
    return LV_OK;
}

int lv_create_device(const int32_t *d_rowptr, const int32_t *d_col, const float *d_w, int32_t V,
                     int64_t E, const lv_opts *opts, lv_handle **out) {
    if (!d_rowptr || (E > 0 && (!d_col || !d_w))) return LV_ERR_INVALID;
    lv_handle *h = nullptr;
    int rc = begin_create(opts, V, E, out, &h);
    if (rc) return rc;
    h->owns_input = false;
    h->in_rowptr = const_cast<int32_t *>(d_rowptr);
    h->in_col = const_cast<int32_t *>(d_col);
    h->in_w = const_cast<float *>(d_w);
    rc = finish_create(h);
    if (rc) {
        lv_destroy(h);
        return rc;
    }
    *out = h;
    return LV_OK;
}

const char *lv_last_error(const lv_handle *h) { return h ? h->err.c_str() : "null handle"; }

int lv_reset(lv_handle *h) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    return to_level0(h);
}

int lv_optimise_level(lv_handle *h, float min_gain, int32_t *changed) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    return optimise_level(h, min_gain, changed);
}

int lv_aggregate(lv_handle *h) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    return aggregate(h);
}

int lv_modularity(lv_handle *h, double *q) {
    if (!h || !q) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    return modularity(h, q);
}

int lv_sweep(lv_handle *h, int64_t *moves) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    int64_t m = 0;
    LV_TRY(sweep_and_q(h, &m, nullptr));
    if (moves) *moves = m;
    return LV_OK;
}

int lv_run(lv_handle *h, float min_gain, double *q) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    for (;;) {
        int32_t changed = 0;
        LV_TRY(optimise_level(h, min_gain, &changed));
        if (!changed) break;
        LV_TRY(aggregate(h));
    }
    double qq = 0;
    LV_TRY(modularity(h, &qq));
    if (q) *q = qq;
    return LV_OK;
}

int lv_get_original_to_community(lv_handle *h, int32_t *out, int32_t *num_communities) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    if (out && h->V0 > 0)
        LV_CUDA(h, cudaMemcpyAsync(out, h->orig2comm, sizeof(int32_t) * (size_t)h->V0,
                                   cudaMemcpyDeviceToHost, h->stream));
    LV_TRY(sync(h));
    if (num_communities) *num_communities = h->V;
    return LV_OK;
}

int lv_get_communities(lv_handle *h, int32_t *out) {
    if (!h || !out) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    if (h->V > 0)
        LV_CUDA(h, cudaMemcpyAsync(out, h->comm, sizeof(int32_t) * (size_t)h->V,
                                   cudaMemcpyDeviceToHost, h->stream));
    return sync(h);
}

int lv_set_communities(lv_handle *h, const int32_t *comm) {
    if (!h || !comm) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    if (h->V == 0) return LV_OK;
    int32_t *tmp = h->cls_scratch + SCRATCH_OFF;   // V0 entries of scratch
    LV_CUDA(h, cudaMemcpyAsync(tmp, comm, sizeof(int32_t) * (size_t)h->V, cudaMemcpyHostToDevice,
                               h->stream));
    LV_CUDA(h, cudaMemsetAsync(&h->tot_d->err, 0, sizeof(int), h->stream));
    launch_set_communities(tmp, h->comm, h->newc, h->size, h->k, h->S, h->V, &h->tot_d->err, h->stream);
    h->e_own_valid = false;
    LV_TRY(read_totals(h));
    return LV_OK;
}

int lv_get_level_info(lv_handle *h, int32_t *V, int64_t *E, int32_t *level) {
    if (!h) return LV_ERR_INVALID;
    if (V) *V = h->V;
    if (E) *E = h->E;
    if (level) *level = h->level;
    return LV_OK;
}

int lv_get_level_classes(lv_handle *h, int32_t *vertices, int64_t *entries) {
    if (!h) return LV_ERR_INVALID;
    for (int c = 0; c < NCLS; ++c) {
        if (vertices) vertices[c] = h->cls_off[c + 1] - h->cls_off[c];
        if (entries) entries[c] = h->cls_edges[c];
    }
    return LV_OK;
}

int lv_get_device_name(int32_t device, char *name, int32_t len) {
    if (!name || len <= 0) return LV_ERR_INVALID;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
        cudaGetLastError();
        return LV_ERR_NO_DEVICE;
    }
    std::snprintf(name, (size_t)len, "%s (sm_%d%d, %d SMs)", p.name, p.major, p.minor, p.multiProcessorCount);
    return LV_OK;
}

int lv_get_csr(lv_handle *h, int32_t *rowptr, int32_t *col, int64_t *wfix) {
    if (!h) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    if (h->level == 0) {
        if (rowptr)
            LV_CUDA(h, cudaMemcpyAsync(rowptr, h->cur_rowptr, sizeof(int32_t) * ((size_t)h->V + 1),
                                       cudaMemcpyDeviceToHost, h->stream));
        if (col && h->E > 0)
            LV_CUDA(h, cudaMemcpyAsync(col, h->cur_col, sizeof(int32_t) * (size_t)h->E,
                                       cudaMemcpyDeviceToHost, h->stream));
        if (wfix && h->E > 0) {
            int64_t *tmp = nullptr;
            LV_TRY(dalloc(h, &tmp, (size_t)h->E));
            launch_weights_to_fixed<float>(h->in_w, h->E, h->scale_d, tmp, h->stream);
            cudaError_t e = cudaMemcpyAsync(wfix, tmp, sizeof(int64_t) * (size_t)h->E,
                                            cudaMemcpyDeviceToHost, h->stream);
            cudaStreamSynchronize(h->stream);
            dfree(h, tmp);
            if (e != cudaSuccess) return fail(h, LV_ERR_CUDA, cudaGetErrorString(e));
        }
        return sync(h);
    }
    // aggregated level: gather the (possibly non-contiguous) rows on the host
    const size_t V = (size_t)h->V;
    std::vector<int32_t> st(V + 1), en(V + 1);
    if (V) {
        LV_CUDA(h, cudaMemcpyAsync(st.data(), h->cur_rowptr, sizeof(int32_t) * V, cudaMemcpyDeviceToHost,
                                   h->stream));
        LV_CUDA(h, cudaMemcpyAsync(en.data(), h->cur_rowend, sizeof(int32_t) * V, cudaMemcpyDeviceToHost,
                                   h->stream));
    }
    LV_TRY(sync(h));
    int32_t span = 0;
    for (size_t v = 0; v < V; ++v) span = en[v] > span ? en[v] : span;
    std::vector<int32_t> c((size_t)span);
    std::vector<u64> w((size_t)span);
    if (span) {
        LV_CUDA(h, cudaMemcpyAsync(c.data(), h->cur_col, sizeof(int32_t) * (size_t)span,
                                   cudaMemcpyDeviceToHost, h->stream));
        LV_CUDA(h, cudaMemcpyAsync(w.data(), h->cur_w, sizeof(u64) * (size_t)span, cudaMemcpyDeviceToHost,
                                   h->stream));
    }
    LV_TRY(sync(h));
    int64_t at = 0;
    for (size_t v = 0; v < V; ++v) {
        if (rowptr) rowptr[v] = (int32_t)at;
        for (int32_t e = st[v]; e < en[v]; ++e, ++at) {
            if (col) col[at] = c[(size_t)e];
            if (wfix) wfix[at] = (int64_t)w[(size_t)e];
        }
    }
    if (rowptr) rowptr[V] = (int32_t)at;
    return LV_OK;
}

int lv_get_scale(lv_handle *h, int32_t *scale, uint64_t *total_weight, int32_t *exact) {
    if (!h) return LV_ERR_INVALID;
    if (scale) *scale = h->scale;
    if (total_weight) *total_weight = h->T;
    if (exact) *exact = h->exact;
    return LV_OK;
}

int lv_set_active_model(lv_handle *h, const uint16_t *model, int32_t n_params, float logit_threshold) {
    if (!h || !model || n_params != LV_ACTIVE_MODEL_SIZE) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    if (!h->model) LV_TRY(dalloc(h, &h->model, (size_t)LV_ACTIVE_MODEL_SIZE));
    LV_CUDA(h, cudaMemcpyAsync(h->model, model, sizeof(uint16_t) * LV_ACTIVE_MODEL_SIZE, cudaMemcpyHostToDevice,
                               h->stream));
    h->logit_thr = logit_threshold;
    h->has_model = true;
    return sync(h);
}

int lv_get_traces(lv_handle *h, float *features, uint8_t *labels, int64_t cap, int64_t *n) {
    if (!h || cap < 0) return LV_ERR_INVALID;
    cudaSetDevice(h->device);
    const int64_t rows = h->tr_rows;
    if (n) *n = rows;
    const int64_t m = rows < cap ? rows : cap;
    if (m > 0 && features)
        LV_CUDA(h, cudaMemcpyAsync(features, h->tr_x, sizeof(float) * LV_ACTIVE_FEATURES * (size_t)m,
                                   cudaMemcpyDeviceToHost, h->stream));
    if (m > 0 && labels)
        LV_CUDA(h, cudaMemcpyAsync(labels, h->tr_y, (size_t)m, cudaMemcpyDeviceToHost, h->stream));
    return sync(h);
}

int lv_get_active_stats(lv_handle *h, int64_t *evaluated, int64_t *full_sweeps, int64_t *active_sweeps,
                        double *last_recall, int32_t *fell_back) {
    if (!h) return LV_ERR_INVALID;
    if (evaluated) *evaluated = h->act_evaluated;
    if (full_sweeps) *full_sweeps = h->act_full;
    if (active_sweeps) *active_sweeps = h->act_active;
    if (last_recall) *last_recall = h->act_recall;
    if (fell_back) *fell_back = h->act_fell_back;
    return LV_OK;
}

int lv_get_stats(lv_handle *h, lv_stats *s) {
    if (!h || !s) return LV_ERR_INVALID;
    LV_TRY(sync(h));
    *s = h->st;
    s->kernel_launches = launches_total() - h->launch_base;
    return LV_OK;
}

int lv_get_class_stats(lv_handle *h, lv_class_stats *s) {
    if (!h || !s) return LV_ERR_INVALID;
    LV_TRY(sync(h));
    *s = h->cst;
    return LV_OK;
}

int lv_clear_stats(lv_handle *h) {
    if (!h) return LV_ERR_INVALID;
    LV_TRY(sync(h));
    std::memset(&h->st, 0, sizeof(h->st));
    std::memset(&h->cst, 0, sizeof(h->cst));
    h->launch_base = launches_total();
    h->act_evaluated = h->act_full = h->act_active = 0;
    h->act_recall = -1.0;
    h->act_fell_back = 0;
    return LV_OK;
}

}  // extern "C"
