// lv_common.cuh -- shared device helpers of the Louvain engine (sm_100a).
//
// Arithmetic model.  Every edge weight is an unsigned integer on a 2^-scale
// grid (level 0 converts float32 weights on load; aggregated levels store the
// exact uint64 sums).  k_i, Sigma_tot and e_{i,C} are exact uint64 sums, so
// their value never depends on the order of atomic additions.  The gain of
// the reference (modularity_optimisation.cu:96-102)
//     g(C) = e_C/M + k (S_own - k - S_C) / (2 M^2),  M = T/2
// is compared through G(C) = g(C) * T^2 / 2 = T e_C + k (S_own - k - S_C),
// an exact 128-bit integer (|G| <= 2 T^2 < 2^126 because T <= 2^62).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Tuning knobs (compile-time): edges per lane in flight in the insert loops
// of the group kernels (LV_U_GROUP), the warp kernel (LV_U_WARP), the small
// and medium fallback CTAs (LV_U_FB) and the giant staging CTAs
// (LV_U_STAGE), and table entries per lane in flight in the evaluation loops
// of the group kernels (LV_U_EVAL).
#ifndef LV_U_GROUP
#define LV_U_GROUP 2
#endif
#ifndef LV_U_CTA
#define LV_U_CTA 4
#endif
#ifndef LV_U_EVAL
#define LV_U_EVAL 4
#endif
#ifndef LV_U_WARP
#define LV_U_WARP 4
#endif
#ifndef LV_U_FB
#define LV_U_FB 4
#endif
#ifndef LV_U_STAGE
#define LV_U_STAGE 8
#endif
// The insert loops combine a warp's equal keys before their atomics
// (key_peers: __match_any_sync + __reduce_add_sync): 1 on aggregated levels,
// 2 at every level, 0 never (the code compiled out), 3 never (the code
// compiled in, switched off at run time; for measurement).  0 is the
// default: with 1 the move phase of an R-MAT-24 run took 620 ms instead of
// 306 ms, and merely compiling the code in (3) costs 5 % (256 against 243 ms
// of move phase: the degree > 319 class 119.8 against 111.6 ms).
#ifndef LV_DEDUP
#define LV_DEDUP 0
#endif
// The 64-bit warp kernel sums runs of one community per lane in registers
// before its table adds (1) or adds every entry (0, the default: 1 measured
// no faster on R-MAT-24, 121 against 120 ms for the degree > 319 class).
#ifndef LV_WARP_COMBINE
#define LV_WARP_COMBINE 0
#endif
// The row insert loops of the CTA and group kernels load U entries that all
// lie inside the row without per-entry bound tests (1) or test each (0, the
// default: 1 made the giants' staging 0.8 ms faster and the row queues
// 0.9 ms slower per R-MAT-24 run).
#ifndef LV_ROW_FULLSTEP
#define LV_ROW_FULLSTEP 0
#endif
// The narrow-weight warp kernel issues the next chunk's column and weight
// loads before inserting the current chunk (1), or loads each chunk when it
// gets to it (0, the default: 1 made the degree > 319 class of an R-MAT-24
// run 15 % slower).
#ifndef LV_WARP_PIPE
#define LV_WARP_PIPE 0
#endif
// The narrow-weight warp kernel loads the home-slot keys of its U entries
// together before inserting (1) or probes entry by entry (0).
#ifndef LV_WARP_PREFETCH
#define LV_WARP_PREFETCH 1
#endif

namespace lv {

typedef unsigned long long u64;
typedef long long i64;
typedef __int128 i128;
typedef unsigned __int128 u128;

constexpr unsigned FULL = 0xffffffffu;

// Update-order buckets (modularity_optimisation.cuh:7-8): bucket b holds the
// vertices with BOUNDS[b] < degree <= BOUNDS[b+1]; degree-0 vertices never move.
constexpr int NBUCKETS = 7;

// Work classes: how a vertex is mapped onto threads.  Classes 0..5 equal
// buckets 0..5; bucket 6 (degree > 319) is split by degree into three
// classes that differ only in where their hash table lives.
enum WorkClass {
    CLS_B0 = 0,   // (0,4]       4 lanes / vertex, shared table of 8
    CLS_B1,       // (4,8]       8 lanes, table 16
    CLS_B2,       // (8,16]      16 lanes, table 32
    CLS_B3,       // (16,32]     32 lanes, table 64
    CLS_B4,       // (32,84]     warp table (bucket 4)
    CLS_B5,       // (84,319]    warp table (bucket 5)
    CLS_H1,       // (319,1024]  warp table, CTA fallback (bucket 6)
    CLS_H2,       // (1024,8192] warp table, CTA fallback (bucket 6)
    CLS_HG,       // > 8192      edge chunks staged and merged (bucket 6)
    NCLS
};
// Giants: degree above giant_degree (a tuning knob, lv_opts.giant_degree:
// default HG_MIN_DEG, at least HG_MIN_DEG_LO so that CLS_H1 is unchanged, at
// most HG_MIN_DEG_HI so that a warp's row fits its piece counters).
constexpr int HG_MIN_DEG = 8192;
constexpr int HG_MIN_DEG_LO = 1024, HG_MIN_DEG_HI = 65536;
// class -> update bucket
__host__ __device__ constexpr int class_bucket(int c) { return c < CLS_H1 ? c : 6; }

__host__ __device__ __forceinline__ int degree_class(int32_t d, int32_t giant_degree = HG_MIN_DEG) {
    if (d <= 0) return -1;
    if (d <= 4) return CLS_B0;
    if (d <= 8) return CLS_B1;
    if (d <= 16) return CLS_B2;
    if (d <= 32) return CLS_B3;
    if (d <= 84) return CLS_B4;
    if (d <= 319) return CLS_B5;
    if (d <= 1024) return CLS_H1;
    if (d <= giant_degree) return CLS_H2;
    return CLS_HG;
}

// Device error bits (OR-ed into a device word, read back once per sweep).
enum DevErr { DEVERR_HASH_FULL = 1, DEVERR_BAD_STATE = 2, DEVERR_FALLBACK_FULL = 4 };

__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

__host__ __device__ constexpr int ilog2_c(int x) { return x <= 1 ? 0 : 1 + ilog2_c(x >> 1); }

__host__ __device__ __forceinline__ int ceil_log2_i(int64_t x) {
    int r = 0;
    while ((int64_t(1) << r) < x) r++;
    return r;
}

// Multiplicative hash into a table of 2^lg slots (lg >= 1).
__device__ __forceinline__ uint32_t hash_slot(int32_t key, int lg) {
    return ((uint32_t)key * 0x9E3779B1u) >> (32 - lg);
}

// Hash of the aggregation's tables, independent of hash_slot.  Aggregation
// writes each merged row in the slot order of its table, so with a shared
// hash a chunk of such a row holds keys whose hash_slot top bits nearly
// coincide and the move phase's chunk tables degenerate into one long probe
// run.  Two multiply-xorshift rounds decorrelate the two orders.
__device__ __forceinline__ uint32_t hash_slot_agg(int32_t key, int lg) {
    uint32_t x = (uint32_t)key * 0x2C1B3C6Du;
    x ^= x >> 15;
    x *= 0x297A2D39u;
    x ^= x >> 13;
    return x >> (32 - lg);
}

// H = 0: move-phase tables; H = 1: aggregation tables.
template <int H>
__device__ __forceinline__ uint32_t table_hash(int32_t key, int lg) {
    return H == 0 ? hash_slot(key, lg) : hash_slot_agg(key, lg);
}

// Weight access: level 0 reads float32 and maps it onto the fixed grid
// (exact: w * 2^scale is a power-of-two scaling, then round-to-nearest-even,
// the same rule as the host's llrint(ldexp(w, scale))); later levels read the
// stored uint64 sums, or their 32-bit copy when every sum of the level is
// below 2^32.
__device__ __forceinline__ u64 wfix(const float *w, int64_t e, double scale) {
    return (u64)__double2ll_rn(__dmul_rn((double)__ldg(w + e), scale));
}
__device__ __forceinline__ u64 wfix(const u64 *w, int64_t e, double) { return __ldg(w + e); }
__device__ __forceinline__ u64 wfix(const uint32_t *w, int64_t e, double) { return (u64)__ldg(w + e); }

// The same reads with the streaming (evict-first) cache hint, for row data
// read once per sweep, so that it does not push the gathered per-vertex
// arrays (communities, Sigma_tot) out of L2.
#ifndef LV_STREAM_ROWS
#define LV_STREAM_ROWS 1
#endif
template <typename T>
__device__ __forceinline__ T ld_row(const T *p) {
#if LV_STREAM_ROWS
    return __ldcs(p);
#else
    return __ldg(p);
#endif
}
__device__ __forceinline__ u64 wfix_row(const float *w, int64_t e, double scale) {
    return (u64)__double2ll_rn(__dmul_rn((double)ld_row(w + e), scale));
}
__device__ __forceinline__ u64 wfix_row(const u64 *w, int64_t e, double) { return ld_row(w + e); }
__device__ __forceinline__ u64 wfix_row(const uint32_t *w, int64_t e, double) { return (u64)ld_row(w + e); }

// A level's graph: row v is col/w[rowptr[v] .. rowend[v]).  Level 0 is a
// plain CSR (rowend = rowptr + 1); aggregated levels keep each merged row
// where the merge wrote it, so rows need not be contiguous.
template <typename WT>
struct GraphView {
    const int32_t *rowptr;
    const int32_t *rowend;
    const int32_t *col;
    const WT *w;
    double scale;     // 2^scale (used for float weights only)
    const u64 *w64;   // 32-bit view of an aggregated level: the uint64 sums, read
                      // where the 32-bit copy holds W32_ESC
    int64_t nent;     // entries allocated in col / w (bulk copies stay below it)
};

// The 32-bit copy of an aggregated level holds each sum below W32_ESC as it
// is and W32_ESC (an escape) for larger ones, whose exact value is read from
// the uint64 sums.  A row with an escaped entry other than its self-loop is
// marked (lv_handle::wrow) and decided by the 64-bit kernels, so the
// piece-counter tables only ever see weights below 2^32.
constexpr uint32_t W32_ESC = 0xFFFFFFFFu;

// Exact weight of entry e of a level's row.
__device__ __forceinline__ u64 gw(const GraphView<float> &g, int64_t e) { return wfix(g.w, e, g.scale); }
__device__ __forceinline__ u64 gw(const GraphView<u64> &g, int64_t e) { return __ldg(g.w + e); }
__device__ __forceinline__ u64 gw(const GraphView<uint32_t> &g, int64_t e) {
    const uint32_t x = __ldg(g.w + e);
    return x != W32_ESC ? (u64)x : __ldg(g.w64 + e);
}
// ... with the streaming cache hint (row data read once per sweep)
__device__ __forceinline__ u64 gw_row(const GraphView<float> &g, int64_t e) { return wfix_row(g.w, e, g.scale); }
__device__ __forceinline__ u64 gw_row(const GraphView<u64> &g, int64_t e) { return ld_row(g.w + e); }
__device__ __forceinline__ u64 gw_row(const GraphView<uint32_t> &g, int64_t e) {
    const uint32_t x = ld_row(g.w + e);
    return x != W32_ESC ? (u64)x : __ldg(g.w64 + e);
}

// Row weights as loaded (32 bits for float and the 32-bit view) and their
// exact value: a chunk's weights can be loaded one step ahead of their use
// while holding one register each.
template <typename WT>
struct RawOf { typedef uint32_t T; };
template <>
struct RawOf<u64> { typedef u64 T; };
__device__ __forceinline__ u64 raw_row(const GraphView<u64> &g, int64_t e) { return ld_row(g.w + e); }
__device__ __forceinline__ u64 raw_value(const GraphView<u64> &, int64_t, u64 x) { return x; }
__device__ __forceinline__ uint32_t raw_row(const GraphView<float> &g, int64_t e) {
    return __float_as_uint(ld_row(g.w + e));
}
__device__ __forceinline__ uint32_t raw_row(const GraphView<uint32_t> &g, int64_t e) { return ld_row(g.w + e); }
__device__ __forceinline__ u64 raw_value(const GraphView<float> &g, int64_t, uint32_t x) {
    return (u64)__double2ll_rn(__dmul_rn((double)__uint_as_float(x), g.scale));
}
__device__ __forceinline__ u64 raw_value(const GraphView<uint32_t> &g, int64_t e, uint32_t x) {
    return x != W32_ESC ? (u64)x : __ldg(g.w64 + e);
}

// ---------------------------------------------------------------------------
// 1-D bulk copies (TMA, no tensor map) into shared memory, completed on an
// mbarrier.  Addresses and sizes are multiples of 16 bytes; a CTA launched
// without a cluster is its own cluster of one, so its shared::cta addresses
// are valid shared::cluster destinations.  Waits are bounded: a wait that runs
// out reports false and the caller records a device error.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// one arrival that also announces `bytes` of transfers still to complete
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// generic-proxy accesses of shared memory ordered before later bulk copies
// into it
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait_parity(uint64_t *bar, uint32_t parity, uint32_t max_polls) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < max_polls; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
constexpr uint32_t MBAR_MAX_POLLS = 1u << 22;   // each try_wait may itself suspend for a while

struct StateView {
    int32_t *comm;
    int32_t *newc;
    int32_t *size;
    u64 *k;
    u64 *S;
    u64 T;
    int *err;
    float *feat;   // learned active set: 2 features per vertex, written when set
    const uint8_t *wrow;   // rows with a weight of 2^32 or more (nullptr: none); such a
                           // vertex is decided by the large fallback queue (64-bit sums)
    int dedup;             // aggregated level: the narrow insert loops combine a warp's
                           // equal keys before their shared atomics (key_peers)
};

// Exact 64-bit add to a table value.  In shared memory a 64-bit atomicAdd
// is a compare-and-swap loop that spins when many lanes hit one slot, so it
// is done as two native 32-bit atomic adds: the low word's returned old value
// gives the carry into the high word.  The final hi:lo equals the 64-bit sum
// whatever the order of the adds (read it only after they have all
// completed).  Global tables use the native 64-bit atomic.
// LV_TABLE_SPACE_CHECK = 0: every table add takes the split form, which is
// exact in global memory too (a global table then pays two atomics instead
// of one) and drops the address-space test; it measured no faster (the
// compiler already resolves the test where the table is known to be shared).
#ifndef LV_TABLE_SPACE_CHECK
#define LV_TABLE_SPACE_CHECK 1
#endif
__device__ __forceinline__ void table_add(u64 *p, u64 w) {
    if (!LV_TABLE_SPACE_CHECK || __isShared(p)) {
        unsigned *q = reinterpret_cast<unsigned *>(p);
        const unsigned lo = (unsigned)w, hi = (unsigned)(w >> 32);
        const unsigned old = atomicAdd(q, lo);
        const unsigned carry = (old + lo < old) ? 1u : 0u;
        if (hi | carry) atomicAdd(q + 1, hi + carry);
    } else {
        atomicAdd(p, w);
    }
}

// Insert (key, w) into an open-addressing table with linear probing; works
// for shared and global tables (generic addressing).  A key once written
// never changes, so a stale EMPTY read only costs a failed CAS.  The probe
// count is bounded by the capacity; a full table sets an error bit instead
// of spinning.
template <int H = 0>
__device__ __forceinline__ void table_insert(int32_t *keys, u64 *vals, int lg, int32_t key,
                                             u64 w, int *err) {
    const uint32_t mask = (1u << lg) - 1u;
    uint32_t s = table_hash<H>(key, lg);
    for (uint32_t p = 0; p <= mask; ++p) {
        int32_t k = ((volatile int32_t *)keys)[s];
        if (k == key) { table_add(vals + s, w); return; }
        if (k < 0) {
            int32_t prev = atomicCAS(keys + s, -1, key);
            if (prev < 0 || prev == key) { table_add(vals + s, w); return; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
}

// table_insert that returns the slot it newly claimed for `key` (-1 when the
// key was already present or the table is full).
template <int H = 0>
__device__ __forceinline__ int32_t table_insert_claim(int32_t *keys, u64 *vals, int lg, int32_t key,
                                                      u64 w, int *err) {
    const uint32_t mask = (1u << lg) - 1u;
    uint32_t s = table_hash<H>(key, lg);
    for (uint32_t p = 0; p <= mask; ++p) {
        int32_t k = ((volatile int32_t *)keys)[s];
        if (k == key) { table_add(vals + s, w); return -1; }
        if (k < 0) {
            int32_t prev = atomicCAS(keys + s, -1, key);
            if (prev < 0) { table_add(vals + s, w); return (int32_t)s; }
            if (prev == key) { table_add(vals + s, w); return -1; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
    return -1;
}

// Shared table whose sums are kept as two 32-bit counters of 16-bit pieces:
// lo[s] sums w & 0xFFFF and hi[s] sums w >> 16 of weights below 2^32, so the
// value hi * 2^16 + lo is the exact 64-bit sum as long as a slot takes at
// most 65537 additions (a row or chunk of at most 65536 entries).  Both adds
// are fire-and-forget shared atomics (no returned value to wait for, no
// carry), which is what the move phase's rows need once weights fit 32 bits
// (level 0 with a fixed-point grid below 2^32 and every aggregated level
// whose merged sums, self-loops aside, stay below 2^32).
struct PieceTable {
    int32_t *keys;
    uint32_t *lo;
    uint32_t *hi;
};
constexpr int PIECE_MAX_ADDS = 65536;   // rows or chunks longer than this need 64-bit sums

__device__ __forceinline__ void piece_add(const PieceTable &t, uint32_t s, u64 w) {
    atomicAdd(t.lo + s, (uint32_t)w & 0xFFFFu);
    atomicAdd(t.hi + s, (uint32_t)(w >> 16));
}

__device__ __forceinline__ u64 piece_value(const PieceTable &t, uint32_t s) {
    return ((u64)t.hi[s] << 16) + (u64)t.lo[s];
}

// Insert (key, w) into a piece table (move-phase hash, linear probing,
// bounded by the capacity); returns the slot newly claimed for key, or -1.
// piece_insert_at starts at slot s = hash_slot(key, lg) (computed by the
// caller, who may have loaded its key already to overlap the load latency).
__device__ __forceinline__ int32_t piece_insert_at(const PieceTable &t, int lg, uint32_t s, int32_t key, u64 w,
                                                   int *err) {
    const uint32_t mask = (1u << lg) - 1u;
    for (uint32_t p = 0; p <= mask; ++p) {
        const int32_t k = ((volatile int32_t *)t.keys)[s];
        if (k == key) { piece_add(t, s, w); return -1; }
        if (k < 0) {
            const int32_t prev = atomicCAS(t.keys + s, -1, key);
            if (prev < 0) { piece_add(t, s, w); return (int32_t)s; }
            if (prev == key) { piece_add(t, s, w); return -1; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
    return -1;
}

__device__ __forceinline__ int32_t piece_insert(const PieceTable &t, int lg, int32_t key, u64 w, int *err) {
    return piece_insert_at(t, lg, hash_slot(key, lg), key, w, err);
}

// Warp-level combining of equal keys before the shared atomics.  On
// aggregated levels a row's entries fall into a few communities, so many
// lanes of a warp add to the same slot and their atomics serialise.
// key_peers gives the lanes of the warp holding the same valid key (an
// invalid lane groups alone); the group's weights are summed piecewise with
// redux.sync (a group has at most 32 lanes, so each 16-bit-piece sum stays
// below 2^21), and only the group's lowest lane touches the table.  All 32
// lanes must call these together.
__device__ __forceinline__ unsigned key_peers(int32_t key, bool valid) {
    return __match_any_sync(FULL, valid ? key : (int32_t)(0x80000000u | (threadIdx.x & 31u)));
}
struct Pieces {
    uint32_t lo, hi;   // sum of (w & 0xFFFF) and of (w >> 16) over the group
};
__device__ __forceinline__ Pieces group_pieces(unsigned peers, u64 w) {
    Pieces p;
    p.lo = __reduce_add_sync(peers, (uint32_t)w & 0xFFFFu);
    p.hi = __reduce_add_sync(peers, (uint32_t)(w >> 16));
    return p;
}
// Exact uint64 sum over the group: four 16-bit-piece sums (each below 2^21)
// recombined modulo 2^64, which is the exact sum while that stays below 2^64
// (as every weight sum of a level does).
__device__ __forceinline__ u64 group_sum_u64(unsigned peers, u64 w) {
    const u64 p0 = __reduce_add_sync(peers, (uint32_t)w & 0xFFFFu);
    const u64 p1 = __reduce_add_sync(peers, (uint32_t)(w >> 16) & 0xFFFFu);
    const u64 p2 = __reduce_add_sync(peers, (uint32_t)(w >> 32) & 0xFFFFu);
    const u64 p3 = __reduce_add_sync(peers, (uint32_t)(w >> 48));
    return p0 + (p1 << 16) + (p2 << 32) + (p3 << 48);
}
__device__ __forceinline__ bool group_leader(unsigned peers) {
    return (threadIdx.x & 31u) == (unsigned)(__ffs(peers) - 1);
}
__device__ __forceinline__ void piece_add_p(const PieceTable &t, uint32_t s, Pieces p) {
    atomicAdd(t.lo + s, p.lo);
    atomicAdd(t.hi + s, p.hi);
}
// piece_insert_at for a group's combined pieces (the group counts as one
// add per member towards PIECE_MAX_ADDS, as before combining).
__device__ __forceinline__ int32_t piece_insert_at_p(const PieceTable &t, int lg, uint32_t s, int32_t key, Pieces p,
                                                     int *err) {
    const uint32_t mask = (1u << lg) - 1u;
    for (uint32_t q = 0; q <= mask; ++q) {
        const int32_t k = ((volatile int32_t *)t.keys)[s];
        if (k == key) { piece_add_p(t, s, p); return -1; }
        if (k < 0) {
            const int32_t prev = atomicCAS(t.keys + s, -1, key);
            if (prev < 0) { piece_add_p(t, s, p); return (int32_t)s; }
            if (prev == key) { piece_add_p(t, s, p); return -1; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
    return -1;
}

// Append the slots claimed by this warp's lanes (claimed >= 0) to occ[],
// reserving space with one atomic per warp.  All 32 lanes must call it.
__device__ __forceinline__ void warp_append(int32_t claimed, int32_t *occ, int32_t *nocc) {
    const unsigned bal = __ballot_sync(FULL, claimed >= 0);
    if (!bal) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(bal) - 1;
    int32_t base = 0;
    if (lane == leader) base = atomicAdd(nocc, __popc(bal));
    base = __shfl_sync(FULL, base, leader);
    if (claimed >= 0) occ[base + __popc(bal & ((1u << lane) - 1u))] = claimed;
}

// warp_append for a list of occ_cap entries: *nocc counts every claim, the
// first occ_cap of them are listed.  All 32 lanes must call it.
__device__ __forceinline__ void warp_append_capped(int32_t claimed, int32_t *occ, int32_t *nocc, int32_t occ_cap) {
    const unsigned bal = __ballot_sync(FULL, claimed >= 0);
    if (!bal) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(bal) - 1;
    int32_t base = 0;
    if (lane == leader) base = atomicAdd(nocc, __popc(bal));
    base = __shfl_sync(FULL, base, leader);
    const int32_t i = base + __popc(bal & ((1u << lane) - 1u));
    if (claimed >= 0 && i < occ_cap) occ[i] = claimed;
}

// table_insert that also appends every newly claimed slot to occ[] (count in
// *nocc), so that evaluation and clearing visit only occupied slots.
__device__ __forceinline__ void table_insert_occ(int32_t *keys, u64 *vals, int lg, int32_t key,
                                                 u64 w, int *err, int32_t *occ, int32_t *nocc) {
    const uint32_t mask = (1u << lg) - 1u;
    uint32_t s = hash_slot(key, lg);
    for (uint32_t p = 0; p <= mask; ++p) {
        int32_t k = ((volatile int32_t *)keys)[s];
        if (k == key) { table_add(vals + s, w); return; }
        if (k < 0) {
            int32_t prev = atomicCAS(keys + s, -1, key);
            if (prev < 0) {
                table_add(vals + s, w);
                occ[atomicAdd(nocc, 1)] = (int32_t)s;
                return;
            }
            if (prev == key) { table_add(vals + s, w); return; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
}

// table_insert_occ for tables whose occupied list holds occ_cap slots: a
// claim beyond that is reported as DEVERR_HASH_FULL and not listed.
__device__ __forceinline__ void table_insert_occ_capped(int32_t *keys, u64 *vals, int lg, int32_t key,
                                                        u64 w, int *err, int32_t *occ, int32_t *nocc,
                                                        int32_t occ_cap) {
    const uint32_t mask = (1u << lg) - 1u;
    uint32_t s = hash_slot(key, lg);
    for (uint32_t p = 0; p <= mask; ++p) {
        int32_t k = ((volatile int32_t *)keys)[s];
        if (k == key) { table_add(vals + s, w); return; }
        if (k < 0) {
            int32_t prev = atomicCAS(keys + s, -1, key);
            if (prev < 0) {
                table_add(vals + s, w);
                const int32_t i = atomicAdd(nocc, 1);
                if (i < occ_cap) occ[i] = (int32_t)s;
                else atomicOr(err, DEVERR_HASH_FULL);
                return;
            }
            if (prev == key) { table_add(vals + s, w); return; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
}

// Insert the row col/w[r0..r1) of vertex v, lanes lane, lane+stride, ...,
// into a table, U edges per lane at a time so that U column loads and then U
// community gathers are in flight together.  Self-loops are skipped; the
// weight to the own community is summed into *e_own instead of the table.
// OCC: record newly claimed slots in occ[] / *nocc.
template <int U, bool OCC, typename WT>
__device__ __forceinline__ void insert_row(const GraphView<WT> &g, const int32_t *__restrict__ comm,
                                           int32_t v, int32_t own, int32_t r0, int32_t r1, int lane,
                                           int stride, int32_t *keys, u64 *vals, int lg, int *err,
                                           int32_t *occ, int32_t *nocc, u64 &e_own, bool dedup = false) {
    // dedup (CTA-wide OCC callers only: lane = threadIdx.x, stride a multiple
    // of 32): the loop then runs the same steps in every lane of a warp and a
    // warp's equal keys are combined before the atomics (key_peers)
    const int32_t wlane = (LV_DEDUP && OCC && dedup) ? (lane & 31) : 0;
    for (int32_t base = r0 + lane; base - wlane < r1; base += U * stride) {
        int32_t jj[U];
        u64 ww[U];
        int32_t cc[U];
        if (LV_ROW_FULLSTEP && base + (U - 1) * stride < r1) {
            // all U entries inside the row: no bound tests
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = base + u * stride;
                jj[u] = __ldg(g.col + e);
                ww[u] = gw(g, e);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = jj[u] != v ? __ldg(comm + jj[u]) : -1;
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = base + u * stride;
                jj[u] = -1;
                ww[u] = 0;
                if (e < r1) {
                    jj[u] = __ldg(g.col + e);
                    ww[u] = gw(g, e);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? __ldg(comm + jj[u]) : -1;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (LV_DEDUP && OCC && dedup) {
                const bool valid = cc[u] >= 0 && cc[u] != own;
                if (cc[u] >= 0 && cc[u] == own) e_own += ww[u];
                const unsigned peers = key_peers(cc[u], valid);
                const u64 ws = group_sum_u64(peers, valid ? ww[u] : 0);
                if (valid && group_leader(peers)) table_insert_occ(keys, vals, lg, cc[u], ws, err, occ, nocc);
                continue;
            }
            if (cc[u] < 0) continue;
            if (cc[u] == own) {
                e_own += ww[u];
            } else if (OCC) {
                table_insert_occ(keys, vals, lg, cc[u], ww[u], err, occ, nocc);
            } else {
                table_insert(keys, vals, lg, cc[u], ww[u], err);
            }
        }
    }
}

// insert_row for piece tables (weights below 2^32, at most PIECE_MAX_ADDS
// entries): OCC records every newly claimed slot in occ[] (the first occ_cap
// of them; *nocc counts them all).
template <int U, bool OCC, typename WT>
__device__ __forceinline__ void insert_row_piece(const GraphView<WT> &g, const int32_t *__restrict__ comm,
                                                 int32_t v, int32_t own, int32_t r0, int32_t r1, int lane,
                                                 int stride, const PieceTable &t, int lg, int *err,
                                                 int32_t *occ, int32_t *nocc, int32_t occ_cap, u64 &e_own,
                                                 bool dedup = false) {
    // OCC (CTA-wide callers: lane = threadIdx.x, stride a multiple of 32):
    // the loop runs the same number of steps in every lane of a warp, so the
    // claims of a step are listed with one shared atomic per warp
    const int32_t wlane = OCC ? (lane & 31) : 0;
    for (int32_t base = r0 + lane; base - wlane < r1; base += U * stride) {
        int32_t jj[U];
        u64 ww[U];
        int32_t cc[U];
        if (LV_ROW_FULLSTEP && base + (U - 1) * stride < r1) {
            // all U entries inside the row: no bound tests
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = base + u * stride;
                jj[u] = __ldg(g.col + e);
                ww[u] = gw(g, e);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = jj[u] != v ? __ldg(comm + jj[u]) : -1;
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = base + u * stride;
                jj[u] = -1;
                ww[u] = 0;
                if (e < r1) {
                    jj[u] = __ldg(g.col + e);
                    ww[u] = gw(g, e);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? __ldg(comm + jj[u]) : -1;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            int32_t claimed = -1;
            if (LV_DEDUP && OCC && dedup) {
                // equal keys of the warp combined first (see key_peers)
                const bool valid = cc[u] >= 0 && cc[u] != own;
                if (cc[u] >= 0 && cc[u] == own) e_own += ww[u];
                const unsigned peers = key_peers(cc[u], valid);
                const Pieces pc = group_pieces(peers, valid ? ww[u] : 0);
                if (valid && group_leader(peers))
                    claimed = piece_insert_at_p(t, lg, hash_slot(cc[u], lg), cc[u], pc, err);
            } else if (cc[u] >= 0) {
                if (cc[u] == own) e_own += ww[u];
                else claimed = piece_insert(t, lg, cc[u], ww[u], err);
            }
            if (OCC) warp_append_capped(claimed, occ, nocc, occ_cap);
        }
    }
}

// ---------------------------------------------------------------------------
// Gain comparison.
//
// For vertex v (own community o, weight k, S_o = Sigma_tot[o]) and candidate
// community C with weight e_C from v and Sigma_tot S_C, the reference's gain
// (modularity_optimisation.cu:96-102) scaled by T^2/2 is the integer
//     G(C) = T e_C + k (S_o - k - S_C)                 (|G| < 2^126)
// "Stay" is the initial best with G = 0 (:137-138).  Candidates are compared
// with an FP64 estimate g~ whose error is bounded by
//     |g~ - G| <= 2^-50 (T e_C + k |S_o - k - S_C|)
// (each operand is one rounding away from its integer, the products and the
// sum add three more, each <= 2^-53 relative); when the two intervals
// overlap the exact 128-bit values decide, ties going to the lower id
// (:157,169,182).  The result is the exact argmax.
// ---------------------------------------------------------------------------
struct MoveCtx {
    int32_t own;
    bool own_single;
    u64 T;
    u64 kv;
    u64 sown;
    double Td;
    double kvd;
};

__device__ __forceinline__ MoveCtx move_ctx(int32_t own, bool own_single, u64 T, u64 kv, u64 sown) {
    MoveCtx m;
    m.own = own;
    m.own_single = own_single;
    m.T = T;
    m.kv = kv;
    m.sown = sown;
    m.Td = (double)T;
    m.kvd = (double)kv;
    return m;
}

// Exact G for (e, S); the stay candidate (c == own) has G = 0.
__device__ __forceinline__ i128 exact_gain(const MoveCtx &m, u64 e, u64 S) {
    const u128 te = ((u128)__umul64hi(m.T, e) << 64) | (u128)(m.T * e);
    const i64 d = (i64)m.sown - (i64)m.kv - (i64)S;
    const u64 ad = d < 0 ? (u64)0 - (u64)d : (u64)d;
    const u128 kd = ((u128)__umul64hi(m.kv, ad) << 64) | (u128)(m.kv * ad);
    return d < 0 ? (i128)te - (i128)kd : (i128)te + (i128)kd;
}

// Running best of one thread (or group): FP64 estimate gd of G, community c,
// weight e and Sigma_tot S of c (to recompute G exactly), and e_own, the
// summed weight to the own community.
struct Best {
    double gd;
    u64 e;
    u64 S;
    int32_t c;
    u64 eo;
};

__device__ __forceinline__ Best best_init(int32_t own) {
    Best b;
    b.gd = 0.0;
    b.e = 0;
    b.S = 0;
    b.c = own;
    b.eo = 0;
    return b;
}

__device__ __forceinline__ double gain_err(const MoveCtx &m, const Best &b) {
    if (b.c == m.own) return 0.0;
    const double dd = (double)((i64)m.sown - (i64)m.kv - (i64)b.S);
    return (m.Td * (double)b.e + m.kvd * fabs(dd)) * 0x1p-50;
}

// true iff candidate a is strictly better than b (exact order).
__device__ __forceinline__ bool better(const MoveCtx &m, const Best &a, const Best &b) {
    const double ea = gain_err(m, a), eb = gain_err(m, b);
    if (a.gd - ea > b.gd + eb) return true;
    if (b.gd - eb > a.gd + ea) return false;
    const i128 ga = a.c == m.own ? (i128)0 : exact_gain(m, a.e, a.S);
    const i128 gb = b.c == m.own ? (i128)0 : exact_gain(m, b.e, b.S);
    return ga > gb || (ga == gb && a.c < b.c);
}

// Evaluate one neighbour community c (self-loops excluded) whose Sigma_tot
// Sc and (when the singleton guard needs it) size szc were already loaded.
// Singleton guard (modularity_optimisation.cu:154-155): a singleton may not
// move into a larger-id singleton.
__device__ __forceinline__ bool guard_needs_size(const MoveCtx &m, int32_t c) {
    return m.own_single && c > m.own;
}

__device__ __forceinline__ void eval_loaded(int32_t c, u64 ec, u64 Sc, int32_t szc, const MoveCtx &m,
                                            Best &b) {
    if (c == m.own) { b.eo += ec; return; }
    if (guard_needs_size(m, c) && szc == 1) return;
    Best x;
    x.S = Sc;
    x.e = ec;
    x.c = c;
    x.eo = 0;
    const double dd = (double)((i64)m.sown - (i64)m.kv - (i64)Sc);
    x.gd = fma(m.Td, (double)ec, m.kvd * dd);
    if (better(m, x, b)) { b.gd = x.gd; b.e = x.e; b.S = x.S; b.c = x.c; }
}

__device__ __forceinline__ void eval_candidate(int32_t c, u64 ec, const MoveCtx &m,
                                               const u64 *__restrict__ S,
                                               const int32_t *__restrict__ size, Best &b) {
    if (c == m.own) { b.eo += ec; return; }
    eval_loaded(c, ec, __ldg(S + c), guard_needs_size(m, c) ? __ldg(size + c) : 0, m, b);
}

// Evaluate U table entries per lane at a time: first U keys/sums, then their
// U Sigma_tot (and guard size) gathers, then the comparisons.  Entries come
// from slot indices (OCC: occ[i], else i itself, i < n); each visited slot is
// cleared when CLEAR is set.
template <int U, bool OCC, bool CLEAR>
__device__ __forceinline__ void eval_slots(int32_t *keys, u64 *vals, const int32_t *occ, int32_t n,
                                           int lane, int stride, const MoveCtx &m,
                                           const u64 *__restrict__ S,
                                           const int32_t *__restrict__ size, Best &b) {
    for (int32_t i0 = lane; i0 < n; i0 += U * stride) {
        int32_t cc[U];
        u64 ee[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t i = i0 + u * stride;
            cc[u] = -1;
            ee[u] = 0;
            if (i < n) {
                const int32_t sl = OCC ? occ[i] : i;
                cc[u] = keys[sl];
                if (cc[u] >= 0) {
                    ee[u] = vals[sl];
                    if (CLEAR) {
                        keys[sl] = -1;
                        vals[sl] = 0;
                    }
                }
            }
        }
        u64 SS[U];
        int32_t zz[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool cand = cc[u] >= 0 && cc[u] != m.own;
            SS[u] = cand ? __ldg(S + cc[u]) : 0;
            zz[u] = (cand && guard_needs_size(m, cc[u])) ? __ldg(size + cc[u]) : 0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (cc[u] >= 0) eval_loaded(cc[u], ee[u], SS[u], zz[u], m, b);
    }
}

// Move rule (modularity_optimisation.cu:192): move iff g_best - e_own/M > 0,
// i.e. G_best - T * e_own > 0.  *delta receives the mover's contribution to
// sum_i e_{i->C(i)} when none of its neighbours moves in the same sub-round,
// 2 (e_best - e_own) as a wrapping uint64 (corrected for co-moving neighbours
// by the correction kernel).
__device__ __forceinline__ int32_t move_decision(const MoveCtx &m, const Best &b, u64 *delta) {
    *delta = 0;
    if (b.c == m.own) return m.own;
    const i128 g = exact_gain(m, b.e, b.S);
    const i128 stay = (i128)(((u128)__umul64hi(m.T, b.eo) << 64) | (u128)(m.T * b.eo));
    if (g - stay > 0) {
        *delta = 2 * (b.e - b.eo);
        return b.c;
    }
    return m.own;
}

// Features of the learned active set, recorded at v's evaluation when
// st.feat is set: the fraction of k_v into the own community and the best
// move's gain relative to T k_v, (G_best - T e_own) / (T k_v) in [-1, 1]
// (from the FP64 estimate; the exact rule never reads them).
__device__ __forceinline__ void record_features(const StateView &st, int32_t v, const MoveCtx &m,
                                                const Best &b) {
    if (!st.feat) return;
    float own = 0.0f, gain = 0.0f;
    if (m.kv > 0) {
        const double eo = (double)b.eo;
        own = (float)(eo / m.kvd);
        const double g = (b.c == m.own ? 0.0 : b.gd) - m.Td * eo;
        gain = (float)fmin(1.0, fmax(-1.0, g / (m.Td * m.kvd)));
    }
    st.feat[2 * (size_t)v] = own;
    st.feat[2 * (size_t)v + 1] = gain;
}

// Butterfly reduction inside aligned groups of `width` lanes; every lane of
// the group ends with the group's best and the summed e_own.
// The exact gain of each lane's best lies in [gd - err, gd + err].  A lane
// whose upper bound is below the group's largest lower bound cannot win; when
// one lane per group is left (the usual case) it is the exact argmax and is
// broadcast.  Otherwise (ties or near-ties in some group of the warp) the
// butterfly of exact comparisons decides.
__device__ __forceinline__ void group_reduce_best(const MoveCtx &m, Best &b, int width) {
    const int lane = threadIdx.x & 31;
    const unsigned gmask = width == 32 ? FULL : (((1u << width) - 1u) << (lane & ~(width - 1)));
    const double eb = gain_err(m, b);
    double lo = b.gd - eb;
    u64 eo = b.eo;
    for (int off = width >> 1; off > 0; off >>= 1) {
        lo = fmax(lo, __shfl_xor_sync(FULL, lo, off, width));
        eo += __shfl_xor_sync(FULL, eo, off, width);
    }
    const unsigned alive = __ballot_sync(FULL, b.gd + eb >= lo) & gmask;
    if (!__any_sync(FULL, __popc(alive) != 1)) {
        const int src = (__ffs(alive) - 1) & (width - 1);
        b.gd = __shfl_sync(FULL, b.gd, src, width);
        b.e = __shfl_sync(FULL, b.e, src, width);
        b.S = __shfl_sync(FULL, b.S, src, width);
        b.c = __shfl_sync(FULL, b.c, src, width);
    } else {
        for (int off = width >> 1; off > 0; off >>= 1) {
            Best o;
            o.gd = __shfl_xor_sync(FULL, b.gd, off, width);
            o.e = __shfl_xor_sync(FULL, b.e, off, width);
            o.S = __shfl_xor_sync(FULL, b.S, off, width);
            o.c = __shfl_xor_sync(FULL, b.c, off, width);
            if (better(m, o, b)) { b.gd = o.gd; b.e = o.e; b.S = o.S; b.c = o.c; }
        }
    }
    b.eo = eo;
}

// u128 -> double, round to nearest even (as the host's conversion): the top 64
// significant bits with every lower bit folded into bit 0 round the same way
// as the full value, then an exact power-of-two scale.
__device__ __forceinline__ double u128_to_double_rn(u64 hi, u64 lo) {
    if (hi == 0) return __ull2double_rn(lo);
    const int lz = __clzll((long long)hi);
    const u64 top = lz ? ((hi << lz) | (lo >> (64 - lz))) : hi;
    const u64 rest = lz ? (lo << lz) : lo;
    return ldexp(__ull2double_rn(top | (rest != 0 ? 1ull : 0ull)), 64 - lz);
}

// Q = e_own / T - sum(Sigma_tot^2) / T^2 with the host's FP64 operations, each
// correctly rounded, so the value equals the host's bit for bit
// (calculateModularity, modularity_optimisation.cu:395-401, in exact parts).
__device__ __forceinline__ double q_from_parts_dev(u64 T, u64 e_own, u64 s2_hi, u64 s2_lo) {
    const double td = __ull2double_rn(T);
    const double a = __ddiv_rn(__ull2double_rn(e_own), td);
    const double b = __ddiv_rn(u128_to_double_rn(s2_hi, s2_lo), __dmul_rn(td, td));
    return __dsub_rn(a, b);
}

// Fixed-point analysis of one float32 weight (the oracle's weight_bits):
// need = fractional bits of its exact binary value, top = floor(log2 w) + 1024
// (0 for a zero weight); bad = 1 for a negative, NaN or infinite weight.
__device__ __forceinline__ void weight_bits_dev(float wf, int &need, int &top, int &bad) {
    const uint32_t bits = __float_as_uint(wf);
    const uint32_t ex = (bits >> 23) & 0xFF, man = bits & 0x7FFFFF;
    need = 0;
    top = 0;
    bad = 0;
    if (ex == 0xFF) { bad = 1; return; }
    if ((bits & 0x7FFFFFFFu) == 0) return;
    if (bits >> 31) { bad = 1; return; }
    uint32_t m;
    int ee, t;
    if (ex == 0) { m = man; ee = -149; t = (31 - __clz(man)) - 149; }
    else { m = man | 0x800000u; ee = (int)ex - 150; t = (int)ex - 127; }
    ee += __ffs(m) - 1;
    need = ee < 0 ? -ee : 0;
    top = t + 1024;
}

__device__ __forceinline__ u64 warp_sum_u64(u64 x) {
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(FULL, x, off);
    return x;
}

__device__ __forceinline__ u128 warp_sum_u128(u128 x) {
    for (int off = 16; off > 0; off >>= 1) {
        u64 lo = (u64)x, hi = (u64)(x >> 64);
        lo = __shfl_xor_sync(FULL, lo, off);
        hi = __shfl_xor_sync(FULL, hi, off);
        x += ((u128)hi << 64) | (u128)lo;
    }
    return x;
}

// 128-bit accumulate into two device words with an exact carry.
__device__ __forceinline__ void atomic_add_u128(u64 *hi_lo, u128 x) {
    u64 lo = (u64)x, hi = (u64)(x >> 64);
    u64 old = atomicAdd(hi_lo + 1, lo);
    if (old + lo < old) hi += 1;
    if (hi) atomicAdd(hi_lo, hi);
}

}  // namespace lv
