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
    CLS_B0 = 0,   // (0,4]      4 lanes / vertex, shared table of 8
    CLS_B1,       // (4,8]      8 lanes, table 16
    CLS_B2,       // (8,16]     16 lanes, table 32
    CLS_B3,       // (16,32]    32 lanes, table 64
    CLS_B4,       // (32,84]    32 lanes, table 256
    CLS_B5,       // (84,319]   CTA of 128, table <= 1024
    CLS_H1,       // (319,1024] CTA of 256, table <= 2048
    CLS_H2,       // (1024,4096] CTA of 512, table <= 8192
    CLS_HG,       // > 4096     multi-CTA, table in global memory
    NCLS
};
constexpr int CLASS_MAX_DEG[NCLS] = {4, 8, 16, 32, 84, 319, 1024, 4096, 0x7fffffff};
// class -> update bucket
__host__ __device__ constexpr int class_bucket(int c) { return c < CLS_H1 ? c : 6; }

__host__ __device__ __forceinline__ int degree_class(int32_t d) {
    if (d <= 0) return -1;
    if (d <= 4) return CLS_B0;
    if (d <= 8) return CLS_B1;
    if (d <= 16) return CLS_B2;
    if (d <= 32) return CLS_B3;
    if (d <= 84) return CLS_B4;
    if (d <= 319) return CLS_B5;
    if (d <= 1024) return CLS_H1;
    if (d <= 4096) return CLS_H2;
    return CLS_HG;
}

// Device error bits (OR-ed into a device word, read back once per sweep).
enum DevErr { DEVERR_HASH_FULL = 1, DEVERR_BAD_STATE = 2 };

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

// Weight access: level 0 reads float32 and maps it onto the fixed grid
// (exact: w * 2^scale is a power-of-two scaling, then round-to-nearest-even,
// the same rule as the host's llrint(ldexp(w, scale))); later levels read the
// stored uint64 sums.
__device__ __forceinline__ u64 wfix(const float *w, int64_t e, double scale) {
    return (u64)__double2ll_rn(__dmul_rn((double)__ldg(w + e), scale));
}
__device__ __forceinline__ u64 wfix(const u64 *w, int64_t e, double) { return __ldg(w + e); }

// A level's graph: row v is col/w[rowptr[v] .. rowend[v]).  Level 0 is a
// plain CSR (rowend = rowptr + 1); aggregated levels keep each merged row
// where the merge wrote it, so rows need not be contiguous.
template <typename WT>
struct GraphView {
    const int32_t *rowptr;
    const int32_t *rowend;
    const int32_t *col;
    const WT *w;
    double scale;   // 2^scale (used for float weights only)
};

struct StateView {
    int32_t *comm;
    int32_t *newc;
    int32_t *size;
    u64 *k;
    u64 *S;
    u64 T;
    int *err;
};

// Insert (key, w) into an open-addressing table with linear probing; works
// for shared and global tables (generic addressing).  A key once written
// never changes, so a stale EMPTY read only costs a failed CAS.  The probe
// count is bounded by the capacity; a full table sets an error bit instead
// of spinning.
__device__ __forceinline__ void table_insert(int32_t *keys, u64 *vals, int lg, int32_t key,
                                             u64 w, int *err) {
    const uint32_t mask = (1u << lg) - 1u;
    uint32_t s = hash_slot(key, lg);
    for (uint32_t p = 0; p <= mask; ++p) {
        int32_t k = ((volatile int32_t *)keys)[s];
        if (k == key) { atomicAdd(vals + s, w); return; }
        if (k < 0) {
            int32_t prev = atomicCAS(keys + s, -1, key);
            if (prev < 0 || prev == key) { atomicAdd(vals + s, w); return; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
}

// Exact sum of a uint64 over the lanes in `mask` (redux.sync adds 32-bit
// values): the value is split into 22/22/20-bit slices whose 32-lane sums
// cannot overflow 32 bits.  Lanes of different masks may call it together.
__device__ __forceinline__ u64 redux_add_u64(unsigned mask, u64 x) {
    const unsigned p0 = (unsigned)(x & 0x3FFFFFull);
    const unsigned p1 = (unsigned)((x >> 22) & 0x3FFFFFull);
    const unsigned p2 = (unsigned)(x >> 44);
    const u64 s0 = __reduce_add_sync(mask, p0);
    const u64 s1 = __reduce_add_sync(mask, p1);
    const u64 s2 = __reduce_add_sync(mask, p2);
    return s0 + (s1 << 22) + (s2 << 44);
}

// Warp-aggregated insert: every lane of the warp calls it (uniformly);
// valid lanes holding the same key first combine their weights, and one
// lane per distinct key inserts.  A key shared by many neighbours (the common
// case once communities form) then costs one atomic per warp instead of 32.
__device__ __forceinline__ void warp_insert(int32_t *keys, u64 *vals, int lg, bool valid,
                                            int32_t key, u64 w, int *err) {
    const unsigned act = __ballot_sync(FULL, valid);
    if (!valid) return;
    const unsigned peers = __match_any_sync(act, key);
    const u64 sum = redux_add_u64(peers, w);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) table_insert(keys, vals, lg, key, sum, err);
}

// Candidate ordering of computeMove: larger gain wins, equal gains go to the
// lower community id (modularity_optimisation.cu:157,169,182).
__device__ __forceinline__ bool better(i128 g1, int32_t c1, i128 g2, int32_t c2) {
    return g1 > g2 || (g1 == g2 && c1 < c2);
}

// Evaluate one neighbour community C of vertex v (e_C = summed weight to C,
// self-loops excluded).  The community of v itself only contributes e_own.
// Singleton guard (modularity_optimisation.cu:154-155): a singleton may not
// move into a larger-id singleton.
struct MoveCtx {
    int32_t own;
    bool own_single;
    u64 kv;
    u64 sown;
};

// Running best of one thread (or group): gain, community, and the summed
// weight e_best to that community (used for the exact modularity update);
// e_own is the weight to the vertex's own community.
struct Best {
    i128 g;
    int32_t c;
    u64 eb;
    u64 eo;
};

__device__ __forceinline__ Best best_init(int32_t own) {
    Best b;
    b.g = 0;
    b.c = own;
    b.eb = 0;
    b.eo = 0;
    return b;
}

__device__ __forceinline__ void eval_candidate(int32_t c, u64 ec, const MoveCtx &m, u64 T,
                                               const u64 *__restrict__ S,
                                               const int32_t *__restrict__ size, Best &b) {
    if (c == m.own) { b.eo = ec; return; }
    if (m.own_single && c > m.own && size[c] == 1) return;
    const i64 d = (i64)m.sown - (i64)m.kv - (i64)S[c];
    const i128 g = (i128)((u128)T * (u128)ec) + (i128)(i64)m.kv * (i128)d;
    if (better(g, c, b.g, b.c)) { b.g = g; b.c = c; b.eb = ec; }
}

// Move rule (modularity_optimisation.cu:192): move iff g_best - e_own/M > 0,
// i.e. G_best - T * e_own > 0.  *delta receives the mover's contribution to
// sum_i e_{i->C(i)} when none of its neighbours moves in the same sub-round,
// 2 (e_best - e_own) as a wrapping uint64 (corrected for co-moving neighbours
// by the correction kernel).
__device__ __forceinline__ int32_t move_decision(const Best &b, u64 T, int32_t own, u64 *delta) {
    const i128 stay = (i128)((u128)T * (u128)b.eo);
    if (b.g - stay > 0) {
        *delta = 2 * (b.eb - b.eo);
        return b.c;
    }
    *delta = 0;
    return own;
}

__device__ __forceinline__ i128 shfl_xor_i128(i128 x, int m, int width) {
    u64 lo = (u64)x, hi = (u64)((u128)x >> 64);
    lo = __shfl_xor_sync(FULL, lo, m, width);
    hi = __shfl_xor_sync(FULL, hi, m, width);
    return (i128)(((u128)hi << 64) | (u128)lo);
}

// Butterfly reduction inside aligned groups of `width` lanes; every lane of
// the group ends with the group's best (g, c, e_best) and summed e_own.
__device__ __forceinline__ void group_reduce_best(Best &b, int width) {
    for (int off = width >> 1; off > 0; off >>= 1) {
        const i128 og = shfl_xor_i128(b.g, off, width);
        const int32_t oc = __shfl_xor_sync(FULL, b.c, off, width);
        const u64 ob = __shfl_xor_sync(FULL, b.eb, off, width);
        const u64 oe = __shfl_xor_sync(FULL, b.eo, off, width);
        if (better(og, oc, b.g, b.c)) { b.g = og; b.c = oc; b.eb = ob; }
        b.eo += oe;
    }
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
