// lv_move.cu -- modularity-optimisation kernels (the move sweep), the commit
// of a sub-round and the exact modularity reductions.
//
// Replaces computeMove / computeMoveShared / computeMoveGlobal,
// updateVertexCommunity, computeEdgesSum and calculateToOwnCommunity of
// modularity_optimisation.cu (:23-40, :111-228, :237-249, :365-386).
//
// Work mapping (one kernel family per degree class, all classes of one
// update bucket are decided before that bucket is committed):
//   - classes B0..B4: a group of G lanes (4/8/16/32) per vertex, the group's
//     neighbour-community table in shared memory;
//   - classes B5, H1, H2: one CTA per vertex (persistent grid-stride), table
//     in shared memory sized to the vertex's degree;
//   - class HG: many CTAs per hub, table in global memory (insert kernel over
//     edge chunks, evaluate kernel over slot chunks, final per-hub reduce).
#include "lv_internal.h"

namespace lv {

namespace {

// Sum a per-thread uint64 (wrapping) over the CTA and add it to *total with
// one atomic.  Every thread of the CTA must call it.
template <int THREADS>
__device__ __forceinline__ void block_add_total(u64 x, u64 *total) {
    __shared__ u64 part[THREADS / 32];
    x = warp_sum_u64(x);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        u64 y = threadIdx.x < THREADS / 32 ? part[threadIdx.x] : 0;
        y = warp_sum_u64(y);
        if (threadIdx.x == 0 && y) atomicAdd(total, y);
    }
    __syncthreads();
}

// Queue vertex v (degree d) for the large queue only (64-bit sums, any row):
// the vertices of a 32-bit-view level whose row holds a sum of 2^32 or more.
// One lane calls it.
__device__ __forceinline__ void enqueue_large(const Fallback &f, int32_t v, int32_t d, int *err) {
    const int32_t P = d > FB_KEYS ? (d + FB_KEYS - 1) / FB_KEYS : 1;
    const int32_t first = atomicAdd(f.count, P);
    if (first + P <= f.cap) {
        for (int32_t q = 0; q < P; ++q) {
            f.v[first + q] = v;
            f.p[first + q] = q;
            f.P[first + q] = P;
            f.first[first + q] = first;
            f.src[first + q] = -1;
        }
    } else {
        atomicOr(err, DEVERR_FALLBACK_FULL);
    }
}

// ------------------------------------------------------------------------
// group-per-vertex move kernel (degree <= 84)
// ------------------------------------------------------------------------
template <int G, int CAP, typename WT>
__global__ void __launch_bounds__(256) move_group_kernel(GraphView<WT> g, StateView st,
                                                         const int32_t *__restrict__ list,
                                                         int32_t n, u64 *dE) {
    constexpr int GPB = 256 / G;
    constexpr int LG = ilog2_c(CAP);
    static_assert((1 << LG) == CAP, "CAP must be a power of two");
    __shared__ u64 svals[GPB * CAP];
    __shared__ int32_t skeys[GPB * CAP];
    const int grp = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int idx = blockIdx.x * GPB + grp;
    int32_t *keys = skeys + grp * CAP;
    u64 *vals = svals + grp * CAP;
#pragma unroll
    for (int s = lane; s < CAP; s += G) { keys[s] = -1; vals[s] = 0; }
    __syncwarp();
    const bool active = idx < n;
    int32_t v = 0, own = 0;
    u64 e_own = 0;   // weight to the own community: kept out of the table
    if (active) {
        v = list[idx];
        own = __ldg(st.comm + v);
        insert_row<(CAP > 32 ? LV_U_CTA : LV_U_GROUP), false>(g, st.comm, v, own, g.rowptr[v], g.rowend[v], lane, G,
                                               keys, vals, LG, st.err, nullptr, nullptr, e_own);
    }
    __syncwarp();
    const MoveCtx m = move_ctx(own, active ? __ldg(st.size + own) == 1 : false, st.T,
                               active ? __ldg(st.k + v) : 0, active ? __ldg(st.S + own) : 0);
    Best b = best_init(own);
    b.eo = e_own;
    if (active) eval_slots<(CAP / G > 1 ? (LV_U_EVAL < 2 ? LV_U_EVAL : 2) : 1), false, false>(keys, vals, nullptr, CAP, lane, G, m, st.S, st.size, b);
    group_reduce_best(m, b, G);
    u64 delta = 0;
    if (active && lane == 0) {
        st.newc[v] = move_decision(m, b, &delta);
        record_features(st, v, m, b);
    }
    block_add_total<256>(delta, dE);
}

// move_group_kernel for weights below 2^32: the group's table keeps its sums
// in 16-bit-piece counters (fire-and-forget adds).
template <int G, int CAP, typename WT>
__global__ void __launch_bounds__(256) move_group_narrow_kernel(GraphView<WT> g, StateView st,
                                                                const int32_t *__restrict__ list,
                                                                int32_t n, u64 *dE, Fallback fbl) {
    constexpr int GPB = 256 / G;
    constexpr int LG = ilog2_c(CAP);
    static_assert((1 << LG) == CAP, "CAP must be a power of two");
    __shared__ uint32_t slo[GPB * CAP], shi[GPB * CAP];
    __shared__ int32_t skeys[GPB * CAP];
    const int grp = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int idx = blockIdx.x * GPB + grp;
    PieceTable t;
    t.keys = skeys + grp * CAP;
    t.lo = slo + grp * CAP;
    t.hi = shi + grp * CAP;
#pragma unroll
    for (int s = lane; s < CAP; s += G) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    __syncwarp();
    bool active = idx < n;
    int32_t v = 0, own = 0, r0 = 0, r1 = 0;
    u64 e_own = 0;
    if (active) {
        // the row bounds, the community and the wide-row flag are loaded
        // together (none depends on another)
        v = list[idx];
        r0 = g.rowptr[v];
        r1 = g.rowend[v];
        own = __ldg(st.comm + v);
        if (st.wrow && st.wrow[v]) {
            // a row with a sum of 2^32 or more: decided by the large queue
            if (lane == 0) enqueue_large(fbl, v, r1 - r0, st.err);
            active = false;
        }
    }
    if (active)
        insert_row_piece<(CAP > 32 ? LV_U_CTA : LV_U_GROUP), false>(g, st.comm, v, own, r0, r1, lane, G, t, LG,
                                                                     st.err, nullptr, nullptr, 0, e_own);
    __syncwarp();
    const MoveCtx m = move_ctx(own, active ? __ldg(st.size + own) == 1 : false, st.T,
                               active ? __ldg(st.k + v) : 0, active ? __ldg(st.S + own) : 0);
    Best b = best_init(own);
    b.eo = e_own;
    if (active) {
#pragma unroll
        for (int s = lane; s < CAP; s += G) {
            const int32_t c = t.keys[s];
            if (c < 0) continue;
            const bool cand = c != own;
            const u64 Sc = cand ? __ldg(st.S + c) : 0;
            const int32_t szc = (cand && guard_needs_size(m, c)) ? __ldg(st.size + c) : 0;
            eval_loaded(c, piece_value(t, (uint32_t)s), Sc, szc, m, b);
        }
    }
    group_reduce_best(m, b, G);
    u64 delta = 0;
    if (active && lane == 0) {
        st.newc[v] = move_decision(m, b, &delta);
        record_features(st, v, m, b);
    }
    block_add_total<256>(delta, dE);
}

// CTA-wide reduction of a Best; the result is valid in thread 0.
template <int THREADS>
__device__ __forceinline__ void cta_reduce_best(const MoveCtx &m, Best &b) {
    constexpr int NW = THREADS / 32;
    __shared__ double rgd[NW];
    __shared__ u64 re[NW], rS[NW], reo[NW];
    __shared__ int32_t rc[NW];
    group_reduce_best(m, b, 32);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        rgd[w] = b.gd;
        re[w] = b.e;
        rS[w] = b.S;
        rc[w] = b.c;
        reo[w] = b.eo;
    }
    __syncthreads();
    if (w == 0) {
        if (l < NW) {
            b.gd = rgd[l];
            b.e = re[l];
            b.S = rS[l];
            b.c = rc[l];
            b.eo = reo[l];
        } else {
            b = best_init(m.own);
        }
        group_reduce_best(m, b, 32);
    }
}

// ------------------------------------------------------------------------
// degree > 32: warp per vertex with an optimistic shared table, fallback
// CTAs for vertices with many distinct neighbour communities
// ------------------------------------------------------------------------
// W. A warp per vertex inserts its row into a shared table of
//    min(WARP_CAP, 2^ceil(log2(2 degree))) slots and counts newly claimed
//    slots with a ballot.  Once communities have formed a vertex has few
//    distinct neighbour communities (a few percent of its degree on
//    aggregated levels), so this decides almost every vertex.  A vertex whose
//    count passes WARP_LIMIT, or whose hint says it did at its last
//    evaluation, is queued for a fallback CTA instead: to the first row
//    queue b with degree <= FBQ_MAXDEG(b), else as
//    P = ceil(degree / FB_KEYS) key-space partitions (v, p) to the large queue.
// F. Persistent fallback CTAs take items from their queue.  Small and medium
//    items are whole rows in a table of 2^ceil(log2(2 degree)) slots.  A large
//    item (v, p) streams v's row (or the staged pairs of a giant), keeps the
//    communities whose hash falls in partition p, evaluates them and stores
//    its partial best; the CTA that finishes the last item of v combines the
//    P partials (the items of v are contiguous) and decides.
// Results do not depend on which path decides a vertex.

__device__ __forceinline__ uint32_t part_of(int32_t c, int32_t P) {
    const uint32_t hsh = (uint32_t)c * 0x85EBCA6Bu;
    return (uint32_t)(((u64)(hsh ^ (hsh >> 15)) * (u64)P) >> 32);
}

// Queue vertex v (degree d) for a fallback CTA.  One lane calls it.
__device__ __forceinline__ void enqueue_fallback(const FallbackSet &fs, int32_t v, int32_t d, int *err) {
    if (d <= FBQ_MAXDEG(NFBQ - 1)) {
        int b = 0;
        while (d > FBQ_MAXDEG(b)) ++b;
        const Fallback &f = fs.q[b];
        const int32_t i = atomicAdd(f.count, 1);
        if (i < f.cap) f.v[i] = v;
        else atomicOr(err, DEVERR_FALLBACK_FULL);
        return;
    }
    const Fallback &f = fs.q[NFBQ];
    const int32_t P = (d + FB_KEYS - 1) / FB_KEYS;
    const int32_t first = atomicAdd(f.count, P);
    if (first + P <= f.cap) {
        for (int32_t q = 0; q < P; ++q) {
            f.v[first + q] = v;
            f.p[first + q] = q;
            f.P[first + q] = P;
            f.first[first + q] = first;
            f.src[first + q] = -1;
        }
    } else {
        atomicOr(err, DEVERR_FALLBACK_FULL);
    }
}

// The 64-bit warp kernel loads the home-slot keys of a step's U entries
// together before its inserts (1) or probes entry by entry (0, the default:
// 1 measured 0.3 ms slower per R-MAT-24 run, the degree > 319 class 0.4 ms
// faster and degrees 33-319 0.5 ms slower).
#ifndef LV_WIDE_PREFETCH
#define LV_WIDE_PREFETCH 0
#endif
// The warp kernels load a step that lies wholly inside the row without
// per-entry bound tests (1, the default: the degree > 319 class of an
// R-MAT-24 run 107.1 against 111.5 ms) or test every entry (0).
#ifndef LV_WARP_FULLSTEP
#define LV_WARP_FULLSTEP 1
#endif
// The 64-bit warp kernel counts its claims after every chunk of 32 entries
// (0) or once per step of U chunks (1, the default: 0.6 ms less per R-MAT-24
// run, 111.4 against 111.8 ms for the degree > 319 class).
#ifndef LV_CLAIM_PER_STEP
#define LV_CLAIM_PER_STEP 1
#endif
static_assert(!LV_CLAIM_PER_STEP || WARP_LIMIT_MAX + 32 * LV_U_WARP <= WARP_CAP,
              "claims counted per step fit the warp table");

template <typename WT>
__global__ void __launch_bounds__(256) move_warp_kernel(GraphView<WT> g, StateView st,
                                                        const int32_t *__restrict__ list, int32_t n,
                                                        FallbackSet fs, u64 *dE) {
    constexpr int NW = 8;
    constexpr int LG = ilog2_c(WARP_CAP);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *svals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *skeys = reinterpret_cast<int32_t *>(svals + NW * WARP_CAP);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int32_t *keys = skeys + wid * WARP_CAP;
    u64 *vals = svals + wid * WARP_CAP;
    for (int s = lane; s < WARP_CAP; s += 32) { keys[s] = -1; vals[s] = 0; }
    __syncwarp();
    u64 delta_acc = 0;
    // the next vertex's id, row bounds and community are loaded while the
    // current one is processed (none of them changes during the sub-round)
    // vertices are taken one at a time from a shared cursor (the class lists
    // are sorted by decreasing degree, so the longest rows go first and the
    // warps finish together); the next vertex's id, row bounds and community
    // are loaded while the current one is processed
    int32_t idx = 0;
    if (lane == 0) idx = atomicAdd(fs.warp_next, 1);
    idx = __shfl_sync(FULL, idx, 0);
    int32_t nv = 0, nr0 = 0, nr1 = 0, nown = 0;
    if (idx < n) {
        nv = list[idx];
        nr0 = g.rowptr[nv];
        nr1 = g.rowend[nv];
        nown = __ldg(st.comm + nv);
    }
    while (idx < n) {
        const int32_t v = nv, r0 = nr0, r1 = nr1, own = nown;
        int32_t nidx = 0;
        if (lane == 0) nidx = atomicAdd(fs.warp_next, 1);
        nidx = __shfl_sync(FULL, nidx, 0);
        if (nidx < n) {
            nv = list[nidx];
            nr0 = g.rowptr[nv];
            nr1 = g.rowend[nv];
            nown = __ldg(st.comm + nv);
        }
        idx = nidx;
        const int32_t d = r1 - r0;
        if (d > fs.warp_limit && fs.hint[v]) {
            if (lane == 0) enqueue_fallback(fs, v, d, st.err);
            continue;
        }
        // the vertex's own terms, issued before the edge loop
        const int32_t sz_own = __ldg(st.size + own);
        const u64 k_v = __ldg(st.k + v), s_own = __ldg(st.S + own);
        int lg = ceil_log2_i(2 * (int64_t)d);
        lg = lg < 5 ? 5 : (lg > LG ? LG : lg);
        u64 e_own = 0;
        int32_t nclaim = 0;
        bool overflow = false;
        // LV_WARP_COMBINE: each lane holds its last community and the weight
        // summed to it in registers and adds them to the table only when the
        // community changes (and at the end of the row), so runs of one
        // community in a lane's entries cost one shared add
        int32_t ck = -1;
        u64 cw = 0;
        // U chunks of 32 edges per step: U column and weight loads, then U
        // community gathers, are in flight together.  The claim count is
        // checked after every chunk, so at most WARP_LIMIT + 32 slots of
        // the WARP_CAP-slot table are ever claimed (+ 32 held in registers
        // with LV_WARP_COMBINE, added at the end of the row).
        constexpr int U = LV_U_WARP;
        for (int32_t base = r0 + lane; base < r1 + lane && !overflow; base += 32 * U) {
            int32_t jj[U];
            u64 ww[U];
            int32_t lclaims = 0;   // LV_CLAIM_PER_STEP: this lane's claims in the step
            int32_t cc[U];
            if (LV_WARP_FULLSTEP && base - lane + 32 * U <= r1) {
                // a whole step inside the row (warp-uniform): no bound tests
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int32_t e = base + 32 * u;
                    jj[u] = __ldg(g.col + e);
                    ww[u] = gw(g, e);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) cc[u] = jj[u] != v ? __ldg(st.comm + jj[u]) : -1;
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int32_t e = base + 32 * u;
                    jj[u] = -1;
                    ww[u] = 0;
                    if (e < r1) { jj[u] = __ldg(g.col + e); ww[u] = gw(g, e); }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? __ldg(st.comm + jj[u]) : -1;
            }
            // LV_WIDE_PREFETCH: the U home slots and their keys are loaded
            // together; a key already in its home slot is added without probing
            uint32_t hs[U];
            int32_t kk[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                hs[u] = cc[u] >= 0 ? hash_slot(cc[u], lg) : 0u;
                kk[u] = (LV_WIDE_PREFETCH && cc[u] >= 0 && cc[u] != own) ? ((volatile int32_t *)keys)[hs[u]] : -2;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                int32_t claimed = -1;
                if (LV_DEDUP && st.dedup) {
                    // equal keys of the warp combined before the atomics
                    const bool valid = cc[u] >= 0 && cc[u] != own;
                    if (cc[u] >= 0 && cc[u] == own) e_own += ww[u];
                    const unsigned peers = key_peers(cc[u], valid);
                    const u64 ws = group_sum_u64(peers, valid ? ww[u] : 0);
                    if (valid && group_leader(peers)) claimed = table_insert_claim(keys, vals, lg, cc[u], ws, st.err);
                } else if (LV_WIDE_PREFETCH && !LV_WARP_COMBINE) {
                    // home-slot key loaded with the step's other U (below)
                    if (cc[u] >= 0) {
                        if (cc[u] == own) e_own += ww[u];
                        else if (kk[u] == cc[u]) table_add(vals + hs[u], ww[u]);
                        else claimed = table_insert_claim(keys, vals, lg, cc[u], ww[u], st.err);
                    }
                } else if (cc[u] >= 0) {
                    if (cc[u] == own) {
                        e_own += ww[u];
                    } else if (LV_WARP_COMBINE) {
                        if (cc[u] == ck) {
                            cw += ww[u];
                        } else {
                            if (ck >= 0) claimed = table_insert_claim(keys, vals, lg, ck, cw, st.err);
                            ck = cc[u];
                            cw = ww[u];
                        }
                    } else {
                        claimed = table_insert_claim(keys, vals, lg, cc[u], ww[u], st.err);
                    }
                }
                if (LV_CLAIM_PER_STEP) {
                    lclaims += claimed >= 0 ? 1 : 0;
                } else {
                    nclaim += __popc(__ballot_sync(FULL, claimed >= 0));
                    if (nclaim > fs.warp_limit) { overflow = true; break; }
                }
            }
            if (LV_CLAIM_PER_STEP) {
                // claims counted once per step: at most warp_limit + 32 U
                // (<= 512 = WARP_CAP) distinct keys are ever claimed
                nclaim += (int32_t)__reduce_add_sync(FULL, (unsigned)lclaims);
                if (nclaim > fs.warp_limit) overflow = true;
            }
        }
        if (LV_WARP_COMBINE && !overflow) {
            // the communities still held in registers
            const int32_t claimed = ck >= 0 ? table_insert_claim(keys, vals, lg, ck, cw, st.err) : -1;
            nclaim += __popc(__ballot_sync(FULL, claimed >= 0));
            if (nclaim > fs.warp_limit) overflow = true;
        }
        __syncwarp();
        const int nslots = 1 << lg;
        if (overflow) {
            for (int s = lane; s < nslots; s += 32) {
                if (keys[s] >= 0) { keys[s] = -1; vals[s] = 0; }
            }
            if (lane == 0) {
                fs.hint[v] = 1;
                enqueue_fallback(fs, v, d, st.err);
            }
            __syncwarp();
            continue;
        }
        const MoveCtx m = move_ctx(own, sz_own == 1, st.T, k_v, s_own);
        Best b = best_init(own);
        b.eo = e_own;
        eval_slots<1, false, true>(keys, vals, nullptr, nslots, lane, 32, m, st.S, st.size, b);
        group_reduce_best(m, b, 32);
        if (lane == 0) {
            u64 delta = 0;
            st.newc[v] = move_decision(m, b, &delta);
            record_features(st, v, m, b);
            delta_acc += delta;
        }
        __syncwarp();
    }
    if (lane == 0 && delta_acc) atomicAdd(dE, delta_acc);
}

// The warp kernel for weights below 2^32 (see PieceTable): the same work
// mapping and overflow rule as move_warp_kernel, with the table sums kept in
// 16-bit-piece counters (fire-and-forget adds, no carry) and the claimed slots
// listed, so that evaluation and clearing visit only the vertex's distinct
// neighbour communities (a few dozen on aggregated levels) instead of the
// whole table.  A vertex with more than WARP_OCC_CAP distinct communities is
// evaluated over the whole table.
constexpr int WARP_OCC_CAP = 128;
constexpr int WARP_NSMEM = 8 * (WARP_CAP * 12 + WARP_OCC_CAP * 4 + 16);

template <typename WT>
__global__ void __launch_bounds__(256) move_warp_narrow_kernel(GraphView<WT> g, StateView st,
                                                               const int32_t *__restrict__ list, int32_t n,
                                                               FallbackSet fs, u64 *dE) {
    constexpr int LG = ilog2_c(WARP_CAP);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *base = smem_raw + (size_t)wid * (WARP_CAP * 12 + WARP_OCC_CAP * 4 + 16);
    PieceTable t;
    t.lo = reinterpret_cast<uint32_t *>(base);
    t.hi = t.lo + WARP_CAP;
    t.keys = reinterpret_cast<int32_t *>(t.hi + WARP_CAP);
    int32_t *occ = t.keys + WARP_CAP;
    int32_t *nocc = occ + WARP_OCC_CAP;
    for (int s = lane; s < WARP_CAP; s += 32) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    if (lane == 0) *nocc = 0;
    __syncwarp();
    u64 delta_acc = 0;
    // vertices are taken one at a time from a shared cursor (the class lists
    // are sorted by decreasing degree, so the longest rows go first and the
    // warps finish together); the next vertex's id, row bounds and community
    // are loaded while the current one is processed
    int32_t idx = 0;
    if (lane == 0) idx = atomicAdd(fs.warp_next, 1);
    idx = __shfl_sync(FULL, idx, 0);
    int32_t nv = 0, nr0 = 0, nr1 = 0, nown = 0;
    bool nwide = false;
    if (idx < n) {
        nv = list[idx];
        nr0 = g.rowptr[nv];
        nr1 = g.rowend[nv];
        nown = __ldg(st.comm + nv);
        nwide = st.wrow && st.wrow[nv];
    }
    while (idx < n) {
        const int32_t v = nv, r0 = nr0, r1 = nr1, own = nown;
        const bool wide = nwide;
        int32_t nidx = 0;
        if (lane == 0) nidx = atomicAdd(fs.warp_next, 1);
        nidx = __shfl_sync(FULL, nidx, 0);
        if (nidx < n) {
            nv = list[nidx];
            nr0 = g.rowptr[nv];
            nr1 = g.rowend[nv];
            nown = __ldg(st.comm + nv);
            nwide = st.wrow && st.wrow[nv];
        }
        idx = nidx;
        const int32_t d = r1 - r0;
        if (wide) {   // a sum of 2^32 or more: 64-bit sums in the large queue
            if (lane == 0) enqueue_large(fs.q[NFBQ], v, d, st.err);
            continue;
        }
        if (d > fs.warp_limit && fs.hint[v]) {
            if (lane == 0) enqueue_fallback(fs, v, d, st.err);
            continue;
        }
        const int32_t sz_own = __ldg(st.size + own);
        const u64 k_v = __ldg(st.k + v), s_own = __ldg(st.S + own);
        int lg = ceil_log2_i(2 * (int64_t)d);
        lg = lg < 5 ? 5 : (lg > LG ? LG : lg);
        u64 e_own = 0;
        bool overflow = false;
        // U chunks of 32 edges per step; the claim count is read after every
        // step, so at most WARP_LIMIT + 32 U slots are ever claimed
        constexpr int U = LV_U_WARP;
#if LV_WARP_PIPE
        // the step's column and raw weight loads were issued one step ahead
        int32_t jn[U];
        typename RawOf<WT>::T xn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t e = r0 + lane + 32 * u;
            jn[u] = -1;
            xn[u] = 0;
            if (e < r1) { jn[u] = ld_row(g.col + e); xn[u] = raw_row(g, e); }
        }
#endif
        for (int32_t b0 = r0 + lane; b0 < r1 + lane; b0 += 32 * U) {
            int32_t jj[U];
            u64 ww[U];
#if LV_WARP_PIPE
            typename RawOf<WT>::T xx[U];
#pragma unroll
            for (int u = 0; u < U; ++u) { jj[u] = jn[u]; xx[u] = xn[u]; }
            int32_t cc[U];
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? __ldg(st.comm + jj[u]) : -1;
#else
            int32_t cc[U];
            if (LV_WARP_FULLSTEP && b0 - lane + 32 * U <= r1) {
                // a whole step inside the row (warp-uniform): no bound tests
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int32_t e = b0 + 32 * u;
                    jj[u] = ld_row(g.col + e);
                    ww[u] = gw_row(g, e);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) cc[u] = jj[u] != v ? __ldg(st.comm + jj[u]) : -1;
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int32_t e = b0 + 32 * u;
                    jj[u] = -1;
                    ww[u] = 0;
                    if (e < r1) { jj[u] = ld_row(g.col + e); ww[u] = gw_row(g, e); }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? __ldg(st.comm + jj[u]) : -1;
            }
#endif
#if LV_WARP_PIPE
            // the next step's loads go out before this step's inserts
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = b0 + 32 * (U + u);
                jn[u] = -1;
                xn[u] = 0;
                if (e < r1) { jn[u] = ld_row(g.col + e); xn[u] = raw_row(g, e); }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) ww[u] = jj[u] >= 0 ? raw_value(g, b0 + 32 * u, xx[u]) : 0;
#endif
#if LV_WARP_PREFETCH
            // the U first-probe slots and their keys are loaded together; a
            // key already in its home slot (the common case once a row's few
            // communities are in the table) is then added without probing
            uint32_t hs[U];
            int32_t kk[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                hs[u] = cc[u] >= 0 ? hash_slot(cc[u], lg) : 0u;
                kk[u] = (cc[u] >= 0 && cc[u] != own) ? ((volatile int32_t *)t.keys)[hs[u]] : -2;
            }
            if (LV_DEDUP && st.dedup) {
                // equal keys of the warp combined before the atomics
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    int32_t claimed = -1;
                    const bool valid = cc[u] >= 0 && cc[u] != own;
                    if (cc[u] >= 0 && cc[u] == own) e_own += ww[u];
                    const unsigned peers = key_peers(cc[u], valid);
                    const Pieces pc = group_pieces(peers, valid ? ww[u] : 0);
                    if (valid && group_leader(peers)) {
                        if (kk[u] == cc[u]) piece_add_p(t, hs[u], pc);
                        else claimed = piece_insert_at_p(t, lg, hs[u], cc[u], pc, st.err);
                    }
                    warp_append_capped(claimed, occ, nocc, WARP_OCC_CAP);
                }
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    int32_t claimed = -1;
                    if (cc[u] >= 0) {
                        if (cc[u] == own) e_own += ww[u];
                        else if (kk[u] == cc[u]) piece_add(t, hs[u], ww[u]);
                        else claimed = piece_insert_at(t, lg, hs[u], cc[u], ww[u], st.err);
                    }
                    // one shared atomic per warp for the claims of this step
                    warp_append_capped(claimed, occ, nocc, WARP_OCC_CAP);
                }
            }
#else
#pragma unroll
            for (int u = 0; u < U; ++u) {
                int32_t claimed = -1;
                if (cc[u] >= 0) {
                    if (cc[u] == own) e_own += ww[u];
                    else claimed = piece_insert(t, lg, cc[u], ww[u], st.err);
                }
                warp_append_capped(claimed, occ, nocc, WARP_OCC_CAP);
            }
#endif
            __syncwarp();
            if (*nocc > fs.warp_limit) { overflow = true; break; }
        }
        __syncwarp();
        const int nslots = 1 << lg;
        const int32_t nd = *nocc;
        __syncwarp();
        if (lane == 0) *nocc = 0;
        if (overflow) {
            for (int s2 = lane; s2 < nslots; s2 += 32) {
                if (t.keys[s2] >= 0) { t.keys[s2] = -1; t.lo[s2] = 0; t.hi[s2] = 0; }
            }
            if (lane == 0) {
                fs.hint[v] = 1;
                enqueue_fallback(fs, v, d, st.err);
            }
            __syncwarp();
            continue;
        }
        const MoveCtx m = move_ctx(own, sz_own == 1, st.T, k_v, s_own);
        Best b = best_init(own);
        b.eo = e_own;
        const bool listed = nd <= WARP_OCC_CAP;
        const int32_t nscan = listed ? nd : nslots;
        for (int32_t i = lane; i < nscan; i += 32) {
            const int32_t sl = listed ? occ[i] : i;
            const int32_t c = t.keys[sl];
            if (c < 0) continue;
            const u64 ec = piece_value(t, (uint32_t)sl);
            t.keys[sl] = -1;
            t.lo[sl] = 0;
            t.hi[sl] = 0;
            const bool cand = c != own;
            const u64 Sc = cand ? __ldg(st.S + c) : 0;
            const int32_t szc = (cand && guard_needs_size(m, c)) ? __ldg(st.size + c) : 0;
            eval_loaded(c, ec, Sc, szc, m, b);
        }
        group_reduce_best(m, b, 32);
        if (lane == 0) {
            u64 delta = 0;
            st.newc[v] = move_decision(m, b, &delta);
            record_features(st, v, m, b);
            delta_acc += delta;
        }
        __syncwarp();
    }
    if (lane == 0 && delta_acc) atomicAdd(dE, delta_acc);
}

// Fallback CTAs.  PART = false: items are whole rows of degree <= CAP / 2
// (small and medium queues).  PART = true: key-space partitions of a row or
// of a giant's staged pairs (large queue).  The occupied list holds CAP / 2
// slots; a partition with more distinct communities than that reports
// DEVERR_HASH_FULL.
template <typename WT, int THREADS, int CAP, bool PART>
__global__ void __launch_bounds__(THREADS) move_fallback_kernel(GraphView<WT> g, StateView st,
                                                                Fallback fb, HubGlobal hg,
                                                                uint8_t *hint, int32_t hint_set, u64 *dE) {
    constexpr int OCC_CAP = CAP / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *vals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAP);
    int32_t *occ = keys + CAP;
    __shared__ int32_t nocc, item_sh;
    for (int s = threadIdx.x; s < CAP; s += THREADS) { keys[s] = -1; vals[s] = 0; }
    if (threadIdx.x == 0) nocc = 0;
    __syncthreads();
    const int32_t count = min(*fb.count, fb.cap);
    u64 delta_acc = 0;
    for (;;) {
        if (threadIdx.x == 0) item_sh = atomicAdd(fb.next, 1);
        __syncthreads();
        const int32_t item = item_sh;
        if (item >= count) break;
        const int32_t v = fb.v[item];
        int32_t p = 0, P = 1, first = item, src = -1;
        if (PART) { p = fb.p[item]; P = fb.P[item]; first = fb.first[item]; src = fb.src[item]; }
        const int32_t own = __ldg(st.comm + v);
        u64 e_own = 0;
        if (src < 0) {
            // the vertex's row
            const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
            int lg = P > 1 ? ilog2_c(CAP) : ceil_log2_i(2 * (int64_t)(r1 - r0));
            lg = lg < 3 ? 3 : lg;
            if (!PART) {
                insert_row<LV_U_FB, true>(g, st.comm, v, own, r0, r1, threadIdx.x, THREADS, keys, vals,
                                          lg, st.err, occ, &nocc, e_own, (LV_DEDUP && st.dedup != 0));
            } else if (LV_DEDUP && st.dedup) {
                // warp-uniform steps; a warp's equal keys combined first
                const int lane = threadIdx.x & 31;
                for (int32_t b = r0 + threadIdx.x - lane; b < r1; b += THREADS) {
                    const int32_t e = b + lane;
                    int32_t c = -1;
                    u64 w = 0;
                    if (e < r1) {
                        const int32_t j = __ldg(g.col + e);
                        if (j != v) {
                            c = __ldg(st.comm + j);
                            w = gw(g, e);
                        }
                    }
                    if (c >= 0 && c == own && p == 0) e_own += w;
                    const bool valid = c >= 0 && c != own && (P == 1 || (int32_t)part_of(c, P) == p);
                    const unsigned peers = key_peers(c, valid);
                    const u64 ws = group_sum_u64(peers, valid ? w : 0);
                    if (valid && group_leader(peers))
                        table_insert_occ_capped(keys, vals, lg, c, ws, st.err, occ, &nocc, OCC_CAP);
                }
            } else {
                for (int32_t e = r0 + threadIdx.x; e < r1; e += THREADS) {
                    const int32_t j = __ldg(g.col + e);
                    if (j == v) continue;
                    const int32_t c = __ldg(st.comm + j);
                    if (c == own) {
                        if (p == 0) e_own += gw(g, e);
                    } else if (P == 1 || (int32_t)part_of(c, P) == p) {
                        table_insert_occ_capped(keys, vals, lg, c, gw(g, e), st.err, occ,
                                                &nocc, OCC_CAP);
                    }
                }
            }
        } else {
            // the staged (community, weight) pairs of giant src
            const int32_t n = hg.nocc[src];
            int lg = P > 1 ? ilog2_c(CAP) : ceil_log2_i(2 * (int64_t)n);
            lg = lg < 3 ? 3 : lg;
            const int32_t pb = hg.pbase[src], pe = hg.pbase[src + 1];
            const bool regrouped = hg.poff && P > 1 && P + 2 <= pe - pb && hg.poff[pb] >= 0 && hg.poff[pe - 1] == P &&
                                   hg.poff[pb + P] == n;
            if (regrouped) {
                // partition p's pairs only (giant_regroup_kernel)
                const int32_t i0 = hg.poff[pb + p], i1 = min(hg.poff[pb + p + 1], n);
                const int32_t *sk = hg.stage2_key + hg.occ_off[src];
                const u64 *sv = hg.stage2_val + hg.occ_off[src];
                for (int32_t i = i0 + threadIdx.x; i < i1; i += THREADS)
                    table_insert_occ_capped(keys, vals, lg, sk[i], sv[i], st.err, occ, &nocc, OCC_CAP);
            } else {
                const int32_t *sk = hg.stage_key + hg.occ_off[src];
                const u64 *sv = hg.stage_val + hg.occ_off[src];
                for (int32_t i = threadIdx.x; i < n; i += THREADS) {
                    const int32_t c = sk[i];
                    if (P == 1 || (int32_t)part_of(c, P) == p)
                        table_insert_occ_capped(keys, vals, lg, c, sv[i], st.err, occ, &nocc, OCC_CAP);
                }
            }
            if (p == 0 && threadIdx.x == 0) e_own = hg.eown[src];
        }
        __syncthreads();
        const int32_t nd = min(nocc, OCC_CAP);
        const MoveCtx m = move_ctx(own, __ldg(st.size + own) == 1, st.T, __ldg(st.k + v), __ldg(st.S + own));
        Best b = best_init(own);
        b.eo = e_own;
        eval_slots<1, true, true>(keys, vals, occ, nd, threadIdx.x, THREADS, m, st.S, st.size, b);
        cta_reduce_best<THREADS>(m, b);
        if (threadIdx.x == 0) {
            nocc = 0;
            bool decide = P == 1;
            int32_t distinct = nd;
            Best t = b;
            if (P > 1) {
                fb.gd[item] = b.gd;
                fb.e[item] = b.e;
                fb.S[item] = b.S;
                fb.c[item] = b.c;
                fb.eo[item] = b.eo;
                fb.cnt[item] = nd;
                __threadfence();
                const int32_t done = atomicAdd(fb.done + first, 1);
                decide = done == P - 1;
                if (decide) {
                    __threadfence();
                    t = best_init(own);
                    distinct = 0;
                    for (int32_t q = 0; q < P; ++q) {
                        Best o;
                        o.gd = __ldcg(fb.gd + first + q);
                        o.e = __ldcg(fb.e + first + q);
                        o.S = __ldcg(fb.S + first + q);
                        o.c = __ldcg(fb.c + first + q);
                        o.eo = 0;
                        if (better(m, o, t)) { t.gd = o.gd; t.e = o.e; t.S = o.S; t.c = o.c; }
                        t.eo += __ldcg(fb.eo + first + q);
                        distinct += __ldcg(fb.cnt + first + q);
                    }
                    fb.done[first] = 0;
                }
            }
            if (decide) {
                u64 delta = 0;
                st.newc[v] = move_decision(m, t, &delta);
                record_features(st, v, m, t);
                delta_acc += delta;
                if (src >= 0) {
                    hg.nocc[src] = 0;
                    hg.eown[src] = 0;
                } else {
                    hint[v] = distinct > hint_set ? 1 : 0;
                }
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && delta_acc) atomicAdd(dE, delta_acc);
}

// The row queues' fallback CTAs for weights below 2^32: whole rows of degree
// <= CAP / 2 in a piece table (fire-and-forget adds), evaluated over the
// claimed-slot list.
template <typename WT, int THREADS, int CAP>
__global__ void __launch_bounds__(THREADS) move_rowq_narrow_kernel(GraphView<WT> g, StateView st, Fallback fb,
                                                                   uint8_t *hint, int32_t hint_set, u64 *dE) {
    constexpr int OCC_CAP = CAP / 2;
    static_assert(OCC_CAP <= PIECE_MAX_ADDS, "rows of the queue fit the piece counters");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PieceTable t;
    t.lo = reinterpret_cast<uint32_t *>(smem_raw);
    t.hi = t.lo + CAP;
    t.keys = reinterpret_cast<int32_t *>(t.hi + CAP);
    int32_t *occ = t.keys + CAP;
    __shared__ int32_t nocc, item_sh;
    for (int s = threadIdx.x; s < CAP; s += THREADS) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    if (threadIdx.x == 0) nocc = 0;
    __syncthreads();
    const int32_t count = min(*fb.count, fb.cap);
    u64 delta_acc = 0;
    for (;;) {
        if (threadIdx.x == 0) item_sh = atomicAdd(fb.next, 1);
        __syncthreads();
        const int32_t item = item_sh;
        if (item >= count) break;
        const int32_t v = fb.v[item];
        const int32_t own = __ldg(st.comm + v);
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        int lg = ceil_log2_i(2 * (int64_t)(r1 - r0));
        lg = lg < 3 ? 3 : lg;
        u64 e_own = 0;
        insert_row_piece<LV_U_FB, true>(g, st.comm, v, own, r0, r1, threadIdx.x, THREADS, t, lg, st.err, occ,
                                        &nocc, OCC_CAP, e_own, (LV_DEDUP && st.dedup != 0));
        __syncthreads();
        const int32_t nd = min(nocc, OCC_CAP);
        const MoveCtx m = move_ctx(own, __ldg(st.size + own) == 1, st.T, __ldg(st.k + v), __ldg(st.S + own));
        Best b = best_init(own);
        b.eo = e_own;
        for (int32_t i = threadIdx.x; i < nd; i += THREADS) {
            const int32_t sl = occ[i];
            const int32_t c = t.keys[sl];
            const u64 ec = piece_value(t, (uint32_t)sl);
            t.keys[sl] = -1;
            t.lo[sl] = 0;
            t.hi[sl] = 0;
            const bool cand = c != own;
            const u64 Sc = cand ? __ldg(st.S + c) : 0;
            const int32_t szc = (cand && guard_needs_size(m, c)) ? __ldg(st.size + c) : 0;
            eval_loaded(c, ec, Sc, szc, m, b);
        }
        cta_reduce_best<THREADS>(m, b);
        if (threadIdx.x == 0) {
            nocc = 0;
            u64 delta = 0;
            st.newc[v] = move_decision(m, b, &delta);
            record_features(st, v, m, b);
            delta_acc += delta;
            hint[v] = nd > hint_set ? 1 : 0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && delta_acc) atomicAdd(dE, delta_acc);
}

// move_rowq_narrow_kernel with the rows staged in shared memory by 1-D bulk
// copies (TMA): while the CTA decides one row, the next item's columns and
// weights are already on their way into the other of two staging buffers, so
// the insert loop reads them from shared memory and only the community
// gathers go to global memory.  A bulk copy covers the row rounded out to
// 16-byte boundaries (entries [r0 & ~3, (r1 + 3) & ~3)), clipped to the last
// whole 16 bytes of the arrays; entries past the clip are read from global
// memory.  The host uses this form only for 4-byte weights whose column and
// weight arrays start on 16-byte boundaries.
template <int THREADS, int CAP>
struct RowqStage {
    static constexpr int SB = CAP / 2 + 4;   // staged entries per buffer (row + alignment)
    static constexpr int TABLE = CAP * 12 + (CAP / 2) * 4;
    static constexpr int BYTES = TABLE + 2 * SB * 8 + 2 * 8 + 8 * 4;
};

template <typename WT, int THREADS, int CAP>
__global__ void __launch_bounds__(THREADS) move_rowq_staged_kernel(GraphView<WT> g, StateView st, Fallback fb,
                                                                   uint8_t *hint, int32_t hint_set, u64 *dE) {
    static_assert(sizeof(WT) == 4, "staged rows hold 4-byte weights");
    constexpr int OCC_CAP = CAP / 2;
    constexpr int SB = RowqStage<THREADS, CAP>::SB;
    constexpr int U = LV_U_FB;
    static_assert(OCC_CAP <= PIECE_MAX_ADDS, "rows of the queue fit the piece counters");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PieceTable t;
    t.lo = reinterpret_cast<uint32_t *>(smem_raw);
    t.hi = t.lo + CAP;
    t.keys = reinterpret_cast<int32_t *>(t.hi + CAP);
    int32_t *occ = t.keys + CAP;
    int32_t *scol = reinterpret_cast<int32_t *>(smem_raw + RowqStage<THREADS, CAP>::TABLE);   // [2][SB]
    uint32_t *sw = reinterpret_cast<uint32_t *>(scol + 2 * SB);                               // [2][SB]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sw + 2 * SB);                                // [2]
    int32_t *info = reinterpret_cast<int32_t *>(bar + 2);   // [2][4]: item, r0, r1, staged count
    __shared__ int32_t nocc;
    __shared__ int timed_out;
    for (int s = threadIdx.x; s < CAP; s += THREADS) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    const int32_t count = min(*fb.count, fb.cap);
    const int64_t clip = g.nent & ~(int64_t)3;   // bulk copies end at or before this entry
    // thread 0 takes the next item and starts its row's bulk copy into buffer b
    auto fetch = [&](int b) {
        const int32_t item = atomicAdd(fb.next, 1);
        int32_t r0 = 0, r1 = 0, nst = 0;
        if (item < count) {
            const int32_t v = fb.v[item];
            r0 = g.rowptr[v];
            r1 = g.rowend[v];
            const int64_t a0 = (int64_t)(r0 & ~3);
            int64_t a1 = ((int64_t)r1 + 3) & ~(int64_t)3;
            if (a1 > clip) a1 = clip;
            nst = a1 > a0 ? (int32_t)(a1 - a0) : 0;
            if (nst > SB) nst = 0;   // cannot happen for rows of this queue; read them from global memory
            fence_proxy_async_smem();
            mbar_arrive_expect(bar + b, (uint32_t)nst * 8u);
            if (nst > 0) {
                bulk_g2s(scol + b * SB, g.col + a0, (uint32_t)nst * 4u, bar + b);
                bulk_g2s(sw + b * SB, g.w + a0, (uint32_t)nst * 4u, bar + b);
            }
        }
        info[4 * b] = item;
        info[4 * b + 1] = r0;
        info[4 * b + 2] = r1;
        info[4 * b + 3] = nst;
    };
    if (threadIdx.x == 0) {
        nocc = 0;
        timed_out = 0;
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) fetch(0);
    __syncthreads();
    u64 delta_acc = 0;
    uint32_t phase = 0;   // bit b: parity of buffer b's next completion
    int b = 0;
    for (;;) {
        const int32_t item = info[4 * b];
        if (item >= count) break;
        const int32_t r0 = info[4 * b + 1], r1 = info[4 * b + 2], nst = info[4 * b + 3];
        // the next item's copy goes out before this row is waited for
        if (threadIdx.x == 0) fetch(b ^ 1);
        if (!mbar_wait_parity(bar + b, (phase >> b) & 1u, MBAR_MAX_POLLS)) timed_out = 1;
        __syncthreads();
        if (timed_out) break;
        phase ^= 1u << b;
        const int32_t v = fb.v[item];
        const int32_t own = __ldg(st.comm + v);
        const int32_t a0 = r0 & ~3;                        // staged entry i is entry a0 + i
        const int32_t *rc = scol + b * SB;
        const uint32_t *rw = sw + b * SB;
        const int32_t send = a0 + nst;                     // first entry not staged
        int lg = ceil_log2_i(2 * (int64_t)(r1 - r0));
        lg = lg < 3 ? 3 : lg;
        u64 e_own = 0;
        const int lane = threadIdx.x & 31;
        for (int32_t base = r0 + threadIdx.x; base - lane < r1; base += U * THREADS) {
            int32_t jj[U];
            uint32_t xx[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = base + u * THREADS;
                jj[u] = -1;
                xx[u] = 0;
                if (e < r1) {
                    if (e < send) { jj[u] = rc[e - a0]; xx[u] = rw[e - a0]; }
                    else { jj[u] = __ldg(g.col + e); xx[u] = raw_row(g, e); }
                }
            }
            int32_t cc[U];
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? __ldg(st.comm + jj[u]) : -1;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const u64 w = cc[u] >= 0 ? raw_value(g, base + u * THREADS, xx[u]) : 0;
                int32_t claimed = -1;
                if (LV_DEDUP && st.dedup) {
                    const bool valid = cc[u] >= 0 && cc[u] != own;
                    if (cc[u] >= 0 && cc[u] == own) e_own += w;
                    const unsigned peers = key_peers(cc[u], valid);
                    const Pieces pc = group_pieces(peers, valid ? w : 0);
                    if (valid && group_leader(peers))
                        claimed = piece_insert_at_p(t, lg, hash_slot(cc[u], lg), cc[u], pc, st.err);
                } else if (cc[u] >= 0) {
                    if (cc[u] == own) e_own += w;
                    else claimed = piece_insert(t, lg, cc[u], w, st.err);
                }
                warp_append_capped(claimed, occ, &nocc, OCC_CAP);
            }
        }
        __syncthreads();
        const int32_t nd = min(nocc, OCC_CAP);
        const MoveCtx m = move_ctx(own, __ldg(st.size + own) == 1, st.T, __ldg(st.k + v), __ldg(st.S + own));
        Best bb = best_init(own);
        bb.eo = e_own;
        for (int32_t i = threadIdx.x; i < nd; i += THREADS) {
            const int32_t sl = occ[i];
            const int32_t c = t.keys[sl];
            const u64 ec = piece_value(t, (uint32_t)sl);
            t.keys[sl] = -1;
            t.lo[sl] = 0;
            t.hi[sl] = 0;
            const bool cand = c != own;
            const u64 Sc = cand ? __ldg(st.S + c) : 0;
            const int32_t szc = (cand && guard_needs_size(m, c)) ? __ldg(st.size + c) : 0;
            eval_loaded(c, ec, Sc, szc, m, bb);
        }
        cta_reduce_best<THREADS>(m, bb);
        if (threadIdx.x == 0) {
            nocc = 0;
            u64 delta = 0;
            st.newc[v] = move_decision(m, bb, &delta);
            record_features(st, v, m, bb);
            delta_acc += delta;
            hint[v] = nd > hint_set ? 1 : 0;
        }
        __syncthreads();
        b ^= 1;
    }
    if (timed_out) {
        // a copy that did not complete in time: report it, and give the
        // copies still in flight (buffer b's and, when the next item was
        // valid, the other buffer's) a bounded time to land before the CTA's
        // shared memory is released
        if (threadIdx.x == 0) {
            atomicOr(st.err, DEVERR_BAD_STATE);
            mbar_wait_parity(bar + b, (phase >> b) & 1u, MBAR_MAX_POLLS);
            if (info[4 * (b ^ 1)] < count) mbar_wait_parity(bar + (b ^ 1), (phase >> (b ^ 1)) & 1u, MBAR_MAX_POLLS);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && delta_acc) atomicAdd(dE, delta_acc);
}

// ------------------------------------------------------------------------
// giants (degree > 8192): staged two-level reduction
// ------------------------------------------------------------------------
// G1. One CTA per chunk of STAGE_CHUNK edges of a giant reduces the chunk in
//     shared memory and appends its distinct (community, weight) pairs to the
//     giant's staging area (room for `degree` pairs); the weight to the
//     giant's own community goes to eown[h].
// G2. Persistent CTAs merge each giant's staged pairs in a shared table and
//     decide its move; a giant with more staged pairs than the table holds
//     is queued as key-space partitions of its staged pairs (fallback items
//     with src = h), which the fallback kernel then decides.
// giant_stage_kernel for weights below 2^32: the chunk's table keeps its sums
// in 16-bit-piece counters (fire-and-forget adds; a chunk has STAGE_CHUNK
// entries, far below PIECE_MAX_ADDS).
template <typename WT>
__global__ void __launch_bounds__(STAGE_THREADS) giant_stage_narrow_kernel(GraphView<WT> g, StateView st,
                                                                           HubGlobal hg) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LCAP = 2 * STAGE_CHUNK;
    constexpr int LLG = ilog2_c(LCAP);
    static_assert(STAGE_CHUNK <= PIECE_MAX_ADDS, "chunks fit the piece counters");
    PieceTable t;
    t.lo = reinterpret_cast<uint32_t *>(smem_raw);
    t.hi = t.lo + LCAP;
    t.keys = reinterpret_cast<int32_t *>(t.hi + LCAP);
    int32_t *locc = t.keys + LCAP;
    __shared__ int32_t lnocc, base;
    for (int s = threadIdx.x; s < LCAP; s += STAGE_THREADS) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    if (threadIdx.x == 0) lnocc = 0;
    __syncthreads();
    // persistent over the chunks: the table is initialised once and after
    // each chunk only its claimed slots are cleared (a chunk of an aggregated
    // level touches a few dozen of the 2 STAGE_CHUNK slots)
    for (int32_t ch = blockIdx.x; ch < hg.n_echunks; ch += gridDim.x) {
        const int32_t h = hg.echunk_hub[ch];
        const int32_t v = hg.hubs[h];
        if (st.wrow && st.wrow[v]) continue;   // staged by giant_stage_kernel (64-bit sums)
        const int32_t r1 = g.rowend[v];
        const int32_t e0 = g.rowptr[v] + hg.echunk_e0[ch];
        const int32_t e1 = min(e0 + STAGE_CHUNK, r1);
        const int32_t own = __ldg(st.comm + v);
        u64 e_own = 0;
        insert_row_piece<LV_U_STAGE, true>(g, st.comm, v, own, e0, e1, threadIdx.x, STAGE_THREADS, t, LLG, st.err,
                                           locc, &lnocc, STAGE_CHUNK, e_own, (LV_DEDUP && st.dedup != 0));
        block_add_total<STAGE_THREADS>(e_own, hg.eown + h);   // contains the barrier
        const int32_t n = min(lnocc, STAGE_CHUNK);
        if (threadIdx.x == 0) base = atomicAdd(hg.nocc + h, n);
        __syncthreads();
        int32_t *sk = hg.stage_key + hg.occ_off[h] + base;
        u64 *sv = hg.stage_val + hg.occ_off[h] + base;
        for (int32_t i = threadIdx.x; i < n; i += STAGE_THREADS) {
            const uint32_t sl = (uint32_t)locc[i];
            sk[i] = t.keys[sl];
            sv[i] = piece_value(t, sl);
            t.keys[sl] = -1;
            t.lo[sl] = 0;
            t.hi[sl] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) lnocc = 0;
        __syncthreads();
    }
}

template <typename WT>
__global__ void __launch_bounds__(STAGE_THREADS) giant_stage_kernel(GraphView<WT> g, StateView st,
                                                                    HubGlobal hg, const uint8_t *only) {
    // only != nullptr: just the giants marked there (the rest are staged by
    // the narrow kernel).  Persistent over the chunks, as the narrow kernel:
    // the table is initialised once and after each chunk only its claimed
    // slots are cleared.
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LCAP = 2 * STAGE_CHUNK;
    constexpr int LLG = ilog2_c(LCAP);
    u64 *lvals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *lkeys = reinterpret_cast<int32_t *>(lvals + LCAP);
    int32_t *locc = lkeys + LCAP;   // claimed slots of the chunk (at most STAGE_CHUNK)
    __shared__ int32_t lnocc, base;
    for (int s = threadIdx.x; s < LCAP; s += STAGE_THREADS) { lkeys[s] = -1; lvals[s] = 0; }
    if (threadIdx.x == 0) lnocc = 0;
    __syncthreads();
    for (int32_t ch = blockIdx.x; ch < hg.n_echunks; ch += gridDim.x) {
        const int32_t h = hg.echunk_hub[ch];
        const int32_t v = hg.hubs[h];
        if (only && !only[v]) continue;
        const int32_t r1 = g.rowend[v];
        const int32_t e0 = g.rowptr[v] + hg.echunk_e0[ch];
        const int32_t e1 = min(e0 + STAGE_CHUNK, r1);
        const int32_t own = __ldg(st.comm + v);
        u64 e_own = 0;
        insert_row<LV_U_STAGE, true>(g, st.comm, v, own, e0, e1, threadIdx.x, STAGE_THREADS, lkeys, lvals, LLG,
                                     st.err, locc, &lnocc, e_own, (LV_DEDUP && st.dedup != 0));
        block_add_total<STAGE_THREADS>(e_own, hg.eown + h);   // contains the barrier
        const int32_t n = min(lnocc, STAGE_CHUNK);
        if (threadIdx.x == 0) base = atomicAdd(hg.nocc + h, n);
        __syncthreads();
        int32_t *sk = hg.stage_key + hg.occ_off[h] + base;
        u64 *sv = hg.stage_val + hg.occ_off[h] + base;
        for (int32_t i = threadIdx.x; i < n; i += STAGE_THREADS) {
            const int32_t sl = locc[i];
            sk[i] = lkeys[sl];
            sv[i] = lvals[sl];
            lkeys[sl] = -1;
            lvals[sl] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) lnocc = 0;
        __syncthreads();
    }
}

// Giants with more staged pairs than the merge table holds are decided by
// P = ceil(n / FB_KEYS) large-queue items, item p keeping the pairs whose
// key falls in partition p.  Before the merges, one CTA per such giant
// regroups its n staged pairs by partition (a counting sort: partition
// sizes, their offsets, then a scatter into stage2), so that each item reads
// its own n / P pairs instead of all n.  A giant whose P would exceed
// REGROUP_PMAX keeps the filtering path (poff[pbase] = -1).
constexpr int REGROUP_THREADS = 1024;
constexpr int REGROUP_PMAX = 4096;

__global__ void __launch_bounds__(REGROUP_THREADS) giant_regroup_kernel(HubGlobal hg) {
    __shared__ int32_t cnt[REGROUP_PMAX];
    const int32_t h = blockIdx.x;
    const int32_t pb = hg.pbase[h], pe = hg.pbase[h + 1];   // pe - pb = Pmax + 2
    const int32_t cap = hg.hub_cap[h];
    const int32_t n = min(hg.nocc[h], cap);
    if (2 * (int64_t)n <= HG_MERGE_CAP) return;   // merged in shared memory; no items
    const int32_t P = (n + FB_KEYS - 1) / FB_KEYS;
    if (P > REGROUP_PMAX || P + 2 > pe - pb) {
        if (threadIdx.x == 0) hg.poff[pb] = -1;
        return;
    }
    for (int32_t p = threadIdx.x; p < P; p += REGROUP_THREADS) cnt[p] = 0;
    __syncthreads();
    const int64_t o = hg.occ_off[h];
    const int32_t *sk = hg.stage_key + o;
    const u64 *sv = hg.stage_val + o;
    for (int32_t i = threadIdx.x; i < n; i += REGROUP_THREADS) atomicAdd(&cnt[part_of(sk[i], P)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        // exclusive offsets; cnt[p] becomes partition p's write cursor
        int32_t run = 0;
        for (int32_t p = 0; p < P; ++p) {
            const int32_t c = cnt[p];
            hg.poff[pb + p] = run;
            cnt[p] = run;
            run += c;
        }
        hg.poff[pb + P] = run;        // = n
        hg.poff[pe - 1] = P;
    }
    __syncthreads();
    int32_t *dk = hg.stage2_key + o;
    u64 *dv = hg.stage2_val + o;
    for (int32_t i = threadIdx.x; i < n; i += REGROUP_THREADS) {
        const int32_t c = sk[i];
        const int32_t pos = atomicAdd(&cnt[part_of(c, P)], 1);   // < n: the cursors stay in their partitions
        dk[pos] = c;
        dv[pos] = sv[i];
    }
}

// Two instances: CAP = HG_MERGE_CAP decides the giants with
// n_min < n <= HG_MERGE_CAP / 2 staged pairs and queues the larger ones; a
// smaller instance (more CTAs per SM) runs first and takes n <= CAP / 2.
template <int THREADS, int CAP>
__global__ void __launch_bounds__(THREADS) giant_merge_kernel(StateView st, HubGlobal hg, Fallback fb,
                                                              u64 *dE, int32_t n_min) {
    // fb: the large fallback queue
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *vals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAP);
    int32_t *occ = keys + CAP;
    __shared__ int32_t nocc;
    for (int s = threadIdx.x; s < CAP; s += THREADS) { keys[s] = -1; vals[s] = 0; }
    if (threadIdx.x == 0) nocc = 0;
    __syncthreads();
    u64 delta_sum = 0;
    for (int32_t h = blockIdx.x; h < hg.nhubs; h += gridDim.x) {
        const int32_t n = hg.nocc[h];
        if (2 * (int64_t)n > HG_MERGE_CAP && CAP == HG_MERGE_CAP) {
            // too many staged pairs for one shared table: queue key-space
            // partitions of the staged pairs for the fallback kernel
            if (threadIdx.x == 0) {
                const int32_t P = (n + FB_KEYS - 1) / FB_KEYS;
                const int32_t first = atomicAdd(fb.count, P);
                if (first + P <= fb.cap) {
                    for (int32_t q = 0; q < P; ++q) {
                        fb.v[first + q] = hg.hubs[h];
                        fb.p[first + q] = q;
                        fb.P[first + q] = P;
                        fb.first[first + q] = first;
                        fb.src[first + q] = h;
                    }
                } else {
                    atomicOr(st.err, DEVERR_FALLBACK_FULL);
                }
            }
            continue;
        }
        if (n <= n_min || 2 * (int64_t)n > CAP) continue;   // the other instance's range
        const int32_t v = hg.hubs[h];
        const int32_t own = __ldg(st.comm + v);
        int lg = ceil_log2_i(2 * (int64_t)n);
        lg = lg < 3 ? 3 : lg;
        const int32_t *sk = hg.stage_key + hg.occ_off[h];
        const u64 *sv = hg.stage_val + hg.occ_off[h];
        for (int32_t i = threadIdx.x; i < n; i += THREADS)
            table_insert_occ(keys, vals, lg, sk[i], sv[i], st.err, occ, &nocc);
        __syncthreads();
        const MoveCtx m = move_ctx(own, __ldg(st.size + own) == 1, st.T, __ldg(st.k + v), __ldg(st.S + own));
        Best b = best_init(own);
        if (threadIdx.x == 0) b.eo = hg.eown[h];
        eval_slots<1, true, true>(keys, vals, occ, nocc, threadIdx.x, THREADS, m, st.S, st.size, b);
        cta_reduce_best<THREADS>(m, b);
        if (threadIdx.x == 0) {
            u64 delta = 0;
            st.newc[v] = move_decision(m, b, &delta);
            record_features(st, v, m, b);
            delta_sum += delta;
            nocc = 0;
            hg.nocc[h] = 0;
            hg.eown[h] = 0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && delta_sum) atomicAdd(dE, delta_sum);
}

// ------------------------------------------------------------------------
// correction of the modularity update for neighbours that moved together
// ------------------------------------------------------------------------
// For a mover u and a neighbour j != u that moved in the same sub-round, the
// per-vertex updates 2(e_best - e_own) assumed j static; the exact change of
// the pair's two CSR entries differs by
//   w_uj ([n_u = n_j] - [n_u = c_j] - [c_u = n_j] + [c_u = c_j])
// from each side (c = community before, n = after the sub-round).  Vertices
// outside the sub-round's bucket have newc == comm, so "j moved" is newc[j] !=
// comm[j].  Sums wrap in uint64; the final total is exact.
__device__ __forceinline__ u64 pair_correction(int32_t cu, int32_t nu, int32_t cj, int32_t nj, u64 w) {
    const int t = (int)(nu == nj) - (int)(nu == cj) - (int)(cu == nj) + (int)(cu == cj);
    return (u64)(i64)t * w;
}

template <int G, typename WT>
__global__ void __launch_bounds__(256) corr_group_kernel(GraphView<WT> g, const int32_t *__restrict__ comm,
                                                         const int32_t *__restrict__ newc,
                                                         const int32_t *__restrict__ list, int32_t n,
                                                         u64 *dE) {
    const int grp = threadIdx.x / G, lane = threadIdx.x % G;
    const int32_t idx = blockIdx.x * (256 / G) + grp;
    u64 acc = 0;
    if (idx < n) {
        const int32_t u = list[idx];
        const int32_t cu = comm[u], nu = newc[u];
        if (cu != nu) {
            const int32_t r0 = g.rowptr[u], r1 = g.rowend[u];
            for (int32_t e = r0 + lane; e < r1; e += G) {
                const int32_t j = __ldg(g.col + e);
                if (j == u) continue;
                const int32_t cj = comm[j], nj = newc[j];
                if (cj != nj) acc += pair_correction(cu, nu, cj, nj, gw(g, e));
            }
        }
    }
    block_add_total<256>(acc, dE);
}

// Rows of T threads each.  A pass checks CORR_BATCH vertices of the list at
// once (one per lane of warp 0), gathers the ones that moved in shared
// memory, and then scans only their rows, so a sub-round with few movers
// costs one parallel check per CORR_BATCH vertices instead of a serial check
// per vertex.
constexpr int CORR_BATCH = 32;

template <int T, typename WT>
__global__ void __launch_bounds__(T) corr_cta_kernel(GraphView<WT> g, const int32_t *__restrict__ comm,
                                                     const int32_t *__restrict__ newc,
                                                     const int32_t *__restrict__ list, int32_t n,
                                                     u64 *dE) {
    __shared__ int32_t movers[CORR_BATCH];
    __shared__ int32_t nm;
    u64 acc = 0;
    for (int32_t base = blockIdx.x * CORR_BATCH; base < n; base += gridDim.x * CORR_BATCH) {
        if (threadIdx.x < 32) {
            const int32_t idx = base + threadIdx.x;
            bool moved = false;
            int32_t u = 0;
            if (idx < n) {
                u = list[idx];
                moved = comm[u] != newc[u];
            }
            const unsigned bal = __ballot_sync(FULL, moved);
            if (moved) movers[__popc(bal & ((1u << threadIdx.x) - 1u))] = u;
            if (threadIdx.x == 0) nm = __popc(bal);
        }
        __syncthreads();
        const int32_t cnt = nm;
        for (int32_t k = 0; k < cnt; ++k) {
            const int32_t u = movers[k];
            const int32_t cu = comm[u], nu = newc[u];
            const int32_t r0 = g.rowptr[u], r1 = g.rowend[u];
            for (int32_t e = r0 + threadIdx.x; e < r1; e += T) {
                const int32_t j = __ldg(g.col + e);
                if (j == u) continue;
                const int32_t cj = comm[j], nj = newc[j];
                if (cj != nj) acc += pair_correction(cu, nu, cj, nj, gw(g, e));
            }
        }
        __syncthreads();   // movers / nm are rewritten by the next pass
    }
    block_add_total<T>(acc, dE);
}

// ------------------------------------------------------------------------
// commit of one sub-round (updateVertexCommunity + Sigma_tot update)
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) commit_kernel(StateView st, const int32_t *__restrict__ list,
                                                     int32_t n, u64 *moves) {
    const int32_t i = blockIdx.x * 256 + threadIdx.x;
    u64 mv = 0;
    if (i < n) {
        const int32_t v = list[i];
        const int32_t nc = st.newc[v], oc = st.comm[v];
        if (nc != oc) {
            mv = 1;
            st.comm[v] = nc;
            atomicAdd(st.size + nc, 1);
            atomicSub(st.size + oc, 1);
            const u64 kv = st.k[v];
            atomicAdd(st.S + nc, kv);
            atomicAdd(st.S + oc, (u64)0 - kv);
        }
    }
    block_add_total<256>(mv, moves);
}

// ------------------------------------------------------------------------
// row reductions: k_i (mode 0) and sum_i e_{i->C(i)} (mode 1)
// ------------------------------------------------------------------------
template <int G, int MODE, typename WT>
__global__ void __launch_bounds__(256) row_reduce_group_kernel(GraphView<WT> g,
                                                               const int32_t *__restrict__ comm,
                                                               u64 *k, u64 *total,
                                                               const int32_t *__restrict__ list,
                                                               int32_t n) {
    const int grp = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int32_t idx = blockIdx.x * (256 / G) + grp;
    u64 acc = 0;
    int32_t v = 0;
    if (idx < n) {
        v = list[idx];
        const int32_t own = MODE == 1 ? comm[v] : 0;
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        for (int32_t e = r0 + lane; e < r1; e += G) {
            if (MODE == 1) {
                if (comm[__ldg(g.col + e)] == own) acc += gw(g, e);
            } else {
                acc += gw(g, e);
            }
        }
    }
    if (MODE == 0) {
        for (int off = G >> 1; off > 0; off >>= 1) acc += __shfl_xor_sync(FULL, acc, off, G);
        if (idx < n && lane == 0) k[v] = acc;
    } else {
        block_add_total<256>(acc, total);
    }
}

template <int THREADS, int MODE, typename WT>
__global__ void __launch_bounds__(THREADS) row_reduce_cta_kernel(GraphView<WT> g,
                                                                 const int32_t *__restrict__ comm,
                                                                 u64 *k, u64 *total,
                                                                 const int32_t *__restrict__ list,
                                                                 int32_t n) {
    __shared__ u64 part[THREADS / 32];
    u64 grand = 0;
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t v = list[idx];
        const int32_t own = MODE == 1 ? comm[v] : 0;
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        u64 acc = 0;
        for (int32_t e = r0 + threadIdx.x; e < r1; e += THREADS) {
            if (MODE == 1) {
                if (comm[__ldg(g.col + e)] == own) acc += gw(g, e);
            } else {
                acc += gw(g, e);
            }
        }
        if (MODE == 0) {
            acc = warp_sum_u64(acc);
            if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
            __syncthreads();
            if (threadIdx.x == 0) {
                u64 y = 0;
                for (int w = 0; w < THREADS / 32; ++w) y += part[w];
                k[v] = y;
            }
            __syncthreads();
        } else {
            grand += acc;
        }
    }
    if (MODE == 1) block_add_total<THREADS>(grand, total);
}

__global__ void __launch_bounds__(256) s2_kernel(const u64 *__restrict__ S, int32_t V,
                                                 u64 *total_hi_lo) {
    __shared__ u64 plo[8], phi[8];
    u128 acc = 0;
    for (int32_t c = blockIdx.x * 256 + threadIdx.x; c < V; c += gridDim.x * 256) {
        const u64 x = S[c];
        acc += (u128)x * (u128)x;
    }
    acc = warp_sum_u128(acc);
    if ((threadIdx.x & 31) == 0) {
        plo[threadIdx.x >> 5] = (u64)acc;
        phi[threadIdx.x >> 5] = (u64)(acc >> 64);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        u128 y = 0;
        for (int w = 0; w < 8; ++w) y += ((u128)phi[w] << 64) | (u128)plo[w];
        if (y) atomic_add_u128(total_hi_lo, y);
    }
}

inline unsigned nblocks(int64_t items, int per_block) {
    return (unsigned)((items + per_block - 1) / per_block);
}

}  // namespace

__host__ __device__ constexpr int FBQ_SMEM(int b) { return 2 * FBQ_MAXDEG(b) * 14; }

// Giants decided by several large-queue items have their staged pairs
// regrouped by key partition first (1), or every item filters all of the
// giant's pairs (0).
#ifndef LV_GIANT_REGROUP
#define LV_GIANT_REGROUP 1
#endif

// Rows of the narrow row queues staged by bulk copies (1) or read with
// plain loads (0).  0 is the default: on R-MAT-22's first level-0 sweep the
// staged 256-thread queue kernel took 595 us against 474 us (its rows are
// already read by coalesced loads; the staging adds barrier and
// shared-memory waits, issue-active 43 % against 53 %).
#ifndef LV_ROWQ_STAGE
#define LV_ROWQ_STAGE 0
#endif

template <typename WT, int B>
static void set_row_queue_attrs(DeviceInfo &di) {
    constexpr int T = FBQ_THREADS(B), CAP = 2 * FBQ_MAXDEG(B), SM = FBQ_SMEM(B);
    cudaFuncSetAttribute(move_fallback_kernel<WT, T, CAP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
    cudaFuncSetAttribute(move_rowq_narrow_kernel<WT, T, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
    int o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, move_fallback_kernel<WT, T, CAP, false>, T, SM);
    di.occ_fbq[B] = o > 0 ? o : 1;
    o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, move_rowq_narrow_kernel<WT, T, CAP>, T, SM);
    di.occ_fbq_narrow[B] = o > 0 ? o : 1;
    if constexpr (sizeof(WT) == 4) {
        constexpr int SS = RowqStage<T, CAP>::BYTES;
        cudaFuncSetAttribute(move_rowq_staged_kernel<WT, T, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, SS);
        o = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, move_rowq_staged_kernel<WT, T, CAP>, T, SS);
        di.occ_fbq_staged[B] = o > 0 ? o : 1;
    }
}

template <typename WT, int B>
static void launch_row_queue(const GraphView<WT> &g, const StateView &st, const FallbackSet &fs,
                             const DeviceInfo &di, u64 *dE, cudaStream_t s, bool narrow) {
    constexpr int T = FBQ_THREADS(B), CAP = 2 * FBQ_MAXDEG(B), SM = FBQ_SMEM(B);
    if constexpr (sizeof(WT) == 4) {
        // bulk copies need 16-byte aligned arrays
        const bool aligned = (((uintptr_t)g.col | (uintptr_t)g.w) & 15u) == 0;
        if (LV_ROWQ_STAGE && narrow && aligned) {
            move_rowq_staged_kernel<WT, T, CAP><<<di.sms * di.occ_fbq_staged[B], T, RowqStage<T, CAP>::BYTES, s>>>(
                g, st, fs.q[B], fs.hint, fs.hint_set, dE);
            note_launches(1);
            return;
        }
    }
    if (narrow)
        move_rowq_narrow_kernel<WT, T, CAP><<<di.sms * di.occ_fbq_narrow[B], T, SM, s>>>(g, st, fs.q[B], fs.hint,
                                                                                        fs.hint_set, dE);
    else
        move_fallback_kernel<WT, T, CAP, false><<<di.sms * di.occ_fbq[B], T, SM, s>>>(g, st, fs.q[B], HubGlobal(),
                                                                                    fs.hint, fs.hint_set, dE);
    note_launches(1);
}

template <typename WT>
static void set_attrs_for(DeviceInfo &di) {
    set_row_queue_attrs<WT, 0>(di);
    set_row_queue_attrs<WT, 1>(di);
    set_row_queue_attrs<WT, 2>(di);
    set_row_queue_attrs<WT, 3>(di);
    cudaFuncSetAttribute(move_fallback_kernel<WT, FB_THREADS, FB_CAP, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, FB_SMEM);
    cudaFuncSetAttribute(giant_stage_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, STAGE_SMEM);
    cudaFuncSetAttribute(giant_stage_narrow_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, STAGE_SMEM);
    {
        int o2 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, giant_stage_narrow_kernel<WT>, STAGE_THREADS, STAGE_SMEM);
        di.occ_stage_narrow = o2 > 0 ? o2 : 1;
        o2 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, giant_stage_kernel<WT>, STAGE_THREADS, STAGE_SMEM);
        di.occ_stage = o2 > 0 ? o2 : 1;
    }
    cudaFuncSetAttribute(move_warp_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, WARP_SMEM);
#ifdef LV_WIDE_CARVEOUT
    // measurement knob: preferred shared-memory share of the 64-bit warp
    // kernel (72: three CTAs per SM with 92 KB of L1 instead of four with
    // 60 KB measured the same, 119.7 ms for the degree > 319 class)
    cudaFuncSetAttribute(move_warp_kernel<WT>, cudaFuncAttributePreferredSharedMemoryCarveout, LV_WIDE_CARVEOUT);
#endif
    cudaFuncSetAttribute(move_warp_narrow_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, WARP_NSMEM);
    // The SM's L1 / shared-memory split follows the shared memory its
    // resident CTAs need, in steps (…, 132, 164, 196, 228 KB of shared
    // memory; L1 gets the rest of 256 KB).  Four narrow warp CTAs (53 KB
    // each) would take the 228 KB step and leave 28 KB of L1 for the
    // community and Sigma_tot gathers; preferring the 164 KB step runs three
    // CTAs per SM with 92 KB of L1, which measured faster (degrees 33-84 at
    // level 0: 9.45 against 10.05 ms per R-MAT-24 run).
#ifndef LV_NARROW_CARVEOUT
#define LV_NARROW_CARVEOUT 72
#endif
    if (LV_NARROW_CARVEOUT > 0)
        cudaFuncSetAttribute(move_warp_narrow_kernel<WT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             LV_NARROW_CARVEOUT);
    int o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, move_warp_kernel<WT>, 256, WARP_SMEM);
    di.occ_warp = o > 0 ? o : 1;
    o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, move_warp_narrow_kernel<WT>, 256, WARP_NSMEM);
    di.occ_warp_narrow = o > 0 ? o : 1;
}

void init_kernel_attributes(DeviceInfo &di) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev);
    set_attrs_for<u64>(di);
    set_attrs_for<uint32_t>(di);
    set_attrs_for<float>(di);
    cudaFuncSetAttribute(giant_merge_kernel<HG_MERGE_THREADS, HG_MERGE_CAP>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, HG_MERGE_SMEM);
    cudaFuncSetAttribute(giant_merge_kernel<MERGE_S_THREADS, MERGE_S_CAP>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, MERGE_S_CAP * 14);
    int o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, giant_merge_kernel<MERGE_S_THREADS, MERGE_S_CAP>,
                                                  MERGE_S_THREADS, MERGE_S_CAP * 14);
    di.occ_merge_s = o > 0 ? o : 1;
}

template <typename WT>
static void launch_fallback_large(const GraphView<WT> &g, const StateView &st, const HubGlobal &hg,
                                  const FallbackSet &fs, const DeviceInfo &di, u64 *dE, cudaStream_t s);

template <typename WT>
void launch_move_class(int cls, const GraphView<WT> &g, const StateView &st, const int32_t *list,
                       int32_t n, const DeviceInfo &di, u64 *dE, cudaStream_t s, bool narrow,
                       const FallbackSet &fs) {
    if (n <= 0) return;
    // rows marked in st.wrow go to the large queue, decided right after
    const bool large = narrow && st.wrow;
    if (large) {
        cudaMemsetAsync(fs.q[NFBQ].count, 0, 2 * sizeof(int32_t), s);   // count, next
        cudaMemsetAsync(fs.q[NFBQ].done, 0, sizeof(int32_t) * (size_t)fs.q[NFBQ].cap, s);
    }
#define LV_GROUP(G, CAP)                                                                              \
    do {                                                                                              \
        if (narrow)                                                                                   \
            move_group_narrow_kernel<G, CAP, WT><<<nblocks(n, 256 / G), 256, 0, s>>>(g, st, list, n, dE, \
                                                                                    fs.q[NFBQ]);     \
        else move_group_kernel<G, CAP, WT><<<nblocks(n, 256 / G), 256, 0, s>>>(g, st, list, n, dE);   \
        note_launches(1);                                                                             \
    } while (0)
    switch (cls) {
    case CLS_B0: LV_GROUP(4, 8); break;
    case CLS_B1: LV_GROUP(8, 16); break;
    case CLS_B2: LV_GROUP(16, 32); break;
    case CLS_B3: LV_GROUP(32, 64); break;
    default: break;
    }
#undef LV_GROUP
    if (large) launch_fallback_large<WT>(g, st, HubGlobal(), fs, di, dE, s);
}

template <typename WT>
static void launch_fallback_large(const GraphView<WT> &g, const StateView &st, const HubGlobal &hg,
                                  const FallbackSet &fs, const DeviceInfo &di, u64 *dE, cudaStream_t s) {
    move_fallback_kernel<WT, FB_THREADS, FB_CAP, true><<<di.sms, FB_THREADS, FB_SMEM, s>>>(
        g, st, fs.q[NFBQ], hg, fs.hint, fs.hint_set, dE);
    note_launches(1);
}

template <typename WT>
void launch_move_giants(const GraphView<WT> &g, const StateView &st, const HubGlobal &hg,
                        const FallbackSet &fs, const DeviceInfo &di, u64 *dE, cudaStream_t s, bool narrow) {
    if (hg.nhubs <= 0) return;
    cudaMemsetAsync(fs.q[NFBQ].count, 0, 2 * sizeof(int32_t), s);   // count, next
    // The staging counters, the own-community sums and the partition done
    // counters are returned to zero by the kernel that consumes them; they are
    // cleared here as well, so that a sweep that ended early (a device error,
    // an item the full large queue could not take) cannot leave a count that
    // makes the next staging pass append beyond a giant's area.
    cudaMemsetAsync(hg.nocc, 0, sizeof(int32_t) * (size_t)hg.nhubs, s);
    cudaMemsetAsync(hg.eown, 0, sizeof(u64) * (size_t)hg.nhubs, s);
    cudaMemsetAsync(fs.q[NFBQ].done, 0, sizeof(int32_t) * (size_t)fs.q[NFBQ].cap, s);
    if (narrow) {
        giant_stage_narrow_kernel<WT><<<(unsigned)imin64(hg.n_echunks, (int64_t)di.sms * di.occ_stage_narrow),
                                        STAGE_THREADS, STAGE_SMEM, s>>>(g, st, hg);
        note_launches(1);
        if (st.wrow) {
            giant_stage_kernel<WT><<<(unsigned)imin64(hg.n_echunks, (int64_t)di.sms * di.occ_stage), STAGE_THREADS,
                                     STAGE_SMEM, s>>>(g, st, hg, st.wrow);
            note_launches(1);
        }
    } else {
        giant_stage_kernel<WT><<<(unsigned)imin64(hg.n_echunks, (int64_t)di.sms * di.occ_stage), STAGE_THREADS,
                                 STAGE_SMEM, s>>>(g, st, hg, nullptr);
        note_launches(1);
    }
    if (LV_GIANT_REGROUP && hg.poff) {
        giant_regroup_kernel<<<hg.nhubs, REGROUP_THREADS, 0, s>>>(hg);
        note_launches(1);
    }
#if LV_MERGE_SMALL
    giant_merge_kernel<MERGE_S_THREADS, MERGE_S_CAP>
        <<<(unsigned)imin64(hg.nhubs, (int64_t)di.sms * di.occ_merge_s), MERGE_S_THREADS, MERGE_S_CAP * 14, s>>>(
            st, hg, fs.q[NFBQ], dE, -1);
    note_launches(1);
    const int32_t big_min = MERGE_S_CAP / 2;
#else
    const int32_t big_min = -1;
#endif
    giant_merge_kernel<HG_MERGE_THREADS, HG_MERGE_CAP>
        <<<(unsigned)imin64(hg.nhubs, di.sms), HG_MERGE_THREADS, HG_MERGE_SMEM, s>>>(st, hg, fs.q[NFBQ], dE,
                                                                                   big_min);
    note_launches(1);
    launch_fallback_large<WT>(g, st, hg, fs, di, dE, s);
}

template <typename WT>
void launch_move_wide(const GraphView<WT> &g, const StateView &st, const int32_t *list, int32_t n,
                      const FallbackSet &fs, const DeviceInfo &di, u64 *dE, cudaStream_t s,
                      int32_t max_degree, bool narrow) {
    if (n <= 0) return;
    // the queues' (count, next) pairs are contiguous; the large queue's done
    // counters are cleared as in launch_move_giants
    cudaMemsetAsync(fs.q[0].count, 0, (2 * (NFBQ + 1) + 1) * sizeof(int32_t), s);   // + the warp cursor
    if (max_degree > fs.warp_limit || (narrow && st.wrow))
        cudaMemsetAsync(fs.q[NFBQ].done, 0, sizeof(int32_t) * (size_t)fs.q[NFBQ].cap, s);
    if (narrow) {
        const unsigned grid = (unsigned)imin64((n + 7) / 8, (int64_t)di.sms * di.occ_warp_narrow);
        move_warp_narrow_kernel<WT><<<grid, 256, WARP_NSMEM, s>>>(g, st, list, n, fs, dE);
    } else {
        const unsigned grid = (unsigned)imin64((n + 7) / 8, (int64_t)di.sms * di.occ_warp);
        move_warp_kernel<WT><<<grid, 256, WARP_SMEM, s>>>(g, st, list, n, fs, dE);
    }
    note_launches(1);
    if (max_degree <= fs.warp_limit) {   // no vertex can overflow its warp table
        if (narrow && st.wrow) launch_fallback_large<WT>(g, st, HubGlobal(), fs, di, dE, s);
        return;
    }
    launch_fallback_large<WT>(g, st, HubGlobal(), fs, di, dE, s);
    launch_row_queue<WT, 3>(g, st, fs, di, dE, s, narrow);
    launch_row_queue<WT, 2>(g, st, fs, di, dE, s, narrow);
    launch_row_queue<WT, 1>(g, st, fs, di, dE, s, narrow);
    launch_row_queue<WT, 0>(g, st, fs, di, dE, s, narrow);
}

template <typename WT>
void launch_correction(int cls, const GraphView<WT> &g, const StateView &st, const int32_t *list,
                       int32_t n, const DeviceInfo &di, u64 *dE, cudaStream_t s) {
    if (n <= 0) return;
    switch (cls) {
    case CLS_B0: corr_group_kernel<4, WT><<<nblocks(n, 64), 256, 0, s>>>(g, st.comm, st.newc, list, n, dE); break;
    case CLS_B1: corr_group_kernel<8, WT><<<nblocks(n, 32), 256, 0, s>>>(g, st.comm, st.newc, list, n, dE); break;
    case CLS_B2: corr_group_kernel<16, WT><<<nblocks(n, 16), 256, 0, s>>>(g, st.comm, st.newc, list, n, dE); break;
    case CLS_B3:
    case CLS_B4: corr_group_kernel<32, WT><<<nblocks(n, 8), 256, 0, s>>>(g, st.comm, st.newc, list, n, dE); break;
    case CLS_B5:
        corr_cta_kernel<128, WT><<<(unsigned)imin64(nblocks(n, CORR_BATCH), (int64_t)di.sms * 16), 128, 0, s>>>(g, st.comm, st.newc, list, n, dE);
        break;
    case CLS_H1:
        corr_cta_kernel<256, WT><<<(unsigned)imin64(nblocks(n, CORR_BATCH), (int64_t)di.sms * 8), 256, 0, s>>>(g, st.comm, st.newc, list, n, dE);
        break;
    default:
        corr_cta_kernel<512, WT><<<(unsigned)imin64(nblocks(n, CORR_BATCH), (int64_t)di.sms * 4), 512, 0, s>>>(g, st.comm, st.newc, list, n, dE);
        break;
    }
    note_launches(1);
}

void launch_commit(const StateView &st, const int32_t *list, int32_t n, u64 *moves, cudaStream_t s) {
    if (n <= 0) return;
    commit_kernel<<<nblocks(n, 256), 256, 0, s>>>(st, list, n, moves); note_launches(1);
}

template <typename WT>
void launch_row_reduce(int cls, int mode, const GraphView<WT> &g, const int32_t *comm, u64 *k,
                       u64 *total, const int32_t *list, int32_t n, const DeviceInfo &di,
                       cudaStream_t s) {
    if (n <= 0) return;
#define LV_RR(G)                                                                             \
    do {                                                                                     \
        if (mode == 0)                                                                       \
            row_reduce_group_kernel<G, 0, WT><<<nblocks(n, 256 / G), 256, 0, s>>>(g, comm, k, total, list, n); \
        else                                                                                 \
            row_reduce_group_kernel<G, 1, WT><<<nblocks(n, 256 / G), 256, 0, s>>>(g, comm, k, total, list, n); \
        note_launches(1);                                                                    \
    } while (0)
#define LV_RRC(T)                                                                            \
    do {                                                                                     \
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * (2048 / T));            \
        if (mode == 0)                                                                       \
            row_reduce_cta_kernel<T, 0, WT><<<grid, T, 0, s>>>(g, comm, k, total, list, n);  \
        else                                                                                 \
            row_reduce_cta_kernel<T, 1, WT><<<grid, T, 0, s>>>(g, comm, k, total, list, n);  \
        note_launches(1);                                                                    \
    } while (0)
    switch (cls) {
    case CLS_B0: LV_RR(4); break;
    case CLS_B1: LV_RR(8); break;
    case CLS_B2: LV_RR(16); break;
    case CLS_B3:
    case CLS_B4: LV_RR(32); break;
    case CLS_B5: LV_RRC(128); break;
    case CLS_H1: LV_RRC(256); break;
    default: LV_RRC(512); break;
    }
#undef LV_RR
#undef LV_RRC
}

void launch_s2(const u64 *S, int32_t V, u64 *total_hi_lo, cudaStream_t s) {
    if (V <= 0) return;
    unsigned grid = (unsigned)imin64(nblocks(V, 256), 148 * 8);
    s2_kernel<<<grid, 256, 0, s>>>(S, V, total_hi_lo); note_launches(1);
}

template void launch_move_class<float>(int, const GraphView<float> &, const StateView &,
                                       const int32_t *, int32_t, const DeviceInfo &, u64 *,
                                       cudaStream_t, bool, const FallbackSet &);
template void launch_move_class<u64>(int, const GraphView<u64> &, const StateView &,
                                     const int32_t *, int32_t, const DeviceInfo &, u64 *,
                                     cudaStream_t, bool, const FallbackSet &);
template void launch_move_wide<float>(const GraphView<float> &, const StateView &, const int32_t *,
                                      int32_t, const FallbackSet &, const DeviceInfo &, u64 *,
                                      cudaStream_t, int32_t, bool);
template void launch_move_wide<u64>(const GraphView<u64> &, const StateView &, const int32_t *,
                                    int32_t, const FallbackSet &, const DeviceInfo &, u64 *,
                                    cudaStream_t, int32_t, bool);
template void launch_move_giants<float>(const GraphView<float> &, const StateView &,
                                        const HubGlobal &, const FallbackSet &, const DeviceInfo &,
                                        u64 *, cudaStream_t, bool);
template void launch_move_giants<u64>(const GraphView<u64> &, const StateView &, const HubGlobal &,
                                      const FallbackSet &, const DeviceInfo &, u64 *, cudaStream_t, bool);
template void launch_correction<float>(int, const GraphView<float> &, const StateView &,
                                       const int32_t *, int32_t, const DeviceInfo &, u64 *,
                                       cudaStream_t);
template void launch_correction<u64>(int, const GraphView<u64> &, const StateView &,
                                     const int32_t *, int32_t, const DeviceInfo &, u64 *,
                                     cudaStream_t);
template void launch_row_reduce<float>(int, int, const GraphView<float> &, const int32_t *, u64 *,
                                       u64 *, const int32_t *, int32_t, const DeviceInfo &,
                                       cudaStream_t);
template void launch_row_reduce<u64>(int, int, const GraphView<u64> &, const int32_t *, u64 *,
                                     u64 *, const int32_t *, int32_t, const DeviceInfo &,
                                     cudaStream_t);

template void launch_move_class<uint32_t>(int, const GraphView<uint32_t> &, const StateView &,
                                     const int32_t *, int32_t, const DeviceInfo &, u64 *,
                                     cudaStream_t, bool, const FallbackSet &);
template void launch_move_wide<uint32_t>(const GraphView<uint32_t> &, const StateView &, const int32_t *,
                                    int32_t, const FallbackSet &, const DeviceInfo &, u64 *,
                                    cudaStream_t, int32_t, bool);
template void launch_move_giants<uint32_t>(const GraphView<uint32_t> &, const StateView &, const HubGlobal &,
                                      const FallbackSet &, const DeviceInfo &, u64 *, cudaStream_t, bool);
template void launch_correction<uint32_t>(int, const GraphView<uint32_t> &, const StateView &,
                                     const int32_t *, int32_t, const DeviceInfo &, u64 *,
                                     cudaStream_t);
template void launch_row_reduce<uint32_t>(int, int, const GraphView<uint32_t> &, const int32_t *, u64 *,
                                     u64 *, const int32_t *, int32_t, const DeviceInfo &,
                                     cudaStream_t);

}  // namespace lv
