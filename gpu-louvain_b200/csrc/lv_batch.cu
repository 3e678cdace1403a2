// lv_batch.cu -- many independent graphs in one persistent launch
// (lv_batch_create / lv_batch_run).
//
// Every graph of a batch goes through the level loop of gpulouvain.cu:30-37
// with the rule of lv_run: sweeps of the seven degree-bucket sub-rounds
// (modularity_optimisation.cu:284-363) with exact gains, the sweep loop's stop
// rule, exact aggregation (community_aggregation.cu:248-347) and the final
// modularity.  A graph's partition, modularity, level and sweep counts are
// therefore what lv_create + lv_run (and the CPU oracle) give for that graph
// alone.
//
// Execution.  One CTA runs one graph from start to finish; CTAs take graphs
// from a device queue ordered by decreasing entry count, so one launch covers
// the whole batch and the large graphs start first.  A graph's state lives in
// slices of batch-wide arrays at the graph's own vertex and entry offsets, and
// the steps of the level loop are separated by CTA barriers instead of kernel
// launches and host round trips.  Vertex ids stay global at every level: the
// level-L vertices of a graph whose first vertex is v0 are v0 .. v0 + V_L - 1.
//
// Tables.  A vertex of degree <= DW (or a merged row of at most DW entries)
// is handled by a lane group or a warp with a table in shared memory; a larger
// one by the whole CTA, with the CTA's shared table when 2 * min(degree, V)
// slots fit, else with the graph's own global table of 2^ceil(log2(2 V0))
// slots.  Every table is empty between uses.
//
// Coherence.  Rows of aggregated levels and the community state are written
// inside the launch, so they are read with ordinary (coherent) loads; only the
// caller's level-0 CSR goes through the read-only cache.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/louvain_b200.h"
#include "lv_internal.h"

namespace lv {
namespace {

// 512 threads and 2 CTAs per SM (64 registers): 16 warps per graph shorten
// the largest graphs' latency, which bounds the launch, and 32 resident warps
// per SM raise throughput; measured against 256 x 3 (80 registers) on the
// 4096-graph batch: 469 ms vs 713 ms per launch.
#ifndef LV_BATCH_THREADS
#define LV_BATCH_THREADS 512
#endif
#ifndef LV_BATCH_MINB
#define LV_BATCH_MINB 2
#endif
constexpr int BT = LV_BATCH_THREADS;   // threads per CTA
constexpr int BW = BT / 32;            // warps per CTA
constexpr int WTAB = 256;           // slots of one warp's table
constexpr int DW = WTAB / 2;        // degree / merged-row bound served by a warp table
constexpr int CTAB = BW * WTAB;     // slots of the CTA table (the warp tables together)
// Iteration caps that keep a launch bounded; a graph that reaches one stops
// with LV_ERR_DEVICE (the rule itself has no cap: with min_gain <= 0 a sweep
// loop that keeps moving at zero gain would not end).
constexpr int SWEEP_CAP = 4096;
constexpr int LEVEL_CAP = 256;

struct BatchParams {
    // the caller's block-diagonal CSR (read-only during the launch)
    const int32_t *rowptr;
    const int32_t *col;
    const float *w;
    const int32_t *gptr;       // [G + 1] first vertex of each graph
    const int32_t *order;      // [G] graphs by decreasing entry count
    const int64_t *tbl_off;    // [G + 1] first slot of each graph's global table
    int32_t G;
    int32_t max_sweeps;
    double min_gain;
    // per vertex (V entries; mstart / roff: V + G, the slice of graph g starts at v0 + g)
    int32_t *comm, *newc, *size, *blist, *newid, *members, *o2c, *mstart, *roff;
    int32_t *rs[2], *re[2];    // aggregated levels: row v = [rs[v], re[v])
    u64 *k, *S;
    // per entry (E entries): aggregated rows, ping-pong
    int32_t *colb[2];
    u64 *wb[2];
    int32_t *tkeys;            // global tables (-1 / 0 between uses)
    u64 *tvals;
    int32_t *next;             // queue head
    // results
    int32_t *out_comm;         // [V] community of each vertex, numbered within its graph
    double *q;
    int32_t *nc, *status, *levels;
    int64_t *sweeps, *edge_sweeps, *vertex_sweeps, *moves;
    u64 *t_start, *t_end;      // %globaltimer (ns) around each graph
};

struct BatchSmem {
    u64 vals[CTAB];
    int32_t keys[CTAB];
    u64 red[2 * BW];
    double bgd[BW];
    u64 be[BW], bS[BW], beo[BW];
    int32_t bc[BW];
    int32_t scan[BW];
    int32_t bcnt[16], boff[16], bcur[16];   // bucket b: [2b] degree <= DW, [2b + 1] larger
    int32_t gi, err, nbig, cnt;
};

// A graph's current level and totals (the same in every thread of the CTA).
struct GState {
    int32_t g, v0, V0, V;
    int64_t e0;     // first entry of the graph in the caller's CSR
    int64_t E;      // entries of the current level
    int64_t tbl;    // first slot of the graph's global table
    u64 T;
    double scale;
    int cur;        // -1: level 0 (the caller's CSR), else the buffer of the level's rows
};

struct Acc {
    int status;
    int32_t levels;
    int64_t sweeps, edge_sweeps, vertex_sweeps, moves;
    double q;
};

// Level views: row bounds, column and fixed-point weight of an entry.
template <typename WT>
struct Lv;
template <>
struct Lv<float> {
    const int32_t *rp;
    const int32_t *col;
    const float *w;
    double scale;
    __device__ __forceinline__ int32_t r0(int32_t v) const { return __ldg(rp + v); }
    __device__ __forceinline__ int32_t r1(int32_t v) const { return __ldg(rp + v + 1); }
    __device__ __forceinline__ int32_t c(int64_t e) const { return __ldg(col + e); }
    __device__ __forceinline__ u64 x(int64_t e) const { return wfix(w, e, scale); }
};
template <>
struct Lv<u64> {
    const int32_t *rs;
    const int32_t *re;
    const int32_t *col;
    const u64 *w;
    __device__ __forceinline__ int32_t r0(int32_t v) const { return rs[v]; }
    __device__ __forceinline__ int32_t r1(int32_t v) const { return re[v]; }
    __device__ __forceinline__ int32_t c(int64_t e) const { return col[e]; }
    __device__ __forceinline__ u64 x(int64_t e) const { return w[e]; }
};

// Update-order bucket of a degree (modularity_optimisation.cuh:7-8).
__device__ __forceinline__ int bucket_of(int32_t d) {
    if (d <= 0) return -1;
    if (d <= 4) return 0;
    if (d <= 8) return 1;
    if (d <= 16) return 2;
    if (d <= 32) return 3;
    if (d <= 84) return 4;
    if (d <= 319) return 5;
    return 6;
}

__device__ __forceinline__ u64 globaltimer() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int table_lg(int32_t bound) {
    const int lg = ceil_log2_i(2 * (int64_t)bound);
    return lg < 1 ? 1 : lg;
}

// ---- CTA-wide reductions and scan (every thread gets the result) ----
__device__ __forceinline__ u64 block_sum_u64(u64 x, BatchSmem &sm) {
    x = warp_sum_u64(x);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = x;
    __syncthreads();
    u64 t = 0;
    for (int i = 0; i < BW; ++i) t += sm.red[i];
    return t;
}

__device__ __forceinline__ u128 block_sum_u128(u128 x, BatchSmem &sm) {
    x = warp_sum_u128(x);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        sm.red[2 * (threadIdx.x >> 5)] = (u64)(x >> 64);
        sm.red[2 * (threadIdx.x >> 5) + 1] = (u64)x;
    }
    __syncthreads();
    u128 t = 0;
    for (int i = 0; i < BW; ++i) t += ((u128)sm.red[2 * i] << 64) | (u128)sm.red[2 * i + 1];
    return t;
}

__device__ __forceinline__ int block_max_i32(int x, BatchSmem &sm) {
    for (int off = 16; off > 0; off >>= 1) x = max(x, __shfl_xor_sync(FULL, x, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sm.scan[threadIdx.x >> 5] = x;
    __syncthreads();
    int t = sm.scan[0];
    for (int i = 1; i < BW; ++i) t = max(t, sm.scan[i]);
    return t;
}

// Exclusive scan of get(0 .. n-1); put(i, prefix, value) for each i; returns
// the total.  Each index is read and written by the same thread.
template <class Get, class Put>
__device__ int32_t block_scan(int32_t n, Get get, Put put, BatchSmem &sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t carry = 0;
    for (int32_t base = 0; base < n; base += BT) {
        const int32_t i = base + threadIdx.x;
        const int32_t x = i < n ? get(i) : 0;
        int32_t inc = x;
        for (int off = 1; off < 32; off <<= 1) {
            const int32_t y = __shfl_up_sync(FULL, inc, off);
            if (lane >= off) inc += y;
        }
        __syncthreads();
        if (lane == 31) sm.scan[warp] = inc;
        __syncthreads();
        int32_t pre = 0, tot = 0;
        for (int j = 0; j < BW; ++j) {
            const int32_t t = sm.scan[j];
            pre += j < warp ? t : 0;
            tot += t;
        }
        if (i < n) put(i, carry + pre + inc - x, x);
        carry += tot;
    }
    __syncthreads();
    return carry;
}

// ---- move phase ----
// Vertices of one bucket with degree <= 2^(LG-1): a group of W lanes per
// vertex (32/W vertices per warp at a time) and a table of 2^LG slots per
// group inside the warp's table.  U entries per lane are in flight at a
// time (U column loads, then U community gathers), and the next vertex's
// row bounds and community are loaded while the current one is evaluated.
template <typename WT, int W, int LG, int U>
__device__ void decide_groups(const Lv<WT> &L, const BatchParams &P, const GState &gs,
                              const int32_t *list, int32_t n, BatchSmem &sm) {
    constexpr int GPW = 32 / W;
    constexpr int NSLOT = 1 << LG;
    constexpr int EU = (NSLOT / W) < 4 ? (NSLOT / W) : 4;   // table slots per lane in flight
    constexpr int32_t STRIDE = BW * GPW;
    static_assert(GPW * NSLOT <= WTAB, "group tables fit the warp's table");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane / W, gl = lane % W;
    int32_t *keys = sm.keys + warp * WTAB + grp * NSLOT;
    u64 *vals = sm.vals + warp * WTAB + grp * NSLOT;
    int32_t i = warp * GPW + grp;
    int32_t v = -1, own = -1, r0 = 0, r1 = 0;
    u64 kv = 0;
    if (i < n) {
        v = list[i];
        r0 = L.r0(v);
        r1 = L.r1(v);
        own = P.comm[v];
        kv = P.k[v];
    }
    for (int32_t i0 = warp * GPW; i0 < n; i0 += STRIDE) {
        const int32_t inext = i + STRIDE;
        const int32_t vnext = inext < n ? list[inext] : -1;
        u64 sown = 0;
        bool single = false;
        if (v >= 0) {
            sown = P.S[own];
            single = P.size[own] == 1;
        }
        u64 eo = 0;
        for (int32_t base = r0 + gl; base < r1; base += U * W) {
            int32_t jj[U];
            u64 xx[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t e = base + u * W;
                jj[u] = -1;
                xx[u] = 0;
                if (e < r1) {
                    jj[u] = L.c(e);
                    xx[u] = L.x(e);
                }
            }
            int32_t cc[U];
#pragma unroll
            for (int u = 0; u < U; ++u) cc[u] = (jj[u] >= 0 && jj[u] != v) ? P.comm[jj[u]] : -1;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (cc[u] < 0) continue;
                if (cc[u] == own) eo += xx[u];
                else table_insert<0>(keys, vals, LG, cc[u], xx[u], &sm.err);
            }
        }
        // the next vertex's row bounds, community and weight (its id has arrived)
        int32_t nr0 = 0, nr1 = 0, nown = -1;
        u64 nkv = 0;
        if (vnext >= 0) {
            nr0 = L.r0(vnext);
            nr1 = L.r1(vnext);
            nown = P.comm[vnext];
            nkv = P.k[vnext];
        }
        __syncwarp();
        const MoveCtx m = move_ctx(own, single, gs.T, kv, sown);
        Best b = best_init(own);
        b.eo = eo;
        for (int s0 = gl; s0 < NSLOT; s0 += EU * W) {
            int32_t cc[EU];
            u64 ee[EU];
#pragma unroll
            for (int u = 0; u < EU; ++u) {
                const int s = s0 + u * W;
                cc[u] = keys[s];
                ee[u] = 0;
                if (cc[u] >= 0) {
                    ee[u] = vals[s];
                    keys[s] = -1;
                    vals[s] = 0;
                }
            }
            u64 SS[EU];
            int32_t zz[EU];
#pragma unroll
            for (int u = 0; u < EU; ++u) {
                SS[u] = cc[u] >= 0 ? P.S[cc[u]] : 0;
                zz[u] = (cc[u] >= 0 && guard_needs_size(m, cc[u])) ? P.size[cc[u]] : 0;
            }
#pragma unroll
            for (int u = 0; u < EU; ++u)
                if (cc[u] >= 0) eval_loaded(cc[u], ee[u], SS[u], zz[u], m, b);
        }
        __syncwarp();
        group_reduce_best(m, b, W);
        if (v >= 0 && gl == 0) {
            u64 d;
            P.newc[v] = move_decision(m, b, &d);
        }
        i = inext;
        v = vnext;
        r0 = nr0;
        r1 = nr1;
        own = nown;
        kv = nkv;
    }
}

// One vertex of degree > DW by the whole CTA.
template <typename WT>
__device__ void decide_cta(const Lv<WT> &L, const BatchParams &P, const GState &gs, int32_t v,
                           BatchSmem &sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t r0 = L.r0(v), r1 = L.r1(v);
    const int32_t own = P.comm[v];
    const u64 kv = P.k[v], sown = P.S[own];
    const bool single = P.size[own] == 1;
    const int lg = table_lg(min(r1 - r0, gs.V));
    int32_t *keys = sm.keys;
    u64 *vals = sm.vals;
    if ((1 << lg) > CTAB) {
        keys = P.tkeys + gs.tbl;
        vals = P.tvals + gs.tbl;
    }
    u64 eo = 0;
    for (int32_t e = r0 + threadIdx.x; e < r1; e += BT) {
        const int32_t j = L.c(e);
        if (j == v) continue;
        const u64 x = L.x(e);
        const int32_t c = P.comm[j];
        if (c == own) eo += x;
        else table_insert<0>(keys, vals, lg, c, x, &sm.err);
    }
    __syncthreads();
    const MoveCtx m = move_ctx(own, single, gs.T, kv, sown);
    Best b = best_init(own);
    b.eo = eo;
    for (int32_t s = threadIdx.x; s < (1 << lg); s += BT) {
        const int32_t c = keys[s];
        if (c < 0) continue;
        const u64 ec = vals[s];
        keys[s] = -1;
        vals[s] = 0;
        eval_loaded(c, ec, P.S[c], guard_needs_size(m, c) ? P.size[c] : 0, m, b);
    }
    group_reduce_best(m, b, 32);
    if (lane == 0) {
        sm.bgd[warp] = b.gd;
        sm.be[warp] = b.e;
        sm.bS[warp] = b.S;
        sm.bc[warp] = b.c;
        sm.beo[warp] = b.eo;
    }
    __syncthreads();
    if (warp == 0) {
        Best x = best_init(own);
        if (lane < BW) {
            x.gd = sm.bgd[lane];
            x.e = sm.be[lane];
            x.S = sm.bS[lane];
            x.c = sm.bc[lane];
            x.eo = sm.beo[lane];
        }
        group_reduce_best(m, x, 32);
        if (lane == 0) {
            u64 d;
            P.newc[v] = move_decision(m, x, &d);
        }
    }
    __syncthreads();
}

// Exact change of sum_i e_{i->C(i)} when one sub-round's decisions commit.
// For a mover v (o -> n) and a neighbour x != v the pair's term changes by
// w ([n == C'(x)] - [o == C(x)]): counted twice from v's row when x stays
// (the entry in x's row is not visited), once from each row when x moves
// too.  Between sub-rounds newc == comm, so newc[x] != comm[x] marks a mover
// of this sub-round.  Lane groups of 8 per vertex; wrapping uint64 sum.
template <typename WT>
__device__ __forceinline__ u64 commit_delta(const Lv<WT> &L, const BatchParams &P, const int32_t *list,
                                            int32_t n) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 d = 0;
    for (int32_t i0 = warp * 4; i0 < n; i0 += BW * 4) {
        const int32_t i = i0 + (lane >> 3);
        if (i >= n) continue;
        const int32_t v = list[i];
        const int32_t nv = P.newc[v], ov = P.comm[v];
        if (nv == ov) continue;
        const int32_t r1 = L.r1(v);
        for (int32_t e = L.r0(v) + (lane & 7); e < r1; e += 8) {
            const int32_t x = L.c(e);
            if (x == v) continue;
            const u64 w = L.x(e);
            const int32_t cx = P.comm[x], nx = P.newc[x];
            if (nx != cx) {
                if (nv == nx) d += w;
                if (ov == cx) d -= w;
            } else {
                if (nv == cx) d += 2 * w;
                if (ov == cx) d -= 2 * w;
            }
        }
    }
    return d;
}

// updateVertexCommunity (modularity_optimisation.cu:237-249) for one
// sub-round's vertices, with exact Sigma_tot and size updates.
__device__ __forceinline__ int32_t commit_list(const BatchParams &P, const int32_t *list, int32_t n) {
    int32_t moved = 0;
    for (int32_t i = threadIdx.x; i < n; i += BT) {
        const int32_t v = list[i];
        const int32_t nc = P.newc[v], oc = P.comm[v];
        if (nc == oc) continue;
        P.comm[v] = nc;
        atomicSub(P.size + oc, 1);
        atomicAdd(P.size + nc, 1);
        const u64 kv = P.k[v];
        atomicAdd(P.S + oc, (u64)0 - kv);
        atomicAdd(P.S + nc, kv);
        ++moved;
    }
    return moved;
}

// One sweep: the seven sub-rounds, each deciding against the state committed
// before it.  Returns the number of moves; *de receives the exact change of
// sum_i e_{i->C(i)}.
template <typename WT>
__device__ int64_t sweep(const Lv<WT> &L, const BatchParams &P, const GState &gs, BatchSmem &sm, u64 *de) {
    int32_t moved = 0;
    u64 d = 0;
    const int32_t *bl = P.blist + gs.v0;
    for (int b = 0; b < NBUCKETS; ++b) {
        const int32_t o = sm.boff[2 * b], ns = sm.bcnt[2 * b], nb = sm.bcnt[2 * b + 1];
        if (ns + nb == 0) continue;
        switch (b) {
        case 0: decide_groups<WT, 4, 3, 1>(L, P, gs, bl + o, ns, sm); break;
        case 1: decide_groups<WT, 4, 4, 2>(L, P, gs, bl + o, ns, sm); break;
        case 2: decide_groups<WT, 8, 5, 2>(L, P, gs, bl + o, ns, sm); break;
        case 3: decide_groups<WT, 8, 6, 4>(L, P, gs, bl + o, ns, sm); break;
        default: decide_groups<WT, 32, 8, 4>(L, P, gs, bl + o, ns, sm); break;
        }
        if (nb) {
            __syncthreads();
            for (int32_t i = 0; i < nb; ++i) decide_cta(L, P, gs, bl[o + ns + i], sm);
        }
        __syncthreads();
        d += commit_delta(L, P, bl + o, ns + nb);
        __syncthreads();
        moved += commit_list(P, bl + o, ns + nb);
        __syncthreads();
    }
    *de = block_sum_u64(d, sm);
    return (int64_t)block_sum_u64((u64)moved, sm);
}

// sum_i e_{i->C(i)} over whole rows, self-loops included
// (calculateToOwnCommunity, modularity_optimisation.cu:365-393).
template <typename WT>
__device__ u64 own_weight(const Lv<WT> &L, const BatchParams &P, const GState &gs, BatchSmem &sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 eo = 0;
    for (int32_t i0 = warp * 4; i0 < gs.V; i0 += BW * 4) {
        const int32_t i = i0 + (lane >> 3);
        if (i >= gs.V) continue;
        const int32_t v = gs.v0 + i;
        const int32_t cv = P.comm[v];
        const int32_t r1 = L.r1(v);
        for (int32_t e = L.r0(v) + (lane & 7); e < r1; e += 8)
            if (P.comm[L.c(e)] == cv) eo += L.x(e);
    }
    return block_sum_u64(eo, sm);
}

// calculateModularity (modularity_optimisation.cu:395-401) from the exact
// sum_i e_{i->C(i)} and a pass over Sigma_tot.
__device__ double modularity_from(u64 e_own, const BatchParams &P, const GState &gs, BatchSmem &sm) {
    u128 s2 = 0;
    for (int32_t i = threadIdx.x; i < gs.V; i += BT) {
        const u64 s = P.S[gs.v0 + i];
        s2 += (u128)s * (u128)s;
    }
    const u128 ts = block_sum_u128(s2, sm);
    return q_from_parts_dev(gs.T, e_own, (u64)(ts >> 64), (u64)ts);
}

// Level set-up: k_i (level 0; aggregation writes it for later levels),
// singleton communities, Sigma_tot = k, and the bucket lists.
template <typename WT>
__device__ void level_setup(const Lv<WT> &L, const BatchParams &P, GState &gs, BatchSmem &sm,
                            bool level0) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t v0 = gs.v0, V = gs.V;
    if (level0) {
        u64 tot = 0;
        for (int32_t i0 = warp * 4; i0 < V; i0 += BW * 4) {
            const int32_t i = i0 + (lane >> 3);
            u64 s = 0;
            if (i < V) {
                const int32_t r1 = L.r1(v0 + i);
                for (int32_t e = L.r0(v0 + i) + (lane & 7); e < r1; e += 8) s += L.x(e);
            }
            for (int off = 4; off > 0; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
            if (i < V && (lane & 7) == 0) {
                P.k[v0 + i] = s;
                tot += s;
            }
        }
        gs.T = block_sum_u64(tot, sm);
    }
    for (int32_t i = threadIdx.x; i < V; i += BT) {
        const int32_t v = v0 + i;
        P.comm[v] = v;
        P.newc[v] = v;
        P.size[v] = 1;
        P.S[v] = P.k[v];
    }
    if (threadIdx.x < 16) sm.bcnt[threadIdx.x] = 0;
    __syncthreads();
    for (int32_t i = threadIdx.x; i < V; i += BT) {
        const int32_t d = L.r1(v0 + i) - L.r0(v0 + i);
        const int b = bucket_of(d);
        if (b >= 0) atomicAdd(&sm.bcnt[2 * b + (d > DW ? 1 : 0)], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t o = 0;
        for (int j = 0; j < 2 * NBUCKETS; ++j) {
            sm.boff[j] = o;
            sm.bcur[j] = o;
            o += sm.bcnt[j];
        }
    }
    __syncthreads();
    for (int32_t i = threadIdx.x; i < V; i += BT) {
        const int32_t d = L.r1(v0 + i) - L.r0(v0 + i);
        const int b = bucket_of(d);
        if (b >= 0) P.blist[v0 + atomicAdd(&sm.bcur[2 * b + (d > DW ? 1 : 0)], 1)] = v0 + i;
    }
    __syncthreads();
}

// optimiseModularity (modularity_optimisation.cu:284-363): sweeps while the
// sweep's gain >= min_gain (the first always runs), stopping after a sweep
// without moves; changed = some sweep gained (> 0).  Then
// originalToCommunity <- C(originalToCommunity) (:251-257, :361).
template <typename WT>
__device__ int optimise_level(const Lv<WT> &L, const BatchParams &P, const GState &gs, BatchSmem &sm,
                              Acc &acc) {
    u64 e_own = own_weight(L, P, gs, sm);
    double q_before = modularity_from(e_own, P, gs, sm);
    double gain = P.min_gain;
    int changed = 0, sw = 0;
    while (gain >= P.min_gain) {
        if (P.max_sweeps > 0 && sw >= P.max_sweeps) break;
        if (sw >= SWEEP_CAP) {
            acc.status = LV_ERR_DEVICE;
            break;
        }
        u64 de = 0;
        const int64_t moves = sweep(L, P, gs, sm, &de);
        ++sw;
        acc.moves += moves;
        if (sm.err) {
            acc.status = LV_ERR_DEVICE;
            break;
        }
        e_own += de;
        const double q_after = modularity_from(e_own, P, gs, sm);
        gain = __dsub_rn(q_after, q_before);
        if (gain > 0) changed = 1;
        q_before = q_after;
        if (moves == 0) break;
    }
    acc.sweeps += sw;
    acc.edge_sweeps += (int64_t)sw * gs.E;
    acc.vertex_sweeps += (int64_t)sw * gs.V;
    acc.q = q_before;
    for (int32_t u = threadIdx.x; u < gs.V0; u += BT) {
        const int32_t x = P.o2c[gs.v0 + u];
        P.o2c[gs.v0 + u] = P.comm[x];
    }
    __syncthreads();
    return changed;
}

// aggregateCommunities (community_aggregation.cu:248-347): nonempty
// communities renumbered in ascending old id; each new vertex's row is the sum
// of its members' rows keyed by the neighbours' new ids (intra-community
// entries become one self-loop); new k = row sum; originalToCommunity <-
// newID (:222-228).  Rows are written at the offset of their bound (the sum of
// the members' degrees) inside the graph's entry range and stay there.
template <typename WT>
__device__ void aggregate(const Lv<WT> &L, const BatchParams &P, GState &gs, BatchSmem &sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nb = gs.cur < 0 ? 0 : 1 - gs.cur;
    const int32_t v0 = gs.v0, V = gs.V;
    int32_t *ms = P.mstart + v0 + gs.g;
    int32_t *ro = P.roff + v0 + gs.g;
    int32_t *nid = P.newid;
    const int32_t nv = block_scan(
        V, [&](int32_t i) { return P.size[v0 + i] > 0 ? 1 : 0; },
        [&](int32_t i, int32_t pre, int32_t x) { nid[v0 + i] = x ? pre : -1; }, sm);
    for (int32_t i = threadIdx.x; i <= nv; i += BT) {
        ms[i] = 0;
        ro[i] = 0;
    }
    __syncthreads();
    for (int32_t i = threadIdx.x; i < V; i += BT) {
        const int32_t v = v0 + i;
        const int32_t c = nid[P.comm[v]];
        atomicAdd(ms + c, 1);
        atomicAdd(ro + c, L.r1(v) - L.r0(v));
    }
    __syncthreads();
    block_scan(nv + 1, [&](int32_t i) { return ms[i]; }, [&](int32_t i, int32_t pre, int32_t) { ms[i] = pre; }, sm);
    block_scan(nv + 1, [&](int32_t i) { return ro[i]; }, [&](int32_t i, int32_t pre, int32_t) { ro[i] = pre; }, sm);
    for (int32_t i = threadIdx.x; i < nv; i += BT) P.newc[v0 + i] = ms[i];
    __syncthreads();
    for (int32_t i = threadIdx.x; i < V; i += BT) {
        const int32_t v = v0 + i;
        const int32_t pos = atomicAdd(P.newc + v0 + nid[P.comm[v]], 1);
        P.members[v0 + pos] = v;
    }
    if (threadIdx.x == 0) sm.nbig = 0;
    __syncthreads();

    int32_t *ocol = P.colb[nb];
    u64 *ow = P.wb[nb];
    int32_t *ors = P.rs[nb], *ore = P.re[nb];
    u64 enew = 0;
    // merged rows of bound <= DW: one warp each, table in the warp's slots
    for (int32_t c = warp; c < nv; c += BW) {
        const int32_t bound = ro[c + 1] - ro[c];
        if (bound > DW) {
            if (lane == 0) P.blist[v0 + atomicAdd(&sm.nbig, 1)] = c;
            continue;
        }
        const int lg = table_lg(min(bound, nv));
        int32_t *keys = sm.keys + warp * WTAB;
        u64 *vals = sm.vals + warp * WTAB;
        for (int32_t j = ms[c]; j < ms[c + 1]; ++j) {
            const int32_t m = P.members[v0 + j];
            const int32_t r1 = L.r1(m);
            for (int32_t e = L.r0(m) + lane; e < r1; e += 32)
                table_insert<1>(keys, vals, lg, nid[P.comm[L.c(e)]], L.x(e), &sm.err);
        }
        __syncwarp();
        const int64_t base = gs.e0 + ro[c];
        int32_t cnt = 0;
        u64 ks = 0;
        for (int s0 = 0; s0 < (1 << lg); s0 += 32) {
            const int s = s0 + lane;
            const int32_t key = s < (1 << lg) ? keys[s] : -1;
            const unsigned bal = __ballot_sync(FULL, key >= 0);
            if (key >= 0) {
                const int32_t pos = cnt + __popc(bal & ((1u << lane) - 1u));
                const u64 x = vals[s];
                if (pos < bound) {
                    ocol[base + pos] = v0 + key;
                    ow[base + pos] = x;
                } else {
                    atomicOr(&sm.err, DEVERR_BAD_STATE);
                }
                ks += x;
                keys[s] = -1;
                vals[s] = 0;
            }
            cnt += __popc(bal);
        }
        __syncwarp();
        ks = warp_sum_u64(ks);
        if (lane == 0) {
            ors[v0 + c] = (int32_t)base;
            ore[v0 + c] = (int32_t)(base + cnt);
            P.k[v0 + c] = ks;
            enew += (u64)cnt;
        }
    }
    __syncthreads();
    // larger merged rows: the whole CTA, one at a time
    const int32_t nbig = sm.nbig;
    for (int32_t t = 0; t < nbig; ++t) {
        const int32_t c = P.blist[v0 + t];
        const int32_t bound = ro[c + 1] - ro[c];
        const int lg = table_lg(min(bound, nv));
        int32_t *keys = sm.keys;
        u64 *vals = sm.vals;
        if ((1 << lg) > CTAB) {
            keys = P.tkeys + gs.tbl;
            vals = P.tvals + gs.tbl;
        }
        for (int32_t j = ms[c] + warp; j < ms[c + 1]; j += BW) {
            const int32_t m = P.members[v0 + j];
            const int32_t r1 = L.r1(m);
            for (int32_t e = L.r0(m) + lane; e < r1; e += 32)
                table_insert<1>(keys, vals, lg, nid[P.comm[L.c(e)]], L.x(e), &sm.err);
        }
        if (threadIdx.x == 0) sm.cnt = 0;
        __syncthreads();
        const int64_t base = gs.e0 + ro[c];
        u64 ks = 0;
        for (int32_t s0 = 0; s0 < (1 << lg); s0 += BT) {
            const int32_t s = s0 + threadIdx.x;
            const int32_t key = s < (1 << lg) ? keys[s] : -1;
            const unsigned bal = __ballot_sync(FULL, key >= 0);
            int32_t wbase = 0;
            if (lane == 0 && bal) wbase = atomicAdd(&sm.cnt, __popc(bal));
            wbase = __shfl_sync(FULL, wbase, 0);
            if (key >= 0) {
                const int32_t pos = wbase + __popc(bal & ((1u << lane) - 1u));
                const u64 x = vals[s];
                if (pos < bound) {
                    ocol[base + pos] = v0 + key;
                    ow[base + pos] = x;
                } else {
                    atomicOr(&sm.err, DEVERR_BAD_STATE);
                }
                ks += x;
                keys[s] = -1;
                vals[s] = 0;
            }
        }
        const u64 ktot = block_sum_u64(ks, sm);
        if (threadIdx.x == 0) {
            const int32_t cnt = sm.cnt;
            ors[v0 + c] = (int32_t)base;
            ore[v0 + c] = (int32_t)(base + cnt);
            P.k[v0 + c] = ktot;
            enew += (u64)cnt;
        }
        __syncthreads();
    }
    const u64 etot = block_sum_u64(enew, sm);
    for (int32_t u = threadIdx.x; u < gs.V0; u += BT) {
        const int32_t x = P.o2c[v0 + u];
        P.o2c[v0 + u] = v0 + nid[x];
    }
    gs.V = nv;
    gs.E = (int64_t)etot;
    gs.cur = nb;
    __syncthreads();
}

// The whole level loop of one graph (gpulouvain.cu:30-37).
__device__ void run_graph(const BatchParams &P, int32_t g, BatchSmem &sm) {
    GState gs;
    gs.g = g;
    gs.v0 = P.gptr[g];
    gs.V0 = P.gptr[g + 1] - gs.v0;
    gs.V = gs.V0;
    gs.e0 = __ldg(P.rowptr + gs.v0);
    gs.E = (int64_t)__ldg(P.rowptr + gs.v0 + gs.V0) - gs.e0;
    gs.tbl = P.tbl_off[g];
    gs.T = 0;
    gs.scale = 1.0;
    gs.cur = -1;
    if (threadIdx.x == 0) {
        sm.err = 0;
        P.t_start[g] = globaltimer();
    }
    for (int s = threadIdx.x; s < CTAB; s += BT) {
        sm.keys[s] = -1;
        sm.vals[s] = 0;
    }
    // column range of the graph and the fixed-point scale (orc_choose_scale)
    int need = 0, top = 0, bad = 0;
    for (int64_t e = gs.e0 + threadIdx.x; e < gs.e0 + gs.E; e += BT) {
        const int32_t j = __ldg(P.col + e);
        if (j < gs.v0 || j >= gs.v0 + gs.V0) bad = 1;
        int n, t, b;
        weight_bits_dev(__ldg(P.w + e), n, t, b);
        need = max(need, n);
        top = max(top, t);
        bad |= b;
    }
    need = block_max_i32(need, sm);
    top = block_max_i32(top, sm);
    bad = block_max_i32(bad, sm);
    Acc acc{};
    acc.status = LV_OK;
    acc.q = 0.0;
    if (bad) {
        acc.status = LV_ERR_INVALID;
    } else {
        const int tp = top ? top - 1024 : 0;
        const int cap = 61 - tp - ceil_log2_i(gs.E > 0 ? gs.E : 1);
        const int sc = need < cap ? need : cap;
        if (sc < 0) acc.status = LV_ERR_TOO_LARGE;
        else gs.scale = ldexp(1.0, sc);
    }
    if (acc.status == LV_OK) {
        for (int32_t u = threadIdx.x; u < gs.V0; u += BT) P.o2c[gs.v0 + u] = gs.v0 + u;
        const Lv<float> L0{P.rowptr, P.col, P.w, gs.scale};
        level_setup(L0, P, gs, sm, true);
        int changed = optimise_level(L0, P, gs, sm, acc);
        acc.levels = 1;
        if (changed && acc.status == LV_OK) aggregate(L0, P, gs, sm);
        while (changed && acc.status == LV_OK) {
            if (sm.err) {
                acc.status = LV_ERR_DEVICE;
                break;
            }
            if (acc.levels >= LEVEL_CAP) {
                acc.status = LV_ERR_DEVICE;
                break;
            }
            const Lv<u64> L{P.rs[gs.cur], P.re[gs.cur], P.colb[gs.cur], P.wb[gs.cur]};
            level_setup(L, P, gs, sm, false);
            changed = optimise_level(L, P, gs, sm, acc);
            acc.levels += 1;
            if (changed && acc.status == LV_OK) aggregate(L, P, gs, sm);
        }
    }
    if (acc.status != LV_OK) {
        // leave the graph's global table empty for the next run
        const int64_t n = P.tbl_off[g + 1] - gs.tbl;
        for (int64_t s = threadIdx.x; s < n; s += BT) {
            P.tkeys[gs.tbl + s] = -1;
            P.tvals[gs.tbl + s] = 0;
        }
    }
    for (int32_t u = threadIdx.x; u < gs.V0; u += BT)
        P.out_comm[gs.v0 + u] = acc.status == LV_OK ? P.o2c[gs.v0 + u] - gs.v0 : -1;
    if (threadIdx.x == 0) {
        P.q[g] = acc.q;
        P.nc[g] = acc.status == LV_OK ? gs.V : 0;
        P.status[g] = acc.status;
        P.levels[g] = acc.levels;
        P.sweeps[g] = acc.sweeps;
        P.edge_sweeps[g] = acc.edge_sweeps;
        P.vertex_sweeps[g] = acc.vertex_sweeps;
        P.moves[g] = acc.moves;
        P.t_end[g] = globaltimer();
    }
    __syncthreads();
}

__global__ void __launch_bounds__(BT, LV_BATCH_MINB) batch_kernel(const __grid_constant__ BatchParams P) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    BatchSmem &sm = *reinterpret_cast<BatchSmem *>(batch_smem);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) sm.gi = atomicAdd(P.next, 1);
        __syncthreads();
        const int32_t gi = sm.gi;
        if (gi >= P.G) break;
        run_graph(P, P.order[gi], sm);
    }
}

// first entry of each graph: out[g] = rowptr[gptr[g]]
__global__ void graph_entries_kernel(const int32_t *rowptr, const int32_t *gptr, int32_t G,
                                     int32_t *out) {
    for (int32_t g = blockIdx.x * 256 + threadIdx.x; g <= G; g += gridDim.x * 256)
        out[g] = rowptr[gptr[g]];
}

__global__ void fill_tables_kernel(int32_t *keys, u64 *vals, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        keys[i] = -1;
        vals[i] = 0;
    }
}

}  // namespace
}  // namespace lv

using namespace lv;

struct lv_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    lv_opts opts{};
    std::string err;
    int32_t G = 0, V = 0;
    int64_t E = 0;
    std::vector<int32_t> gptr_h;
    std::vector<int64_t> entries_h;   // [G] entries per graph
    bool owns_input = false;
    const int32_t *rowptr = nullptr, *col = nullptr;
    const float *w = nullptr;
    BatchParams P{};
    int64_t tbl_total = 0;
    std::vector<void *> allocs;
    int grid = 1;
    bool ran = false;
    bool tables_dirty = false;
    float last_ms = 0;
    int64_t last_edge_sweeps = 0, last_vertex_sweeps = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

int bfail(lv_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    return code;
}

template <typename T>
int balloc(lv_batch *b, T **p, size_t n) {
    void *q = nullptr;
    if (pool_alloc(b->device, &q, sizeof(T) * (n ? n : 1), b->stream) != cudaSuccess)
        return bfail(b, LV_ERR_NOMEM, "device allocation failed");
    b->allocs.push_back(q);
    *p = (T *)q;
    return LV_OK;
}

#define LVB_TRY(expr)           \
    do {                        \
        int rc__ = (expr);      \
        if (rc__) return rc__;  \
    } while (0)

#define LVB_CUDA(b, call)                                                                      \
    do {                                                                                       \
        cudaError_t e__ = (call);                                                              \
        if (e__ != cudaSuccess) {                                                              \
            cudaGetLastError();                                                                \
            return bfail((b), LV_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
        }                                                                                      \
    } while (0)

int batch_sync(lv_batch *b) {
    LVB_CUDA(b, cudaStreamSynchronize(b->stream));
    LVB_CUDA(b, cudaGetLastError());
    return LV_OK;
}

int batch_begin(const int32_t *graph_ptr, int32_t G, int32_t V, int64_t E, const lv_opts *opts,
                lv_batch **out, lv_batch **bp) {
    if (!out) return LV_ERR_INVALID;
    *out = nullptr;
    if (G < 0 || V < 0 || E < 0 || (G > 0 && !graph_ptr)) return LV_ERR_INVALID;
    if (E > 0x7fffffffLL || (int64_t)V + G >= 0x7fffffffLL) return LV_ERR_TOO_LARGE;
    if (G > 0 && (graph_ptr[0] != 0 || graph_ptr[G] != V)) return LV_ERR_INVALID;
    for (int32_t g = 0; g < G; ++g) {
        if (graph_ptr[g + 1] < graph_ptr[g]) return LV_ERR_INVALID;
        if (graph_ptr[g + 1] - graph_ptr[g] > LV_BATCH_MAX_GRAPH_VERTICES) return LV_ERR_TOO_LARGE;
    }
    if (G == 0 && V != 0) return LV_ERR_INVALID;
    lv_batch *b = new lv_batch();
    lv_default_opts(&b->opts);
    if (opts) {
        size_t n = opts->struct_size && opts->struct_size < sizeof(lv_opts) ? opts->struct_size : sizeof(lv_opts);
        std::memcpy(&b->opts, opts, n);
        b->opts.struct_size = sizeof(lv_opts);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        delete b;
        return LV_ERR_NO_DEVICE;
    }
    if (b->opts.device < 0 || b->opts.device >= ndev) {
        delete b;
        return LV_ERR_INVALID;
    }
    b->device = b->opts.device;
    cudaSetDevice(b->device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return LV_ERR_CUDA;
    }
    cudaEventCreate(&b->ev0);
    cudaEventCreate(&b->ev1);
    b->G = G;
    b->V = V;
    b->E = E;
    b->gptr_h.assign(graph_ptr, graph_ptr + (G > 0 ? G + 1 : 0));
    *bp = b;
    return LV_OK;
}

int batch_finish(lv_batch *b) {
    const int32_t G = b->G, V = b->V;
    const int64_t E = b->E;
    BatchParams &P = b->P;
    // whole-CSR checks: offsets, column ids, weights
    int32_t *chk = nullptr;
    LVB_TRY(balloc(b, &chk, 8 + (size_t)G + 1));
    LVB_CUDA(b, cudaMemsetAsync(chk, 0, sizeof(int32_t) * 8, b->stream));
    launch_validate_csr(b->rowptr, b->col, V, E, chk, b->stream);
    launch_weight_scan(b->w, E, chk + 4, b->stream);
    int32_t *gptr_d = nullptr;
    LVB_TRY(balloc(b, &gptr_d, (size_t)G + 1));
    if (G > 0) {
        LVB_CUDA(b, cudaMemcpyAsync(gptr_d, b->gptr_h.data(), sizeof(int32_t) * ((size_t)G + 1),
                                    cudaMemcpyHostToDevice, b->stream));
    }
    std::vector<int32_t> hchk(8 + (size_t)G + 1, 0);
    LVB_CUDA(b, cudaMemcpyAsync(hchk.data(), chk, sizeof(int32_t) * 8, cudaMemcpyDeviceToHost, b->stream));
    LVB_TRY(batch_sync(b));
    if (hchk[0]) return bfail(b, LV_ERR_INVALID, "malformed CSR (offsets or column ids)");
    if (hchk[6]) return bfail(b, LV_ERR_WEIGHT, "negative, NaN or infinite edge weight");
    // entries per graph, processing order (decreasing entries), table layout
    if (G > 0) {
        graph_entries_kernel<<<(G + 256) / 256, 256, 0, b->stream>>>(b->rowptr, gptr_d, G, chk + 8);
        note_launches(1);
        LVB_CUDA(b, cudaMemcpyAsync(hchk.data() + 8, chk + 8, sizeof(int32_t) * ((size_t)G + 1),
                                    cudaMemcpyDeviceToHost, b->stream));
        LVB_TRY(batch_sync(b));
    }
    b->entries_h.assign(G, 0);
    for (int32_t g = 0; g < G; ++g) b->entries_h[g] = (int64_t)hchk[8 + g + 1] - hchk[8 + g];
    std::vector<int32_t> order(G);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t c) { return b->entries_h[a] > b->entries_h[c]; });
    std::vector<int64_t> toff((size_t)G + 1, 0);
    for (int32_t g = 0; g < G; ++g) {
        const int32_t vg = b->gptr_h[g + 1] - b->gptr_h[g];
        toff[g + 1] = toff[g] + ((int64_t)1 << ceil_log2_i(2 * (int64_t)(vg > 0 ? vg : 1)));
    }
    b->tbl_total = toff[G];
    int32_t *order_d = nullptr;
    int64_t *toff_d = nullptr;
    LVB_TRY(balloc(b, &order_d, (size_t)G));
    LVB_TRY(balloc(b, &toff_d, (size_t)G + 1));
    if (G > 0) {
        LVB_CUDA(b, cudaMemcpyAsync(order_d, order.data(), sizeof(int32_t) * G, cudaMemcpyHostToDevice, b->stream));
        LVB_CUDA(b, cudaMemcpyAsync(toff_d, toff.data(), sizeof(int64_t) * ((size_t)G + 1),
                                    cudaMemcpyHostToDevice, b->stream));
    }
    const size_t nv = (size_t)V + 1, nvg = (size_t)V + G + 1, ne = (size_t)E + 1;
    P.rowptr = b->rowptr;
    P.col = b->col;
    P.w = b->w;
    P.gptr = gptr_d;
    P.order = order_d;
    P.tbl_off = toff_d;
    P.G = G;
    P.max_sweeps = b->opts.max_sweeps;
    LVB_TRY(balloc(b, &P.comm, nv));
    LVB_TRY(balloc(b, &P.newc, nv));
    LVB_TRY(balloc(b, &P.size, nv));
    LVB_TRY(balloc(b, &P.blist, nv));
    LVB_TRY(balloc(b, &P.newid, nv));
    LVB_TRY(balloc(b, &P.members, nv));
    LVB_TRY(balloc(b, &P.o2c, nv));
    LVB_TRY(balloc(b, &P.mstart, nvg));
    LVB_TRY(balloc(b, &P.roff, nvg));
    for (int i = 0; i < 2; ++i) {
        LVB_TRY(balloc(b, &P.rs[i], nv));
        LVB_TRY(balloc(b, &P.re[i], nv));
        LVB_TRY(balloc(b, &P.colb[i], ne));
        LVB_TRY(balloc(b, &P.wb[i], ne));
    }
    LVB_TRY(balloc(b, &P.k, nv));
    LVB_TRY(balloc(b, &P.S, nv));
    LVB_TRY(balloc(b, &P.tkeys, (size_t)b->tbl_total));
    LVB_TRY(balloc(b, &P.tvals, (size_t)b->tbl_total));
    LVB_TRY(balloc(b, &P.next, 4));
    LVB_TRY(balloc(b, &P.out_comm, nv));
    LVB_TRY(balloc(b, &P.q, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.nc, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.status, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.levels, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.sweeps, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.edge_sweeps, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.vertex_sweeps, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.moves, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.t_start, (size_t)G + 1));
    LVB_TRY(balloc(b, &P.t_end, (size_t)G + 1));
    if (b->tbl_total > 0) {
        fill_tables_kernel<<<148 * 8, 256, 0, b->stream>>>(P.tkeys, P.tvals, b->tbl_total);
        note_launches(1);
    }
    int occ = 1, sms = 148;
    cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BatchSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, BT, sizeof(BatchSmem));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    cudaGetLastError();
    const int64_t slots = (int64_t)(occ > 0 ? occ : 1) * (sms > 0 ? sms : 148);
    b->grid = (int)std::max<int64_t>(1, std::min<int64_t>(slots, G));
    return batch_sync(b);
}

}  // namespace

extern "C" {

int lv_batch_destroy(lv_batch *b) {
    if (!b) return LV_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->owns_input) {
        pool_free(b->device, (void *)b->rowptr, b->stream);
        pool_free(b->device, (void *)b->col, b->stream);
        pool_free(b->device, (void *)b->w, b->stream);
    }
    for (void *p : b->allocs) pool_free(b->device, p, b->stream);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) {
        cudaStreamSynchronize(b->stream);
        cudaStreamDestroy(b->stream);
    }
    delete b;
    return LV_OK;
}

int lv_batch_create(const int32_t *rowptr, const int32_t *col, const float *w, int32_t V, int64_t E,
                    const int32_t *graph_ptr, int32_t num_graphs, const lv_opts *opts, lv_batch **out) {
    if (!rowptr || (E > 0 && (!col || !w))) return LV_ERR_INVALID;
    lv_batch *b = nullptr;
    int rc = batch_begin(graph_ptr, num_graphs, V, E, opts, out, &b);
    if (rc) return rc;
    b->owns_input = true;
    void *p = nullptr;
    rc = pool_alloc(b->device, &p, sizeof(int32_t) * ((size_t)V + 1), b->stream) == cudaSuccess ? 0 : LV_ERR_NOMEM;
    b->rowptr = (const int32_t *)p;
    if (!rc) {
        rc = pool_alloc(b->device, &p, sizeof(int32_t) * (size_t)(E ? E : 1), b->stream) == cudaSuccess ? 0 : LV_ERR_NOMEM;
        b->col = (const int32_t *)p;
    }
    if (!rc) {
        rc = pool_alloc(b->device, &p, sizeof(float) * (size_t)(E ? E : 1), b->stream) == cudaSuccess ? 0 : LV_ERR_NOMEM;
        b->w = (const float *)p;
    }
    if (!rc && cudaMemcpyAsync((void *)b->rowptr, rowptr, sizeof(int32_t) * ((size_t)V + 1),
                               cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
        rc = LV_ERR_CUDA;
    if (!rc && E > 0 && cudaMemcpyAsync((void *)b->col, col, sizeof(int32_t) * (size_t)E,
                                        cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
        rc = LV_ERR_CUDA;
    if (!rc && E > 0 && cudaMemcpyAsync((void *)b->w, w, sizeof(float) * (size_t)E,
                                        cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
        rc = LV_ERR_CUDA;
    if (!rc) rc = batch_finish(b);
    if (rc) {
        lv_batch_destroy(b);
        return rc;
    }
    *out = b;
    return LV_OK;
}

int lv_batch_create_device(const int32_t *d_rowptr, const int32_t *d_col, const float *d_w, int32_t V,
                           int64_t E, const int32_t *graph_ptr, int32_t num_graphs, const lv_opts *opts,
                           lv_batch **out) {
    if (!d_rowptr || (E > 0 && (!d_col || !d_w))) return LV_ERR_INVALID;
    lv_batch *b = nullptr;
    int rc = batch_begin(graph_ptr, num_graphs, V, E, opts, out, &b);
    if (rc) return rc;
    b->owns_input = false;
    b->rowptr = d_rowptr;
    b->col = d_col;
    b->w = d_w;
    rc = batch_finish(b);
    if (rc) {
        lv_batch_destroy(b);
        return rc;
    }
    *out = b;
    return LV_OK;
}

const char *lv_batch_last_error(const lv_batch *b) { return b ? b->err.c_str() : "null batch"; }

int lv_batch_run(lv_batch *b, float min_gain) {
    if (!b) return LV_ERR_INVALID;
    cudaSetDevice(b->device);
    b->err.clear();
    if (b->tables_dirty && b->tbl_total > 0) {
        fill_tables_kernel<<<148 * 8, 256, 0, b->stream>>>(b->P.tkeys, b->P.tvals, b->tbl_total);
        note_launches(1);
        b->tables_dirty = false;
    }
    b->P.min_gain = (double)min_gain;
    LVB_CUDA(b, cudaMemsetAsync(b->P.next, 0, sizeof(int32_t), b->stream));
    cudaEventRecord(b->ev0, b->stream);
    if (b->G > 0) {
        batch_kernel<<<b->grid, BT, sizeof(BatchSmem), b->stream>>>(b->P);
        note_launches(1);
    }
    cudaEventRecord(b->ev1, b->stream);
    LVB_TRY(batch_sync(b));
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    b->ran = true;
    // per-graph status and edge-sweeps
    std::vector<int32_t> st(b->G);
    std::vector<int64_t> es(b->G), vs(b->G);
    if (b->G > 0) {
        LVB_CUDA(b, cudaMemcpyAsync(st.data(), b->P.status, sizeof(int32_t) * b->G, cudaMemcpyDeviceToHost, b->stream));
        LVB_CUDA(b, cudaMemcpyAsync(es.data(), b->P.edge_sweeps, sizeof(int64_t) * b->G, cudaMemcpyDeviceToHost,
                                    b->stream));
        LVB_CUDA(b, cudaMemcpyAsync(vs.data(), b->P.vertex_sweeps, sizeof(int64_t) * b->G,
                                    cudaMemcpyDeviceToHost, b->stream));
        LVB_TRY(batch_sync(b));
    }
    int64_t tot = 0, vtot = 0;
    int32_t failed = 0, first = -1;
    for (int32_t g = 0; g < b->G; ++g) {
        tot += es[g];
        vtot += vs[g];
        if (st[g] != LV_OK) {
            if (first < 0) first = g;
            ++failed;
        }
    }
    b->last_edge_sweeps = tot;
    b->last_vertex_sweeps = vtot;
    if (failed) {
        b->tables_dirty = true;
        return bfail(b, LV_ERR_DEVICE,
                     std::to_string(failed) + " graph(s) failed (first: graph " + std::to_string(first) + ", " +
                         lv_status_string(st[first]) + "); see the per-graph status");
    }
    return LV_OK;
}

int lv_batch_get_results(lv_batch *b, int32_t *communities, double *modularity, int32_t *num_communities,
                         int32_t *status) {
    if (!b) return LV_ERR_INVALID;
    if (!b->ran) return bfail(b, LV_ERR_INVALID, "lv_batch_run has not run");
    cudaSetDevice(b->device);
    if (communities && b->V > 0)
        LVB_CUDA(b, cudaMemcpyAsync(communities, b->P.out_comm, sizeof(int32_t) * b->V, cudaMemcpyDeviceToHost,
                                    b->stream));
    if (b->G > 0) {
        if (modularity)
            LVB_CUDA(b, cudaMemcpyAsync(modularity, b->P.q, sizeof(double) * b->G, cudaMemcpyDeviceToHost, b->stream));
        if (num_communities)
            LVB_CUDA(b, cudaMemcpyAsync(num_communities, b->P.nc, sizeof(int32_t) * b->G, cudaMemcpyDeviceToHost,
                                        b->stream));
        if (status)
            LVB_CUDA(b, cudaMemcpyAsync(status, b->P.status, sizeof(int32_t) * b->G, cudaMemcpyDeviceToHost,
                                        b->stream));
    }
    return batch_sync(b);
}

int lv_batch_get_graph_stats(lv_batch *b, int32_t *levels, int64_t *sweeps, int64_t *edge_sweeps,
                             double *latency_ms) {
    if (!b) return LV_ERR_INVALID;
    if (!b->ran) return bfail(b, LV_ERR_INVALID, "lv_batch_run has not run");
    cudaSetDevice(b->device);
    const size_t G = (size_t)b->G;
    if (G == 0) return LV_OK;
    if (levels)
        LVB_CUDA(b, cudaMemcpyAsync(levels, b->P.levels, sizeof(int32_t) * G, cudaMemcpyDeviceToHost, b->stream));
    if (sweeps)
        LVB_CUDA(b, cudaMemcpyAsync(sweeps, b->P.sweeps, sizeof(int64_t) * G, cudaMemcpyDeviceToHost, b->stream));
    if (edge_sweeps)
        LVB_CUDA(b, cudaMemcpyAsync(edge_sweeps, b->P.edge_sweeps, sizeof(int64_t) * G, cudaMemcpyDeviceToHost,
                                    b->stream));
    std::vector<u64> t0, t1;
    if (latency_ms) {
        t0.resize(G);
        t1.resize(G);
        LVB_CUDA(b, cudaMemcpyAsync(t0.data(), b->P.t_start, sizeof(u64) * G, cudaMemcpyDeviceToHost, b->stream));
        LVB_CUDA(b, cudaMemcpyAsync(t1.data(), b->P.t_end, sizeof(u64) * G, cudaMemcpyDeviceToHost, b->stream));
    }
    LVB_TRY(batch_sync(b));
    if (latency_ms)
        for (size_t g = 0; g < G; ++g) latency_ms[g] = (double)(t1[g] - t0[g]) * 1e-6;
    return LV_OK;
}

int lv_batch_get_stats(lv_batch *b, double *device_ms, int64_t *edge_sweeps, int64_t *vertex_sweeps,
                       int32_t *ctas) {
    if (!b) return LV_ERR_INVALID;
    if (device_ms) *device_ms = b->last_ms;
    if (edge_sweeps) *edge_sweeps = b->last_edge_sweeps;
    if (vertex_sweeps) *vertex_sweeps = b->last_vertex_sweeps;
    if (ctas) *ctas = b->grid;
    return LV_OK;
}

}  // extern "C"
