// lv_agg.cu -- community aggregation kernels.
//
// Replaces fillArrays / orderVertices / mergeCommunity{Shared,Global} /
// compressEdges / updateOriginalToCommunity of community_aggregation.cu
// (:47-74, :76-228).  The result is the same graph as the reference's
// aggregateCommunities (:248-347): non-empty communities are renumbered in
// ascending old id, each new vertex's row holds one entry per neighbouring
// new community with the summed weight (intra-community weight becomes a
// self-loop counting both directions), and the new vertex weight equals
// Sigma_tot.  Sums are exact uint64, so the rows are identical whatever the
// order of the atomic additions; only the order of entries inside a row is
// unspecified (it is in the reference too).
//
// Pipeline (all on the device, three small host reads per level):
//   flag/newid scan -> lab[v] = newid[C(v)] -> members grouped by community
//   -> member-order prefix P of degrees -> permute every row into the
//   community-grouped "virtual edge" array (key = lab[neighbour], weight)
//   -> per-community hash merge written back in place -> scan of the
//   distinct counts -> compaction into the next level's CSR.
#include "lv_internal.h"

namespace lv {

namespace {

inline unsigned grid_for(int64_t n, int64_t cap = 148 * 16) {
    int64_t b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (unsigned)(b < cap ? b : cap);
}
inline unsigned nblocks(int64_t items, int per_block) {
    return (unsigned)((items + per_block - 1) / per_block);
}

__global__ void flag_kernel(const int32_t *__restrict__ size, int32_t V, int32_t *flag) {
    for (int32_t c = blockIdx.x * 256 + threadIdx.x; c < V; c += gridDim.x * 256)
        flag[c] = size[c] > 0 ? 1 : 0;
}

__global__ void label_kernel(const int32_t *__restrict__ comm, const int32_t *__restrict__ newid,
                             int32_t V, int32_t *lab) {
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256)
        lab[v] = newid[comm[v]];
}

// Vertices grouped by community: one warp-aggregated cursor increment per
// distinct community in the warp (a giant community would otherwise
// serialise on its cursor).
__global__ void members_kernel(const int32_t *__restrict__ comm, const int32_t *__restrict__ mstart,
                               const int32_t *__restrict__ rowptr, const int32_t *__restrict__ rowend,
                               int32_t V, int32_t *cursor,
                               int32_t *members, int32_t *mslot, int32_t *degm) {
    const int lane = threadIdx.x & 31;
    for (int32_t base = blockIdx.x * 256; base < V; base += gridDim.x * 256) {
        const int32_t v = base + threadIdx.x;
        const bool valid = v < V;
        const int32_t c = valid ? comm[v] : -1;
        const unsigned peers = __match_any_sync(FULL, c);
        const int leader = __ffs(peers) - 1;
        int32_t pos = 0;
        if (lane == leader && valid) pos = atomicAdd(cursor + c, __popc(peers));
        pos = __shfl_sync(FULL, pos, leader);
        if (valid) {
            const int32_t m = mstart[c] + pos + __popc(peers & ((1u << lane) - 1u));
            members[m] = v;
            mslot[v] = m;
            degm[m] = rowend[v] - rowptr[v];
        }
    }
}

// Permute vertex rows into community-grouped order.
template <int G, typename WT>
__global__ void __launch_bounds__(256) permute_group_kernel(GraphView<WT> g,
                                                            const int32_t *__restrict__ lab,
                                                            const int32_t *__restrict__ mslot,
                                                            const int32_t *__restrict__ P,
                                                            const int32_t *__restrict__ list,
                                                            int32_t n, int32_t *vkey, u64 *vw) {
    const int grp = threadIdx.x / G, lane = threadIdx.x % G;
    const int32_t idx = blockIdx.x * (256 / G) + grp;
    if (idx >= n) return;
    const int32_t v = list[idx];
    const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
    const int32_t dst = P[mslot[v]] - r0;
    for (int32_t e = r0 + lane; e < r1; e += G) {
        vkey[dst + e] = lab[__ldg(g.col + e)];
        vw[dst + e] = gw(g, e);
    }
}

template <int T, typename WT>
__global__ void __launch_bounds__(T) permute_cta_kernel(GraphView<WT> g,
                                                        const int32_t *__restrict__ lab,
                                                        const int32_t *__restrict__ mslot,
                                                        const int32_t *__restrict__ P,
                                                        const int32_t *__restrict__ list,
                                                        int32_t n, int32_t *vkey, u64 *vw) {
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t v = list[idx];
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        const int32_t dst = P[mslot[v]] - r0;
        for (int32_t e = r0 + threadIdx.x; e < r1; e += T) {
            vkey[dst + e] = lab[__ldg(g.col + e)];
            vw[dst + e] = gw(g, e);
        }
    }
}

// Merge classes of communities by degree bound (sum of member degrees).
enum AggClass { AC1 = 0, AC2, AC3, AC4, AC5, NAC };
__device__ __forceinline__ int agg_class(int32_t d) {
    if (d <= 0) return -1;
    if (d <= 32) return AC1;
    if (d <= 128) return AC2;
    if (d <= 1024) return AC3;
    if (d <= 4096) return AC4;
    return AC5;
}

__global__ void __launch_bounds__(256) agg_class_count_kernel(const int32_t *__restrict__ size,
                                                              const int32_t *__restrict__ mstart,
                                                              const int32_t *__restrict__ P,
                                                              int32_t V, int32_t *counts) {
    __shared__ int32_t c[NAC];
    if (threadIdx.x < NAC) c[threadIdx.x] = 0;
    __syncthreads();
    for (int32_t x = blockIdx.x * 256 + threadIdx.x; x < V; x += gridDim.x * 256) {
        if (size[x] <= 0) continue;
        const int cls = agg_class(P[mstart[x + 1]] - P[mstart[x]]);
        if (cls >= 0) atomicAdd(c + cls, 1);
    }
    __syncthreads();
    if (threadIdx.x < NAC && c[threadIdx.x]) atomicAdd(counts + threadIdx.x, c[threadIdx.x]);
}

struct AggOffsets {
    int32_t off[NAC];
};

__global__ void __launch_bounds__(256) agg_class_scatter_kernel(
    const int32_t *__restrict__ size, const int32_t *__restrict__ mstart,
    const int32_t *__restrict__ P, int32_t V, AggOffsets offs, int32_t *cursors, int32_t *clist) {
    const int lane = threadIdx.x & 31;
    for (int32_t base = blockIdx.x * 256; base < V; base += gridDim.x * 256) {
        const int32_t x = base + threadIdx.x;
        int cls = -1;
        if (x < V && size[x] > 0) cls = agg_class(P[mstart[x + 1]] - P[mstart[x]]);
        const unsigned peers = __match_any_sync(FULL, cls);
        const int leader = __ffs(peers) - 1;
        int32_t pos = 0;
        if (lane == leader && cls >= 0) pos = atomicAdd(cursors + cls, __popc(peers));
        pos = __shfl_sync(FULL, pos, leader);
        if (cls >= 0) clist[offs.off[cls] + pos + __popc(peers & ((1u << lane) - 1u))] = x;
    }
}

// New vertex weights and the rows of communities without edges.
__global__ void new_vertex_kernel(const int32_t *__restrict__ size,
                                  const int32_t *__restrict__ newid,
                                  const int32_t *__restrict__ mstart,
                                  const int32_t *__restrict__ P, const u64 *__restrict__ S,
                                  int32_t V, u64 *knew, int32_t *newdeg, int32_t *epos_new) {
    for (int32_t c = blockIdx.x * 256 + threadIdx.x; c < V; c += gridDim.x * 256) {
        if (size[c] <= 0) continue;
        const int32_t nid = newid[c];
        knew[nid] = S[c];
        const int32_t a = P[mstart[c]], b = P[mstart[c + 1]];
        if (a == b) {
            newdeg[nid] = 0;
            epos_new[nid] = a;
        }
    }
}

template <int G, int CAP>
__global__ void __launch_bounds__(256) merge_group_kernel(const int32_t *__restrict__ clist,
                                                          int32_t n, const int32_t *__restrict__ mstart,
                                                          const int32_t *__restrict__ P,
                                                          const int32_t *__restrict__ newid,
                                                          int32_t *vkey, u64 *vw, uint32_t *vw32,
                                                          int32_t *newdeg, int32_t *epos_new, int *err,
                                                          int *hiflag, uint8_t *wrow) {
    constexpr int GPB = 256 / G;
    constexpr int LG = (CAP == 64) ? 6 : (CAP == 128) ? 7 : 8;
    static_assert((1 << LG) == CAP, "CAP");
    __shared__ u64 svals[GPB * CAP];
    __shared__ int32_t skeys[GPB * CAP];
    const int grp = threadIdx.x / G, lane = threadIdx.x % G;
    const int32_t idx = blockIdx.x * GPB + grp;
    int32_t *keys = skeys + grp * CAP;
    u64 *vals = svals + grp * CAP;
#pragma unroll
    for (int s = lane; s < CAP; s += G) { keys[s] = -1; vals[s] = 0; }
    __syncwarp();
    const bool active = idx < n;
    int32_t c = 0, a = 0, b = 0;
    if (active) {
        c = clist[idx];
        a = P[mstart[c]];
        b = P[mstart[c + 1]];
    }
    // entries keyed by the community's own new id (its intra-community
    // weight, usually the bulk) are summed in registers
    const int32_t self = active ? newid[c] : -1;
    u64 w_self = 0;
    for (int32_t i = a + lane; i < b; i += G) {
        const int32_t k = vkey[i];
        if (k == self) w_self += vw[i];
        else table_insert<1>(keys, vals, LG, k, vw[i], err);
    }
    for (int off = G >> 1; off > 0; off >>= 1) w_self += __shfl_xor_sync(FULL, w_self, off, G);
    __syncwarp();
    if (active && lane == 0 && w_self) table_insert<1>(keys, vals, LG, self, w_self, err);
    __syncwarp();
    // write the distinct entries back at the start of the range, in slot order
    const int wl = threadIdx.x & 31;
    const unsigned gmask = (G == 32) ? FULL : (((1u << G) - 1u) << (wl & ~(G - 1)));
    int32_t cnt = 0;
    u64 hi = 0;
#pragma unroll
    for (int s0 = 0; s0 < CAP; s0 += G) {
        const int s = s0 + lane;
        const bool occ = active && keys[s] >= 0;
        const unsigned bal = __ballot_sync(FULL, occ) & gmask;
        if (occ) {
            const int32_t pos = a + cnt + __popc(bal & ((1u << wl) - 1u));
            const u64 x = vals[s];
            vkey[pos] = keys[s];
            vw[pos] = x;
            vw32[pos] = x < W32_ESC ? (uint32_t)x : W32_ESC;
            if (keys[s] != self && x >= W32_ESC) hi = 1;   // the self-loop is read as uint64 only
        }
        cnt += __popc(bal);
    }
    if (hi) {
        atomicOr(hiflag, 1);
        wrow[self] = 1;
    }
    if (active && lane == 0) {
        const int32_t nid = newid[c];
        newdeg[nid] = cnt;
        epos_new[nid] = a;
    }
}

template <int T, int CAPMAX>
__global__ void __launch_bounds__(T) merge_cta_kernel(const int32_t *__restrict__ clist, int32_t n,
                                                      const int32_t *__restrict__ mstart,
                                                      const int32_t *__restrict__ P,
                                                      const int32_t *__restrict__ newid,
                                                      int32_t *vkey, u64 *vw, uint32_t *vw32,
                                                      int32_t *newdeg, int32_t *epos_new, int *err,
                                                      int *hiflag, uint8_t *wrow) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *vals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAPMAX);
    __shared__ int32_t cnt;
    for (int s = threadIdx.x; s < CAPMAX; s += T) { keys[s] = -1; vals[s] = 0; }
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t c = clist[idx];
        const int32_t a = P[mstart[c]], b = P[mstart[c + 1]];
        int lg = ceil_log2_i(2 * (int64_t)(b - a));
        lg = lg < 3 ? 3 : lg;
        const int cap = 1 << lg;
        const int32_t self = newid[c];
        u64 w_self = 0;
        for (int32_t i = a + threadIdx.x; i < b; i += T) {
            const int32_t k = vkey[i];
            if (k == self) w_self += vw[i];
            else table_insert<1>(keys, vals, lg, k, vw[i], err);
        }
        w_self = warp_sum_u64(w_self);
        if ((threadIdx.x & 31) == 0 && w_self) table_insert<1>(keys, vals, lg, self, w_self, err);
        __syncthreads();
        for (int s = threadIdx.x; s < cap; s += T) {
            const int32_t key = keys[s];
            if (key >= 0) {
                const int32_t pos = a + atomicAdd(&cnt, 1);
                const u64 x = vals[s];
                vkey[pos] = key;
                vw[pos] = x;
                vw32[pos] = x < W32_ESC ? (uint32_t)x : W32_ESC;
                if (key != self && x >= W32_ESC) {   // the self-loop is read as uint64 only
                    atomicOr(hiflag, 1);
                    wrow[self] = 1;
                }
                keys[s] = -1;
                vals[s] = 0;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int32_t nid = newid[c];
            newdeg[nid] = cnt;
            epos_new[nid] = a;
            cnt = 0;
        }
        __syncthreads();
    }
}

// merge_cta_kernel for a level whose non-self-loop weights are below 2^32:
// the inter-community entries (the only ones that enter the table; the
// community's own key is summed in registers, as a self-loop can be large)
// are summed in 16-bit-piece counters with fire-and-forget adds, and the
// self entry is appended to the merged row after the table's entries.
template <int T, int CAPMAX>
__global__ void __launch_bounds__(T) merge_cta_narrow_kernel(const int32_t *__restrict__ clist, int32_t n,
                                                             const int32_t *__restrict__ mstart,
                                                             const int32_t *__restrict__ P,
                                                             const int32_t *__restrict__ newid,
                                                             int32_t *vkey, u64 *vw, uint32_t *vw32,
                                                             int32_t *newdeg, int32_t *epos_new, int *err,
                                                             int *hiflag, uint8_t *wrow) {
    static_assert(CAPMAX / 2 <= PIECE_MAX_ADDS, "a community's entries fit the piece counters");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PieceTable t;
    t.lo = reinterpret_cast<uint32_t *>(smem_raw);
    t.hi = t.lo + CAPMAX;
    t.keys = reinterpret_cast<int32_t *>(t.hi + CAPMAX);
    __shared__ int32_t cnt;
    __shared__ u64 wpart[T / 32];
    for (int s = threadIdx.x; s < CAPMAX; s += T) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t c = clist[idx];
        const int32_t a = P[mstart[c]], b = P[mstart[c + 1]];
        int lg = ceil_log2_i(2 * (int64_t)(b - a));
        lg = lg < 3 ? 3 : lg;
        const int cap = 1 << lg;
        const int32_t self = newid[c];
        u64 w_self = 0;
        for (int32_t i = a + threadIdx.x; i < b; i += T) {
            const int32_t k = vkey[i];
            if (k == self) w_self += vw[i];
            else piece_insert_at(t, lg, hash_slot_agg(k, lg), k, vw[i], err);
        }
        w_self = warp_sum_u64(w_self);
        if ((threadIdx.x & 31) == 0) wpart[threadIdx.x >> 5] = w_self;
        __syncthreads();
        for (int s = threadIdx.x; s < cap; s += T) {
            const int32_t key = t.keys[s];
            if (key >= 0) {
                const int32_t pos = a + atomicAdd(&cnt, 1);
                const u64 x = piece_value(t, (uint32_t)s);
                vkey[pos] = key;
                vw[pos] = x;
                vw32[pos] = x < W32_ESC ? (uint32_t)x : W32_ESC;
                if (x >= W32_ESC) {
                    atomicOr(hiflag, 1);
                    wrow[self] = 1;
                }
                t.keys[s] = -1;
                t.lo[s] = 0;
                t.hi[s] = 0;
            }
        }
        if (threadIdx.x == 0) {
            u64 ws = 0;
            for (int i = 0; i < T / 32; ++i) ws += wpart[i];
            if (ws) {
                const int32_t pos = a + atomicAdd(&cnt, 1);
                vkey[pos] = self;
                vw[pos] = ws;
                vw32[pos] = ws < W32_ESC ? (uint32_t)ws : W32_ESC;   // the self-loop is read as uint64 only
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int32_t nid = newid[c];
            newdeg[nid] = cnt;
            epos_new[nid] = a;
            cnt = 0;
        }
        __syncthreads();
    }
}

// Insert (key, w) into a community's global table (GSlot layout, move-phase
// hash, linear probing bounded by the capacity); returns the slot newly
// claimed for key, or -1.
__device__ __forceinline__ int32_t gslot_insert_claim(GSlot *t, int lg, int32_t key, u64 w, int *err) {
    const uint32_t mask = (1u << lg) - 1u;
    const uint32_t k1 = (uint32_t)key + 1u;
    uint32_t s = hash_slot(key, lg);
    for (uint32_t p = 0; p <= mask; ++p) {
        const uint32_t cur = ((volatile uint32_t *)&t[s].key1)[0];
        if (cur == k1) { atomicAdd(&t[s].val, w); return -1; }
        if (cur == 0) {
            const uint32_t prev = atomicCAS(&t[s].key1, 0u, k1);
            if (prev == 0) { atomicAdd(&t[s].val, w); return (int32_t)s; }
            if (prev == k1) { atomicAdd(&t[s].val, w); return -1; }
        }
        s = (s + 1u) & mask;
    }
    atomicOr(err, DEVERR_HASH_FULL);
    return -1;
}

// Global-table merge for communities whose degree bound exceeds 4096: one CTA
// per chunk of HG_EDGE_CHUNK entries, reduced first in a chunk-local shared
// table (intra-community entries all carry the community's own key), then
// added once per distinct key to the community's global table.
__global__ void __launch_bounds__(HG_INSERT_THREADS) mergeg_insert_kernel(
    HubGlobal hg, const int32_t *__restrict__ mstart, const int32_t *__restrict__ P,
    const int32_t *__restrict__ newid, const int32_t *__restrict__ vkey,
    const u64 *__restrict__ vw, int *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LCAP = 2 * HG_EDGE_CHUNK;
    constexpr int LLG = ilog2_c(LCAP);
    u64 *lvals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *lkeys = reinterpret_cast<int32_t *>(lvals + LCAP);
    for (int s = threadIdx.x; s < LCAP; s += HG_INSERT_THREADS) { lkeys[s] = -1; lvals[s] = 0; }
    __syncthreads();
    const int32_t h = hg.echunk_hub[blockIdx.x];
    const int32_t c = hg.hubs[h];
    const int32_t b = P[mstart[c + 1]];
    const int32_t i0 = P[mstart[c]] + hg.echunk_e0[blockIdx.x];
    const int32_t i1 = min(i0 + HG_EDGE_CHUNK, b);
    const int32_t self = newid[c];
    u64 w_self = 0;
    for (int32_t i = i0 + threadIdx.x; i < i1; i += HG_INSERT_THREADS) {
        const int32_t k = vkey[i];
        if (k == self) w_self += vw[i];
        else table_insert<1>(lkeys, lvals, LLG, k, vw[i], err);
    }
    w_self = warp_sum_u64(w_self);
    if ((threadIdx.x & 31) == 0 && w_self) table_insert<1>(lkeys, lvals, LLG, self, w_self, err);
    __syncthreads();
    // the chunk table (aggregation hash) is drained in slot order into the
    // community's global table (move-phase hash), so consecutive inserts land
    // far apart; the merged row comes out in claim order, i.e. in the chunk
    // table's slot order, which is independent of the move phase's hash
    GSlot *tbl = hg.slots + hg.tbl_off[h];
    int32_t *occ = hg.occ + hg.occ_off[h];
    const int lg = hg.tbl_lg[h];
    for (int s = threadIdx.x; s < LCAP; s += HG_INSERT_THREADS) {
        const int32_t k = lkeys[s];
        const int32_t claimed = k >= 0 ? gslot_insert_claim(tbl, lg, k, lvals[s], err) : -1;
        warp_append(claimed, occ, hg.nocc + h);
    }
}

// mergeg_insert_kernel for a level whose non-self-loop weights are below
// 2^32: the chunk-local table sums in 16-bit-piece counters (a chunk has
// HG_EDGE_CHUNK entries); the chunk's weight to the community's own key (which
// can be large) is summed over the CTA and added to the global table once.
__global__ void __launch_bounds__(HG_INSERT_THREADS) mergeg_insert_narrow_kernel(
    HubGlobal hg, const int32_t *__restrict__ mstart, const int32_t *__restrict__ P,
    const int32_t *__restrict__ newid, const int32_t *__restrict__ vkey,
    const u64 *__restrict__ vw, int *err) {
    static_assert(HG_EDGE_CHUNK <= PIECE_MAX_ADDS, "chunks fit the piece counters");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LCAP = 2 * HG_EDGE_CHUNK;
    constexpr int LLG = ilog2_c(LCAP);
    constexpr int NW = HG_INSERT_THREADS / 32;
    PieceTable t;
    t.lo = reinterpret_cast<uint32_t *>(smem_raw);
    t.hi = t.lo + LCAP;
    t.keys = reinterpret_cast<int32_t *>(t.hi + LCAP);
    int32_t *locc = t.keys + LCAP;   // claimed slots of the chunk table (at most HG_EDGE_CHUNK)
    __shared__ u64 wpart[NW];
    __shared__ int32_t lnocc;
    for (int s = threadIdx.x; s < LCAP; s += HG_INSERT_THREADS) { t.keys[s] = -1; t.lo[s] = 0; t.hi[s] = 0; }
    if (threadIdx.x == 0) lnocc = 0;
    __syncthreads();
    // persistent over the chunks; after a chunk only its claimed slots are
    // cleared
    for (int32_t ch = blockIdx.x; ch < hg.n_echunks; ch += gridDim.x) {
        const int32_t h = hg.echunk_hub[ch];
        const int32_t c = hg.hubs[h];
        const int32_t b = P[mstart[c + 1]];
        const int32_t i0 = P[mstart[c]] + hg.echunk_e0[ch];
        const int32_t i1 = min(i0 + HG_EDGE_CHUNK, b);
        const int32_t self = newid[c];
        u64 w_self = 0;
        for (int32_t i = i0 + threadIdx.x; i < i1; i += HG_INSERT_THREADS) {
            const int32_t k = vkey[i];
            if (k == self) {
                w_self += vw[i];
            } else {
                const int32_t claimed = piece_insert_at(t, LLG, hash_slot_agg(k, LLG), k, vw[i], err);
                if (claimed >= 0) {
                    const int32_t j = atomicAdd(&lnocc, 1);
                    if (j < HG_EDGE_CHUNK) locc[j] = claimed;
                }
            }
        }
        w_self = warp_sum_u64(w_self);
        if ((threadIdx.x & 31) == 0) wpart[threadIdx.x >> 5] = w_self;
        __syncthreads();
        GSlot *tbl = hg.slots + hg.tbl_off[h];
        int32_t *occ = hg.occ + hg.occ_off[h];
        const int lg = hg.tbl_lg[h];
        if (threadIdx.x < 32) {
            u64 ws = 0;
            if (threadIdx.x == 0)
                for (int i = 0; i < NW; ++i) ws += wpart[i];
            const int32_t claimed = ws ? gslot_insert_claim(tbl, lg, self, ws, err) : -1;
            warp_append(claimed, occ, hg.nocc + h);
        }
        // drained in claim order into the community's global table (its
        // move-phase hash is independent of the chunk table's)
        const int32_t n = min(lnocc, HG_EDGE_CHUNK);
        for (int32_t i0s = 0; i0s < n; i0s += HG_INSERT_THREADS) {
            const int32_t i = i0s + threadIdx.x;
            int32_t claimed = -1;
            if (i < n) {
                const uint32_t sl = (uint32_t)locc[i];
                claimed = gslot_insert_claim(tbl, lg, t.keys[sl], piece_value(t, sl), err);
                t.keys[sl] = -1;
                t.lo[sl] = 0;
                t.hi[sl] = 0;
            }
            warp_append(claimed, occ, hg.nocc + h);
        }
        __syncthreads();
        if (threadIdx.x == 0) lnocc = 0;
        __syncthreads();
    }
}

// Entry i of a community's occupied list becomes entry i of its merged row.
__global__ void __launch_bounds__(256) mergeg_emit_kernel(HubGlobal hg,
                                                          const int32_t *__restrict__ mstart,
                                                          const int32_t *__restrict__ P,
                                                          const int32_t *__restrict__ newid,
                                                          int32_t *vkey, u64 *vw, uint32_t *vw32,
                                                          int *hiflag, uint8_t *wrow) {
    const int32_t bidx = blockIdx.x;
    const int32_t h = hg.schunk_hub[bidx];
    const int32_t c = hg.hubs[h];
    const int32_t a = P[mstart[c]];
    const int32_t self = newid[c];
    GSlot *tbl = hg.slots + hg.tbl_off[h];
    const int32_t *occ = hg.occ + hg.occ_off[h];
    const int32_t s0 = hg.schunk_s0[bidx];
    const int32_t n = min(hg.nocc[h] - s0, HG_SLOT_CHUNK);
    u64 hi = 0;
    for (int32_t i = threadIdx.x; i < n; i += 256) {
        const int32_t sl = occ[s0 + i];
        const GSlot g = tbl[sl];
        const int32_t key = (int32_t)(g.key1 - 1u);
        const u64 x = g.val;
        vkey[a + s0 + i] = key;
        vw[a + s0 + i] = x;
        vw32[a + s0 + i] = x < W32_ESC ? (uint32_t)x : W32_ESC;
        if (key != self && x >= W32_ESC) hi = 1;   // the self-loop is read as uint64 only
        tbl[sl] = GSlot{0u, 0u, 0};
    }
    if (hi) {
        atomicOr(hiflag, 1);
        wrow[self] = 1;
    }
}

__global__ void mergeg_finish_kernel(HubGlobal hg, const int32_t *__restrict__ mstart,
                                     const int32_t *__restrict__ P, const int32_t *__restrict__ newid,
                                     int32_t *newdeg, int32_t *epos_new) {
    for (int32_t h = blockIdx.x * 256 + threadIdx.x; h < hg.nhubs; h += gridDim.x * 256) {
        const int32_t c = hg.hubs[h];
        const int32_t nid = newid[c];
        newdeg[nid] = hg.nocc[h];
        epos_new[nid] = P[mstart[c]];
        hg.nocc[h] = 0;
    }
}


// Rows of the next level stay where the merge wrote them: row c' spans
// [epos_new[c'], epos_new[c'] + newdeg[c']).
__global__ void row_bounds_kernel(const int32_t *__restrict__ epos_new,
                                  const int32_t *__restrict__ newdeg, int32_t Vn, int32_t *start,
                                  int32_t *end) {
    for (int32_t c = blockIdx.x * 256 + threadIdx.x; c < Vn; c += gridDim.x * 256) {
        const int32_t a = epos_new[c];
        start[c] = a;
        end[c] = a + newdeg[c];
    }
}

}  // namespace

constexpr int A3_T = 256, A3_CAP = 2048;
constexpr int A4_T = 512, A4_CAP = 8192;
static int g_occ_a3 = 4, g_occ_a4 = 2, g_occ_mg = 2, g_sms = 148;
// narrow global merge: chunk table + its claimed-slot list
constexpr int HG_INSERT_NSMEM = 2 * HG_EDGE_CHUNK * 12 + HG_EDGE_CHUNK * 4;

void init_agg_attributes() {
    cudaFuncSetAttribute(merge_cta_kernel<A3_T, A3_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         A3_CAP * 12);
    cudaFuncSetAttribute(merge_cta_kernel<A4_T, A4_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         A4_CAP * 12);
    cudaFuncSetAttribute(mergeg_insert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, HG_INSERT_SMEM);
    cudaFuncSetAttribute(mergeg_insert_narrow_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, HG_INSERT_NSMEM);
    {
        int o = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, mergeg_insert_narrow_kernel, HG_INSERT_THREADS, HG_INSERT_NSMEM);
        g_occ_mg = o > 0 ? o : 1;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    cudaFuncSetAttribute(merge_cta_narrow_kernel<A3_T, A3_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         A3_CAP * 12);
    cudaFuncSetAttribute(merge_cta_narrow_kernel<A4_T, A4_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         A4_CAP * 12);
    int o3 = 0, o4 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3, merge_cta_kernel<A3_T, A3_CAP>, A3_T, A3_CAP * 12);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o4, merge_cta_kernel<A4_T, A4_CAP>, A4_T, A4_CAP * 12);
    g_occ_a3 = o3 > 0 ? o3 : 1;
    g_occ_a4 = o4 > 0 ? o4 : 1;
}

// Steps up to the member prefix and the merge classification.
//   flag -> newid (scan, total in scalars[0]), lab, mstart (scan of size),
//   members / mslot / degm, P (scan of degm, total in scalars[1]),
//   class counts in scalars[2..2+NAC).
void agg_prepare(const int32_t *rowptr, const int32_t *rowend, const int32_t *comm,
                 const int32_t *size, int32_t V, AggBuffers &ab, int32_t *mslot, int32_t *degm,
                 int32_t *P, cudaStream_t s) {
    flag_kernel<<<grid_for(V), 256, 0, s>>>(size, V, ab.flag); note_launches(1);
    scan_exclusive_i32(ab.flag, ab.flag, V, ab.scalars + 0, ab.scan_tmp, s);
    label_kernel<<<grid_for(V), 256, 0, s>>>(comm, ab.flag, V, ab.lab); note_launches(1);
    scan_exclusive_i32(size, ab.mstart, V, ab.mstart + V, ab.scan_tmp, s);
    cudaMemsetAsync(ab.cursor, 0, sizeof(int32_t) * (size_t)V, s);
    members_kernel<<<grid_for(V), 256, 0, s>>>(comm, ab.mstart, rowptr, rowend, V, ab.cursor,
                                                ab.members, mslot, degm); note_launches(1);
    scan_exclusive_i32(degm, P, V, P + V, ab.scan_tmp, s);
    cudaMemsetAsync(ab.scalars + 2, 0, sizeof(int32_t) * NAC, s);
    agg_class_count_kernel<<<grid_for(V), 256, 0, s>>>(size, ab.mstart, P, V, ab.scalars + 2); note_launches(1);
}

void agg_classify(const int32_t *size, int32_t V, AggBuffers &ab, const int32_t *P,
                  const int32_t *offsets, cudaStream_t s) {
    AggOffsets o;
    for (int c = 0; c < NAC; ++c) o.off[c] = offsets[c];
    cudaMemsetAsync(ab.cursor, 0, sizeof(int32_t) * NAC, s);
    agg_class_scatter_kernel<<<grid_for(V), 256, 0, s>>>(size, ab.mstart, P, V, o, ab.cursor, ab.clist); note_launches(1);
}

template <typename WT>
void agg_permute(int cls, const GraphView<WT> &g, const AggBuffers &ab, const int32_t *mslot,
                 const int32_t *P, const int32_t *list, int32_t n, int32_t *vkey, u64 *vw,
                 int sms, cudaStream_t s) {
    if (n <= 0) return;
    switch (cls) {
    case CLS_B0: permute_group_kernel<4, WT><<<nblocks(n, 64), 256, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    case CLS_B1: permute_group_kernel<8, WT><<<nblocks(n, 32), 256, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    case CLS_B2: permute_group_kernel<16, WT><<<nblocks(n, 16), 256, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    case CLS_B3:
    case CLS_B4: permute_group_kernel<32, WT><<<nblocks(n, 8), 256, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    case CLS_B5: permute_cta_kernel<128, WT><<<(unsigned)imin64(n, sms * 16), 128, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    case CLS_H1: permute_cta_kernel<256, WT><<<(unsigned)imin64(n, sms * 8), 256, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    default: permute_cta_kernel<512, WT><<<(unsigned)imin64(n, sms * 4), 512, 0, s>>>(g, ab.lab, mslot, P, list, n, vkey, vw); note_launches(1); break;
    }
}
template void agg_permute<float>(int, const GraphView<float> &, const AggBuffers &, const int32_t *,
                                 const int32_t *, const int32_t *, int32_t, int32_t *, u64 *, int,
                                 cudaStream_t);
template void agg_permute<u64>(int, const GraphView<u64> &, const AggBuffers &, const int32_t *,
                               const int32_t *, const int32_t *, int32_t, int32_t *, u64 *, int,
                               cudaStream_t);

void agg_new_vertices(const int32_t *size, const u64 *S, int32_t V, const AggBuffers &ab,
                      const int32_t *P, u64 *knew, cudaStream_t s) {
    new_vertex_kernel<<<grid_for(V), 256, 0, s>>>(size, ab.flag, ab.mstart, P, S, V, knew,
                                                   ab.newdeg, ab.epos_new); note_launches(1);
}

void agg_merge_class(int acls, const AggBuffers &ab, const int32_t *P, const int32_t *list,
                     int32_t n, int32_t *vkey, u64 *vw, uint32_t *vw32, int *err, int *hiflag, uint8_t *wrow,
                     int sms, cudaStream_t s, bool narrow) {
    if (n <= 0) return;
    switch (acls) {
    case AC1:
        merge_group_kernel<8, 64><<<nblocks(n, 32), 256, 0, s>>>(list, n, ab.mstart, P, ab.flag, vkey,
                                                                  vw, vw32, ab.newdeg, ab.epos_new, err, hiflag, wrow); note_launches(1);
        break;
    case AC2:
        merge_group_kernel<32, 256><<<nblocks(n, 8), 256, 0, s>>>(list, n, ab.mstart, P, ab.flag, vkey,
                                                                   vw, vw32, ab.newdeg, ab.epos_new, err, hiflag, wrow); note_launches(1);
        break;
    case AC3:
        if (narrow)
            merge_cta_narrow_kernel<A3_T, A3_CAP><<<(unsigned)imin64(n, (int64_t)sms * g_occ_a3), A3_T, A3_CAP * 12,
                                                    s>>>(list, n, ab.mstart, P, ab.flag, vkey, vw, vw32, ab.newdeg,
                                                         ab.epos_new, err, hiflag, wrow);
        else
            merge_cta_kernel<A3_T, A3_CAP><<<(unsigned)imin64(n, (int64_t)sms * g_occ_a3), A3_T,
                                             A3_CAP * 12, s>>>(list, n, ab.mstart, P, ab.flag, vkey, vw, vw32,
                                                               ab.newdeg, ab.epos_new, err, hiflag, wrow);
        note_launches(1);
        break;
    case AC4:
        if (narrow)
            merge_cta_narrow_kernel<A4_T, A4_CAP><<<(unsigned)imin64(n, (int64_t)sms * g_occ_a4), A4_T, A4_CAP * 12,
                                                    s>>>(list, n, ab.mstart, P, ab.flag, vkey, vw, vw32, ab.newdeg,
                                                         ab.epos_new, err, hiflag, wrow);
        else
            merge_cta_kernel<A4_T, A4_CAP><<<(unsigned)imin64(n, (int64_t)sms * g_occ_a4), A4_T,
                                             A4_CAP * 12, s>>>(list, n, ab.mstart, P, ab.flag, vkey, vw, vw32,
                                                               ab.newdeg, ab.epos_new, err, hiflag, wrow);
        note_launches(1);
        break;
    default: break;
    }
}

void agg_merge_global(const HubGlobal &hg, const AggBuffers &ab, const int32_t *P, int32_t *vkey,
                      u64 *vw, uint32_t *vw32, int *err, int *hiflag, uint8_t *wrow, cudaStream_t s,
                      bool narrow) {
    if (hg.nhubs <= 0) return;
    // the per-community list lengths are zero between uses; cleared here too
    // so that no earlier failure can leave an append offset behind
    cudaMemsetAsync(hg.nocc, 0, sizeof(int32_t) * (size_t)hg.nhubs, s);
    if (narrow)
        mergeg_insert_narrow_kernel<<<(unsigned)imin64(hg.n_echunks, (int64_t)g_sms * g_occ_mg), HG_INSERT_THREADS,
                                      HG_INSERT_NSMEM, s>>>(hg, ab.mstart, P, ab.flag, vkey, vw, err);
    else
        mergeg_insert_kernel<<<hg.n_echunks, HG_INSERT_THREADS, HG_INSERT_SMEM, s>>>(hg, ab.mstart, P, ab.flag, vkey,
                                                                                     vw, err);
    note_launches(1);
    mergeg_emit_kernel<<<hg.n_schunks, 256, 0, s>>>(hg, ab.mstart, P, ab.flag, vkey, vw, vw32, hiflag, wrow); note_launches(1);
    mergeg_finish_kernel<<<grid_for(hg.nhubs), 256, 0, s>>>(hg, ab.mstart, P, ab.flag, ab.newdeg, ab.epos_new); note_launches(1);
}

void agg_row_bounds(const AggBuffers &ab, int32_t Vn, int32_t *start, int32_t *end, cudaStream_t s) {
    if (Vn <= 0) return;
    row_bounds_kernel<<<grid_for(Vn), 256, 0, s>>>(ab.epos_new, ab.newdeg, Vn, start, end); note_launches(1);
}

}  // namespace lv
