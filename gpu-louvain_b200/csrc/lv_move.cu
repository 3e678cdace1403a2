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
    if (G == 32) {
        // one warp per vertex: uniform trip count, warp-aggregated inserts
        int32_t r0 = 0, r1 = 0;
        if (active) {
            v = list[idx];
            own = st.comm[v];
            r0 = g.rowptr[v];
            r1 = g.rowend[v];
        }
        for (int32_t base = r0; base < r1; base += 32) {
            const int32_t e = base + lane;
            bool valid = e < r1;
            int32_t c = 0;
            u64 w = 0;
            if (valid) {
                const int32_t j = __ldg(g.col + e);
                valid = j != v;
                if (valid) { c = st.comm[j]; w = wfix(g.w, e, g.scale); }
            }
            warp_insert(keys, vals, LG, valid, c, w, st.err);
        }
    } else if (active) {
        v = list[idx];
        own = st.comm[v];
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        for (int32_t e = r0 + lane; e < r1; e += G) {
            const int32_t j = __ldg(g.col + e);
            if (j != v) table_insert(keys, vals, LG, st.comm[j], wfix(g.w, e, g.scale), st.err);
        }
    }
    __syncwarp();
    Best b = best_init(own);
    if (active) {
        MoveCtx m;
        m.own = own;
        m.own_single = st.size[own] == 1;
        m.kv = st.k[v];
        m.sown = st.S[own];
#pragma unroll
        for (int s = lane; s < CAP; s += G) {
            const int32_t c = keys[s];
            if (c >= 0) eval_candidate(c, vals[s], m, st.T, st.S, st.size, b);
        }
    }
    group_reduce_best(b, G);
    u64 delta = 0;
    if (active && lane == 0) st.newc[v] = move_decision(b, st.T, own, &delta);
    block_add_total<256>(delta, dE);
}

// CTA-wide reduction of a Best; the result is valid in thread 0.
template <int THREADS>
__device__ __forceinline__ void cta_reduce_best(Best &b, int32_t fill_c) {
    constexpr int NW = THREADS / 32;
    __shared__ u64 rg_lo[NW], rg_hi[NW], reb[NW], reo[NW];
    __shared__ int32_t rc[NW];
    group_reduce_best(b, 32);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        rg_lo[w] = (u64)b.g;
        rg_hi[w] = (u64)((u128)b.g >> 64);
        rc[w] = b.c;
        reb[w] = b.eb;
        reo[w] = b.eo;
    }
    __syncthreads();
    if (w == 0) {
        if (l < NW) {
            b.g = (i128)(((u128)rg_hi[l] << 64) | (u128)rg_lo[l]);
            b.c = rc[l];
            b.eb = reb[l];
            b.eo = reo[l];
        } else {
            b = best_init(fill_c);
        }
        group_reduce_best(b, 32);
    }
}

// ------------------------------------------------------------------------
// CTA-per-vertex move kernel (84 < degree <= 4096), persistent grid-stride
// ------------------------------------------------------------------------
template <int THREADS, int CAPMAX, typename WT>
__global__ void __launch_bounds__(THREADS) move_cta_kernel(GraphView<WT> g, StateView st,
                                                           const int32_t *__restrict__ list,
                                                           int32_t n, u64 *dE) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *vals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAPMAX);
    for (int s = threadIdx.x; s < CAPMAX; s += THREADS) { keys[s] = -1; vals[s] = 0; }
    __syncthreads();
    u64 delta_sum = 0;
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t v = list[idx];
        const int32_t own = st.comm[v];
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        int lg = ceil_log2_i(2 * (int64_t)(r1 - r0));
        lg = lg < 3 ? 3 : lg;
        const int cap = 1 << lg;
        for (int32_t base = r0; base < r1; base += THREADS) {
            const int32_t e = base + threadIdx.x;
            bool valid = e < r1;
            int32_t c = 0;
            u64 w = 0;
            if (valid) {
                const int32_t j = __ldg(g.col + e);
                valid = j != v;
                if (valid) { c = st.comm[j]; w = wfix(g.w, e, g.scale); }
            }
            warp_insert(keys, vals, lg, valid, c, w, st.err);
        }
        __syncthreads();
        MoveCtx m;
        m.own = own;
        m.own_single = st.size[own] == 1;
        m.kv = st.k[v];
        m.sown = st.S[own];
        Best b = best_init(own);
        for (int s = threadIdx.x; s < cap; s += THREADS) {
            const int32_t c = keys[s];
            if (c >= 0) {
                eval_candidate(c, vals[s], m, st.T, st.S, st.size, b);
                keys[s] = -1;
                vals[s] = 0;
            }
        }
        cta_reduce_best<THREADS>(b, own);
        if (threadIdx.x == 0) {
            u64 delta = 0;
            st.newc[v] = move_decision(b, st.T, own, &delta);
            delta_sum += delta;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && delta_sum) atomicAdd(dE, delta_sum);
}

// ------------------------------------------------------------------------
// global-table hub path (degree > 4096)
// ------------------------------------------------------------------------
// One CTA per chunk of HG_EDGE_CHUNK edges of one hub: the chunk is first
// reduced in a shared table (2 * chunk slots), then each distinct key is
// added once to the hub's global table.
template <typename WT>
__global__ void __launch_bounds__(HG_INSERT_THREADS) hubg_insert_kernel(GraphView<WT> g,
                                                                        StateView st, HubGlobal hg) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LCAP = 2 * HG_EDGE_CHUNK;
    constexpr int LLG = ilog2_c(LCAP);
    u64 *lvals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *lkeys = reinterpret_cast<int32_t *>(lvals + LCAP);
    for (int s = threadIdx.x; s < LCAP; s += HG_INSERT_THREADS) { lkeys[s] = -1; lvals[s] = 0; }
    __syncthreads();
    const int32_t h = hg.echunk_hub[blockIdx.x];
    const int32_t v = hg.hubs[h];
    const int32_t r1 = g.rowend[v];
    const int32_t e0 = g.rowptr[v] + hg.echunk_e0[blockIdx.x];
    const int32_t e1 = min(e0 + HG_EDGE_CHUNK, r1);
    for (int32_t base = e0; base < e1; base += HG_INSERT_THREADS) {
        const int32_t e = base + threadIdx.x;
        bool valid = e < e1;
        int32_t c = 0;
        u64 w = 0;
        if (valid) {
            const int32_t j = __ldg(g.col + e);
            valid = j != v;
            if (valid) { c = st.comm[j]; w = wfix(g.w, e, g.scale); }
        }
        warp_insert(lkeys, lvals, LLG, valid, c, w, st.err);
    }
    __syncthreads();
    int32_t *keys = hg.keys + hg.tbl_off[h];
    u64 *vals = hg.vals + hg.tbl_off[h];
    const int lg = hg.tbl_lg[h];
    for (int s = threadIdx.x; s < LCAP; s += HG_INSERT_THREADS) {
        const int32_t c = lkeys[s];
        if (c >= 0) table_insert(keys, vals, lg, c, lvals[s], st.err);
    }
}

__global__ void __launch_bounds__(256) hubg_eval_kernel(StateView st, HubGlobal hg) {
    const int32_t bi = blockIdx.x;
    const int32_t h = hg.schunk_hub[bi];
    const int32_t v = hg.hubs[h];
    const int32_t own = st.comm[v];
    MoveCtx m;
    m.own = own;
    m.own_single = st.size[own] == 1;
    m.kv = st.k[v];
    m.sown = st.S[own];
    int32_t *keys = hg.keys + hg.tbl_off[h];
    u64 *vals = hg.vals + hg.tbl_off[h];
    const int32_t cap = 1 << hg.tbl_lg[h];
    const int32_t s0 = hg.schunk_s0[bi];
    const int32_t s1 = min(s0 + HG_SLOT_CHUNK, cap);
    Best b = best_init(own);
    for (int32_t s = s0 + threadIdx.x; s < s1; s += 256) {
        const int32_t c = keys[s];
        if (c >= 0) {
            eval_candidate(c, vals[s], m, st.T, st.S, st.size, b);
            keys[s] = -1;
            vals[s] = 0;
        }
    }
    cta_reduce_best<256>(b, own);
    if (threadIdx.x == 0) {
        hg.res_g[2 * bi] = (u64)b.g;
        hg.res_g[2 * bi + 1] = (u64)((u128)b.g >> 64);
        hg.res_c[bi] = b.c;
        hg.res_e[bi] = b.eo;
        hg.res_b[bi] = b.eb;
    }
}

__global__ void __launch_bounds__(256) hubg_final_kernel(StateView st, HubGlobal hg, u64 *dE) {
    const int32_t h = (blockIdx.x * 256 + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const bool active = h < hg.nhubs;
    int32_t v = 0, own = 0;
    if (active) {
        v = hg.hubs[h];
        own = st.comm[v];
    }
    Best b = best_init(own);
    if (active) {
        for (int32_t bi = hg.hub_schunk0[h] + lane; bi < hg.hub_schunk0[h + 1]; bi += 32) {
            const i128 og = (i128)(((u128)hg.res_g[2 * bi + 1] << 64) | (u128)hg.res_g[2 * bi]);
            const int32_t oc = hg.res_c[bi];
            if (better(og, oc, b.g, b.c)) { b.g = og; b.c = oc; b.eb = hg.res_b[bi]; }
            b.eo += hg.res_e[bi];
        }
    }
    group_reduce_best(b, 32);
    u64 delta = 0;
    if (active && lane == 0) st.newc[v] = move_decision(b, st.T, own, &delta);
    block_add_total<256>(delta, dE);
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
                if (cj != nj) acc += pair_correction(cu, nu, cj, nj, wfix(g.w, e, g.scale));
            }
        }
    }
    block_add_total<256>(acc, dE);
}

template <int T, typename WT>
__global__ void __launch_bounds__(T) corr_cta_kernel(GraphView<WT> g, const int32_t *__restrict__ comm,
                                                     const int32_t *__restrict__ newc,
                                                     const int32_t *__restrict__ list, int32_t n,
                                                     u64 *dE) {
    u64 acc = 0;
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t u = list[idx];
        const int32_t cu = comm[u], nu = newc[u];
        if (cu == nu) continue;
        const int32_t r0 = g.rowptr[u], r1 = g.rowend[u];
        for (int32_t e = r0 + threadIdx.x; e < r1; e += T) {
            const int32_t j = __ldg(g.col + e);
            if (j == u) continue;
            const int32_t cj = comm[j], nj = newc[j];
            if (cj != nj) acc += pair_correction(cu, nu, cj, nj, wfix(g.w, e, g.scale));
        }
    }
    block_add_total<T>(acc, dE);
}

// ------------------------------------------------------------------------
// commit of one sub-round (updateVertexCommunity + Sigma_tot update)
// ------------------------------------------------------------------------
// Size and Sigma_tot updates are aggregated per warp by destination (and by
// source) community, so many vertices joining one community in a sub-round
// cost one atomic per warp.
__global__ void __launch_bounds__(256) commit_kernel(StateView st, const int32_t *__restrict__ list,
                                                     int32_t n, u64 *moves) {
    const int32_t i = blockIdx.x * 256 + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool mv = false;
    int32_t v = 0, nc = 0, oc = 0;
    u64 kv = 0;
    if (i < n) {
        v = list[i];
        nc = st.newc[v];
        oc = st.comm[v];
        mv = nc != oc;
        if (mv) {
            st.comm[v] = nc;
            kv = st.k[v];
        }
    }
    const unsigned act = __ballot_sync(FULL, mv);
    if (mv) {
        unsigned peers = __match_any_sync(act, nc);
        u64 sum = redux_add_u64(peers, kv);
        if (lane == __ffs(peers) - 1) {
            atomicAdd(st.size + nc, __popc(peers));
            atomicAdd(st.S + nc, sum);
        }
        peers = __match_any_sync(act, oc);
        sum = redux_add_u64(peers, kv);
        if (lane == __ffs(peers) - 1) {
            atomicSub(st.size + oc, __popc(peers));
            atomicAdd(st.S + oc, (u64)0 - sum);
        }
    }
    block_add_total<256>(mv ? 1ull : 0ull, moves);
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
                if (comm[__ldg(g.col + e)] == own) acc += wfix(g.w, e, g.scale);
            } else {
                acc += wfix(g.w, e, g.scale);
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
                if (comm[__ldg(g.col + e)] == own) acc += wfix(g.w, e, g.scale);
            } else {
                acc += wfix(g.w, e, g.scale);
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

// Dynamic shared memory of the CTA kernels: CAPMAX * (8 + 4) bytes.
constexpr int B5_THREADS = 128, B5_CAP = 1024;
constexpr int H1_THREADS = 256, H1_CAP = 2048;
constexpr int H2_THREADS = 512, H2_CAP = 8192;

template <typename WT>
static void set_attrs_for(DeviceInfo &di) {
    auto k5 = move_cta_kernel<B5_THREADS, B5_CAP, WT>;
    auto k6 = move_cta_kernel<H1_THREADS, H1_CAP, WT>;
    auto k7 = move_cta_kernel<H2_THREADS, H2_CAP, WT>;
    cudaFuncSetAttribute(k5, cudaFuncAttributeMaxDynamicSharedMemorySize, B5_CAP * 12);
    cudaFuncSetAttribute(k6, cudaFuncAttributeMaxDynamicSharedMemorySize, H1_CAP * 12);
    cudaFuncSetAttribute(k7, cudaFuncAttributeMaxDynamicSharedMemorySize, H2_CAP * 12);
    cudaFuncSetAttribute(hubg_insert_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         HG_INSERT_SMEM);
    int o5 = 0, o6 = 0, o7 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o5, k5, B5_THREADS, B5_CAP * 12);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o6, k6, H1_THREADS, H1_CAP * 12);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o7, k7, H2_THREADS, H2_CAP * 12);
    di.occ_b5 = o5 > 0 ? o5 : 1;
    di.occ_h1 = o6 > 0 ? o6 : 1;
    di.occ_h2 = o7 > 0 ? o7 : 1;
}

void init_kernel_attributes(DeviceInfo &di) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev);
    set_attrs_for<u64>(di);
    set_attrs_for<float>(di);
}

template <typename WT>
void launch_move_class(int cls, const GraphView<WT> &g, const StateView &st, const int32_t *list,
                       int32_t n, const HubGlobal &hg, const DeviceInfo &di, u64 *dE,
                       cudaStream_t s) {
    if (cls != CLS_HG && n <= 0) return;
    switch (cls) {
    case CLS_B0: move_group_kernel<4, 8, WT><<<nblocks(n, 64), 256, 0, s>>>(g, st, list, n, dE); note_launches(1); break;
    case CLS_B1: move_group_kernel<8, 16, WT><<<nblocks(n, 32), 256, 0, s>>>(g, st, list, n, dE); note_launches(1); break;
    case CLS_B2: move_group_kernel<16, 32, WT><<<nblocks(n, 16), 256, 0, s>>>(g, st, list, n, dE); note_launches(1); break;
    case CLS_B3: move_group_kernel<32, 64, WT><<<nblocks(n, 8), 256, 0, s>>>(g, st, list, n, dE); note_launches(1); break;
    case CLS_B4: move_group_kernel<32, 256, WT><<<nblocks(n, 8), 256, 0, s>>>(g, st, list, n, dE); note_launches(1); break;
    case CLS_B5: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_b5);
        move_cta_kernel<B5_THREADS, B5_CAP, WT><<<grid, B5_THREADS, B5_CAP * 12, s>>>(g, st, list, n, dE); note_launches(1);
        break;
    }
    case CLS_H1: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_h1);
        move_cta_kernel<H1_THREADS, H1_CAP, WT><<<grid, H1_THREADS, H1_CAP * 12, s>>>(g, st, list, n, dE); note_launches(1);
        break;
    }
    case CLS_H2: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_h2);
        move_cta_kernel<H2_THREADS, H2_CAP, WT><<<grid, H2_THREADS, H2_CAP * 12, s>>>(g, st, list, n, dE); note_launches(1);
        break;
    }
    case CLS_HG: {
        if (hg.nhubs <= 0) return;
        hubg_insert_kernel<WT><<<hg.n_echunks, HG_INSERT_THREADS, HG_INSERT_SMEM, s>>>(g, st, hg); note_launches(1);
        hubg_eval_kernel<<<hg.n_schunks, 256, 0, s>>>(st, hg); note_launches(1);
        hubg_final_kernel<<<nblocks((int64_t)hg.nhubs * 32, 256), 256, 0, s>>>(st, hg, dE); note_launches(1);
        break;
    }
    default: break;
    }
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
        corr_cta_kernel<128, WT><<<(unsigned)imin64(n, (int64_t)di.sms * 16), 128, 0, s>>>(g, st.comm, st.newc, list, n, dE);
        break;
    case CLS_H1:
        corr_cta_kernel<256, WT><<<(unsigned)imin64(n, (int64_t)di.sms * 8), 256, 0, s>>>(g, st.comm, st.newc, list, n, dE);
        break;
    default:
        corr_cta_kernel<512, WT><<<(unsigned)imin64(n, (int64_t)di.sms * 4), 512, 0, s>>>(g, st.comm, st.newc, list, n, dE);
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
                                       const int32_t *, int32_t, const HubGlobal &,
                                       const DeviceInfo &, u64 *, cudaStream_t);
template void launch_move_class<u64>(int, const GraphView<u64> &, const StateView &,
                                     const int32_t *, int32_t, const HubGlobal &,
                                     const DeviceInfo &, u64 *, cudaStream_t);
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

}  // namespace lv
