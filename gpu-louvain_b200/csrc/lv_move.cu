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
    u64 e_own = 0;   // weight to the own community: kept out of the table
    if (active) {
        v = list[idx];
        own = __ldg(st.comm + v);
        insert_row<(CAP > 32 ? 4 : 2), false>(g, st.comm, v, own, g.rowptr[v], g.rowend[v], lane, G,
                                               keys, vals, LG, st.err, nullptr, nullptr, e_own);
    }
    __syncwarp();
    const MoveCtx m = move_ctx(own, active ? __ldg(st.size + own) == 1 : false, st.T,
                               active ? __ldg(st.k + v) : 0, active ? __ldg(st.S + own) : 0);
    Best b = best_init(own);
    b.eo = e_own;
    if (active) eval_slots<(CAP / G > 1 ? 2 : 1), false, false>(keys, vals, nullptr, CAP, lane, G, m, st.S, st.size, b);
    group_reduce_best(m, b, G);
    u64 delta = 0;
    if (active && lane == 0) st.newc[v] = move_decision(m, b, &delta);
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
// CTA-per-vertex move kernel (84 < degree <= 4096), persistent grid-stride
// ------------------------------------------------------------------------
template <int THREADS, int CAPMAX, typename WT>
__global__ void __launch_bounds__(THREADS) move_cta_kernel(GraphView<WT> g, StateView st,
                                                           const int32_t *__restrict__ list,
                                                           int32_t n, u64 *dE) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *vals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAPMAX);
    int32_t *occ = keys + CAPMAX;   // occupied slots (at most CAPMAX / 2)
    __shared__ int32_t nocc;
    for (int s = threadIdx.x; s < CAPMAX; s += THREADS) { keys[s] = -1; vals[s] = 0; }
    if (threadIdx.x == 0) nocc = 0;
    __syncthreads();
    u64 delta_sum = 0;
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t v = list[idx];
        const int32_t own = __ldg(st.comm + v);
        const int32_t r0 = g.rowptr[v], r1 = g.rowend[v];
        int lg = ceil_log2_i(2 * (int64_t)(r1 - r0));
        lg = lg < 3 ? 3 : lg;
        u64 e_own = 0;
        insert_row<4, true>(g, st.comm, v, own, r0, r1, threadIdx.x, THREADS, keys, vals, lg, st.err,
                            occ, &nocc, e_own);
        __syncthreads();
        const MoveCtx m = move_ctx(own, __ldg(st.size + own) == 1, st.T, __ldg(st.k + v), __ldg(st.S + own));
        Best b = best_init(own);
        b.eo = e_own;
        eval_slots<4, true, true>(keys, vals, occ, nocc, threadIdx.x, THREADS, m, st.S, st.size, b);
        cta_reduce_best<THREADS>(m, b);
        if (threadIdx.x == 0) {
            u64 delta = 0;
            st.newc[v] = move_decision(m, b, &delta);
            delta_sum += delta;
            nocc = 0;
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
    const int32_t own = __ldg(st.comm + v);
    u64 e_own = 0;
    insert_row<4, false>(g, st.comm, v, own, e0, e1, threadIdx.x, HG_INSERT_THREADS, lkeys, lvals, LLG,
                         st.err, nullptr, nullptr, e_own);
    // the chunk's weight to the own community enters the table once
    e_own = warp_sum_u64(e_own);
    if ((threadIdx.x & 31) == 0 && e_own) table_insert(lkeys, lvals, LLG, own, e_own, st.err);
    __syncthreads();
    int32_t *keys = hg.keys + hg.tbl_off[h];
    u64 *vals = hg.vals + hg.tbl_off[h];
    int32_t *occ = hg.occ + hg.occ_off[h];
    const int lg = hg.tbl_lg[h];
    for (int s = threadIdx.x; s < LCAP; s += HG_INSERT_THREADS) {
        const int32_t c = lkeys[s];
        const int32_t claimed = c >= 0 ? table_insert_claim(keys, vals, lg, c, lvals[s], st.err) : -1;
        warp_append(claimed, occ, hg.nocc + h);
    }
}

__global__ void __launch_bounds__(256) hubg_eval_kernel(StateView st, HubGlobal hg) {
    const int32_t bi = blockIdx.x;
    const int32_t h = hg.schunk_hub[bi];
    const int32_t v = hg.hubs[h];
    const int32_t own = st.comm[v];
    const MoveCtx m = move_ctx(own, st.size[own] == 1, st.T, st.k[v], st.S[own]);
    int32_t *keys = hg.keys + hg.tbl_off[h];
    u64 *vals = hg.vals + hg.tbl_off[h];
    const int32_t s0 = hg.schunk_s0[bi];
    const int32_t n = min(hg.nocc[h] - s0, HG_SLOT_CHUNK);
    Best b = best_init(own);
    eval_slots<4, true, true>(keys, vals, hg.occ + hg.occ_off[h] + s0, n, threadIdx.x, 256, m, st.S,
                              st.size, b);
    cta_reduce_best<256>(m, b);
    if (threadIdx.x == 0) {
        hg.res_g[2 * bi] = (u64)__double_as_longlong(b.gd);
        hg.res_g[2 * bi + 1] = b.S;
        hg.res_c[bi] = b.c;
        hg.res_e[bi] = b.eo;
        hg.res_b[bi] = b.e;
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
    const MoveCtx m = move_ctx(own, active ? st.size[own] == 1 : false, st.T, active ? st.k[v] : 0,
                               active ? st.S[own] : 0);
    Best b = best_init(own);
    if (active) {
        for (int32_t bi = hg.hub_schunk0[h] + lane; bi < hg.hub_schunk0[h + 1]; bi += 32) {
            Best o;
            o.gd = __longlong_as_double((long long)hg.res_g[2 * bi]);
            o.S = hg.res_g[2 * bi + 1];
            o.c = hg.res_c[bi];
            o.e = hg.res_b[bi];
            o.eo = 0;
            if (better(m, o, b)) { b.gd = o.gd; b.e = o.e; b.S = o.S; b.c = o.c; }
            b.eo += hg.res_e[bi];
        }
    }
    group_reduce_best(m, b, 32);
    u64 delta = 0;
    if (active && lane == 0) {
        st.newc[v] = move_decision(m, b, &delta);
        hg.nocc[h] = 0;   // the table and its list are clean again
    }
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

// Dynamic shared memory of the CTA kernels: CAPMAX * (8 + 4) bytes of table
// plus CAPMAX / 2 occupied-slot indices.
constexpr int CTA_SLOT_BYTES = 14;
constexpr int B5_THREADS = 128, B5_CAP = 1024;
constexpr int H1_THREADS = 256, H1_CAP = 2048;
constexpr int H2_THREADS = 512, H2_CAP = 8192;

template <typename WT>
static void set_attrs_for(DeviceInfo &di) {
    auto k5 = move_cta_kernel<B5_THREADS, B5_CAP, WT>;
    auto k6 = move_cta_kernel<H1_THREADS, H1_CAP, WT>;
    auto k7 = move_cta_kernel<H2_THREADS, H2_CAP, WT>;
    cudaFuncSetAttribute(k5, cudaFuncAttributeMaxDynamicSharedMemorySize, B5_CAP * CTA_SLOT_BYTES);
    cudaFuncSetAttribute(k6, cudaFuncAttributeMaxDynamicSharedMemorySize, H1_CAP * CTA_SLOT_BYTES);
    cudaFuncSetAttribute(k7, cudaFuncAttributeMaxDynamicSharedMemorySize, H2_CAP * CTA_SLOT_BYTES);
    cudaFuncSetAttribute(hubg_insert_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         HG_INSERT_SMEM);
    int o5 = 0, o6 = 0, o7 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o5, k5, B5_THREADS, B5_CAP * CTA_SLOT_BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o6, k6, H1_THREADS, H1_CAP * CTA_SLOT_BYTES);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o7, k7, H2_THREADS, H2_CAP * CTA_SLOT_BYTES);
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
        move_cta_kernel<B5_THREADS, B5_CAP, WT><<<grid, B5_THREADS, B5_CAP * CTA_SLOT_BYTES, s>>>(g, st, list, n, dE); note_launches(1);
        break;
    }
    case CLS_H1: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_h1);
        move_cta_kernel<H1_THREADS, H1_CAP, WT><<<grid, H1_THREADS, H1_CAP * CTA_SLOT_BYTES, s>>>(g, st, list, n, dE); note_launches(1);
        break;
    }
    case CLS_H2: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_h2);
        move_cta_kernel<H2_THREADS, H2_CAP, WT><<<grid, H2_THREADS, H2_CAP * CTA_SLOT_BYTES, s>>>(g, st, list, n, dE); note_launches(1);
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
