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

// ------------------------------------------------------------------------
// group-per-vertex move kernel (degree <= 84)
// ------------------------------------------------------------------------
template <int G, int CAP, typename WT>
__global__ void __launch_bounds__(256) move_group_kernel(GraphView<WT> g, StateView st,
                                                         const int32_t *__restrict__ list,
                                                         int32_t n) {
    constexpr int GPB = 256 / G;
    constexpr int LG = (CAP == 8) ? 3 : (CAP == 16) ? 4 : (CAP == 32) ? 5 : (CAP == 64) ? 6
                     : (CAP == 128) ? 7 : 8;
    static_assert((1 << LG) == CAP, "CAP must be a power of two <= 256");
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
    if (active) {
        v = list[idx];
        own = st.comm[v];
        const int32_t r0 = g.rowptr[v], r1 = g.rowptr[v + 1];
        for (int32_t e = r0 + lane; e < r1; e += G) {
            const int32_t j = __ldg(g.col + e);
            if (j != v) table_insert(keys, vals, LG, st.comm[j], wfix(g.w, e, g.scale), st.err);
        }
    }
    __syncwarp();
    i128 best_g = 0;
    int32_t best_c = own;
    u64 e_own = 0;
    if (active) {
        MoveCtx m;
        m.own = own;
        m.own_single = st.size[own] == 1;
        m.kv = st.k[v];
        m.sown = st.S[own];
#pragma unroll
        for (int s = lane; s < CAP; s += G) {
            const int32_t c = keys[s];
            if (c >= 0) eval_candidate(c, vals[s], m, st.T, st.S, st.size, best_g, best_c, e_own);
        }
    }
    group_reduce_best(best_g, best_c, e_own, G);
    if (active && lane == 0) st.newc[v] = move_decision(best_g, best_c, e_own, st.T, own);
}

// CTA-wide reduction of (best_g, best_c, e_own); result valid in thread 0.
template <int THREADS>
__device__ __forceinline__ void cta_reduce_best(i128 &g, int32_t &c, u64 &e, int32_t fill_c) {
    constexpr int NW = THREADS / 32;
    __shared__ u64 rg_lo[NW], rg_hi[NW], re[NW];
    __shared__ int32_t rc[NW];
    group_reduce_best(g, c, e, 32);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        rg_lo[w] = (u64)g;
        rg_hi[w] = (u64)((u128)g >> 64);
        rc[w] = c;
        re[w] = e;
    }
    __syncthreads();
    if (w == 0) {
        if (l < NW) {
            g = (i128)(((u128)rg_hi[l] << 64) | (u128)rg_lo[l]);
            c = rc[l];
            e = re[l];
        } else {
            g = 0;
            c = fill_c;
            e = 0;
        }
        group_reduce_best(g, c, e, 32);
    }
}

// ------------------------------------------------------------------------
// CTA-per-vertex move kernel (84 < degree <= 4096), persistent grid-stride
// ------------------------------------------------------------------------
template <int THREADS, int CAPMAX, typename WT>
__global__ void __launch_bounds__(THREADS) move_cta_kernel(GraphView<WT> g, StateView st,
                                                           const int32_t *__restrict__ list,
                                                           int32_t n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *vals = reinterpret_cast<u64 *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAPMAX);
    for (int s = threadIdx.x; s < CAPMAX; s += THREADS) { keys[s] = -1; vals[s] = 0; }
    __syncthreads();
    for (int32_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
        const int32_t v = list[idx];
        const int32_t own = st.comm[v];
        const int32_t r0 = g.rowptr[v], r1 = g.rowptr[v + 1];
        int lg = ceil_log2_i(2 * (int64_t)(r1 - r0));
        lg = lg < 3 ? 3 : lg;
        const int cap = 1 << lg;
        for (int32_t e = r0 + threadIdx.x; e < r1; e += THREADS) {
            const int32_t j = __ldg(g.col + e);
            if (j != v) table_insert(keys, vals, lg, st.comm[j], wfix(g.w, e, g.scale), st.err);
        }
        __syncthreads();
        MoveCtx m;
        m.own = own;
        m.own_single = st.size[own] == 1;
        m.kv = st.k[v];
        m.sown = st.S[own];
        i128 best_g = 0;
        int32_t best_c = own;
        u64 e_own = 0;
        for (int s = threadIdx.x; s < cap; s += THREADS) {
            const int32_t c = keys[s];
            if (c >= 0) {
                eval_candidate(c, vals[s], m, st.T, st.S, st.size, best_g, best_c, e_own);
                keys[s] = -1;
                vals[s] = 0;
            }
        }
        cta_reduce_best<THREADS>(best_g, best_c, e_own, own);
        if (threadIdx.x == 0) st.newc[v] = move_decision(best_g, best_c, e_own, st.T, own);
        __syncthreads();
    }
}

// ------------------------------------------------------------------------
// global-table hub path (degree > 4096)
// ------------------------------------------------------------------------
template <typename WT>
__global__ void __launch_bounds__(256) hubg_insert_kernel(GraphView<WT> g, StateView st,
                                                          HubGlobal hg) {
    const int32_t h = hg.echunk_hub[blockIdx.x];
    const int32_t v = hg.hubs[h];
    const int32_t r1 = g.rowptr[v + 1];
    const int32_t e0 = g.rowptr[v] + hg.echunk_e0[blockIdx.x];
    const int32_t e1 = min(e0 + HG_EDGE_CHUNK, r1);
    int32_t *keys = hg.keys + hg.tbl_off[h];
    u64 *vals = hg.vals + hg.tbl_off[h];
    const int lg = hg.tbl_lg[h];
    for (int32_t e = e0 + threadIdx.x; e < e1; e += 256) {
        const int32_t j = __ldg(g.col + e);
        if (j != v) table_insert(keys, vals, lg, st.comm[j], wfix(g.w, e, g.scale), st.err);
    }
}

__global__ void __launch_bounds__(256) hubg_eval_kernel(StateView st, HubGlobal hg) {
    const int32_t b = blockIdx.x;
    const int32_t h = hg.schunk_hub[b];
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
    const int32_t s0 = hg.schunk_s0[b];
    const int32_t s1 = min(s0 + HG_SLOT_CHUNK, cap);
    i128 best_g = 0;
    int32_t best_c = own;
    u64 e_own = 0;
    for (int32_t s = s0 + threadIdx.x; s < s1; s += 256) {
        const int32_t c = keys[s];
        if (c >= 0) {
            eval_candidate(c, vals[s], m, st.T, st.S, st.size, best_g, best_c, e_own);
            keys[s] = -1;
            vals[s] = 0;
        }
    }
    cta_reduce_best<256>(best_g, best_c, e_own, own);
    if (threadIdx.x == 0) {
        hg.res_g[2 * b] = (u64)best_g;
        hg.res_g[2 * b + 1] = (u64)((u128)best_g >> 64);
        hg.res_c[b] = best_c;
        hg.res_e[b] = e_own;
    }
}

__global__ void __launch_bounds__(256) hubg_final_kernel(StateView st, HubGlobal hg) {
    const int32_t h = (blockIdx.x * 256 + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const bool active = h < hg.nhubs;
    int32_t v = 0, own = 0;
    i128 best_g = 0;
    int32_t best_c = 0;
    u64 e_own = 0;
    if (active) {
        v = hg.hubs[h];
        own = st.comm[v];
        best_c = own;
        for (int32_t b = hg.hub_schunk0[h] + lane; b < hg.hub_schunk0[h + 1]; b += 32) {
            const i128 og = (i128)(((u128)hg.res_g[2 * b + 1] << 64) | (u128)hg.res_g[2 * b]);
            const int32_t oc = hg.res_c[b];
            if (better(og, oc, best_g, best_c)) { best_g = og; best_c = oc; }
            e_own += hg.res_e[b];
        }
    }
    group_reduce_best(best_g, best_c, e_own, 32);
    if (active && lane == 0) st.newc[v] = move_decision(best_g, best_c, e_own, st.T, own);
}

// ------------------------------------------------------------------------
// commit of one sub-round (updateVertexCommunity + Sigma_tot update)
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) commit_kernel(StateView st, const int32_t *__restrict__ list,
                                                     int32_t n, u64 *moves) {
    const int32_t i = blockIdx.x * 256 + threadIdx.x;
    bool mv = false;
    if (i < n) {
        const int32_t v = list[i];
        const int32_t nc = st.newc[v], oc = st.comm[v];
        if (nc != oc) {
            mv = true;
            st.comm[v] = nc;
            atomicAdd(st.size + nc, 1);
            atomicSub(st.size + oc, 1);
            const u64 kv = st.k[v];
            atomicAdd(st.S + nc, kv);
            atomicAdd(st.S + oc, (u64)0 - kv);
        }
    }
    const unsigned b = __ballot_sync(FULL, mv);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(moves, (u64)__popc(b));
}

// ------------------------------------------------------------------------
// row reductions: k_i (mode 0) and sum_i e_{i->C(i)} (mode 1)
// ------------------------------------------------------------------------
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
}

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
        const int32_t r0 = g.rowptr[v], r1 = g.rowptr[v + 1];
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
        const int32_t r0 = g.rowptr[v], r1 = g.rowptr[v + 1];
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
                       int32_t n, const HubGlobal &hg, const DeviceInfo &di, cudaStream_t s) {
    if (cls != CLS_HG && n <= 0) return;
    switch (cls) {
    case CLS_B0: move_group_kernel<4, 8, WT><<<nblocks(n, 64), 256, 0, s>>>(g, st, list, n); note_launches(1); break;
    case CLS_B1: move_group_kernel<8, 16, WT><<<nblocks(n, 32), 256, 0, s>>>(g, st, list, n); note_launches(1); break;
    case CLS_B2: move_group_kernel<16, 32, WT><<<nblocks(n, 16), 256, 0, s>>>(g, st, list, n); note_launches(1); break;
    case CLS_B3: move_group_kernel<32, 64, WT><<<nblocks(n, 8), 256, 0, s>>>(g, st, list, n); note_launches(1); break;
    case CLS_B4: move_group_kernel<32, 256, WT><<<nblocks(n, 8), 256, 0, s>>>(g, st, list, n); note_launches(1); break;
    case CLS_B5: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_b5);
        move_cta_kernel<B5_THREADS, B5_CAP, WT><<<grid, B5_THREADS, B5_CAP * 12, s>>>(g, st, list, n); note_launches(1);
        break;
    }
    case CLS_H1: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_h1);
        move_cta_kernel<H1_THREADS, H1_CAP, WT><<<grid, H1_THREADS, H1_CAP * 12, s>>>(g, st, list, n); note_launches(1);
        break;
    }
    case CLS_H2: {
        unsigned grid = (unsigned)imin64(n, (int64_t)di.sms * di.occ_h2);
        move_cta_kernel<H2_THREADS, H2_CAP, WT><<<grid, H2_THREADS, H2_CAP * 12, s>>>(g, st, list, n); note_launches(1);
        break;
    }
    case CLS_HG: {
        if (hg.nhubs <= 0) return;
        hubg_insert_kernel<WT><<<hg.n_echunks, 256, 0, s>>>(g, st, hg); note_launches(1);
        hubg_eval_kernel<<<hg.n_schunks, 256, 0, s>>>(st, hg); note_launches(1);
        hubg_final_kernel<<<nblocks((int64_t)hg.nhubs * 32, 256), 256, 0, s>>>(st, hg); note_launches(1);
        break;
    }
    default: break;
    }
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
                                       const DeviceInfo &, cudaStream_t);
template void launch_move_class<u64>(int, const GraphView<u64> &, const StateView &,
                                     const int32_t *, int32_t, const HubGlobal &,
                                     const DeviceInfo &, cudaStream_t);
template void launch_row_reduce<float>(int, int, const GraphView<float> &, const int32_t *, u64 *,
                                       u64 *, const int32_t *, int32_t, const DeviceInfo &,
                                       cudaStream_t);
template void launch_row_reduce<u64>(int, int, const GraphView<u64> &, const int32_t *, u64 *,
                                     u64 *, const int32_t *, int32_t, const DeviceInfo &,
                                     cudaStream_t);

}  // namespace lv
