// lv_prims.cu -- device primitives of the engine: exclusive scan, degree
// classification, state initialisation, weight analysis and CSR checks.
//
// These replace the Thrust calls of the reference (sequence / fill /
// partition / exclusive_scan / reduce at modularity_optimisation.cu:290-349
// and community_aggregation.cu:267-343, utils.cu:84-87).  The degree
// classification runs once per level on the device (the reference partitions
// the vertex list 7 times per sweep with a predicate that reads CSR offsets
// from pinned host memory).
#include <atomic>

#include <cub/cub.cuh>

#include "lv_internal.h"

namespace lv {

namespace {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Exclusive scan of one value per thread across the block; returns the
// thread's exclusive prefix and writes the block total to *total.
template <int THREADS>
__device__ __forceinline__ int32_t block_exclusive_scan(int32_t x, int32_t *total) {
    __shared__ int32_t wsum[THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t incl = x;
    for (int off = 1; off < 32; off <<= 1) {
        int32_t y = __shfl_up_sync(FULL, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int32_t t = lane < THREADS / 32 ? wsum[lane] : 0;
        int32_t ti = t;
        for (int off = 1; off < 32; off <<= 1) {
            int32_t y = __shfl_up_sync(FULL, ti, off);
            if (lane >= off) ti += y;
        }
        if (lane < THREADS / 32) wsum[lane] = ti - t;
        if (lane == 31) *total = ti;
    }
    __syncthreads();
    const int32_t r = wsum[w] + incl - x;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_partials_kernel(const int32_t *in, int64_t n,
                                                                     int32_t *partials) {
    __shared__ int32_t tot;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
        if (base + i < n) s += in[base + i];
    block_exclusive_scan<SCAN_THREADS>(s, &tot);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) scan_top_kernel(int32_t *partials, int64_t nb,
                                                        int32_t *total_dev) {
    __shared__ int32_t tot;
    int32_t running = 0;
    for (int64_t base = 0; base < nb; base += 1024) {
        const int64_t i = base + threadIdx.x;
        const int32_t x = i < nb ? partials[i] : 0;
        const int32_t ex = block_exclusive_scan<1024>(x, &tot);
        if (i < nb) partials[i] = running + ex;
        running += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total_dev) *total_dev = running;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_apply_kernel(const int32_t *in, int32_t *out,
                                                                  int64_t n,
                                                                  const int32_t *partials) {
    __shared__ int32_t tot;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int32_t v[SCAN_ITEMS];
    int32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    int32_t run = block_exclusive_scan<SCAN_THREADS>(s, &tot) + partials[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

// ---- degree classes ----
// counts[0..NCLS) = vertices per class; counts[NCLS..) reinterpreted as
// uint64 edge totals per class.
__global__ void __launch_bounds__(256) class_count_kernel(const int32_t *__restrict__ rowptr,
                                                          const int32_t *__restrict__ rowend,
                                                          int32_t V, int32_t giant_degree, int32_t *counts) {
    __shared__ int32_t c[NCLS];
    __shared__ u64 es[NCLS];
    if (threadIdx.x < NCLS) { c[threadIdx.x] = 0; es[threadIdx.x] = 0; }
    __syncthreads();
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256) {
        const int32_t d = rowend[v] - rowptr[v];
        const int cls = degree_class(d, giant_degree);
        if (cls >= 0) {
            atomicAdd(c + cls, 1);
            atomicAdd(es + cls, (u64)d);
        }
    }
    __syncthreads();
    u64 *esum = reinterpret_cast<u64 *>(counts + NCLS + (NCLS & 1));
    if (threadIdx.x < NCLS && c[threadIdx.x]) {
        atomicAdd(counts + threadIdx.x, c[threadIdx.x]);
        atomicAdd(esum + threadIdx.x, es[threadIdx.x]);
    }
}

struct ClassOffsets {
    int32_t off[NCLS];
};

// Also sets the move phase's fallback hint: at the start of a level every
// vertex is a singleton community, so a row with more than warp_limit
// entries has (up to duplicates) more distinct neighbour communities.
__global__ void __launch_bounds__(256) class_scatter_kernel(const int32_t *__restrict__ rowptr,
                                                            const int32_t *__restrict__ rowend,
                                                            int32_t V, int32_t giant_degree, int32_t warp_limit,
                                                            ClassOffsets offs, int32_t *cursors, int32_t *list,
                                                            uint8_t *hint) {
    const int lane = threadIdx.x & 31;
    for (int32_t base = blockIdx.x * 256; base < V; base += gridDim.x * 256) {
        const int32_t v = base + threadIdx.x;
        const int32_t d = v < V ? rowend[v] - rowptr[v] : 0;
        const int cls = v < V ? degree_class(d, giant_degree) : -1;
        if (v < V) hint[v] = d > warp_limit ? 1 : 0;
        const unsigned peers = __match_any_sync(FULL, cls);
        const int leader = __ffs(peers) - 1;
        int32_t pos = 0;
        if (lane == leader && cls >= 0) pos = atomicAdd(cursors + cls, __popc(peers));
        pos = __shfl_sync(FULL, pos, leader);
        if (cls >= 0) {
            const int rank = __popc(peers & ((1u << lane) - 1u));
            list[offs.off[cls] + pos + rank] = v;
        }
    }
}

__global__ void fill_i32_kernel(int32_t *p, int64_t n, int32_t v) {
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        p[i] = v;
}

__global__ void iota_i32_kernel(int32_t *p, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        p[i] = (int32_t)i;
}

__global__ void level_init_kernel(int32_t *comm, int32_t *newc, int32_t *size, const u64 *k,
                                  u64 *S, int32_t V) {
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256) {
        comm[v] = v;
        newc[v] = v;
        size[v] = 1;
        S[v] = k[v];
    }
}

__global__ void zero_state_kernel(int32_t *size, u64 *S, int32_t V) {
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256) {
        size[v] = 0;
        S[v] = 0;
    }
}

__global__ void set_comm_kernel(const int32_t *comm_in, int32_t *comm, int32_t *newc,
                                int32_t *size, const u64 *k, u64 *S, int32_t V, int *err) {
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256) {
        const int32_t c = comm_in[v];
        if (c < 0 || c >= V) {
            atomicOr(err, DEVERR_BAD_STATE);
            continue;
        }
        comm[v] = c;
        newc[v] = c;
        atomicAdd(size + c, 1);
        atomicAdd(S + c, k[v]);
    }
}

__global__ void compose_map_kernel(int32_t *orig2comm, const int32_t *map, int32_t V0) {
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V0; v += gridDim.x * 256)
        orig2comm[v] = map[orig2comm[v]];
}

template <typename WT>
__global__ void to_fixed_kernel(const WT *w, int64_t E, double scale, int64_t *out) {
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < E; e += (int64_t)gridDim.x * 256)
        out[e] = (int64_t)wfix(w, e, scale);
}

// Fractional bits / magnitude / validity of float weights; the same rule as
// the oracle's weight_bits().
__global__ void weight_scan_kernel(const float *__restrict__ w, int64_t E, int32_t *out) {
    int need = 0, top = 0, bad = 0;
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < E; e += (int64_t)gridDim.x * 256) {
        int n, t, b;
        weight_bits_dev(w[e], n, t, b);
        need = max(need, n);
        top = max(top, t);
        bad |= b;
    }
    for (int off = 16; off > 0; off >>= 1) {
        need = max(need, __shfl_xor_sync(FULL, need, off));
        top = max(top, __shfl_xor_sync(FULL, top, off));
        bad |= __shfl_xor_sync(FULL, bad, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (need) atomicMax(out + 0, need);
        if (top) atomicMax(out + 1, top);
        if (bad) atomicOr(out + 2, bad);
    }
}

__global__ void total_weight_kernel(const float *__restrict__ w, int64_t E, double scale,
                                    u64 *total) {
    __shared__ u64 part[8];
    u64 acc = 0;
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < E; e += (int64_t)gridDim.x * 256)
        acc += wfix(w, e, scale);
    acc = warp_sum_u64(acc);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        u64 y = 0;
        for (int i = 0; i < 8; ++i) y += part[i];
        if (y) atomicAdd(total, y);
    }
}

__global__ void validate_csr_kernel(const int32_t *__restrict__ rowptr,
                                    const int32_t *__restrict__ col, int32_t V, int64_t E,
                                    int *err) {
    const int64_t tid = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * 256;
    int bad = 0;
    if (tid == 0 && (rowptr[0] != 0 || (int64_t)rowptr[V] != E)) bad |= 1;
    for (int64_t v = tid; v < V; v += stride)
        if (rowptr[v + 1] < rowptr[v]) bad |= 1;
    for (int64_t e = tid; e < E; e += stride) {
        const int32_t c = col[e];
        if (c < 0 || c >= V) bad |= 2;
    }
    if (bad) atomicOr(err, bad);
}

inline unsigned grid_for(int64_t n, int64_t cap = 148 * 16) {
    int64_t b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (unsigned)(b < cap ? b : cap);
}

}  // namespace

static std::atomic<long long> g_launches{0};
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_total() { return g_launches.load(std::memory_order_relaxed); }

int64_t scan_tmp_elems(int64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

void scan_exclusive_i32(const int32_t *in, int32_t *out, int64_t n, int32_t *total_dev,
                        int32_t *tmp, cudaStream_t s) {
    if (n <= 0) {
        if (total_dev) cudaMemsetAsync(total_dev, 0, sizeof(int32_t), s);
        return;
    }
    const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    scan_partials_kernel<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, tmp); note_launches(1);
    scan_top_kernel<<<1, 1024, 0, s>>>(tmp, nb, total_dev); note_launches(1);
    scan_apply_kernel<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, tmp); note_launches(1);
}

void launch_class_count(const int32_t *rowptr, const int32_t *rowend, int32_t V, int32_t giant_degree,
                        int32_t *counts, cudaStream_t s) {
    cudaMemsetAsync(counts, 0, sizeof(int32_t) * CLASS_COUNT_WORDS, s);
    if (V <= 0) return;
    class_count_kernel<<<grid_for(V), 256, 0, s>>>(rowptr, rowend, V, giant_degree, counts); note_launches(1);
}

void launch_class_scatter(const int32_t *rowptr, const int32_t *rowend, int32_t V, int32_t giant_degree,
                          int32_t warp_limit, const int32_t *offsets, int32_t *cursors, int32_t *list,
                          uint8_t *hint, cudaStream_t s) {
    cudaMemsetAsync(cursors, 0, sizeof(int32_t) * NCLS, s);
    if (V <= 0) return;
    ClassOffsets o;
    for (int c = 0; c < NCLS; ++c) o.off[c] = offsets[c];
    class_scatter_kernel<<<grid_for(V), 256, 0, s>>>(rowptr, rowend, V, giant_degree, warp_limit, o, cursors, list,
                                                     hint);
    note_launches(1);
}

namespace {
__global__ void degree_key_kernel(const int32_t *__restrict__ rowptr, const int32_t *__restrict__ rowend,
                                  const int32_t *__restrict__ list, int32_t n, int32_t maxdeg, int32_t *keys) {
    for (int32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const int32_t v = list[i];
        const int32_t d = rowend[v] - rowptr[v];
        keys[i] = maxdeg - (d < maxdeg ? d : maxdeg);
    }
}

int key_bits(int32_t maxdeg) {
    int b = 1;
    while (b < 31 && ((int64_t)1 << b) <= (int64_t)maxdeg) ++b;
    return b;
}
}  // namespace

size_t sort_by_degree_temp_bytes(int32_t n, int32_t maxdeg) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const int32_t *)nullptr, (int32_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int64_t)n, 0, key_bits(maxdeg));
    return bytes;
}

void sort_by_degree_desc(const int32_t *rowptr, const int32_t *rowend, int32_t *list, int32_t n, int32_t maxdeg,
                         int32_t *keys, int32_t *keys_alt, int32_t *vals_alt, void *temp, size_t temp_bytes,
                         cudaStream_t s) {
    if (n <= 1) return;
    degree_key_kernel<<<grid_for(n), 256, 0, s>>>(rowptr, rowend, list, n, maxdeg, keys);
    note_launches(1);
    cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_alt, list, vals_alt, (int64_t)n, 0, key_bits(maxdeg),
                                    s);
    cudaMemcpyAsync(list, vals_alt, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
}

void launch_fill_i32(int32_t *p, int64_t n, int32_t v, cudaStream_t s) {
    if (n <= 0) return;
    fill_i32_kernel<<<grid_for(n), 256, 0, s>>>(p, n, v); note_launches(1);
}

void launch_iota_i32(int32_t *p, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    iota_i32_kernel<<<grid_for(n), 256, 0, s>>>(p, n); note_launches(1);
}

void launch_level_init(int32_t *comm, int32_t *newc, int32_t *size, const u64 *k, u64 *S,
                       int32_t V, cudaStream_t s) {
    if (V <= 0) return;
    level_init_kernel<<<grid_for(V), 256, 0, s>>>(comm, newc, size, k, S, V); note_launches(1);
}

void launch_set_communities(const int32_t *comm_in, int32_t *comm, int32_t *newc, int32_t *size,
                            const u64 *k, u64 *S, int32_t V, int *err, cudaStream_t s) {
    if (V <= 0) return;
    zero_state_kernel<<<grid_for(V), 256, 0, s>>>(size, S, V); note_launches(1);
    set_comm_kernel<<<grid_for(V), 256, 0, s>>>(comm_in, comm, newc, size, k, S, V, err); note_launches(1);
}

void launch_compose_map(int32_t *orig2comm, const int32_t *map, int32_t V0, cudaStream_t s) {
    if (V0 <= 0) return;
    compose_map_kernel<<<grid_for(V0), 256, 0, s>>>(orig2comm, map, V0); note_launches(1);
}

template <typename WT>
void launch_weights_to_fixed(const WT *w, int64_t E, double scale, int64_t *out, cudaStream_t s) {
    if (E <= 0) return;
    to_fixed_kernel<WT><<<grid_for(E), 256, 0, s>>>(w, E, scale, out); note_launches(1);
}
template void launch_weights_to_fixed<float>(const float *, int64_t, double, int64_t *, cudaStream_t);
template void launch_weights_to_fixed<u64>(const u64 *, int64_t, double, int64_t *, cudaStream_t);

void launch_weight_scan(const float *w, int64_t E, int32_t *out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(int32_t) * 3, s);
    if (E <= 0) return;
    weight_scan_kernel<<<grid_for(E), 256, 0, s>>>(w, E, out); note_launches(1);
}

void launch_total_weight(const float *w, int64_t E, double scale, u64 *total, cudaStream_t s) {
    cudaMemsetAsync(total, 0, sizeof(u64), s);
    if (E <= 0) return;
    total_weight_kernel<<<grid_for(E), 256, 0, s>>>(w, E, scale, total); note_launches(1);
}

void launch_validate_csr(const int32_t *rowptr, const int32_t *col, int32_t V, int64_t E, int *err,
                         cudaStream_t s) {
    validate_csr_kernel<<<grid_for(V > E ? V : E), 256, 0, s>>>(rowptr, col, V, E, err); note_launches(1);
}

}  // namespace lv

namespace lv {
namespace {
__global__ void gather_degrees_kernel(const int32_t *__restrict__ rowptr,
                                      const int32_t *__restrict__ rowend,
                                      const int32_t *__restrict__ list, int32_t n, int32_t *out) {
    for (int32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const int32_t v = list[i];
        out[i] = rowend[v] - rowptr[v];
    }
}
__global__ void gather_cdeg_kernel(const int32_t *__restrict__ mstart, const int32_t *__restrict__ P,
                                   const int32_t *__restrict__ list, int32_t n, int32_t *out) {
    for (int32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const int32_t c = list[i];
        out[i] = P[mstart[c + 1]] - P[mstart[c]];
    }
}
}  // namespace

void launch_gather_degrees(const int32_t *rowptr, const int32_t *rowend, const int32_t *list,
                           int32_t n, int32_t *out, cudaStream_t s) {
    if (n <= 0) return;
    gather_degrees_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rowptr, rowend, list, n, out); note_launches(1);
}

void launch_gather_cdeg(const int32_t *mstart, const int32_t *P, const int32_t *list, int32_t n,
                        int32_t *out, cudaStream_t s) {
    if (n <= 0) return;
    gather_cdeg_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mstart, P, list, n, out); note_launches(1);
}
}  // namespace lv
