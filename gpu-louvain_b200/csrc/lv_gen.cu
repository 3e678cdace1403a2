// lv_gen.cu -- seeded R-MAT graphs drawn on the device (input generation for
// the benchmark; not part of the Louvain path).  Produces exactly the CSR of
// the host generator lv_gen_rmat: rows ascending, (a < b) keys deduplicated,
// self-loops dropped, the same per-edge weights.  Sorting uses CUB.
#include <cub/cub.cuh>

#include "../../include/louvain_b200.h"
#include "lv_rng.h"

namespace {

typedef unsigned long long u64;

__global__ void rmat_draw_kernel(lvrng::RmatParams p, int64_t n, u64 *keys) {
    const u64 selfmark = (1ull << (2 * p.scale)) - 1ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t u, v;
        lvrng::rmat_edge(p, (uint64_t)i, &u, &v);
        if (u == v) {
            keys[i] = selfmark;
        } else {
            const uint32_t x = u < v ? u : v, y = u < v ? v : u;
            keys[i] = ((u64)x << p.scale) | y;
        }
    }
}

// dhi[a] = #keys with first endpoint a, dlo[b] = #keys with second endpoint b
__global__ void degree_kernel(const u64 *keys, int64_t nk, int scale, int32_t *dlo, int32_t *dhi) {
    const u64 mask = (1ull << scale) - 1ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk;
         i += (int64_t)gridDim.x * blockDim.x) {
        atomicAdd(dhi + (keys[i] >> scale), 1);
        atomicAdd(dlo + (keys[i] & mask), 1);
    }
}

__global__ void sum_deg_kernel(const int32_t *dlo, const int32_t *dhi, int32_t V, int32_t *deg) {
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
        deg[v] = dlo[v] + dhi[v];
}

// keys sorted by (first, second): the key at i is the (i - segstart)-th
// larger neighbour of `first`.  swapped = 1: keys sorted by (second, first)
// give the smaller neighbours of `second`.
__global__ void fill_kernel(const u64 *keys, int64_t nk, int scale, int swapped,
                            const int32_t *rowptr, const int32_t *dlo, uint64_t wkey,
                            int weight_mode, int32_t *col, float *w) {
    const u64 mask = (1ull << scale) - 1ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(keys[i] >> scale), other = (uint32_t)(keys[i] & mask);
        // first index of this row's segment (binary search on the sorted keys)
        int64_t lo = 0, hi = i;
        const u64 rowkey = (u64)row << scale;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (keys[mid] < rowkey) lo = mid + 1; else hi = mid;
        }
        const int64_t rank = i - lo;
        const int64_t pos = (int64_t)rowptr[row] + (swapped ? 0 : dlo[row]) + rank;
        const uint32_t a = swapped ? other : row, b = swapped ? row : other;
        col[pos] = (int32_t)other;
        w[pos] = weight_mode == 1 ? lvrng::edge_weight(wkey, a, b) : 1.0f;
    }
}

__global__ void swap_kernel(const u64 *in, int64_t nk, int scale, u64 *out) {
    const u64 mask = (1ull << scale) - 1ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = ((in[i] & mask) << scale) | (in[i] >> scale);
}

}  // namespace

extern "C" {

void lv_free_device(void *p) {
    if (p) cudaFree(p);
}

int lv_gen_rmat_device(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b,
                       double c, int32_t weight_mode, int32_t device, int32_t *Vout, int64_t *Eout,
                       int32_t **d_rowptr, int32_t **d_col, float **d_w) {
    if (scale < 1 || scale > 30 || edge_factor < 1 || !Vout || !Eout || !d_rowptr || !d_col || !d_w ||
        !lvrng::rmat_probabilities_ok(a, b, c))
        return LV_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return LV_ERR_NO_DEVICE;
    const int64_t n = (int64_t)edge_factor << scale;
    const int32_t V = (int32_t)(1u << scale);
    const int bits = 2 * scale;
    const lvrng::RmatParams p = lvrng::rmat_params(scale, a, b, c, seed);
    u64 *k1 = nullptr, *k2 = nullptr;
    void *tmp = nullptr;
    int32_t *dlo = nullptr, *dhi = nullptr, *rp = nullptr, *cl = nullptr;
    // the distinct-key count is 64-bit: edge_factor << scale reaches 2^31 and more
    int64_t *nsel = nullptr;
    float *wt = nullptr;
    size_t tmp_bytes = 0, t1 = 0, t2 = 0, t3 = 0;
    int rc = LV_OK;
    int64_t nk = 0;
    int64_t h_nsel = 0;
    const unsigned grid = 148 * 16;
#define GEN_CHECK(x)                                  \
    do {                                              \
        if ((x) != cudaSuccess) { rc = LV_ERR_CUDA; goto done; } \
    } while (0)
    GEN_CHECK(cudaMalloc(&k1, sizeof(u64) * (size_t)n));
    GEN_CHECK(cudaMalloc(&k2, sizeof(u64) * (size_t)n));
    GEN_CHECK(cudaMalloc(&nsel, sizeof(int64_t) * 2));
    rmat_draw_kernel<<<grid, 256>>>(p, n, k1);
    cub::DeviceRadixSort::SortKeys(nullptr, t1, k1, k2, (int64_t)n, 0, bits);
    cub::DeviceSelect::Unique(nullptr, t2, k2, k1, nsel, (int64_t)n);
    cub::DeviceScan::ExclusiveSum(nullptr, t3, dlo, rp, V + 1);
    tmp_bytes = t1 > t2 ? t1 : t2;
    tmp_bytes = tmp_bytes > t3 ? tmp_bytes : t3;
    GEN_CHECK(cudaMalloc(&tmp, tmp_bytes));
    GEN_CHECK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, k1, k2, (int64_t)n, 0, bits));
    GEN_CHECK(cub::DeviceSelect::Unique(tmp, tmp_bytes, k2, k1, nsel, (int64_t)n));
    GEN_CHECK(cudaMemcpy(&h_nsel, nsel, sizeof(int64_t), cudaMemcpyDeviceToHost));
    nk = h_nsel;
    {
        // drop the self-loop marker (the largest key) if present
        u64 last = 0;
        if (nk > 0) {
            GEN_CHECK(cudaMemcpy(&last, k1 + nk - 1, sizeof(u64), cudaMemcpyDeviceToHost));
            if (last == (1ull << bits) - 1ull) nk -= 1;
        }
    }
    if (2 * nk > 0x7fffffffLL) { rc = LV_ERR_TOO_LARGE; goto done; }
    GEN_CHECK(cudaMalloc(&dlo, sizeof(int32_t) * ((size_t)V + 1)));
    GEN_CHECK(cudaMalloc(&dhi, sizeof(int32_t) * ((size_t)V + 1)));
    GEN_CHECK(cudaMalloc(&rp, sizeof(int32_t) * ((size_t)V + 1)));
    GEN_CHECK(cudaMalloc(&cl, sizeof(int32_t) * (size_t)(2 * nk + 1)));
    GEN_CHECK(cudaMalloc(&wt, sizeof(float) * (size_t)(2 * nk + 1)));
    GEN_CHECK(cudaMemset(dlo, 0, sizeof(int32_t) * ((size_t)V + 1)));
    GEN_CHECK(cudaMemset(dhi, 0, sizeof(int32_t) * ((size_t)V + 1)));
    degree_kernel<<<grid, 256>>>(k1, nk, scale, dlo, dhi);
    sum_deg_kernel<<<grid, 256>>>(dlo, dhi, V, dhi);   // dhi <- total degree (dlo kept)
    GEN_CHECK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, dhi, rp, V + 1));
    {
        const uint64_t wkey = lvrng::stream_key(seed, lvrng::WEIGHT_STREAM);
        fill_kernel<<<grid, 256>>>(k1, nk, scale, 0, rp, dlo, wkey, weight_mode, cl, wt);
        swap_kernel<<<grid, 256>>>(k1, nk, scale, k2);
        GEN_CHECK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, k2, k1, (int64_t)nk, 0, bits));
        fill_kernel<<<grid, 256>>>(k1, nk, scale, 1, rp, dlo, wkey, weight_mode, cl, wt);
    }
    GEN_CHECK(cudaDeviceSynchronize());
    GEN_CHECK(cudaGetLastError());
done:
#undef GEN_CHECK
    if (k1) cudaFree(k1);
    if (k2) cudaFree(k2);
    if (tmp) cudaFree(tmp);
    if (dlo) cudaFree(dlo);
    if (dhi) cudaFree(dhi);
    if (nsel) cudaFree(nsel);
    if (rc != LV_OK) {
        if (rp) cudaFree(rp);
        if (cl) cudaFree(cl);
        if (wt) cudaFree(wt);
        return rc;
    }
    *Vout = V;
    *Eout = 2 * nk;
    *d_rowptr = rp;
    *d_col = cl;
    *d_w = wt;
    return LV_OK;
}

}  // extern "C"
