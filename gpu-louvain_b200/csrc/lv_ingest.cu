// lv_ingest.cu -- CSR build on the device from Matrix Market entries in file
// order (lv_csr_from_entries_device, used by lv_read_mtx_device).
//
// The reference builds its CSR on the host (utils.cu:32-59): entry "v1 v2 w"
// appends (v2, w) to v1's list and, unless v1 == v2, (v1, w) to v2's list, and
// each row keeps file order.  Here every entry becomes one or two directed
// entries numbered in that order (an exclusive scan of 1 + [v1 != v2]), the
// directed entries are stably radix-sorted by row, and the sorted order gives
// each row's entries in file order: the same CSR as lv_read_mtx's host build.
#include <cub/cub.cuh>

#include "../../include/louvain_b200.h"

namespace {

__global__ void entry_count_kernel(const int32_t *__restrict__ a, const int32_t *__restrict__ b, int64_t n,
                                   int32_t V, int32_t *cnt, int *err) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = a[i], y = b[i];
        if (x < 0 || x >= V || y < 0 || y >= V) {
            atomicOr(err, 1);
            cnt[i] = 0;
            continue;
        }
        cnt[i] = x != y ? 2 : 1;
    }
}

// directed entry d = pos[i] (v1 -> v2) and d + 1 (v2 -> v1, off-diagonal only)
__global__ void entry_expand_kernel(const int32_t *__restrict__ a, const int32_t *__restrict__ b,
                                    const float *__restrict__ w, const int64_t *__restrict__ pos, int64_t n,
                                    int32_t V, int32_t *row, int32_t *idx, int32_t *dcol, float *dw,
                                    int32_t *deg) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = a[i], y = b[i];
        if (x < 0 || x >= V || y < 0 || y >= V) continue;
        const int64_t d = pos[i];
        const float wv = w[i];
        row[d] = x;
        idx[d] = (int32_t)d;
        dcol[d] = y;
        dw[d] = wv;
        atomicAdd(deg + x, 1);
        if (x != y) {
            row[d + 1] = y;
            idx[d + 1] = (int32_t)(d + 1);
            dcol[d + 1] = x;
            dw[d + 1] = wv;
            atomicAdd(deg + y, 1);
        }
    }
}

__global__ void entry_gather_kernel(const int32_t *__restrict__ idx, int64_t E, const int32_t *__restrict__ dcol,
                                    const float *__restrict__ dw, int32_t *col, float *w) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < E; j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = idx[j];
        col[j] = dcol[d];
        w[j] = dw[d];
    }
}

int bits_for(int32_t V) {
    int b = 1;
    while (b < 31 && ((int64_t)1 << b) < (int64_t)V) ++b;
    return b;
}

}  // namespace

extern "C" int lv_csr_from_entries_device(int32_t device, int32_t V, int64_t nnz, const int32_t *v1, const int32_t *v2,
                                          const float *w, int64_t *Eout, int32_t **d_rowptr, int32_t **d_col,
                                          float **d_w) {
    if (V < 0 || nnz < 0 || !Eout || !d_rowptr || !d_col || !d_w || (nnz > 0 && (!v1 || !v2 || !w)))
        return LV_ERR_INVALID;
    if (nnz > 0 && V == 0) return LV_ERR_INVALID;
    if (nnz > 0x7fffffffLL) return LV_ERR_TOO_LARGE;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return LV_ERR_NO_DEVICE;
    }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return LV_ERR_CUDA;
    }
    const size_t n = (size_t)(nnz > 0 ? nnz : 1);
    int32_t *a = nullptr, *b = nullptr, *cnt = nullptr, *row = nullptr, *idx = nullptr, *row2 = nullptr,
            *idx2 = nullptr, *dcol = nullptr, *deg = nullptr, *rp = nullptr, *cl = nullptr;
    float *ww = nullptr, *dw = nullptr, *wt = nullptr;
    int64_t *pos = nullptr, *tot = nullptr;
    int *err = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int64_t E = 0;
    int h_err = 0;
    int rc = LV_OK;
    const unsigned grid = 148 * 16;
#define ING_CHECK(x)                                                                         \
    do {                                                                                     \
        const cudaError_t e__ = (x);                                                         \
        if (e__ != cudaSuccess) {                                                            \
            rc = e__ == cudaErrorMemoryAllocation ? LV_ERR_NOMEM : LV_ERR_CUDA;              \
            goto done;                                                                       \
        }                                                                                    \
    } while (0)
    ING_CHECK(cudaMalloc(&rp, sizeof(int32_t) * ((size_t)V + 1)));
    ING_CHECK(cudaMalloc(&deg, sizeof(int32_t) * ((size_t)V + 1)));
    ING_CHECK(cudaMemsetAsync(deg, 0, sizeof(int32_t) * ((size_t)V + 1), s));
    ING_CHECK(cudaMalloc(&err, sizeof(int)));
    ING_CHECK(cudaMemsetAsync(err, 0, sizeof(int), s));
    ING_CHECK(cudaMalloc(&tot, sizeof(int64_t)));
    if (nnz > 0) {
        ING_CHECK(cudaMalloc(&a, sizeof(int32_t) * n));
        ING_CHECK(cudaMalloc(&b, sizeof(int32_t) * n));
        ING_CHECK(cudaMalloc(&ww, sizeof(float) * n));
        ING_CHECK(cudaMalloc(&cnt, sizeof(int32_t) * (n + 1)));   // cnt[n] = 0: pos[n] is the total
        ING_CHECK(cudaMalloc(&pos, sizeof(int64_t) * (n + 1)));
        ING_CHECK(cudaMemcpyAsync(a, v1, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        ING_CHECK(cudaMemcpyAsync(b, v2, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        ING_CHECK(cudaMemcpyAsync(ww, w, sizeof(float) * n, cudaMemcpyHostToDevice, s));
        ING_CHECK(cudaMemsetAsync(cnt + n, 0, sizeof(int32_t), s));
        entry_count_kernel<<<grid, 256, 0, s>>>(a, b, nnz, V, cnt, err);
        // the directed total reaches 2 nnz, beyond int32 for nnz >= 2^30: the
        // scan accumulates in int64 (an ExclusiveSum would accumulate in the
        // int32 input type and wrap before the E check below)
        ING_CHECK(cub::DeviceScan::ExclusiveScan(nullptr, tmp_bytes, cnt, pos, ::cuda::std::plus<>{}, (int64_t)0,
                                                 (int64_t)nnz + 1, s));
        ING_CHECK(cudaMalloc(&tmp, tmp_bytes));
        ING_CHECK(cub::DeviceScan::ExclusiveScan(tmp, tmp_bytes, cnt, pos, ::cuda::std::plus<>{}, (int64_t)0,
                                                 (int64_t)nnz + 1, s));
        ING_CHECK(cudaMemcpyAsync(&E, pos + nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        ING_CHECK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        ING_CHECK(cudaStreamSynchronize(s));
        if (h_err) { rc = LV_ERR_INVALID; goto done; }
        if (E > 0x7fffffffLL) { rc = LV_ERR_TOO_LARGE; goto done; }
    }
    {
        const size_t ne = (size_t)(E > 0 ? E : 1);
        ING_CHECK(cudaMalloc(&cl, sizeof(int32_t) * ne));
        ING_CHECK(cudaMalloc(&wt, sizeof(float) * ne));
        if (E > 0) {
            ING_CHECK(cudaMalloc(&row, sizeof(int32_t) * ne));
            ING_CHECK(cudaMalloc(&idx, sizeof(int32_t) * ne));
            ING_CHECK(cudaMalloc(&row2, sizeof(int32_t) * ne));
            ING_CHECK(cudaMalloc(&idx2, sizeof(int32_t) * ne));
            ING_CHECK(cudaMalloc(&dcol, sizeof(int32_t) * ne));
            ING_CHECK(cudaMalloc(&dw, sizeof(float) * ne));
            entry_expand_kernel<<<grid, 256, 0, s>>>(a, b, ww, pos, nnz, V, row, idx, dcol, dw, deg);
            size_t t2 = 0;
            const int bits = bits_for(V);
            ING_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, t2, row, row2, idx, idx2, (int64_t)E, 0, bits, s));
            if (t2 > tmp_bytes) {
                cudaFree(tmp);
                tmp = nullptr;
                tmp_bytes = t2;
                ING_CHECK(cudaMalloc(&tmp, tmp_bytes));
            }
            // stable: equal rows keep the directed (file) order
            ING_CHECK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, row, row2, idx, idx2, (int64_t)E, 0, bits, s));
            entry_gather_kernel<<<grid, 256, 0, s>>>(idx2, E, dcol, dw, cl, wt);
        }
        size_t t3 = 0;
        ING_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, t3, deg, rp, (int64_t)V + 1, s));
        if (t3 > tmp_bytes) {
            if (tmp) cudaFree(tmp);
            tmp = nullptr;
            tmp_bytes = t3;
            ING_CHECK(cudaMalloc(&tmp, tmp_bytes));
        }
        ING_CHECK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, deg, rp, (int64_t)V + 1, s));
        ING_CHECK(cudaStreamSynchronize(s));
        ING_CHECK(cudaGetLastError());
    }
done:
#undef ING_CHECK
    for (void *p : {(void *)a, (void *)b, (void *)ww, (void *)cnt, (void *)pos, (void *)tot, (void *)err, tmp,
                    (void *)row, (void *)idx, (void *)row2, (void *)idx2, (void *)dcol, (void *)dw, (void *)deg})
        if (p) cudaFree(p);
    cudaStreamDestroy(s);
    if (rc != LV_OK) {
        cudaGetLastError();
        if (rp) cudaFree(rp);
        if (cl) cudaFree(cl);
        if (wt) cudaFree(wt);
        return rc;
    }
    *Eout = E;
    *d_rowptr = rp;
    *d_col = cl;
    *d_w = wt;
    return LV_OK;
}
