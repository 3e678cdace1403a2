// lv_noalloc.cu -- modularity of a given partition without any device
// allocation (lv_modularity_noalloc).
//
// Some callers cannot allocate device memory at the moment they want a
// modularity value: a process whose device memory is wholly owned by another
// allocator (a framework's caching allocator, or a fixed pool sized to the
// whole GPU), or a latency-critical loop that cannot afford the device-wide
// synchronisation that cudaMalloc / cudaFree imply.  lv_create and
// lv_modularity allocate their working set per handle, so this entry point
// computes the same number with its working memory in one file-scope device
// array instead.
//
// The computation is the engine's modularity reduction (sum_i e_{i->C(i)} over
// the CSR, Sigma_tot per community, sum of Sigma_tot^2) on the same
// fixed-point grid and with the same FP64 formula, so for the same CSR and
// partition it returns exactly what lv_create_device + lv_set_communities +
// lv_modularity return.
#include <cmath>
#include <cstdio>

#include "../../include/louvain_b200.h"
#include "lv_internal.h"

namespace lv {
namespace {

// Working memory shared by every call on a device: a header (the weight
// scan words, error bits and the exact totals) followed by Sigma_tot of up
// to LV_NOALLOC_MAX_VERTICES communities.  Every GPU that loads the library
// holds it until the process exits.
struct NoallocHeader {
    int32_t scan[4];   // max fractional bits, top exponent + 1024, bad-weight flag, unused
    int32_t err;       // CSR check bits (1, 2) and community-id check bit (4)
    int32_t pad;
    u64 T;             // total weight on the fixed grid
    u64 e_own;         // sum_i e_{i->C(i)}
    u64 s2[2];         // hi, lo of sum_C Sigma_tot^2
};
constexpr int NOALLOC_HEADER_BYTES = 256;
static_assert(sizeof(NoallocHeader) <= NOALLOC_HEADER_BYTES, "header fits its slot");
constexpr size_t NOALLOC_BYTES = NOALLOC_HEADER_BYTES + sizeof(u64) * (size_t)LV_NOALLOC_MAX_VERTICES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

__global__ void noalloc_clear_kernel(u64 *words, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        words[i] = 0;
}

// Warp per vertex: k_v (row weight) and the weight to the own community;
// Sigma_tot[C(v)] += k_v.  Community ids outside [0, V) set error bit 4.
__global__ void __launch_bounds__(256) noalloc_modularity_kernel(const int32_t *__restrict__ rowptr,
                                                               const int32_t *__restrict__ col,
                                                               const float *__restrict__ w,
                                                               const int32_t *__restrict__ comm,
                                                               int32_t V, double scale, u64 *S,
                                                               NoallocHeader *hdr) {
    __shared__ u64 part[8];
    const int lane = threadIdx.x & 31;
    const int32_t warps = gridDim.x * 8;
    u64 own_sum = 0;
    for (int32_t v = blockIdx.x * 8 + (threadIdx.x >> 5); v < V; v += warps) {
        const int32_t cv = comm[v];
        if (cv < 0 || cv >= V) {
            if (lane == 0) atomicOr(&hdr->err, 4);
            continue;
        }
        const int32_t r0 = rowptr[v], r1 = rowptr[v + 1];
        u64 k = 0, eo = 0;
        for (int32_t e = r0 + lane; e < r1; e += 32) {
            const u64 x = wfix(w, e, scale);
            k += x;
            if (comm[__ldg(col + e)] == cv) eo += x;
        }
        k = warp_sum_u64(k);
        if (lane == 0 && k) atomicAdd(S + cv, k);
        own_sum += eo;
    }
    own_sum = warp_sum_u64(own_sum);
    if (lane == 0) part[threadIdx.x >> 5] = own_sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        u64 y = 0;
        for (int i = 0; i < 8; ++i) y += part[i];
        if (y) atomicAdd(&hdr->e_own, y);
    }
}

inline unsigned noalloc_grid(int64_t items, int per_block) {
    const int64_t b = (items + per_block - 1) / per_block;
    return (unsigned)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

int noalloc_fail(char *err, int32_t err_len, int code, const char *msg) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", msg);
    return code;
}

// Device address of the scratch array on the current device.  The host-side
// name of the array is not a device address, so every call asks the runtime
// for it (a cheap lookup) instead of keeping it: an address kept across calls
// would dangle after the caller resets the device (cudaDeviceReset reloads the
// module, possibly elsewhere).
int noalloc_scratch(void **out, char *err, int32_t err_len) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return noalloc_fail(err, err_len, LV_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
    *out = p;
    return LV_OK;
}

int noalloc_read(cudaStream_t s, void *dev_hdr, NoallocHeader *h, char *err, int32_t err_len) {
    cudaError_t e = cudaMemcpyAsync(h, dev_hdr, sizeof(NoallocHeader), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "CUDA error: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return LV_ERR_CUDA;
    }
    return LV_OK;
}

}  // namespace
}  // namespace lv

using namespace lv;

extern "C" int lv_modularity_noalloc(const int32_t *d_rowptr, const int32_t *d_col, const float *d_w,
                                     int32_t V, int64_t E, const int32_t *d_comm, void *stream,
                                     double *q, char *err, int32_t err_len) {
    if (err && err_len > 0) err[0] = '\0';
    if (!q || V < 0 || E < 0 || (V > 0 && (!d_rowptr || !d_comm)) || (E > 0 && (!d_col || !d_w)))
        return noalloc_fail(err, err_len, LV_ERR_INVALID, "invalid argument");
    // a CSR without vertices has no entries (lv_create_device rejects it too)
    if (V == 0 && E > 0) return noalloc_fail(err, err_len, LV_ERR_INVALID, "malformed CSR: entries without vertices");
    if (V > LV_NOALLOC_MAX_VERTICES) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "V = %d exceeds LV_NOALLOC_MAX_VERTICES = %d (the size of the built-in scratch array)",
                      V, LV_NOALLOC_MAX_VERTICES);
        return noalloc_fail(err, err_len, LV_ERR_TOO_LARGE, msg);
    }
    if (E > 0x7fffffffLL) return noalloc_fail(err, err_len, LV_ERR_TOO_LARGE, "E exceeds 2^31 - 1");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return noalloc_fail(err, err_len, LV_ERR_NO_DEVICE, "no usable CUDA device");
    }
    void *base = nullptr;
    int rc = noalloc_scratch(&base, err, err_len);
    if (rc != LV_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    NoallocHeader *dh = (NoallocHeader *)base;
    u64 *S = (u64 *)((unsigned char *)base + NOALLOC_HEADER_BYTES);
    // the array keeps the previous call's contents: clear the header and
    // Sigma_tot[0, V)
    const int64_t words = NOALLOC_HEADER_BYTES / 8 + (int64_t)V;
    noalloc_clear_kernel<<<noalloc_grid(words, 256), 256, 0, s>>>((u64 *)base, words);
    note_launches(1);
    if (V > 0) launch_validate_csr(d_rowptr, d_col, V, E, &dh->err, s);
    launch_weight_scan(d_w, E, dh->scan, s);
    NoallocHeader h;
    rc = noalloc_read(s, dh, &h, err, err_len);
    if (rc != LV_OK) return rc;
    if (h.err) return noalloc_fail(err, err_len, LV_ERR_INVALID, "malformed CSR (offsets or column ids)");
    if (h.scan[2]) return noalloc_fail(err, err_len, LV_ERR_WEIGHT, "negative, NaN or infinite edge weight");
    // fixed-point scale: the rule of lv_create / lv_create_device
    const int need = h.scan[0];
    const int top = h.scan[1] ? h.scan[1] - 1024 : 0;
    const int cap = 61 - top - ceil_log2_i(E > 0 ? E : 1);
    const int sc = need < cap ? need : cap;
    if (sc < 0) return noalloc_fail(err, err_len, LV_ERR_TOO_LARGE, "total edge weight exceeds the fixed-point range");
    const double scale_d = std::ldexp(1.0, sc);
    launch_total_weight(d_w, E, scale_d, &dh->T, s);
    if (V > 0) {
        noalloc_modularity_kernel<<<noalloc_grid(V, 8), 256, 0, s>>>(d_rowptr, d_col, d_w, d_comm, V, scale_d,
                                                                    S, dh);
        note_launches(1);
        launch_s2(S, V, dh->s2, s);
    }
    rc = noalloc_read(s, dh, &h, err, err_len);
    if (rc != LV_OK) return rc;
    if (h.err) return noalloc_fail(err, err_len, LV_ERR_INVALID, "community id outside [0, V)");
    // the FP64 formula of lv_modularity: e_own / T - sum(S^2) / T^2
    const u128 s2 = ((u128)h.s2[0] << 64) | (u128)h.s2[1];
    const double td = (double)h.T;
    const double a = (double)h.e_own / td;
    const double b = (double)s2 / (td * td);
    *q = a - b;
    return LV_OK;
}
