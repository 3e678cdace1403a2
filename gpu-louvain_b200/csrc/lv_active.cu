// lv_active.cu -- learned active-set proposal: the per-vertex move predictor
// (a 5-16-1 MLP, bf16 weights, fp32 accumulation), its inference and
// compaction kernels, the move-trace recorder and the training kernels.
//
// The plain method evaluates every vertex in every sweep.  After the first
// sweeps of a level most vertices stay where they are, so the engine's learned
// mode (lv_opts.active_set) evaluates only the vertices the predictor proposes.
// Every move still uses the exact gain rule.  Periodic full sweeps measure the
// predictor's recall, and the plain sweep takes over for the rest of the
// level when the recall falls below lv_opts.active_min_recall.
//
// Features of vertex v (recorded by the move kernels when v is evaluated):
//   x0 = log2(1 + degree) / 16
//   x1 = weight from v into its own community / k_v   (last evaluation)
//   x2 = (G_best - T e_own) / (T k_v), clamped to [-1, 1] (last evaluation)
//   x3 = 1 if v moved in the previous sweep
//   x4 = fraction of v's row entries whose vertex moved in the previous sweep
// Model: h = relu(W1 x + b1) (16 units), logit = W2 . h + b2; parameters in
// the order W1[16][5], b1[16], W2[16], b2 (LV_ACTIVE_MODEL_SIZE = 113).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/louvain_b200.h"
#include "lv_internal.h"

namespace lv {

namespace {

constexpr int NF = LV_ACTIVE_FEATURES;
constexpr int NH = LV_ACTIVE_HIDDEN;
constexpr int NP = LV_ACTIVE_MODEL_SIZE;
constexpr int OFF_B1 = NH * NF, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH;
static_assert(OFF_B2 + 1 == NP, "model layout");

__device__ __forceinline__ float bf16_bits_to_float(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

__device__ __forceinline__ void load_model(const uint16_t *wq, float *w) {
    for (int i = threadIdx.x; i < NP; i += blockDim.x) w[i] = bf16_bits_to_float(wq[i]);
}

__device__ __forceinline__ float mlp_logit(const float *w, const float *x) {
    float z = w[OFF_B2];
#pragma unroll
    for (int h = 0; h < NH; ++h) {
        float a = w[OFF_B1 + h];
#pragma unroll
        for (int f = 0; f < NF; ++f) a = fmaf(w[h * NF + f], x[f], a);
        z = fmaf(w[OFF_W2 + h], fmaxf(a, 0.0f), z);
    }
    return z;
}

__device__ __forceinline__ void vertex_features(int32_t deg, const float *feat, const uint8_t *moved,
                                                const int32_t *nmoved, int32_t v, float *x) {
    x[0] = log2f(1.0f + (float)deg) * 0.0625f;
    x[1] = feat[2 * (size_t)v];
    x[2] = feat[2 * (size_t)v + 1];
    x[3] = moved[v] ? 1.0f : 0.0f;
    x[4] = fminf(1.0f, (float)nmoved[v] / (float)(deg > 0 ? deg : 1));
}

__device__ __forceinline__ int class_at(const ActiveClassOffsets &co, int32_t p) {
    int c = 0;
#pragma unroll
    for (int i = 1; i < NCLS; ++i) c += p >= co.off[i] ? 1 : 0;
    return c;
}

// One position of the level's vertex list per thread.  Vertices of class
// >= keep_cls are always active.  alist != nullptr: active vertices are
// compacted into alist at their class's offset (acnt[c] counts them) and,
// when fresh is given, marked fresh (evaluated since the last full sweep);
// pred != nullptr: pred[v] = active.
__global__ void __launch_bounds__(256) active_select_kernel(const int32_t *__restrict__ list, int32_t n,
                                                            ActiveClassOffsets co, const int32_t *__restrict__ rowptr,
                                                            const int32_t *__restrict__ rowend,
                                                            const float *__restrict__ feat,
                                                            const uint8_t *__restrict__ moved,
                                                            const int32_t *__restrict__ nmoved,
                                                            const uint16_t *__restrict__ model, float logit_thr,
                                                            int keep_cls, int32_t *alist, int32_t *acnt,
                                                            uint8_t *pred, uint8_t *fresh) {
    __shared__ float w[NP];
    __shared__ int32_t lc[NCLS], base[NCLS];
    load_model(model, w);
    if (threadIdx.x < NCLS) lc[threadIdx.x] = 0;
    __syncthreads();
    const int32_t p = blockIdx.x * 256 + threadIdx.x;
    int c = -1, rank = 0;
    int32_t v = -1;
    bool act = false;
    if (p < n) {
        v = list[p];
        c = class_at(co, p);
        if (c >= keep_cls) {
            act = true;
        } else {
            float x[NF];
            vertex_features(rowend[v] - rowptr[v], feat, moved, nmoved, v, x);
            act = mlp_logit(w, x) > logit_thr;
        }
        if (pred) pred[v] = act ? 1 : 0;
        if (alist && act) {
            rank = atomicAdd(&lc[c], 1);
            if (fresh) fresh[v] = 1;
        }
    }
    if (!alist) return;
    __syncthreads();
    if (threadIdx.x < NCLS && lc[threadIdx.x]) base[threadIdx.x] = atomicAdd(acnt + threadIdx.x, lc[threadIdx.x]);
    __syncthreads();
    if (act) alist[co.off[c] + base[c] + rank] = v;
}

// moved[v] = comm[v] != prev[v]; counts[0] += movers.  When pred is given
// (a full sweep measuring the predictor), the recall counts only the fresh
// vertices (evaluated in an active sweep since the last full sweep, whose
// features are current): counts[3] += fresh movers, counts[1] += fresh
// movers with pred[v] set; fresh is then cleared.
__global__ void __launch_bounds__(256) active_moved_kernel(const int32_t *__restrict__ comm,
                                                           const int32_t *__restrict__ prev, int32_t V,
                                                           uint8_t *moved, const uint8_t *__restrict__ pred,
                                                           uint8_t *fresh, u64 *counts) {
    u64 m = 0, fm = 0, hit = 0;
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256) {
        const bool mv = comm[v] != prev[v];
        moved[v] = mv ? 1 : 0;
        m += mv ? 1 : 0;
        if (pred) {
            const bool f = fresh[v] != 0;
            if (f) fresh[v] = 0;
            if (mv && f) {
                fm += 1;
                if (pred[v]) hit += 1;
            }
        }
    }
    m = warp_sum_u64(m);
    fm = warp_sum_u64(fm);
    hit = warp_sum_u64(hit);
    if ((threadIdx.x & 31) == 0) {
        if (m) atomicAdd(counts, m);
        if (fm) atomicAdd(counts + 3, fm);
        if (hit) atomicAdd(counts + 1, hit);
    }
}

// Trace recorder: vertex v is sampled when draw(key, v) < thr; its current
// features go to the next free row of the trace (rows beyond cap are counted
// but not stored).
__global__ void __launch_bounds__(256) trace_sample_kernel(int32_t V, const int32_t *__restrict__ rowptr,
                                                           const int32_t *__restrict__ rowend,
                                                           const float *__restrict__ feat,
                                                           const uint8_t *__restrict__ moved,
                                                           const int32_t *__restrict__ nmoved, u64 thr, u64 key,
                                                           float *tx, int32_t *tv, int64_t cap, u64 *tcount) {
    for (int32_t v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256) {
        u64 z = key + (u64)v * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        if (z >= thr) continue;
        const u64 idx = atomicAdd(tcount, 1ull);
        if ((int64_t)idx >= cap) continue;
        float x[NF];
        vertex_features(rowend[v] - rowptr[v], feat, moved, nmoved, v, x);
        for (int f = 0; f < NF; ++f) tx[idx * NF + f] = x[f];
        tv[idx] = v;
    }
}

// Labels of trace rows [r0, r1): did the sampled vertex move in the sweep
// that followed its sampling.
__global__ void trace_label_kernel(const int32_t *__restrict__ tv, const uint8_t *__restrict__ moved, int64_t r0,
                                   const u64 *__restrict__ tcount, int64_t cap, uint8_t *ty) {
    const int64_t r1 = (int64_t)*tcount < cap ? (int64_t)*tcount : cap;
    for (int64_t i = r0 + (int64_t)blockIdx.x * 256 + threadIdx.x; i < r1; i += (int64_t)gridDim.x * 256)
        ty[i] = moved[tv[i]];
}

// nmoved[x] += 1 for every row entry (v, x), x != v, of every vertex v that
// moved in the sweep: a warp takes 32 vertices and walks the movers' rows
// with its lanes.
__global__ void __launch_bounds__(256) nbr_moved_kernel(const int32_t *__restrict__ rowptr,
                                                        const int32_t *__restrict__ rowend,
                                                        const int32_t *__restrict__ col, int32_t V,
                                                        const uint8_t *__restrict__ moved, int32_t *nmoved) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * 8;
    for (int64_t base = ((int64_t)blockIdx.x * 8 + (threadIdx.x >> 5)) * 32; base < V; base += warps * 32) {
        const int64_t v = base + lane;
        unsigned bal = __ballot_sync(FULL, v < V && moved[v]);
        while (bal) {
            const int src = __ffs(bal) - 1;
            bal &= bal - 1;
            const int32_t u = (int32_t)(base + src);
            const int32_t r1 = rowend[u];
            for (int32_t e = rowptr[u] + lane; e < r1; e += 32) {
                const int32_t x = col[e];
                if (x != u) atomicAdd(nmoved + x, 1);
            }
        }
    }
}

inline unsigned grid_of(int64_t n, int64_t cap = 148 * 16) {
    int64_t b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (unsigned)(b < cap ? b : cap);
}

}  // namespace

void launch_active_select(const int32_t *list, int32_t n, const ActiveClassOffsets &co, const int32_t *rowptr,
                          const int32_t *rowend, const float *feat, const uint8_t *moved, const int32_t *nmoved,
                          const uint16_t *model, float logit_thr, int keep_cls, int32_t *alist, int32_t *acnt,
                          uint8_t *pred, uint8_t *fresh, cudaStream_t s) {
    if (n <= 0) return;
    active_select_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(list, n, co, rowptr, rowend, feat, moved, nmoved,
                                                                    model, logit_thr, keep_cls, alist, acnt, pred,
                                                                    fresh);
    note_launches(1);
}

void launch_active_moved(const int32_t *comm, const int32_t *prev, int32_t V, uint8_t *moved, const uint8_t *pred,
                         uint8_t *fresh, u64 *counts, cudaStream_t s) {
    if (V <= 0) return;
    active_moved_kernel<<<grid_of(V), 256, 0, s>>>(comm, prev, V, moved, pred, fresh, counts);
    note_launches(1);
}

void launch_trace_sample(int32_t V, const int32_t *rowptr, const int32_t *rowend, const float *feat,
                         const uint8_t *moved, const int32_t *nmoved, u64 thr, u64 key, float *tx, int32_t *tv,
                         int64_t cap, u64 *tcount, cudaStream_t s) {
    if (V <= 0) return;
    trace_sample_kernel<<<grid_of(V), 256, 0, s>>>(V, rowptr, rowend, feat, moved, nmoved, thr, key, tx, tv, cap,
                                                   tcount);
    note_launches(1);
}

void launch_nbr_moved(const int32_t *rowptr, const int32_t *rowend, const int32_t *col, int32_t V,
                      const uint8_t *moved, int32_t *nmoved, cudaStream_t s) {
    if (V <= 0) return;
    cudaMemsetAsync(nmoved, 0, sizeof(int32_t) * (size_t)V, s);
    nbr_moved_kernel<<<grid_of(((int64_t)V + 7) / 8), 256, 0, s>>>(rowptr, rowend, col, V, moved, nmoved);
    note_launches(1);
}

void launch_trace_label(const int32_t *tv, const uint8_t *moved, int64_t r0, const u64 *tcount, int64_t cap,
                        uint8_t *ty, cudaStream_t s) {
    if (cap <= r0) return;
    trace_label_kernel<<<grid_of(cap - r0, 148 * 4), 256, 0, s>>>(tv, moved, r0, tcount, cap, ty);
    note_launches(1);
}

// ---------------------------------------------------------------------------
// training: mini-batch Adam on the weighted binary cross-entropy of the move
// labels.  The forward and backward passes use the bf16 copy of the weights
// with fp32 accumulation; Adam updates an fp32 master copy and rounds it to
// bf16 after every step.  Gradients are summed in a fixed order (per thread,
// then per block in thread order, then over blocks in block order), so a run
// is reproducible bit for bit.
// ---------------------------------------------------------------------------
namespace {

constexpr int TR_THREADS = 64;
constexpr int TR_BLOCKS = 256;
constexpr int NG = NP + 1;   // gradient entries + the loss

__global__ void __launch_bounds__(TR_THREADS) mlp_grad_kernel(const float *__restrict__ x,
                                                              const uint8_t *__restrict__ y, int64_t n,
                                                              int64_t b0, int64_t bn, u64 pa, u64 pc,
                                                              const uint16_t *__restrict__ wq, float pos_w,
                                                              float *part) {
    __shared__ float w[NP];
    __shared__ float acc[TR_THREADS][NG];
    load_model(wq, w);
    __syncthreads();
    float g[NG];
#pragma unroll
    for (int i = 0; i < NG; ++i) g[i] = 0.0f;
    const int64_t stride = (int64_t)TR_BLOCKS * TR_THREADS;
    for (int64_t i = b0 + (int64_t)blockIdx.x * TR_THREADS + threadIdx.x; i < b0 + bn; i += stride) {
        const int64_t j = (int64_t)(((u128)pa * (u128)(u64)i + (u128)pc) % (u128)(u64)n);
        float xs[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) xs[f] = x[j * NF + f];
        const float t = y[j] ? 1.0f : 0.0f;
        float a[NH];
        float z = w[OFF_B2];
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            float s = w[OFF_B1 + h];
#pragma unroll
            for (int f = 0; f < NF; ++f) s = fmaf(w[h * NF + f], xs[f], s);
            a[h] = s;
            z = fmaf(w[OFF_W2 + h], fmaxf(s, 0.0f), z);
        }
        const float wt = y[j] ? pos_w : 1.0f;
        const float p = 1.0f / (1.0f + expf(-z));
        g[NP] += wt * (fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z))) - t * z);
        const float gz = wt * (p - t);
        g[OFF_B2] += gz;
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            g[OFF_W2 + h] += gz * fmaxf(a[h], 0.0f);
            const float dh = a[h] > 0.0f ? gz * w[OFF_W2 + h] : 0.0f;
            g[OFF_B1 + h] += dh;
#pragma unroll
            for (int f = 0; f < NF; ++f) g[h * NF + f] += dh * xs[f];
        }
    }
#pragma unroll
    for (int i = 0; i < NG; ++i) acc[threadIdx.x][i] = g[i];
    __syncthreads();
    for (int i = threadIdx.x; i < NG; i += TR_THREADS) {
        float sum = 0.0f;
        for (int t = 0; t < TR_THREADS; ++t) sum += acc[t][i];
        part[(size_t)blockIdx.x * NG + i] = sum;
    }
}

__global__ void mlp_adam_kernel(const float *__restrict__ part, float inv_bn, float lr, float c1, float c2,
                                float *master, float *m1, float *m2, uint16_t *wq, float *loss_out) {
    const int i = threadIdx.x;
    if (i >= NG) return;
    float sum = 0.0f;
    for (int b = 0; b < TR_BLOCKS; ++b) sum += part[(size_t)b * NG + i];
    if (i == NP) {
        *loss_out = sum * inv_bn;
        return;
    }
    const float gr = sum * inv_bn;
    const float a = 0.9f * m1[i] + 0.1f * gr;
    const float b = 0.999f * m2[i] + 0.001f * gr * gr;
    m1[i] = a;
    m2[i] = b;
    const float mw = master[i] - lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
    master[i] = mw;
    wq[i] = __bfloat16_as_ushort(__float2bfloat16_rn(mw));
}

__global__ void mlp_logit_kernel(const uint16_t *__restrict__ wq, const float *__restrict__ x, int64_t n,
                                 float *out) {
    __shared__ float w[NP];
    load_model(wq, w);
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        float xs[NF];
        for (int f = 0; f < NF; ++f) xs[f] = x[i * NF + f];
        out[i] = mlp_logit(w, xs);
    }
}

// float -> bf16 bits, round to nearest even (finite inputs)
uint16_t host_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

uint64_t mix64h(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t gcd_u64(uint64_t a, uint64_t b) {
    while (b) {
        const uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

struct DevBuf {
    std::vector<void *> p;
    ~DevBuf() {
        for (void *q : p) cudaFree(q);
    }
    template <typename T>
    bool get(T **out, size_t n) {
        void *q = nullptr;
        if (cudaMalloc(&q, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        p.push_back(q);
        *out = (T *)q;
        return true;
    }
};

}  // namespace
}  // namespace lv

using namespace lv;

extern "C" {

int lv_active_train(const float *x, const uint8_t *y, int64_t n, int32_t epochs, int32_t batch, float lr,
                    float pos_weight, uint64_t seed, int32_t device, uint16_t *model_out, float *epoch_loss) {
    if (!x || !y || n <= 0 || epochs < 1 || batch < 1 || !(lr > 0.0f) || !(pos_weight > 0.0f) || !model_out)
        return LV_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return LV_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return LV_ERR_INVALID;
    cudaSetDevice(device);
    // initial weights: uniform in +-1/sqrt(fan_in) from the seed, zero hidden
    // biases, output bias at the log-odds of the positive rate
    std::vector<float> master(NP, 0.0f);
    for (int i = 0; i < NP; ++i) {
        const double u = (double)(mix64h(seed ^ (0x51ED2701ull + (uint64_t)i * 0x9E3779B97F4A7C15ull)) >> 11) * 0x1.0p-53;
        if (i < OFF_B1) master[i] = (float)((2.0 * u - 1.0) / std::sqrt((double)NF));
        else if (i >= OFF_W2 && i < OFF_B2) master[i] = (float)((2.0 * u - 1.0) / std::sqrt((double)NH));
    }
    int64_t pos = 0;
    for (int64_t i = 0; i < n; ++i) pos += y[i] ? 1 : 0;
    const double rate = ((double)pos * pos_weight + 0.5) / ((double)pos * pos_weight + (double)(n - pos) + 1.0);
    master[OFF_B2] = (float)std::log(rate / (1.0 - rate));
    std::vector<uint16_t> wq_h(NP);
    for (int i = 0; i < NP; ++i) wq_h[i] = host_bf16(master[i]);
    const int64_t steps_per_epoch = (n + batch - 1) / batch;
    const int64_t steps = steps_per_epoch * epochs;
    DevBuf B;
    float *dx = nullptr, *part = nullptr, *dm = nullptr, *m1 = nullptr, *m2 = nullptr, *loss = nullptr;
    uint8_t *dy = nullptr;
    uint16_t *wq = nullptr;
    if (!B.get(&dx, (size_t)n * NF) || !B.get(&dy, (size_t)n) || !B.get(&part, (size_t)TR_BLOCKS * NG) ||
        !B.get(&dm, NP) || !B.get(&m1, NP) || !B.get(&m2, NP) || !B.get(&wq, NP) || !B.get(&loss, (size_t)steps))
        return LV_ERR_NOMEM;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return LV_ERR_CUDA;
    cudaMemcpyAsync(dx, x, sizeof(float) * (size_t)n * NF, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dy, y, (size_t)n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dm, master.data(), sizeof(float) * NP, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(wq, wq_h.data(), sizeof(uint16_t) * NP, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(m1, 0, sizeof(float) * NP, s);
    cudaMemsetAsync(m2, 0, sizeof(float) * NP, s);
    int64_t k = 0;
    double b1p = 1.0, b2p = 1.0;
    for (int ep = 0; ep < epochs; ++ep) {
        // a fresh visiting order each epoch: i -> (pa i + pc) mod n, gcd(pa, n) = 1
        uint64_t pa = (mix64h(seed + 0xE9 + (uint64_t)ep) % (uint64_t)n) | 1ull;
        for (int tries = 0; gcd_u64(pa, (uint64_t)n) != 1; ++tries)
            pa = tries < 1000 ? ((pa + 2) % (uint64_t)n | 1ull) : 1ull;
        const uint64_t pc = mix64h(seed * 31 + (uint64_t)ep) % (uint64_t)n;
        for (int64_t st = 0; st < steps_per_epoch; ++st, ++k) {
            const int64_t b0 = st * batch, bn = std::min<int64_t>(batch, n - b0);
            b1p *= 0.9;
            b2p *= 0.999;
            mlp_grad_kernel<<<TR_BLOCKS, TR_THREADS, 0, s>>>(dx, dy, n, b0, bn, pa, pc, wq, pos_weight, part);
            mlp_adam_kernel<<<1, 128, 0, s>>>(part, 1.0f / (float)bn, lr, (float)(1.0 / (1.0 - b1p)),
                                              (float)(1.0 / (1.0 - b2p)), dm, m1, m2, wq, loss + k);
            note_launches(2);
        }
    }
    std::vector<float> lh((size_t)steps);
    cudaMemcpyAsync(wq_h.data(), wq, sizeof(uint16_t) * NP, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(lh.data(), loss, sizeof(float) * (size_t)steps, cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return LV_ERR_CUDA;
    std::memcpy(model_out, wq_h.data(), sizeof(uint16_t) * NP);
    if (epoch_loss) {
        for (int ep = 0; ep < epochs; ++ep) {
            double sum = 0.0;
            for (int64_t st = 0; st < steps_per_epoch; ++st) {
                const int64_t bn = std::min<int64_t>(batch, n - st * batch);
                sum += (double)lh[(size_t)(ep * steps_per_epoch + st)] * (double)bn;
            }
            epoch_loss[ep] = (float)(sum / (double)n);
        }
    }
    return LV_OK;
}

int lv_active_predict(const uint16_t *model, const float *x, int64_t n, int32_t device, float *logits) {
    if (!model || !x || n < 0 || !logits) return LV_ERR_INVALID;
    if (n == 0) return LV_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return LV_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return LV_ERR_INVALID;
    cudaSetDevice(device);
    DevBuf B;
    uint16_t *wq = nullptr;
    float *dx = nullptr, *dz = nullptr;
    if (!B.get(&wq, NP) || !B.get(&dx, (size_t)n * NF) || !B.get(&dz, (size_t)n)) return LV_ERR_NOMEM;
    cudaMemcpy(wq, model, sizeof(uint16_t) * NP, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, x, sizeof(float) * (size_t)n * NF, cudaMemcpyHostToDevice);
    mlp_logit_kernel<<<grid_of(n), 256>>>(wq, dx, n, dz);
    note_launches(1);
    if (cudaMemcpy(logits, dz, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return LV_ERR_CUDA;
    }
    return LV_OK;
}

}  // extern "C"
