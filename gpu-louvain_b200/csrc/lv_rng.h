// lv_rng.h -- counter-based generator shared by the host generators, the
// device R-MAT kernel and the Python test helpers (same integer arithmetic
// everywhere, so a seed names one graph).
//   mix64        : the splitmix64 finaliser (Steele, Lea, Flood 2014)
//   stream_key   : mix64(seed ^ (stream << 32))
//   draw(key, i) : mix64(key + i * 0x9E3779B97F4A7C15)
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define LVRNG_HD __host__ __device__ __forceinline__
#else
#define LVRNG_HD inline
#endif

namespace lvrng {

constexpr uint64_t WEIGHT_STREAM = 0xFFFF;

LVRNG_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
LVRNG_HD uint64_t stream_key(uint64_t seed, uint64_t stream) { return mix64(seed ^ (stream << 32)); }
LVRNG_HD uint64_t draw(uint64_t key, uint64_t i) { return mix64(key + i * 0x9E3779B97F4A7C15ull); }

// Weight of undirected edge (a < b): uniform on [0.5, 1.5) from 24 random
// bits, (m + 2^23) * 2^-24 rounded to float32 (a multiple of 2^-24).
LVRNG_HD float edge_weight(uint64_t wkey, uint32_t a, uint32_t b) {
    const uint64_t h = draw(wkey, ((uint64_t)a << 32) | b);
    const uint32_t m = (uint32_t)(h >> 40);
    return (float)(m + 8388608u) * 5.9604644775390625e-08f;
}

// R-MAT: level l (0 = most significant bit) uses 32 bits of draw(key_{l/2}, i):
// quadrant q = [x >= ta] + [x >= tb] + [x >= tc]; row bit q>>1, column bit q&1.
struct RmatParams {
    int scale;
    uint32_t ta, tb, tc;
    uint64_t keys[16];
};

// Valid quadrant probabilities: a, b, c >= 0 and d = 1 - a - b - c > 0 (the
// thresholds below are 32-bit fixed-point cumulative sums, so a + b + c must
// stay below 1); NaN fails every comparison.
inline bool rmat_probabilities_ok(double a, double b, double c) {
    return a >= 0.0 && b >= 0.0 && c >= 0.0 && a + b + c < 1.0;
}

inline RmatParams rmat_params(int scale, double a, double b, double c, uint64_t seed) {
    RmatParams p;
    p.scale = scale;
    p.ta = (uint32_t)(a * 4294967296.0);
    p.tb = (uint32_t)((a + b) * 4294967296.0);
    p.tc = (uint32_t)((a + b + c) * 4294967296.0);
    for (int i = 0; i < 16; ++i) p.keys[i] = stream_key(seed, (uint64_t)(1 + i));
    return p;
}

LVRNG_HD void rmat_edge(const RmatParams &p, uint64_t i, uint32_t *u, uint32_t *v) {
    uint32_t uu = 0, vv = 0;
    for (int pr = 0; 2 * pr < p.scale; ++pr) {
        const uint64_t r = draw(p.keys[pr], i);
        for (int half = 0; half < 2; ++half) {
            if (2 * pr + half >= p.scale) break;
            const uint32_t x = (uint32_t)(r >> (32 * half));
            const uint32_t q = (uint32_t)(x >= p.ta) + (uint32_t)(x >= p.tb) + (uint32_t)(x >= p.tc);
            uu = (uu << 1) | (q >> 1);
            vv = (vv << 1) | (q & 1u);
        }
    }
    *u = uu;
    *v = vv;
}

// Planted partition: vertex v is in block floor(v*B/V); block b starts at
// ceil(b*V/B).
LVRNG_HD int64_t block_start(int64_t b, int64_t V, int64_t B) { return (b * V + B - 1) / B; }

LVRNG_HD bool planted_intra(uint64_t key, uint64_t i, int64_t V, int64_t B, uint32_t *u, uint32_t *v) {
    const uint64_t r = draw(key, i);
    const int64_t uu = (int64_t)(((r & 0xffffffffull) * (uint64_t)V) >> 32);
    const int64_t blk = uu * B / V;
    const int64_t s0 = block_start(blk, V, B), s1 = block_start(blk + 1, V, B);
    const int64_t vv = s0 + (int64_t)(((r >> 32) * (uint64_t)(s1 - s0)) >> 32);
    *u = (uint32_t)uu;
    *v = (uint32_t)vv;
    return true;
}

LVRNG_HD bool planted_inter(uint64_t key, uint64_t i, int64_t V, int64_t B, uint32_t *u, uint32_t *v) {
    const uint64_t r = draw(key, i);
    const int64_t uu = (int64_t)(((r & 0xffffffffull) * (uint64_t)V) >> 32);
    const int64_t blk = uu * B / V;
    const int64_t s0 = block_start(blk, V, B), s1 = block_start(blk + 1, V, B);
    const int64_t rest = V - (s1 - s0);
    if (rest <= 0) return false;
    const int64_t x = (int64_t)(((r >> 32) * (uint64_t)rest) >> 32);
    *u = (uint32_t)uu;
    *v = (uint32_t)(x < s0 ? x : x + (s1 - s0));
    return true;
}

}  // namespace lvrng
