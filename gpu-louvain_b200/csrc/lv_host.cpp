// lv_host.cpp -- host-side I/O and seeded graph generators (no GPU needed).
//
//   lv_read_mtx           readInputData (utils.cu:9-62): symmetric Matrix Market
//                         -> CSR in file order, parsed from an mmap'd buffer.
//   lv_write_mtx          symmetric Matrix Market writer (i > j, 1-based).
//   lv_print_communities  printOriginalToCommunity (modularity_optimisation.cu:403-418).
//   lv_gen_rmat / lv_gen_planted   seeded synthetic inputs (counter-based RNG,
//                         identical on the host, the device and in numpy).
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/louvain_b200.h"
#include "lv_rng.h"

namespace {

// ---------------------------------------------------------------------------
// Matrix Market reader
// ---------------------------------------------------------------------------
struct Mapped {
    const char *p = nullptr;
    size_t n = 0;
    int fd = -1;
    ~Mapped() {
        if (p) munmap((void *)p, n);
        if (fd >= 0) close(fd);
    }
};

inline const char *skip_ws(const char *p, const char *end) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
    return p;
}

inline bool parse_i64(const char *&p, const char *end, long long *out) {
    p = skip_ws(p, end);
    bool neg = false;
    if (p < end && (*p == '-' || *p == '+')) { neg = *p == '-'; ++p; }
    if (p >= end || *p < '0' || *p > '9') return false;
    long long v = 0;
    while (p < end && *p >= '0' && *p <= '9') { v = v * 10 + (*p - '0'); ++p; }
    *out = neg ? -v : v;
    return true;
}

// Fast path of the decimal -> float conversion: a token of the form
// [+-]digits[.digits][(e|E)[+-]digits] with at most 19 significant digits
// whose value m * 10^k has m < 2^53 and |k| <= 22.  Then m and 10^|k| are
// exact doubles and one multiplication or division gives d, the double
// nearest the decimal value x (Clinger's fast path).  Rounding d to float
// gives the float nearest x unless d is exactly halfway between two
// adjacent floats (a boundary that d can reach by rounding while x lies on
// one side of it): every midpoint is a double, so for any other d, x and d
// lie on the same side of every midpoint.  Returns false (the caller uses
// strtof) for every other token, a midpoint d, or a d outside the normal
// float range.
inline bool fast_f32(const char *p, const char *q, float *out) {
    static const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                      1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
    bool neg = false;
    if (p < q && (*p == '+' || *p == '-')) { neg = *p == '-'; ++p; }
    uint64_t m = 0;
    int sig = 0, frac = 0, digits = 0;
    for (; p < q && *p >= '0' && *p <= '9'; ++p, ++digits) {
        if (m == 0 && *p == '0') continue;   // leading zeros
        if (++sig > 19) return false;
        m = m * 10 + (uint64_t)(*p - '0');
    }
    if (p < q && *p == '.') {
        for (++p; p < q && *p >= '0' && *p <= '9'; ++p, ++digits) {
            ++frac;
            if (m == 0 && *p == '0') continue;
            if (++sig > 19) return false;
            m = m * 10 + (uint64_t)(*p - '0');
        }
    }
    if (digits == 0) return false;
    int ex = 0;
    if (p < q && (*p == 'e' || *p == 'E')) {
        ++p;
        bool eneg = false;
        if (p < q && (*p == '+' || *p == '-')) { eneg = *p == '-'; ++p; }
        if (p >= q || *p < '0' || *p > '9') return false;
        for (; p < q && *p >= '0' && *p <= '9'; ++p) {
            if (ex > 1000) return false;
            ex = ex * 10 + (*p - '0');
        }
        if (eneg) ex = -ex;
    }
    if (p != q) return false;
    if (m == 0) {
        *out = neg ? -0.0f : 0.0f;
        return true;
    }
    const int k = ex - frac;
    if (m >= (1ull << 53) || k < -22 || k > 22) return false;
    const double d = k >= 0 ? (double)m * kPow10[k] : (double)m / kPow10[-k];
    uint64_t bits;
    std::memcpy(&bits, &d, sizeof bits);
    const int e2 = (int)((bits >> 52) & 0x7ff) - 1023;
    if (e2 < -126 || e2 > 127) return false;                 // subnormal or overflowing float
    if ((bits & 0x1fffffffull) == 0x10000000ull) return false;   // a float midpoint
    const float f = (float)d;
    *out = neg ? -f : f;
    return true;
}

// Decimal -> float with the rounding of strtof (the reference reads with
// `file >> w` into a float): the fast path above, else strtof on the token
// copied to a NUL-terminated buffer.
inline bool parse_f32(const char *&p, const char *end, float *out) {
    p = skip_ws(p, end);
    const char *q = p;
    while (q < end && !(*q == ' ' || *q == '\t' || *q == '\r' || *q == '\n')) ++q;
    size_t len = (size_t)(q - p);
    if (len == 0 || len > 120) return false;
    if (fast_f32(p, q, out)) {
        p = q;
        return true;
    }
    char buf[128];
    std::memcpy(buf, p, len);
    buf[len] = 0;
    char *e = nullptr;
    errno = 0;
    float v = std::strtof(buf, &e);
    if (e == buf) return false;
    *out = v;
    p = q;
    return true;
}

// The entries of the data section as the reference reads them: a stream of
// whitespace-separated tokens, `v1 v2 [w]` per entry (utils.cu:20-31).
int parse_entries(const char *p, const char *end, long long nnz, bool pattern, int32_t V, int32_t *ea,
                  int32_t *eb, float *ew) {
    for (long long i = 0; i < nnz; ++i) {
        long long a, b;
        float wv = 1.0f;
        if (!parse_i64(p, end, &a) || !parse_i64(p, end, &b)) return LV_ERR_IO;
        if (!pattern && !parse_f32(p, end, &wv)) return LV_ERR_IO;
        a -= 1;
        b -= 1;
        if (a < 0 || b < 0 || a >= V || b >= V) return LV_ERR_INVALID;
        ea[i] = (int32_t)a;
        eb[i] = (int32_t)b;
        ew[i] = wv;
    }
    return LV_OK;
}

constexpr int PARSE_SEQUENTIAL = -1;

// Tokens on the line [p, eol), up to 4.
inline int line_tokens(const char *p, const char *eol) {
    int n = 0;
    bool in = false;
    for (; p < eol && n < 4; ++p) {
        const bool ws = *p == ' ' || *p == '\t' || *p == '\r';
        if (!ws && !in) ++n;
        in = !ws;
    }
    return n;
}

// The same entries parsed by all host threads.  The data section is cut into
// byte ranges at line starts; a first pass counts each range's entries, a
// second parses them into their file-order positions.  This equals the
// token-stream reading when every non-blank line holds exactly one entry (2
// tokens for pattern files, 3 otherwise); on any other layout, and on any
// parse or range error (whose code depends on file order), the caller falls
// back to the sequential reading (PARSE_SEQUENTIAL).  Small files are read
// sequentially.
int parse_entries_parallel(const char *p, const char *end, long long nnz, bool pattern, int32_t V,
                           int32_t *ea, int32_t *eb, float *ew) {
    const size_t n = (size_t)(end - p);
    const int T = omp_get_max_threads();
    if (T < 2 || n < ((size_t)1 << 22) || nnz < 100000) return PARSE_SEQUENTIAL;
    const int want = pattern ? 2 : 3;
    std::vector<const char *> cut((size_t)T + 1);
    cut[0] = p;
    cut[(size_t)T] = end;
    for (int t = 1; t < T; ++t) {
        const char *c = p + n / (size_t)T * (size_t)t;
        if (c < cut[(size_t)t - 1]) c = cut[(size_t)t - 1];
        const char *nl = c < end ? (const char *)std::memchr(c, '\n', (size_t)(end - c)) : nullptr;
        cut[(size_t)t] = nl ? nl + 1 : end;
    }
    std::vector<long long> cnt((size_t)T, 0);
    std::vector<int> bad((size_t)T, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        const char *q = cut[(size_t)t], *e = cut[(size_t)t + 1];
        long long c = 0;
        while (q < e) {
            const char *nl = (const char *)std::memchr(q, '\n', (size_t)(e - q));
            const char *eol = nl ? nl : e;
            const int k = line_tokens(q, eol);
            if (k == want) ++c;
            else if (k != 0) { bad[(size_t)t] = 1; break; }
            q = nl ? nl + 1 : e;
        }
        cnt[(size_t)t] = c;
    }
    long long total = 0;
    std::vector<long long> first((size_t)T + 1, 0);
    for (int t = 0; t < T; ++t) {
        if (bad[(size_t)t]) return PARSE_SEQUENTIAL;
        first[(size_t)t] = total;
        total += cnt[(size_t)t];
    }
    if (total < nnz) return PARSE_SEQUENTIAL;
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        const char *q = cut[(size_t)t], *e = cut[(size_t)t + 1];
        long long i = first[(size_t)t];
        while (q < e && i < nnz) {
            const char *nl = (const char *)std::memchr(q, '\n', (size_t)(e - q));
            const char *eol = nl ? nl : e;
            if (line_tokens(q, eol) != 0) {
                const char *r = q;
                long long a, b;
                float wv = 1.0f;
                if (!parse_i64(r, eol, &a) || !parse_i64(r, eol, &b) || (!pattern && !parse_f32(r, eol, &wv)) ||
                    a < 1 || b < 1 || a > V || b > V) {
                    bad[(size_t)t] = 1;
                    break;
                }
                ea[i] = (int32_t)(a - 1);
                eb[i] = (int32_t)(b - 1);
                ew[i] = wv;
                ++i;
            }
            q = nl ? nl + 1 : e;
        }
    }
    for (int t = 0; t < T; ++t)
        if (bad[(size_t)t]) return PARSE_SEQUENTIAL;
    return LV_OK;
}

constexpr char CSR_MAGIC[8] = {'L', 'V', 'C', 'S', 'R', '0', '0', '2'};
struct CsrHeader {
    char magic[8];
    int64_t V;
    int64_t E;
    float m_ref;
    uint32_t pad;
    int64_t src_size;       // size of the file the CSR was read from (0: unknown)
    int64_t src_mtime_ns;   // its modification time in nanoseconds (0: unknown)
};

}  // namespace

extern "C" {

void lv_free_host(void *p) { std::free(p); }

int lv_write_csr_stamped(const char *path, int32_t V, int64_t E, const int32_t *rowptr, const int32_t *col,
                         const float *w, float m_ref, int64_t src_size, int64_t src_mtime_ns) {
    if (!path || V < 0 || E < 0 || !rowptr || (E > 0 && (!col || !w))) return LV_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) return LV_ERR_IO;
    CsrHeader h{};
    std::memcpy(h.magic, CSR_MAGIC, 8);
    h.V = V;
    h.E = E;
    h.m_ref = m_ref;
    h.src_size = src_size;
    h.src_mtime_ns = src_mtime_ns;
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
              std::fwrite(rowptr, sizeof(int32_t), (size_t)V + 1, f) == (size_t)V + 1 &&
              (E == 0 || (std::fwrite(col, sizeof(int32_t), (size_t)E, f) == (size_t)E &&
                          std::fwrite(w, sizeof(float), (size_t)E, f) == (size_t)E));
    ok = (std::fclose(f) == 0) && ok;
    return ok ? LV_OK : LV_ERR_IO;
}

int lv_write_csr(const char *path, int32_t V, int64_t E, const int32_t *rowptr, const int32_t *col, const float *w,
                 float m_ref) {
    return lv_write_csr_stamped(path, V, E, rowptr, col, w, m_ref, 0, 0);
}

int lv_read_csr_stamp(const char *path, int64_t *src_size, int64_t *src_mtime_ns) {
    if (!path || !src_size || !src_mtime_ns) return LV_ERR_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) return LV_ERR_IO;
    CsrHeader h;
    const bool ok = std::fread(&h, sizeof h, 1, f) == 1 && std::memcmp(h.magic, CSR_MAGIC, 8) == 0;
    std::fclose(f);
    if (!ok) return LV_ERR_IO;
    *src_size = h.src_size;
    *src_mtime_ns = h.src_mtime_ns;
    return LV_OK;
}

int lv_read_csr(const char *path, int32_t *Vout, int64_t *Eout, int32_t **rowptr, int32_t **col, float **w,
                float *m_ref) {
    if (!path || !Vout || !Eout || !rowptr || !col || !w) return LV_ERR_INVALID;
    Mapped m;
    m.fd = open(path, O_RDONLY);
    if (m.fd < 0) return LV_ERR_IO;
    struct stat sb;
    if (fstat(m.fd, &sb) != 0 || (size_t)sb.st_size < sizeof(CsrHeader)) return LV_ERR_IO;
    m.n = (size_t)sb.st_size;
    void *mp = mmap(nullptr, m.n, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (mp == MAP_FAILED) return LV_ERR_IO;
    m.p = (const char *)mp;
    CsrHeader h;
    std::memcpy(&h, m.p, sizeof h);
    if (std::memcmp(h.magic, CSR_MAGIC, 8) != 0 || h.V < 0 || h.V > 0x7ffffffeLL || h.E < 0 || h.E > 0x7fffffffLL)
        return LV_ERR_IO;
    const size_t need = sizeof h + 4 * ((size_t)h.V + 1) + 8 * (size_t)h.E;
    if (m.n != need) return LV_ERR_IO;
    int32_t *rp = (int32_t *)std::malloc(4 * ((size_t)h.V + 1));
    int32_t *cl = (int32_t *)std::malloc(4 * (size_t)(h.E > 0 ? h.E : 1));
    float *wt = (float *)std::malloc(4 * (size_t)(h.E > 0 ? h.E : 1));
    if (!rp || !cl || !wt) {
        std::free(rp); std::free(cl); std::free(wt);
        return LV_ERR_NOMEM;
    }
    // copied and checked (offsets non-decreasing from 0 to E, columns in
    // [0, V)) by all host threads, in 1 MB-sized pieces
    const char *const q0 = m.p + sizeof h;
    const char *const q1 = q0 + 4 * ((size_t)h.V + 1);
    const char *const q2 = q1 + 4 * (size_t)h.E;
    constexpr int64_t PIECE = 1 << 18;   // 4-byte words
    const int64_t nrp = h.V + 1, ne = h.E;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t s0 = 0; s0 < nrp; s0 += PIECE) {
        const int64_t s1 = s0 + PIECE < nrp ? s0 + PIECE : nrp;
        std::memcpy(rp + s0, q0 + 4 * s0, 4 * (size_t)(s1 - s0));
    }
#pragma omp parallel for schedule(dynamic, 4) reduction(| : bad)
    for (int64_t s0 = 0; s0 < ne; s0 += PIECE) {
        const int64_t s1 = s0 + PIECE < ne ? s0 + PIECE : ne;
        std::memcpy(cl + s0, q1 + 4 * s0, 4 * (size_t)(s1 - s0));
        std::memcpy(wt + s0, q2 + 4 * s0, 4 * (size_t)(s1 - s0));
        for (int64_t e = s0; e < s1; ++e) bad |= (cl[e] < 0 || cl[e] >= h.V) ? 1 : 0;
    }
    bad |= (rp[0] != 0 || (int64_t)rp[h.V] != h.E) ? 1 : 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t v = 0; v < h.V; ++v) bad |= rp[v + 1] < rp[v] ? 1 : 0;
    if (bad) {
        std::free(rp); std::free(cl); std::free(wt);
        return LV_ERR_IO;
    }
    *Vout = (int32_t)h.V;
    *Eout = h.E;
    *rowptr = rp;
    *col = cl;
    *w = wt;
    if (m_ref) *m_ref = h.m_ref;
    return LV_OK;
}

}  // extern "C"

namespace {

// The entries of a Matrix Market file in malloc'd arrays, freed with the
// object unless released to a caller.  They are not initialised when
// allocated: the parsing threads fault their pages in as they fill them.
struct Entries {
    int32_t *a = nullptr, *b = nullptr;
    float *w = nullptr;
    size_t n = 0;
    Entries() = default;
    Entries(const Entries &) = delete;
    Entries &operator=(const Entries &) = delete;
    ~Entries() { std::free(a); std::free(b); std::free(w); }
    bool alloc(size_t k) {
        const size_t c = k > 0 ? k : 1;
        a = (int32_t *)std::malloc(sizeof(int32_t) * c);
        b = (int32_t *)std::malloc(sizeof(int32_t) * c);
        w = (float *)std::malloc(sizeof(float) * c);
        n = k;
        return a && b && w;
    }
    void release() { a = b = nullptr; w = nullptr; }
};

// The header and the entries of a Matrix Market file, in file order
// (0-based): the vertex count is the size line's second number.
int read_mtx_entries(const char *path, int32_t *Vout, Entries &en) {
    Mapped m;
    m.fd = open(path, O_RDONLY);
    if (m.fd < 0) return LV_ERR_IO;
    struct stat sb;
    if (fstat(m.fd, &sb) != 0) return LV_ERR_IO;
    m.n = (size_t)sb.st_size;
    if (m.n == 0) return LV_ERR_IO;
    void *mp = mmap(nullptr, m.n, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (mp == MAP_FAILED) return LV_ERR_IO;
    m.p = (const char *)mp;
    const char *p = m.p, *end = m.p + m.n;
    bool pattern = false;
    // header: '%' lines are comments (utils.cu:14-16); blank lines skipped
    for (;;) {
        if (p >= end) return LV_ERR_IO;
        const char *eol = (const char *)std::memchr(p, '\n', (size_t)(end - p));
        if (!eol) eol = end;
        if (*p == '%') {
            if ((size_t)(eol - p) >= 14 && std::strncmp(p, "%%MatrixMarket", 14) == 0) {
                std::string line(p, eol);
                if (line.find("pattern") != std::string::npos) pattern = true;
            }
            p = eol < end ? eol + 1 : end;
            continue;
        }
        const char *q = skip_ws(p, eol);
        if (q == eol) {   // blank line
            p = eol < end ? eol + 1 : end;
            continue;
        }
        break;
    }
    long long rows = 0, cols = 0, nnz = 0;
    // size line "rows cols nnz"; the vertex count is the second number (utils.cu:18)
    if (!parse_i64(p, end, &rows) || !parse_i64(p, end, &cols) || !parse_i64(p, end, &nnz))
        return LV_ERR_IO;
    if (cols < 0 || nnz < 0) return LV_ERR_IO;
    if (cols > 0x7ffffffeLL) return LV_ERR_TOO_LARGE;
    // an entry takes at least 4 bytes ("1 2" and a line break; the last may
    // lack the break), so a size line that promises more entries than the
    // rest of the file can hold is a short file: rejected before the entry
    // arrays are sized by it
    if (nnz > (long long)((size_t)(end - p) / 4) + 1) return LV_ERR_IO;
    const int32_t V = (int32_t)cols;
    if (!en.alloc((size_t)nnz)) return LV_ERR_NOMEM;
    int prc = parse_entries_parallel(p, end, nnz, pattern, V, en.a, en.b, en.w);
    if (prc == PARSE_SEQUENTIAL) prc = parse_entries(p, end, nnz, pattern, V, en.a, en.b, en.w);
    if (prc != LV_OK) return prc;
    *Vout = V;
    return LV_OK;
}

// M as the reference accumulates it: a sequential float sum of every entry's
// weight, counted twice for off-diagonal entries, halved (utils.cu:36-46).
float reference_m(const Entries &en) {
    float M = 0;
    for (size_t i = 0; i < en.n; ++i) {
        if (en.a[i] != en.b[i]) M += en.w[i];
        M += en.w[i];
    }
    return M / 2;
}

int read_mtx_host_csr(const char *path, int32_t *Vout, int64_t *Eout, int32_t **rowptr_out, int32_t **col_out,
                      float **w_out, float *m_ref);

}  // namespace

extern "C" {

int lv_read_mtx(const char *path, int32_t *Vout, int64_t *Eout, int32_t **rowptr_out,
                int32_t **col_out, float **w_out, float *m_ref) {
    if (!path || !Vout || !Eout || !rowptr_out || !col_out || !w_out) return LV_ERR_INVALID;
    try {
        return read_mtx_host_csr(path, Vout, Eout, rowptr_out, col_out, w_out, m_ref);
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
}

}  // extern "C"

namespace {

// lv_read_mtx's body; its allocations may throw std::bad_alloc, which the
// entry point turns into LV_ERR_NOMEM
int read_mtx_host_csr(const char *path, int32_t *Vout, int64_t *Eout, int32_t **rowptr_out, int32_t **col_out,
                      float **w_out, float *m_ref) {
    int32_t V = 0;
    Entries en;
    const int prc = read_mtx_entries(path, &V, en);
    if (prc != LV_OK) return prc;
    const long long nnz = (long long)en.n;
    const int32_t *ea = en.a, *eb = en.b;
    const float *ew = en.w;
    // entry "v1 v2 w" gives row v1 the pair (v2, w) and, unless it is a
    // self-loop, row v2 the pair (v1, w); each row keeps file order
    // (utils.cu:32-59).  T threads take contiguous ranges of entries: each
    // counts its pairs per row, the counts become per-thread offsets inside
    // each row (thread t's pairs of a row follow those of threads < t), and
    // each thread writes its range in order.  Fewer threads when the
    // per-thread counts would pass 1 GB.
    const float M = reference_m(en);
    int T = omp_get_max_threads() > 0 ? omp_get_max_threads() : 1;
    if (T > 32) T = 32;
    if (nnz < (1 << 16)) T = 1;
    while (T > 1 && (double)T * (double)V * 4.0 > (double)(1ll << 30)) T /= 2;
    const size_t Vs = (size_t)V;
    std::unique_ptr<uint32_t[]> cnt(new uint32_t[(size_t)T * Vs + 1]);
    std::unique_ptr<int64_t[]> deg(new int64_t[Vs + 1]);
    auto range = [&](int t, long long *lo, long long *hi) {
        *lo = nnz * t / T;
        *hi = nnz * (t + 1) / T;
    };
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        uint32_t *c = cnt.get() + (size_t)t * Vs;
        std::fill(c, c + Vs, 0u);
        long long lo, hi;
        range(t, &lo, &hi);
        for (long long i = lo; i < hi; ++i) {
            const int32_t a = ea[(size_t)i], b = eb[(size_t)i];
            c[(size_t)a]++;
            if (a != b) c[(size_t)b]++;
        }
    }
    int64_t E = 0;
#pragma omp parallel for num_threads(T) schedule(static) reduction(+ : E)
    for (int64_t v = 0; v < (int64_t)V; ++v) {
        int64_t d = 0;
        for (int t = 0; t < T; ++t) d += cnt[(size_t)t * Vs + (size_t)v];
        deg[(size_t)v] = d;
        E += d;
    }
    if (E > 0x7fffffffLL) return LV_ERR_TOO_LARGE;
    // per-thread offsets inside each row (every partial sum is <= E < 2^31)
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t v = 0; v < (int64_t)V; ++v) {
        uint32_t run = 0;
        for (int t = 0; t < T; ++t) {
            const uint32_t c = cnt[(size_t)t * Vs + (size_t)v];
            cnt[(size_t)t * Vs + (size_t)v] = run;
            run += c;
        }
    }
    int32_t *rp = (int32_t *)std::malloc(sizeof(int32_t) * (Vs + 1));
    int32_t *cl = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
    float *wt = (float *)std::malloc(sizeof(float) * (size_t)(E > 0 ? E : 1));
    if (!rp || !cl || !wt) {
        std::free(rp); std::free(cl); std::free(wt);
        return LV_ERR_NOMEM;
    }
    int64_t acc = 0;
    for (int32_t v = 0; v < V; ++v) {
        rp[v] = (int32_t)acc;
        acc += deg[(size_t)v];
    }
    rp[V] = (int32_t)acc;
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        uint32_t *c = cnt.get() + (size_t)t * Vs;
        long long lo, hi;
        range(t, &lo, &hi);
        for (long long i = lo; i < hi; ++i) {
            const int32_t a = ea[(size_t)i], b = eb[(size_t)i];
            const float wv = ew[(size_t)i];
            const int64_t pa = (int64_t)rp[a] + c[(size_t)a]++;
            cl[pa] = b;
            wt[pa] = wv;
            if (a != b) {
                const int64_t pb = (int64_t)rp[b] + c[(size_t)b]++;
                cl[pb] = a;
                wt[pb] = wv;
            }
        }
    }
    *Vout = V;
    *Eout = E;
    *rowptr_out = rp;
    *col_out = cl;
    *w_out = wt;
    if (m_ref) *m_ref = M;
    return LV_OK;
}

}  // namespace

extern "C" {

int lv_read_mtx_entries(const char *path, int32_t *Vout, int64_t *nnz_out, int32_t **v1, int32_t **v2, float **w) {
    if (!path || !Vout || !nnz_out || !v1 || !v2 || !w) return LV_ERR_INVALID;
    int32_t V = 0;
    Entries en;
    try {
        const int prc = read_mtx_entries(path, &V, en);
        if (prc != LV_OK) return prc;
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
    *Vout = V;
    *nnz_out = (int64_t)en.n;
    *v1 = en.a;
    *v2 = en.b;
    *w = en.w;
    en.release();   // the caller frees them (lv_free_host)
    return LV_OK;
}

int lv_read_mtx_device(const char *path, int32_t device, int32_t *Vout, int64_t *Eout, int32_t **d_rowptr,
                       int32_t **d_col, float **d_w, float *m_ref) {
    if (!path || !Vout || !Eout || !d_rowptr || !d_col || !d_w) return LV_ERR_INVALID;
    int32_t V = 0;
    Entries en;
    try {
        const int prc = read_mtx_entries(path, &V, en);
        if (prc != LV_OK) return prc;
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
    const int rc = lv_csr_from_entries_device(device, V, (int64_t)en.n, en.a, en.b, en.w, Eout, d_rowptr, d_col,
                                              d_w);
    if (rc != LV_OK) return rc;
    *Vout = V;
    if (m_ref) *m_ref = reference_m(en);
    return LV_OK;
}

// ---------------------------------------------------------------------------
// predictor files of the learned active-set mode
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

// The value after `"key"` and a colon in the JSON text, or nullptr.  The
// files are the flat objects train_active_set.py writes; a key is matched
// only where it is followed by a colon (a key name inside a string value is
// not).
const char *json_value(const std::string &text, const char *key) {
    const std::string k = std::string("\"") + key + "\"";
    for (size_t at = text.find(k); at != std::string::npos; at = text.find(k, at + 1)) {
        size_t i = at + k.size();
        while (i < text.size() && (text[i] == ' ' || text[i] == '\t' || text[i] == '\r' || text[i] == '\n')) ++i;
        if (i < text.size() && text[i] == ':') {
            ++i;
            while (i < text.size() && (text[i] == ' ' || text[i] == '\t' || text[i] == '\r' || text[i] == '\n'))
                ++i;
            return text.c_str() + i;
        }
    }
    return nullptr;
}

bool json_number(const std::string &text, const char *key, double *out) {
    const char *v = json_value(text, key);
    if (!v) return false;
    char *e = nullptr;
    const double x = std::strtod(v, &e);
    if (e == v || !std::isfinite(x)) return false;
    *out = x;
    return true;
}

}  // namespace

extern "C" {

static int read_active_model_body(const char *path, uint16_t *model, int32_t cap, int32_t *n_params,
                                  float *logit_threshold, lv_opts *opts);

int lv_read_active_model(const char *path, uint16_t *model, int32_t cap, int32_t *n_params,
                         float *logit_threshold, lv_opts *opts) {
    if (!path || !model || !n_params || !logit_threshold || cap < 0) return LV_ERR_INVALID;
    try {
        return read_active_model_body(path, model, cap, n_params, logit_threshold, opts);
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
}

static int read_active_model_body(const char *path, uint16_t *model, int32_t cap, int32_t *n_params,
                                  float *logit_threshold, lv_opts *opts) {
    std::string text;
    {
        FILE *f = std::fopen(path, "rb");
        if (!f) return LV_ERR_IO;
        char buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) {
            text.append(buf, got);
            if (text.size() > ((size_t)1 << 24)) {   // far beyond any predictor file
                std::fclose(f);
                return LV_ERR_IO;
            }
        }
        std::fclose(f);
    }
    const char *v = json_value(text, "model_bf16");
    if (!v || *v != '[') return LV_ERR_IO;
    ++v;
    int32_t n = 0;
    for (;;) {
        while (*v == ' ' || *v == '\t' || *v == '\r' || *v == '\n') ++v;
        if (*v == ']') break;
        if (*v < '0' || *v > '9') return LV_ERR_IO;
        char *e = nullptr;
        const long x = std::strtol(v, &e, 10);
        if (x < 0 || x > 65535) return LV_ERR_IO;
        if (n >= LV_ACTIVE_MODEL_SIZE) return LV_ERR_INVALID;   // more parameters than the model has
        if (n < cap) model[n] = (uint16_t)x;
        ++n;
        v = e;
        while (*v == ' ' || *v == '\t' || *v == '\r' || *v == '\n') ++v;
        if (*v == ',') ++v;
        else if (*v != ']') return LV_ERR_IO;
    }
    if (n != LV_ACTIVE_MODEL_SIZE) return LV_ERR_INVALID;
    if (cap < n) return LV_ERR_INVALID;
    double thr = 0;
    if (!json_number(text, "logit_threshold", &thr)) return LV_ERR_IO;
    *n_params = n;
    *logit_threshold = (float)thr;
    if (opts) {
        double x = 0;
        opts->active_set = 1;
        if (json_number(text, "full_every", &x) && x >= 1 && x <= 1e6) opts->active_full_every = (int32_t)x;
        if (json_number(text, "active_start", &x) && x >= 0 && x <= 1) opts->active_start = (float)x;
        if (json_number(text, "min_recall", &x) && x >= 0 && x <= 1) opts->active_min_recall = (float)x;
    }
    return LV_OK;
}

int lv_write_mtx(const char *path, int32_t V, int64_t n_edges, const int32_t *u, const int32_t *v,
                 const float *w) {
    if (!path || V < 0 || n_edges < 0 || (n_edges > 0 && (!u || !v))) return LV_ERR_INVALID;
    FILE *f = std::fopen(path, "w");
    if (!f) return LV_ERR_IO;
    std::vector<char> buf(1 << 22);
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n");
    std::fprintf(f, "%d %d %lld\n", V, V, (long long)n_edges);
    // lines "a b w" (larger id first, 1-based, %.9g: the float reads back
    // exactly) formatted by all host threads, a block of entries at a time,
    // each thread into its own buffer; the buffers are written in order
    constexpr int64_t BLOCK = 1 << 20;
    constexpr size_t LINE_MAX_BYTES = 64;   // two ints, a %.9g float, 2 blanks and a break
    const int T = omp_get_max_threads() > 0 ? omp_get_max_threads() : 1;
    const int64_t per = (BLOCK + T - 1) / T;
    std::unique_ptr<char[]> out(new (std::nothrow) char[(size_t)T * (size_t)per * LINE_MAX_BYTES]);
    if (!out) {
        std::fclose(f);
        return LV_ERR_NOMEM;
    }
    std::vector<size_t> len((size_t)T);
    bool ok = true;
    for (int64_t b0 = 0; b0 < n_edges && ok; b0 += BLOCK) {
        const int64_t b1 = b0 + BLOCK < n_edges ? b0 + BLOCK : n_edges;
#pragma omp parallel for num_threads(T) schedule(static, 1)
        for (int t = 0; t < T; ++t) {
            const int64_t i0 = b0 + per * t, i1 = i0 + per < b1 ? i0 + per : b1;
            char *const o = out.get() + (size_t)t * (size_t)per * LINE_MAX_BYTES;
            char *q = o;
            for (int64_t i = i0; i < i1; ++i) {
                int32_t a = u[i], b = v[i];
                if (a < b) std::swap(a, b);
                q += std::snprintf(q, LINE_MAX_BYTES, "%d %d %.9g\n", a + 1, b + 1, w ? (double)w[i] : 1.0);
            }
            len[(size_t)t] = i1 > i0 ? (size_t)(q - o) : 0;
        }
        for (int t = 0; t < T && ok; ++t)
            ok = len[(size_t)t] == 0 ||
                 std::fwrite(out.get() + (size_t)t * (size_t)per * LINE_MAX_BYTES, 1, len[(size_t)t], f) ==
                     len[(size_t)t];
    }
    const int rc = std::fclose(f);
    return rc == 0 && ok ? LV_OK : LV_ERR_IO;
}

// Stable LSD radix sort of n 64-bit keys on bits [lo, hi), 8 bits per pass,
// all host threads.  The buffers are left uninitialised so that the threads
// that fill them also fault their pages in (a zero-filled std::vector would
// touch every page from one thread first).
static void radix_sort_key_bits(std::unique_ptr<uint64_t[]> &a, size_t n, int lo, int hi) {
    if (n < 2 || hi <= lo) return;
    std::unique_ptr<uint64_t[]> b(new uint64_t[n]);
    const int nt = omp_get_max_threads() > 0 ? omp_get_max_threads() : 1;
    std::vector<size_t> hist((size_t)nt * 256);
    for (int shift = lo; shift < hi; shift += 8) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num();
            const size_t i0 = n * t / nt, i1 = n * (t + 1) / nt;
            size_t *h = hist.data() + (size_t)t * 256;
            for (size_t i = i0; i < i1; ++i) h[(a[i] >> shift) & 255]++;
        }
        size_t run = 0;
        for (int d = 0; d < 256; ++d)
            for (int t = 0; t < nt; ++t) {
                const size_t c = hist[(size_t)t * 256 + d];
                hist[(size_t)t * 256 + d] = run;
                run += c;
            }
#pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num();
            const size_t i0 = n * t / nt, i1 = n * (t + 1) / nt;
            size_t *h = hist.data() + (size_t)t * 256;
            for (size_t i = i0; i < i1; ++i) b[h[(a[i] >> shift) & 255]++] = a[i];
        }
        a.swap(b);
    }
}

// The lines of consecutive community ranges are formatted by all host
// threads into their own buffers (ranges of about equal member counts), then
// written in order.  Every buffer is allocated before the threads start, so
// an allocation failure returns LV_ERR_NOMEM instead of ending the process.
static int print_communities_impl(const char *path, const int32_t *orig2comm, int32_t V0,
                                  int32_t num_communities) {
    // vertices grouped by community with members in increasing id: keys
    // (community << 32 | vertex) in vertex order, stably sorted on the
    // community bits only (the same order as a counting sort, built by all
    // host threads)
    const size_t nv = V0 > 0 ? (size_t)V0 : 1;
    std::unique_ptr<uint64_t[]> key(new uint64_t[nv]);
    int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
    for (int32_t v = 0; v < V0; ++v) {
        const int32_t c = orig2comm[v];
        if (c < 0 || c >= num_communities) bad = 1;
        key[(size_t)v] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)v;
    }
    if (bad) return LV_ERR_INVALID;
    int cbits = 0;
    while (cbits < 31 && ((int64_t)1 << cbits) < (int64_t)num_communities) ++cbits;
    radix_sort_key_bits(key, (size_t)V0, 32, 32 + cbits);
    // start[c] = first position whose community is >= c (empty communities
    // get an empty range); mem = the members in that order
    std::unique_ptr<int64_t[]> start(new int64_t[(size_t)num_communities + 1]);
    std::unique_ptr<int32_t[]> mem(new int32_t[nv]);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)V0; ++i) {
        const int32_t c = (int32_t)(key[(size_t)i] >> 32);
        mem[(size_t)i] = (int32_t)(uint32_t)key[(size_t)i];
        const int32_t prev = i > 0 ? (int32_t)(key[(size_t)i - 1] >> 32) : -1;
        for (int32_t x = prev + 1; x <= c; ++x) start[(size_t)x] = i;
    }
    {
        const int32_t last = V0 > 0 ? (int32_t)(key[(size_t)V0 - 1] >> 32) : -1;
        for (int32_t x = last + 1; x <= num_communities; ++x) start[(size_t)x] = V0;
    }
    key.reset();
    const int T = omp_get_max_threads() > 0 ? omp_get_max_threads() : 1;
    const int64_t per = ((int64_t)V0 + num_communities) / T + 1;
    std::vector<int32_t> cut((size_t)T + 1, num_communities);
    cut[0] = 0;
    for (int t = 1, c = 0; t < T; ++t) {
        while (c < num_communities && start[(size_t)c] + c < per * t) ++c;
        cut[(size_t)t] = c;
    }
    // at most 11 characters per number plus a separator
    std::vector<std::unique_ptr<char[]>> buf((size_t)T);
    for (int t = 0; t < T; ++t) {
        const int32_t c0 = cut[(size_t)t], c1 = cut[(size_t)t + 1];
        if (c1 <= c0) continue;
        buf[(size_t)t].reset(new (std::nothrow)
                                 char[(size_t)(start[(size_t)c1] - start[(size_t)c0] + (c1 - c0)) * 12]);
        if (!buf[(size_t)t]) return LV_ERR_NOMEM;
    }
    // decimal digits of x >= 0 at p, two per division from a table of
    // "00".."99"; returns the end
    static const char kPairs[201] =
        "00010203040506070809101112131415161718192021222324252627282930313233343536373839"
        "40414243444546474849505152535455565758596061626364656667686970717273747576777879"
        "8081828384858687888990919293949596979899";
    auto put_int = [](char *p, int64_t x) {
        uint64_t u = (uint64_t)x;
        int n = 1;
        for (uint64_t t = u; t >= 10; t /= 10) ++n;
        char *const e = p + n;
        char *q = e;
        while (u >= 100) {
            const unsigned r = (unsigned)(u % 100);
            u /= 100;
            q -= 2;
            q[0] = kPairs[2 * r];
            q[1] = kPairs[2 * r + 1];
        }
        if (u >= 10) {
            q -= 2;
            q[0] = kPairs[2 * u];
            q[1] = kPairs[2 * u + 1];
        } else {
            *--q = (char)('0' + u);
        }
        return e;
    };
    std::vector<size_t> len((size_t)T, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        const int32_t c0 = cut[(size_t)t], c1 = cut[(size_t)t + 1];
        if (c1 <= c0) continue;
        char *const o = buf[(size_t)t].get();
        char *q = o;
        for (int32_t c = c0; c < c1; ++c) {
            q = put_int(q, (int64_t)c + 1);
            for (int64_t i = start[(size_t)c]; i < start[(size_t)c + 1]; ++i) {
                *q++ = ' ';
                q = put_int(q, (int64_t)mem[(size_t)i] + 1);
            }
            *q++ = '\n';
        }
        len[(size_t)t] = (size_t)(q - o);
    }
    FILE *f = path ? std::fopen(path, "w") : stdout;
    if (!f) return LV_ERR_IO;
    char head[32];
    char *he = put_int(head, num_communities);
    *he++ = '\n';
    bool ok = std::fwrite(head, 1, (size_t)(he - head), f) == (size_t)(he - head);
    for (int t = 0; t < T && ok; ++t)
        ok = len[(size_t)t] == 0 || std::fwrite(buf[(size_t)t].get(), 1, len[(size_t)t], f) == len[(size_t)t];
    std::fflush(f);
    if (path) ok = (std::fclose(f) == 0) && ok;
    return ok ? LV_OK : LV_ERR_IO;
}

int lv_print_communities(const char *path, const int32_t *orig2comm, int32_t V0,
                         int32_t num_communities) {
    if (V0 < 0 || num_communities < 0 || (V0 > 0 && !orig2comm)) return LV_ERR_INVALID;
    try {
        return print_communities_impl(path, orig2comm, V0, num_communities);
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// generators
// ---------------------------------------------------------------------------
namespace {

int ceil_log2_host(int64_t x) {
    int r = 0;
    while ((int64_t(1) << r) < x) ++r;
    return r < 1 ? 1 : r;
}

// Parallel LSD radix sort of 64-bit keys whose significant bits are < nbits.
void radix_sort_u64(std::vector<uint64_t> &a, int nbits) {
    const size_t n = a.size();
    if (n < 2) return;
    std::vector<uint64_t> b(n);
    const int nt = omp_get_max_threads();
    std::vector<size_t> hist((size_t)nt * 256);
    for (int shift = 0; shift < nbits; shift += 8) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num();
            const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            size_t *h = hist.data() + (size_t)t * 256;
            for (size_t i = lo; i < hi; ++i) h[(a[i] >> shift) & 255]++;
        }
        size_t run = 0;
        for (int d = 0; d < 256; ++d)
            for (int t = 0; t < nt; ++t) {
                size_t c = hist[(size_t)t * 256 + d];
                hist[(size_t)t * 256 + d] = run;
                run += c;
            }
#pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num();
            const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            size_t *h = hist.data() + (size_t)t * 256;
            for (size_t i = lo; i < hi; ++i) b[h[(a[i] >> shift) & 255]++] = a[i];
        }
        a.swap(b);
    }
}

// keys = (lo << sh) | hi with lo < hi, sorted and unique -> symmetric CSR
// with ascending rows.
int keys_to_csr(const std::vector<uint64_t> &keys, int sh, int32_t V, int32_t weight_mode,
                uint64_t seed, int64_t *Eout, int32_t **rowptr, int32_t **col, float **w) {
    const uint64_t mask = (sh >= 64) ? ~0ull : ((1ull << sh) - 1);
    const int64_t nk = (int64_t)keys.size();
    const int64_t E = 2 * nk;
    if (E > 0x7fffffffLL) return LV_ERR_TOO_LARGE;
    std::vector<int64_t> dlo((size_t)V + 1, 0), dhi((size_t)V + 1, 0);
    for (int64_t i = 0; i < nk; ++i) {
        const int32_t a = (int32_t)(keys[(size_t)i] >> sh), b = (int32_t)(keys[(size_t)i] & mask);
        dhi[(size_t)a]++;   // a's larger neighbours
        dlo[(size_t)b]++;   // b's smaller neighbours
    }
    std::vector<int64_t> clo((size_t)V), chi((size_t)V);   // before the mallocs: a throw leaks nothing
    int32_t *rp = (int32_t *)std::malloc(sizeof(int32_t) * ((size_t)V + 1));
    int32_t *cl = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
    float *wt = (float *)std::malloc(sizeof(float) * (size_t)(E > 0 ? E : 1));
    if (!rp || !cl || !wt) {
        std::free(rp); std::free(cl); std::free(wt);
        return LV_ERR_NOMEM;
    }
    int64_t acc = 0;
    for (int32_t v = 0; v < V; ++v) {
        rp[v] = (int32_t)acc;
        clo[(size_t)v] = acc;
        chi[(size_t)v] = acc + dlo[(size_t)v];
        acc += dlo[(size_t)v] + dhi[(size_t)v];
    }
    rp[V] = (int32_t)acc;
    const uint64_t wkey = lvrng::stream_key(seed, lvrng::WEIGHT_STREAM);
    for (int64_t i = 0; i < nk; ++i) {
        const int32_t a = (int32_t)(keys[(size_t)i] >> sh), b = (int32_t)(keys[(size_t)i] & mask);
        const float wv = weight_mode == 1 ? lvrng::edge_weight(wkey, (uint32_t)a, (uint32_t)b) : 1.0f;
        const int64_t pa = chi[(size_t)a]++, pb = clo[(size_t)b]++;
        cl[pa] = b;
        wt[pa] = wv;
        cl[pb] = a;
        wt[pb] = wv;
    }
    *Eout = E;
    *rowptr = rp;
    *col = cl;
    *w = wt;
    return LV_OK;
}

}  // namespace

extern "C" {

static int gen_rmat_body(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b, double c,
                         int32_t weight_mode, int32_t *Vout, int64_t *Eout, int32_t **rowptr, int32_t **col,
                         float **w) {
    const int64_t n = (int64_t)edge_factor << scale;
    const lvrng::RmatParams rp = lvrng::rmat_params(scale, a, b, c, seed);
    std::vector<uint64_t> keys((size_t)n);
    int64_t kept = 0;
    const int nt = omp_get_max_threads();
    std::vector<int64_t> cnt((size_t)nt + 1, 0);
#pragma omp parallel num_threads(nt)
    {
        const int t = omp_get_thread_num();
        const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
        int64_t k = lo;
        for (int64_t i = lo; i < hi; ++i) {
            uint32_t u, v;
            lvrng::rmat_edge(rp, (uint64_t)i, &u, &v);
            if (u == v) continue;
            const uint32_t x = u < v ? u : v, y = u < v ? v : u;
            keys[(size_t)k++] = ((uint64_t)x << scale) | y;
        }
        cnt[(size_t)t + 1] = k - lo;
    }
    // compact the per-thread runs
    {
        int64_t dst = 0;
        for (int t = 0; t < nt; ++t) {
            const int64_t lo = n * t / nt;
            if (dst != lo) std::memmove(&keys[(size_t)dst], &keys[(size_t)lo], sizeof(uint64_t) * (size_t)cnt[(size_t)t + 1]);
            dst += cnt[(size_t)t + 1];
        }
        kept = dst;
    }
    keys.resize((size_t)kept);
    radix_sort_u64(keys, 2 * scale);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    const int32_t V = (int32_t)(1u << scale);
    int rc = keys_to_csr(keys, scale, V, weight_mode, seed, Eout, rowptr, col, w);
    if (rc == LV_OK) *Vout = V;
    return rc;
}

int lv_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b, double c,
                int32_t weight_mode, int32_t *Vout, int64_t *Eout, int32_t **rowptr, int32_t **col,
                float **w) {
    if (scale < 1 || scale > 30 || edge_factor < 1 || !Vout || !Eout || !rowptr || !col || !w ||
        !lvrng::rmat_probabilities_ok(a, b, c))
        return LV_ERR_INVALID;
    try {
        return gen_rmat_body(scale, edge_factor, seed, a, b, c, weight_mode, Vout, Eout, rowptr, col, w);
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
}

}  // extern "C"

namespace {

// The sorted, unique undirected pairs (lo << 32 | hi) of a planted-partition
// draw; false for invalid arguments.
bool planted_keys(int32_t V, int32_t blocks, double d_in, double d_out, uint64_t seed,
                  std::vector<uint64_t> &keys) {
    if (V < 1 || blocks < 1 || blocks > V || !(d_in >= 0.0) || !(d_out >= 0.0)) return false;
    // the draws of a graph whose CSR could hold int32 offsets at most
    // (2 entries per pair); NaN and infinite degrees fail here too
    if (!((double)V * (d_in + d_out) / 2.0 <= (double)(1ll << 30))) return false;
    const int64_t m_in = (int64_t)std::llround((double)V * d_in / 2.0);
    const int64_t m_out = (int64_t)std::llround((double)V * d_out / 2.0);
    keys.clear();
    keys.reserve((size_t)(m_in + m_out));
    const uint64_t k1 = lvrng::stream_key(seed, 1), k2 = lvrng::stream_key(seed, 2);
    for (int64_t i = 0; i < m_in + m_out; ++i) {
        uint32_t u, v;
        bool ok = i < m_in ? lvrng::planted_intra(k1, (uint64_t)i, V, blocks, &u, &v)
                           : lvrng::planted_inter(k2, (uint64_t)(i - m_in), V, blocks, &u, &v);
        if (!ok || u == v) continue;
        const uint32_t x = u < v ? u : v, y = u < v ? v : u;
        keys.push_back(((uint64_t)x << 32) | y);
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    return true;
}

}  // namespace

extern "C" {

int lv_gen_planted(int32_t V, int32_t blocks, double d_in, double d_out, uint64_t seed,
                   int32_t weight_mode, int64_t *Eout, int32_t **rowptr, int32_t **col, float **w) {
    if (!Eout || !rowptr || !col || !w) return LV_ERR_INVALID;
    try {
        std::vector<uint64_t> keys;
        if (!planted_keys(V, blocks, d_in, d_out, seed, keys)) return LV_ERR_INVALID;
        return keys_to_csr(keys, 32, V, weight_mode, seed, Eout, rowptr, col, w);
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
}

int lv_gen_planted_batch(int32_t G, const int32_t *V, const int32_t *blocks, const double *d_in,
                         const double *d_out, const uint64_t *seeds, int32_t weight_mode, int32_t *Vtot,
                         int64_t *Etot, int32_t **rowptr, int32_t **col, float **w, int32_t **graph_ptr) {
    if (G < 0 || !Vtot || !Etot || !rowptr || !col || !w || !graph_ptr ||
        (G > 0 && (!V || !blocks || !d_in || !d_out || !seeds)))
        return LV_ERR_INVALID;
    struct One {
        int32_t *rp = nullptr, *cl = nullptr;
        float *wt = nullptr;
        int64_t E = 0;
        int rc = LV_OK;
    };
    std::vector<One> parts((size_t)G);
    try {
#pragma omp parallel for schedule(dynamic, 1)
        for (int32_t i = 0; i < G; ++i) {
            std::vector<uint64_t> keys;
            One &o = parts[(size_t)i];
            try {
                if (!planted_keys(V[i], blocks[i], d_in[i], d_out[i], seeds[i], keys)) o.rc = LV_ERR_INVALID;
                else o.rc = keys_to_csr(keys, 32, V[i], weight_mode, seeds[i], &o.E, &o.rp, &o.cl, &o.wt);
            } catch (const std::bad_alloc &) {
                o.rc = LV_ERR_NOMEM;
            }
        }
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
    int rc = LV_OK;
    int64_t nv = 0, ne = 0;
    for (int32_t i = 0; i < G; ++i) {
        if (parts[(size_t)i].rc != LV_OK && rc == LV_OK) rc = parts[(size_t)i].rc;
        nv += V[i];
        ne += parts[(size_t)i].E;
    }
    if (rc == LV_OK && (nv >= 0x7fffffffLL - G || ne > 0x7fffffffLL)) rc = LV_ERR_TOO_LARGE;
    int32_t *rp = nullptr, *cl = nullptr, *gp = nullptr;
    float *wt = nullptr;
    if (rc == LV_OK) {
        rp = (int32_t *)std::malloc(sizeof(int32_t) * ((size_t)nv + 1));
        cl = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(ne > 0 ? ne : 1));
        wt = (float *)std::malloc(sizeof(float) * (size_t)(ne > 0 ? ne : 1));
        gp = (int32_t *)std::malloc(sizeof(int32_t) * ((size_t)G + 1));
        if (!rp || !cl || !wt || !gp) rc = LV_ERR_NOMEM;
    }
    if (rc == LV_OK) {
        std::vector<int64_t> v0((size_t)G + 1, 0), e0((size_t)G + 1, 0);
        for (int32_t i = 0; i < G; ++i) {
            v0[(size_t)i + 1] = v0[(size_t)i] + V[i];
            e0[(size_t)i + 1] = e0[(size_t)i] + parts[(size_t)i].E;
        }
        rp[0] = 0;
#pragma omp parallel for schedule(dynamic, 1)
        for (int32_t i = 0; i < G; ++i) {
            const One &o = parts[(size_t)i];
            const int64_t vb = v0[(size_t)i], eb = e0[(size_t)i];
            for (int32_t v = 1; v <= V[i]; ++v) rp[vb + v] = (int32_t)(eb + o.rp[v]);
            for (int64_t e = 0; e < o.E; ++e) {
                cl[eb + e] = (int32_t)(vb + o.cl[e]);
                wt[eb + e] = o.wt[e];
            }
        }
        for (int32_t i = 0; i <= G; ++i) gp[i] = (int32_t)v0[(size_t)i];
    }
    for (One &o : parts) {
        std::free(o.rp); std::free(o.cl); std::free(o.wt);
    }
    if (rc != LV_OK) {
        std::free(rp); std::free(cl); std::free(wt); std::free(gp);
        return rc;
    }
    *Vtot = (int32_t)nv;
    *Etot = ne;
    *rowptr = rp;
    *col = cl;
    *w = wt;
    *graph_ptr = gp;
    return LV_OK;
}


// LFR-like benchmark graph (the construction of Lancichinetti, Fortunato and
// Radicchi, Phys. Rev. E 78, 046110 (2008), simplified): degrees from a
// power law of exponent tau1 on [kmin, kmax] with kmin chosen for the mean
// degree, community sizes from a power law of exponent tau2 on [cmin, cmax]
// (the last community absorbs the remainder), each vertex with
// round((1 - mu) d) stubs inside its community (at most size - 1) and the
// rest outside; stubs are paired uniformly at random (intra stubs within
// their community, inter stubs over the whole graph), self-loops and repeated
// pairs are dropped, and vertex ids are a random permutation of the
// community order.  Unit weights.  comm_out (may be NULL) receives each
// vertex's planted community (malloc'd, V entries).
static int gen_lfr_body(int32_t V, double tau1, double mean_degree, int32_t kmax, double tau2, int32_t cmin,
                        int32_t cmax, double mu, uint64_t seed, int64_t *Eout, int32_t **rowptr, int32_t **col,
                        float **w, int32_t **comm_out);

int lv_gen_lfr(int32_t V, double tau1, double mean_degree, int32_t kmax, double tau2, int32_t cmin,
               int32_t cmax, double mu, uint64_t seed, int64_t *Eout, int32_t **rowptr, int32_t **col,
               float **w, int32_t **comm_out) {
    // the comparisons are written so that NaN fails them
    if (V < 2 || !(tau1 > 1.0 && tau1 < 1e3) || !(tau2 > 1.0 && tau2 < 1e3) || !(mean_degree >= 1.0) ||
        kmax < 2 || cmin < 2 || cmax < cmin || !(mu >= 0.0 && mu <= 1.0) || !Eout || !rowptr || !col || !w)
        return LV_ERR_INVALID;
    if (V >= (1 << 26)) return LV_ERR_TOO_LARGE;
    // about V * mean_degree stubs, one CSR entry each: more than an int32 CSR
    // holds is too large (and a huge mean would only exhaust host memory)
    if ((double)V * mean_degree > (double)(1ll << 30)) return LV_ERR_TOO_LARGE;
    try {
        return gen_lfr_body(V, tau1, mean_degree, kmax, tau2, cmin, cmax, mu, seed, Eout, rowptr, col, w,
                            comm_out);
    } catch (const std::bad_alloc &) {
        return LV_ERR_NOMEM;
    }
}

static int gen_lfr_body(int32_t V, double tau1, double mean_degree, int32_t kmax, double tau2, int32_t cmin,
                        int32_t cmax, double mu, uint64_t seed, int64_t *Eout, int32_t **rowptr, int32_t **col,
                        float **w, int32_t **comm_out) {
    // continuous power-law sample on [a, b] with exponent t from u in [0, 1)
    auto plaw = [](double u, double a, double b, double t) {
        const double e = 1.0 - t;
        const double lo = std::pow(a, e), hi = std::pow(b, e);
        return std::pow(lo + u * (hi - lo), 1.0 / e);
    };
    auto unit = [](uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; };
    // kmin for the requested mean (bisection on the continuous mean)
    auto mean_of = [&](double a) {
        const double e1 = 1.0 - tau1, e2 = 2.0 - tau1, b = (double)kmax;
        return (e1 / e2) * (std::pow(b, e2) - std::pow(a, e2)) / (std::pow(b, e1) - std::pow(a, e1));
    };
    double lo = 1.0, hi = (double)kmax;
    for (int it = 0; it < 100; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mean_of(mid) < mean_degree) lo = mid;
        else hi = mid;
    }
    const double kmin = 0.5 * (lo + hi);
    const uint64_t kdeg = lvrng::stream_key(seed, 11), kcom = lvrng::stream_key(seed, 12),
                   kperm = lvrng::stream_key(seed, 13), kin = lvrng::stream_key(seed, 14),
                   kout = lvrng::stream_key(seed, 15);
    // community sizes
    std::vector<int32_t> csize;
    int64_t tot = 0;
    for (uint64_t i = 0; tot < V; ++i) {
        int32_t c = (int32_t)std::lround(plaw(unit(lvrng::draw(kcom, i)), cmin, cmax, tau2));
        if (c > V - tot) c = (int32_t)(V - tot);
        csize.push_back(c);
        tot += c;
    }
    if (csize.size() > 1 && csize.back() < cmin) {
        csize[csize.size() - 2] += csize.back();
        csize.pop_back();
    }
    const int32_t nc = (int32_t)csize.size();
    std::vector<int32_t> cstart((size_t)nc + 1, 0);
    for (int32_t c = 0; c < nc; ++c) cstart[(size_t)c + 1] = cstart[(size_t)c] + csize[(size_t)c];
    // community-order position -> vertex id: sort by random keys
    const int vb = ceil_log2_host(V);
    std::vector<uint64_t> pk((size_t)V);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < V; ++i) pk[(size_t)i] = ((lvrng::draw(kperm, (uint64_t)i) >> vb) << vb) | (uint64_t)i;
    radix_sort_u64(pk, 64);
    std::vector<int32_t> vid((size_t)V);   // position -> vertex id
    for (int32_t i = 0; i < V; ++i) vid[(size_t)(pk[(size_t)i] & ((1ull << vb) - 1))] = i;
    // degrees and stubs; position p is in community cpos[p]
    std::vector<int32_t> cpos((size_t)V);
    for (int32_t c = 0; c < nc; ++c)
        for (int32_t p = cstart[(size_t)c]; p < cstart[(size_t)c + 1]; ++p) cpos[(size_t)p] = c;
    std::vector<int32_t> din((size_t)V), dout((size_t)V);
#pragma omp parallel for schedule(static)
    for (int32_t p = 0; p < V; ++p) {
        int32_t d = (int32_t)std::lround(plaw(unit(lvrng::draw(kdeg, (uint64_t)p)), kmin, (double)kmax, tau1));
        if (d < 1) d = 1;
        int32_t a = (int32_t)std::lround((1.0 - mu) * d);
        const int32_t cap = csize[(size_t)cpos[(size_t)p]] - 1;
        if (a > cap) a = cap;
        din[(size_t)p] = a;
        dout[(size_t)p] = d - a;
    }
    const int cb = ceil_log2_host(nc);
    const int rb = 64 - vb - cb;
    if (rb < 12) return LV_ERR_TOO_LARGE;
    std::vector<uint64_t> sin, sout;
    {
        int64_t ni = 0, no = 0;
        for (int32_t p = 0; p < V; ++p) { ni += din[(size_t)p]; no += dout[(size_t)p]; }
        sin.reserve((size_t)ni);
        sout.reserve((size_t)no);
        uint64_t j = 0;
        for (int32_t p = 0; p < V; ++p) {
            for (int32_t s = 0; s < din[(size_t)p]; ++s, ++j) {
                const uint64_t r = lvrng::draw(kin, j) >> (64 - rb);
                sin.push_back(((uint64_t)cpos[(size_t)p] << (64 - cb)) | (r << vb) | (uint64_t)p);
            }
        }
        j = 0;
        for (int32_t p = 0; p < V; ++p)
            for (int32_t s = 0; s < dout[(size_t)p]; ++s, ++j)
                sout.push_back(((lvrng::draw(kout, j) >> vb) << vb) | (uint64_t)p);
    }
    radix_sort_u64(sin, 64);
    radix_sort_u64(sout, 64);
    const uint64_t vmask = (1ull << vb) - 1;
    std::vector<uint64_t> keys;
    keys.reserve((sin.size() + sout.size()) / 2 + 1);
    auto add = [&](uint64_t a, uint64_t b) {
        const int32_t u = vid[(size_t)(a & vmask)], v = vid[(size_t)(b & vmask)];
        if (u == v) return;
        const uint32_t x = (uint32_t)(u < v ? u : v), y = (uint32_t)(u < v ? v : u);
        keys.push_back(((uint64_t)x << 32) | y);
    };
    for (size_t i = 0; i + 1 < sin.size();) {
        if ((sin[i] >> (64 - cb)) != (sin[i + 1] >> (64 - cb))) {   // odd stub count: skip one
            ++i;
            continue;
        }
        add(sin[i], sin[i + 1]);
        i += 2;
    }
    for (size_t i = 0; i + 1 < sout.size(); i += 2) add(sout[i], sout[i + 1]);
    radix_sort_u64(keys, 64);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if (comm_out) {
        int32_t *cm = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)V);
        if (!cm) return LV_ERR_NOMEM;
        for (int32_t p = 0; p < V; ++p) cm[vid[(size_t)p]] = cpos[(size_t)p];
        *comm_out = cm;
    }
    return keys_to_csr(keys, 32, V, 0, seed, Eout, rowptr, col, w);
}
}  // extern "C"
