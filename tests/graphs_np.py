"""numpy restatement of the seeded generators (lv_rng.h), used by the tests to
check the C/CUDA generators bit for bit on small sizes."""
import numpy as np

U64 = np.uint64
C1, C2, GOLD = U64(0xBF58476D1CE4E5B9), U64(0x94D049BB133111EB), U64(0x9E3779B97F4A7C15)
WEIGHT_STREAM = 0xFFFF


def mix64(z):
    z = np.asarray(z, dtype=U64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> U64(30))) * C1
        z = (z ^ (z >> U64(27))) * C2
    return z ^ (z >> U64(31))


def stream_key(seed, stream):
    return mix64(np.array([U64(seed) ^ (U64(stream) << U64(32))], dtype=U64))[0]


def draw(key, i):
    with np.errstate(over="ignore"):
        return mix64(U64(key) + np.asarray(i, dtype=U64) * GOLD)


def edge_weight(seed, a, b):
    h = draw(stream_key(seed, WEIGHT_STREAM), (np.asarray(a, U64) << U64(32)) | np.asarray(b, U64))
    m = (h >> U64(40)).astype(np.uint32)
    return (m + np.uint32(8388608)).astype(np.float32) * np.float32(5.9604644775390625e-08)


def keys_to_csr(a, b, V, seed, weights):
    a = a.astype(np.int64)
    b = b.astype(np.int64)
    w = edge_weight(seed, a, b) if weights == "uniform" else np.ones(len(a), np.float32)
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    ww = np.concatenate([w, w])
    order = np.lexsort((dst, src))
    src, dst, ww = src[order], dst[order], ww[order]
    rowptr = np.zeros(V + 1, np.int64)
    np.add.at(rowptr, src + 1, 1)
    rowptr = np.cumsum(rowptr)
    return rowptr.astype(np.int32), dst.astype(np.int32), ww.astype(np.float32)


def rmat(scale, ef=16, seed=1, a=0.57, b=0.19, c=0.19, weights="uniform"):
    n = ef << scale
    i = np.arange(n, dtype=U64)
    u = np.zeros(n, U64)
    v = np.zeros(n, U64)
    ta = int(a * 4294967296.0)
    tb = int((a + b) * 4294967296.0)
    tc = int((a + b + c) * 4294967296.0)
    for p in range((scale + 1) // 2):
        r = draw(stream_key(seed, 1 + p), i)
        for half in range(2):
            if 2 * p + half >= scale:
                break
            x = ((r >> U64(32 * half)) & U64(0xFFFFFFFF)).astype(np.int64)
            q = (x >= ta).astype(np.int64) + (x >= tb) + (x >= tc)
            u = (u << U64(1)) | (q >> 1).astype(U64)
            v = (v << U64(1)) | (q & 1).astype(U64)
    m = u != v
    x = np.minimum(u[m], v[m])
    y = np.maximum(u[m], v[m])
    keys = np.unique((x << U64(32)) | y)
    return keys_to_csr(keys >> U64(32), keys & U64(0xFFFFFFFF), 1 << scale, seed, weights)


def planted(V=10000, blocks=64, d_in=16.0, d_out=2.0, seed=0, weights="unit"):
    m_in = int(round(V * d_in / 2.0))
    m_out = int(round(V * d_out / 2.0))

    def start(b):
        return (b * V + blocks - 1) // blocks

    pairs = []
    r = draw(stream_key(seed, 1), np.arange(m_in, dtype=U64))
    uu = (((r & U64(0xFFFFFFFF)) * U64(V)) >> U64(32)).astype(np.int64)
    blk = uu * blocks // V
    s0, s1 = start(blk), start(blk + 1)
    vv = s0 + (((r >> U64(32)) * (s1 - s0).astype(U64)) >> U64(32)).astype(np.int64)
    pairs.append((uu, vv, np.ones(m_in, bool)))
    r = draw(stream_key(seed, 2), np.arange(m_out, dtype=U64))
    uu = (((r & U64(0xFFFFFFFF)) * U64(V)) >> U64(32)).astype(np.int64)
    blk = uu * blocks // V
    s0, s1 = start(blk), start(blk + 1)
    rest = V - (s1 - s0)
    ok = rest > 0
    x = (((r >> U64(32)) * np.maximum(rest, 0).astype(U64)) >> U64(32)).astype(np.int64)
    vv = np.where(x < s0, x, x + (s1 - s0))
    pairs.append((uu, vv, ok))
    u = np.concatenate([p[0][p[2]] for p in pairs])
    v = np.concatenate([p[1][p[2]] for p in pairs])
    m = u != v
    x, y = np.minimum(u[m], v[m]), np.maximum(u[m], v[m])
    keys = np.unique((x.astype(U64) << U64(32)) | y.astype(U64))
    return keys_to_csr(keys >> U64(32), keys & U64(0xFFFFFFFF), V, seed, weights)


def csr_from_edges(V, edges):
    """CSR in the MTX reader's convention from (u, v, w) entries in file order."""
    rows = [[] for _ in range(V)]
    for u, v, w in edges:
        rows[u].append((v, w))
        if u != v:
            rows[v].append((u, w))
    rowptr = np.zeros(V + 1, np.int32)
    for i in range(V):
        rowptr[i + 1] = rowptr[i] + len(rows[i])
    col = np.array([c for r in rows for c, _ in r], np.int32)
    w = np.array([x for r in rows for _, x in r], np.float32)
    return rowptr, col, w
