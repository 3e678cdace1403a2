"""Host-side parts of the engine library (no GPU): the MTX reader against
the oracle's restatement of readInputData, writers, the verbose printer and
the generators against their numpy restatement."""
import os
import subprocess

import numpy as np
import pytest


def test_generators_match_numpy(lvb, gnp):
    for sc, seed in ((6, 1), (10, 2), (13, 7)):
        a = gnp.rmat(sc, seed=seed)
        b = lvb.gen_rmat(sc, seed=seed)
        for x, y in zip(a, (b.rowptr, b.col, b.w)):
            assert np.array_equal(x, y)
    a = gnp.planted(3000, 20, 12.0, 3.0, 4, "uniform")
    b = lvb.gen_planted(3000, 20, 12.0, 3.0, 4, "uniform")
    for x, y in zip(a, (b.rowptr, b.col, b.w)):
        assert np.array_equal(x, y)


def test_rmat_weights_on_grid(lvb):
    g = lvb.gen_rmat(10)
    w = g.w.astype(np.float64)
    assert w.min() >= 0.5 and w.max() < 1.5
    assert np.all(w * 2 ** 24 == np.round(w * 2 ** 24))


@pytest.mark.parametrize("kind", ["planted", "rmat"])
def test_mtx_roundtrip_and_reader_parity(lvb, orc, tmp_path, kind):
    g = lvb.gen_planted(500, 8, 10.0, 2.0, 1, "uniform") if kind == "planted" else lvb.gen_rmat(9)
    p = str(tmp_path / "g.mtx")
    lvb.write_mtx(p, g)
    r = lvb.read_mtx(p)
    rp, cl, w, m = orc.read_mtx(p)
    assert np.array_equal(r.rowptr, rp) and np.array_equal(r.col, cl) and np.array_equal(r.w, w)
    assert r.m_ref == m
    # same graph as the generator's (row order differs: file order)
    for v in range(g.V):
        a = sorted(zip(g.col[g.rowptr[v]:g.rowptr[v + 1]], g.w[g.rowptr[v]:g.rowptr[v + 1]]))
        b = sorted(zip(r.col[r.rowptr[v]:r.rowptr[v + 1]], r.w[r.rowptr[v]:r.rowptr[v + 1]]))
        assert a == b


def test_reader_edge_cases(lvb, orc, tmp_path):
    p = tmp_path / "e.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n%c\n\n3 3 3\n1 1 4\n3 1 1e-3\n2 3 7\n")
    r = lvb.read_mtx(str(p))
    rp, cl, w, m = orc.read_mtx(str(p))
    assert np.array_equal(r.rowptr, rp) and np.array_equal(r.col, cl) and np.array_equal(r.w, w)
    assert list(r.rowptr) == [0, 2, 3, 5]
    p2 = tmp_path / "pat.mtx"
    p2.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 2\n")
    r2 = lvb.read_mtx(str(p2))
    assert list(r2.w) == [1.0] * 4
    p3 = tmp_path / "bad.mtx"
    p3.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 2\n2 1 1\n")
    with pytest.raises(lvb.LouvainError):
        lvb.read_mtx(str(p3))
    p4 = tmp_path / "range.mtx"
    p4.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 1\n4 1 1\n")
    with pytest.raises(lvb.LouvainError):
        lvb.read_mtx(str(p4))
    with pytest.raises(lvb.LouvainError):
        lvb.read_mtx(str(tmp_path / "missing.mtx"))
    p5 = tmp_path / "empty.mtx"
    p5.write_text("%%MatrixMarket matrix coordinate real symmetric\n0 0 0\n")
    r5 = lvb.read_mtx(str(p5))
    assert r5.V == 0 and r5.E == 0


HDR = "%%MatrixMarket matrix coordinate real symmetric\n"


@pytest.mark.parametrize("name,text,status", [
    # a size line promising more entries than the file can hold: an I/O error,
    # not an attempt to size the entry arrays by it
    ("huge_nnz", HDR + "3 3 99999999999999\n1 2 1.0\n", 7),
    ("short_file", HDR + "3 3 5\n1 2 1.0\n", 7),
    ("truncated_entry", HDR + "3 3 2\n1 2 1.0\n2", 7),
    ("missing_weight", HDR + "3 3 1\n1 2\n", 7),
    ("bad_weight", HDR + "3 3 1\n1 2 abc\n", 7),
    ("negative_size", HDR + "3 -5 1\n1 2 1.0\n", 7),
    ("no_size_line", HDR, 7),
    ("zero_index", HDR + "3 3 1\n0 2 1.0\n", 1),
    ("negative_index", HDR + "3 3 1\n-1 2 1.0\n", 1),
    ("index_past_v", HDR + "3 3 1\n1 4 1.0\n", 1),
    ("index_overflows_int64", HDR + "3 3 1\n1 99999999999999999999 1.0\n", 1),
    ("entries_without_vertices", HDR + "0 0 1\n1 1 1.0\n", 1),
    ("vertices_past_int32", HDR + "3 2147483648 1\n1 2 1.0\n", 3),
])
def test_reader_rejects_malformed_files(lvb, tmp_path, name, text, status):
    p = tmp_path / (name + ".mtx")
    p.write_text(text)
    with pytest.raises(lvb.LouvainError) as ei:
        lvb.read_mtx(str(p))
    assert ei.value.status == status


def test_reader_line_endings_and_separators(lvb, tmp_path):
    ref = None
    for name, text in (("lf", HDR + "3 3 2\n1 2 1.0\n2 3 2.0\n"),
                       ("crlf", HDR.replace("\n", "\r\n") + "3 3 2\r\n1 2 1.0\r\n2 3 2.0\r\n"),
                       ("tabs", HDR + "3\t3\t2\n1\t2\t1.0\n2\t3\t2.0\n"),
                       ("no_final_break", HDR + "3 3 2\n1 2 1.0\n2 3 2.0")):
        p = tmp_path / (name + ".mtx")
        p.write_text(text)
        g = lvb.read_mtx(str(p))
        got = (list(g.rowptr), list(g.col), list(g.w))
        assert got == ([0, 1, 3, 4], [1, 0, 2, 1], [1.0, 1.0, 2.0, 2.0]), name


def test_print_communities_format(lvb, tmp_path):
    # printOriginalToCommunity: V_final, then "c+1 members+1..." for every
    # community id (empty ones included), members in increasing id
    p = str(tmp_path / "map.txt")
    lvb.print_communities(np.array([2, 0, 2, 0, 2], np.int32), 4, p)
    assert open(p).read() == "4\n1 2 4\n2\n3 1 3 5\n4\n"


def test_cli_usage(lvb):
    r = subprocess.run([lvb.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stdout == "Usage: ./gpulouvain -f mtx-matrix-file -g min-gain [-v]\n"
    r = subprocess.run([lvb.CLI_PATH, "-f", "x.mtx"], capture_output=True, text=True)
    assert r.returncode == 1


def test_lfr_generator(lvb):
    """LFR-like graphs: symmetric simple CSR, the requested mean degree (less
    the dropped repeated pairs and odd stubs), the maximum degree, community
    sizes within bounds, and about 1 - mu of the entries inside communities;
    a seed names one graph."""
    V, mu = 50000, 0.3
    g, comm = lvb.gen_lfr(V, mu, seed=4)
    g2, comm2 = lvb.gen_lfr(V, mu, seed=4)
    assert np.array_equal(g.rowptr, g2.rowptr) and np.array_equal(g.col, g2.col)
    assert np.array_equal(comm, comm2)
    deg = np.diff(g.rowptr)
    row = np.repeat(np.arange(V), deg)
    assert (g.col != row).all()                                   # no self-loops
    fwd = set(zip(row.tolist(), g.col.tolist()))
    assert len(fwd) == g.E and all((b, a) in fwd for a, b in list(fwd)[:20000])
    assert 17.0 < deg.mean() < 21.0 and deg.max() <= 2000
    sizes = np.bincount(comm)
    assert sizes.min() >= 50 and sizes.max() <= 5000 + 50
    intra = (comm[row] == comm[g.col]).mean()
    assert abs(intra - (1 - mu)) < 0.05
    assert (g.w == 1.0).all()


def _same_csr(r, o):
    rp, cl, w, m = o
    return (np.array_equal(r.rowptr, rp) and np.array_equal(r.col, cl) and np.array_equal(r.w, w)
            and r.m_ref == m)


def test_parallel_reader_matches_token_stream(lvb, orc, tmp_path):
    """Files large enough for the multi-threaded reading (one entry per line)
    give exactly the oracle's token-stream reading; so do layouts that force
    the sequential reading (an entry split over two lines), CRLF line ends,
    pattern files and a header line with trailing blanks."""
    g = lvb.gen_rmat(15, seed=3)
    p = tmp_path / "big.mtx"
    lvb.write_mtx(str(p), g)
    assert p.stat().st_size > (1 << 22)
    assert _same_csr(lvb.read_mtx(str(p)), orc.read_mtx(str(p)))
    text = p.read_text()
    head, body = text.split("\n", 2)[:2], text.split("\n", 2)[2]
    lines = body.split("\n")
    # an entry split over two lines (sequential reading)
    a, b, w = lines[5].split()
    split = "\n".join(head) + "\n" + "\n".join(lines[:5] + [a + " " + b, w] + lines[6:])
    q = tmp_path / "split.mtx"
    q.write_text(split)
    assert _same_csr(lvb.read_mtx(str(q)), orc.read_mtx(str(q)))
    # CRLF line ends
    q2 = tmp_path / "crlf.mtx"
    q2.write_bytes(text.replace("\n", "\r\n").encode())
    assert _same_csr(lvb.read_mtx(str(q2)), orc.read_mtx(str(q2)))
    # pattern file: two tokens per line
    pat = "%%MatrixMarket matrix coordinate pattern symmetric\n" + head[1] + "   \n" + "\n".join(
        " ".join(l.split()[:2]) for l in lines if l.strip())
    q3 = tmp_path / "pattern.mtx"
    q3.write_text(pat + "\n")
    r3 = lvb.read_mtx(str(q3))
    assert _same_csr(r3, orc.read_mtx(str(q3))) and (r3.w == 1.0).all()
    # an out-of-range vertex far into the file is still an error
    bad = lines[:]
    bad[len(bad) // 2] = f"{g.V + 7} 1 1.0"
    q4 = tmp_path / "range.mtx"
    q4.write_text("\n".join(head) + "\n" + "\n".join(bad))
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.read_mtx(str(q4))
    assert ex.value.status == lvb.LV_ERR_INVALID


def test_csr_cache_roundtrip(lvb, tmp_path):
    g = lvb.gen_planted(3000, 16, 12.0, 2.0, 5, "uniform")
    g.m_ref = 1234.5
    p = str(tmp_path / "g.lvcsr")
    lvb.write_csr(p, g)
    r = lvb.read_csr(p)
    assert np.array_equal(r.rowptr, g.rowptr) and np.array_equal(r.col, g.col) and np.array_equal(r.w, g.w)
    assert r.m_ref == np.float32(1234.5)
    raw = open(p, "rb").read()
    hdr = 48                                   # magic, V, E, m_ref, pad, source size, source mtime
    c0 = hdr + 4 * (g.V + 1)                   # first column word
    last = c0 + 4 * (g.E - 1)                  # last column word
    for broken in (raw[:-4], b"XXXXXXXX" + raw[8:], raw[:64] + (b"\xff" * 4) + raw[68:],
                   raw[:c0] + np.int32(-1).tobytes() + raw[c0 + 4:],            # column below 0
                   raw[:last] + np.int32(g.V).tobytes() + raw[last + 4:],       # column past V
                   raw[:hdr] + np.int32(1).tobytes() + raw[hdr + 4:],           # rowptr[0] != 0
                   raw[:c0 - 4] + np.int32(g.E - 1).tobytes() + raw[c0:]):      # rowptr[V] != E
        q = str(tmp_path / "broken.lvcsr")
        open(q, "wb").write(broken)
        with pytest.raises(lvb.LouvainError) as ex:
            lvb.read_csr(q)
        assert ex.value.status == lvb.LV_ERR_IO


def test_gen_planted_batch_equals_concatenated_graphs(lvb):
    rng = np.random.default_rng(2)
    params = []
    for i in range(40):
        V = int(rng.integers(1, 3000))
        params.append((V, int(rng.integers(1, min(V, 256) + 1)), float(rng.uniform(0, 24)),
                       float(rng.uniform(0, 4)), 77 + i))
    for weights in ("unit", "uniform"):
        got = lvb.gen_planted_batch(params, weights)
        want = lvb.concat_graphs([lvb.gen_planted(*p[:4], seed=p[4], weights=weights) for p in params])
        for x, y in zip(got, want):
            assert np.array_equal(x, y)
    with pytest.raises(lvb.LouvainError):
        lvb.gen_planted_batch([(10, 20, 4.0, 1.0, 1)])   # more blocks than vertices


def test_csr_cache_source_stamp(lvb, tmp_path):
    import ctypes as C
    g = lvb.gen_planted(500, 8, 10.0, 2.0, 3)
    p = str(tmp_path / "s.lvcsr")
    L = lvb.lib()
    P32 = C.POINTER(C.c_int32)
    rc = L.lv_write_csr_stamped(p.encode(), g.V, g.E, g.rowptr.ctypes.data_as(P32), g.col.ctypes.data_as(P32),
                                g.w.ctypes.data_as(C.POINTER(C.c_float)), 1.0, 123456, 1700000000123456789)
    assert rc == lvb.LV_OK
    size, mt = C.c_int64(), C.c_int64()
    assert L.lv_read_csr_stamp(p.encode(), C.byref(size), C.byref(mt)) == lvb.LV_OK
    assert (size.value, mt.value) == (123456, 1700000000123456789)
    r = lvb.read_csr(p)
    assert np.array_equal(r.rowptr, g.rowptr) and np.array_equal(r.col, g.col)
    lvb.write_csr(p, g)           # unstamped
    assert L.lv_read_csr_stamp(p.encode(), C.byref(size), C.byref(mt)) == lvb.LV_OK
    assert (size.value, mt.value) == (0, 0)
    assert L.lv_read_csr_stamp(str(tmp_path / "missing").encode(), C.byref(size), C.byref(mt)) == lvb.LV_ERR_IO


def test_print_communities_large_matches_python(lvb, tmp_path):
    """The multi-threaded writer gives the reference's format byte for byte:
    the community count, then "c+1 m1+1 m2+1 ..." per community with members
    in increasing id (empty communities print just their number)."""
    rng = np.random.default_rng(8)
    V, nc = 200000, 50000
    m = rng.integers(0, nc, V).astype(np.int32)
    p = str(tmp_path / "map.txt")
    lvb.print_communities(m, nc, p)
    order = np.argsort(m, kind="stable")
    bounds = np.searchsorted(m[order], np.arange(nc + 1))
    lines = [str(nc)]
    for c in range(nc):
        mem = order[bounds[c]:bounds[c + 1]] + 1
        lines.append(" ".join([str(c + 1)] + [str(x) for x in mem]))
    assert open(p).read() == "\n".join(lines) + "\n"


@pytest.mark.parametrize("name,call,status", [
    ("rmat_scale_0", lambda L: L.gen_rmat(0), 1),
    ("rmat_scale_31", lambda L: L.gen_rmat(31), 1),
    ("rmat_edge_factor_0", lambda L: L.gen_rmat(5, 0), 1),
    ("rmat_probabilities_over_1", lambda L: L.gen_rmat(5, a=0.5, b=0.3, c=0.3), 1),
    ("rmat_probability_negative", lambda L: L.gen_rmat(5, a=0.7, b=-0.1, c=0.2), 1),
    ("rmat_probability_nan", lambda L: L.gen_rmat(5, a=float("nan")), 1),
    ("planted_no_vertices", lambda L: L.gen_planted(0, 1, 1.0, 1.0, 0, "unit"), 1),
    ("planted_more_blocks_than_vertices", lambda L: L.gen_planted(10, 100, 1.0, 1.0, 0, "unit"), 1),
    ("planted_negative_degree", lambda L: L.gen_planted(100, 4, -1.0, 1.0, 0, "unit"), 1),
    ("planted_nan_degree", lambda L: L.gen_planted(100, 4, float("nan"), 1.0, 0, "unit"), 1),
    # more draws than an int32 CSR can hold: refused before any array is sized
    ("planted_huge_degree", lambda L: L.gen_planted(100, 4, 1e9, 1.0, 0, "unit"), 1),
    ("lfr_mu_above_1", lambda L: L.gen_lfr(1000, 1.5), 1),
    ("lfr_mu_nan", lambda L: L.gen_lfr(1000, float("nan")), 1),
    ("lfr_tau1_1", lambda L: L.gen_lfr(1000, 0.3, tau1=1.0), 1),
    ("lfr_cmin_above_cmax", lambda L: L.gen_lfr(1000, 0.3, cmin=500, cmax=50), 1),
    ("lfr_vertices_past_2_26", lambda L: L.gen_lfr(1 << 26, 0.3), 3),
    ("lfr_stubs_past_int32", lambda L: L.gen_lfr(1 << 20, 0.3, mean_degree=5000.0, kmax=10000), 3),
])
def test_generators_reject_bad_arguments(lvb, name, call, status):
    with pytest.raises(lvb.LouvainError) as ei:
        call(lvb)
    assert ei.value.status == status


def test_generator_weight_names(lvb):
    with pytest.raises(ValueError):
        lvb.gen_planted(100, 4, 4.0, 1.0, 0, "uniformly")
    assert set(lvb.gen_planted(100, 4, 4.0, 1.0, 0, "unit").w.tolist()) == {1.0}


def _weight_tokens(n_random=120000, seed=3):
    """Decimal tokens of many shapes: printed float32 values, random digit
    strings with exponents, decimal forms of values next to float midpoints,
    and edge forms (signs, bare points, subnormal and overflowing values)."""
    rng = np.random.default_rng(seed)
    toks = []
    f = rng.uniform(-1.0, 1.0, n_random // 4).astype(np.float32) * np.float32(10.0) ** rng.integers(-12, 12, n_random // 4)
    for i, x in enumerate(f.tolist()):
        toks.append(("%.9g", "%.8g", "%.17g", "%e")[i % 4] % x)
    for _ in range(n_random // 4):
        nd = int(rng.integers(1, 21))
        digits = "".join(str(int(d)) for d in rng.integers(0, 10, nd))
        cut = int(rng.integers(0, nd + 1))
        tok = digits[:cut] + "." + digits[cut:] if cut < nd else digits
        if rng.random() < 0.5:
            tok += "e%d" % int(rng.integers(-30, 31))
        toks.append(tok)
    # values at and next to float midpoints (the halfway points are exact doubles)
    base = rng.uniform(0.5, 2.0, n_random // 8).astype(np.float32) * np.float32(2.0) ** rng.integers(-100, 100, n_random // 8)
    up = np.nextafter(base, np.float32(np.inf))
    mid = (base.astype(np.float64) + up.astype(np.float64)) / 2.0
    for x in mid.tolist():
        toks.append("%.17g" % x)
        toks.append("%.16g" % x)
        toks.append("%.25g" % x)
        toks.append(repr(float(np.nextafter(x, np.inf))))
    toks += ["0", "-0", "0.0", "-0.000", ".5", "5.", "+1", "1e0", "1E+2", "2.5e-3", "1e-45", "1.4e-45",
             "1.17549435e-38", "1.1754942e-38", "3.4028235e38", "3.4028236e38", "1e39", "123456789012345678",
             "1234567890123456789012", "0.000000000000000000000000001", "9007199254740993", "16777217",
             "0.1", "0.2", "0.3", "1.23782778", "1.5abc", "inf", "nan", "0x1p3"]
    return toks


def _strtof(tokens):
    import ctypes as C
    libc = C.CDLL("libc.so.6")
    libc.strtof.restype = C.c_float
    libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
    return np.array([libc.strtof(t.encode(), None) for t in tokens], np.float32)


@pytest.mark.parametrize("parallel", [False, True])
def test_reader_weights_round_like_strtof(lvb, tmp_path, parallel):
    """Every weight token reads as the float strtof gives (the reference reads
    weights with `>>` into a float): the reader's fast decimal path and its
    strtof fall-back together, on the sequential reading (small file) and on
    the multi-threaded one (over 4 MB and 100,000 entries)."""
    import ctypes as C
    toks = _weight_tokens(200000 if parallel else 4000)
    n = len(toks)
    p = tmp_path / "w.mtx"
    with open(p, "w") as f:
        f.write("%%%%MatrixMarket matrix coordinate real symmetric\n5 5 %d\n" % n)
        for i, t in enumerate(toks):
            f.write("%d %d %s\n" % (1 + i % 5, 1 + (i * 7 + 1) % 5, t))
    if parallel:
        assert os.path.getsize(p) > (1 << 22)
    L = lvb.lib()
    V, m = C.c_int32(), C.c_int64()
    a, b, w = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_float)()
    assert L.lv_read_mtx_entries(str(p).encode(), C.byref(V), C.byref(m), C.byref(a), C.byref(b), C.byref(w)) == 0
    assert m.value == n
    got = np.ctypeslib.as_array(w, shape=(n,)).copy()
    for x in (a, b, w):
        L.lv_free_host(C.cast(x, C.c_void_p))
    want = _strtof(toks)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
