"""CPU checks of the oracle: hand-derived cases, reference conventions,
determinism, and the golden vectors produced by the reference itself."""
import glob
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR


def csr(V, edges, gnp):
    return gnp.csr_from_edges(V, edges)


def test_two_triangles_with_bridge(orc, gnp):
    edges = [(0, 1, 1), (1, 2, 1), (0, 2, 1), (3, 4, 1), (4, 5, 1), (3, 5, 1), (2, 3, 1)]
    rp, cl, w = csr(6, edges, gnp)
    o = orc.Oracle(rp, cl, w, 1)
    q, st = o.run(1e-6)
    o2c = o.original_to_community()
    assert len(set(o2c[:3])) == 1 and len(set(o2c[3:])) == 1 and o2c[0] != o2c[3]
    # T = 14; e_own = 12; S = 7, 7  ->  Q = 12/14 - 98/196
    assert q == pytest.approx(12 / 14 - 98 / 196, abs=1e-15)
    assert orc.modularity_f64(rp, cl, w, o2c) == pytest.approx(q, abs=1e-12)


def test_singleton_guard_and_tie(orc, gnp):
    # single edge: vertex 0 may not join singleton 1 (1 > 0); vertex 1 joins 0
    rp, cl, w = csr(2, [(0, 1, 1)], gnp)
    o = orc.Oracle(rp, cl, w, 1)
    moves = o.sweep()
    assert moves == 1
    assert list(o.communities()) == [0, 0]
    assert o.modularity() == pytest.approx(0.0, abs=1e-15)


def test_isolated_and_self_loops(orc, gnp):
    # vertex 4 isolated; 0 has a self-loop counted once in k and in T
    edges = [(0, 0, 2.0), (0, 1, 1.0), (1, 2, 1.0), (2, 0, 1.0), (3, 3, 1.0)]
    rp, cl, w = csr(5, edges, gnp)
    o = orc.Oracle(rp, cl, w, 1)
    s, T = o.scale()
    assert s == 0 and T == int(sum(w))          # T = sum of CSR weights = 2M
    k = o.vertex_weights()
    assert list(k) == [4, 2, 2, 1, 0]
    q, st = o.run(1e-9)
    o2c = o.original_to_community()
    assert o2c[4] != o2c[0] and o2c[3] != o2c[0]
    assert len(set(o2c[:3])) == 1
    assert orc.modularity_f64(rp, cl, w, o2c) == pytest.approx(q, abs=1e-12)


def ring_of_cliques(k, s, gnp):
    """k cliques of s vertices (unit weights), clique c's last vertex joined to
    clique c+1's first (mod k)."""
    edges = []
    for c in range(k):
        b = c * s
        edges += [(b + i, b + j, 1.0) for i in range(s) for j in range(i + 1, s)]
        edges.append((b + s - 1, ((c + 1) % k) * s, 1.0))
    return csr(k * s, edges, gnp)


def test_ring_of_cliques(orc, gnp):
    # 6 cliques of 5: one community per clique, Q = sum over cliques of
    # l/m - (d/2m)^2 with l = 10 internal edges, d = 22, m = 66
    rp, cl, w = ring_of_cliques(6, 5, gnp)
    o = orc.Oracle(rp, cl, w, 1)
    q, _ = o.run(1e-6)
    m = o.original_to_community()
    assert [len(set(m[c * 5:(c + 1) * 5])) for c in range(6)] == [1] * 6
    assert len(set(m.tolist())) == 6
    assert q == pytest.approx(6 * (10 / 66 - (22 / 132) ** 2), abs=1e-15)
    # 8 cliques of 4: the synchronous sub-rounds end in a local optimum that
    # keeps every clique whole but merges one adjacent pair: 7 communities,
    # Q = 13/56 - (28/112)^2 + 6 (6/56 - (14/112)^2) = 23/32 (one community per
    # clique would give 41/56)
    rp, cl, w = ring_of_cliques(8, 4, gnp)
    o = orc.Oracle(rp, cl, w, 1)
    q, _ = o.run(1e-6)
    m = o.original_to_community()
    assert all(len(set(m[c * 4:(c + 1) * 4])) == 1 for c in range(8))
    labels = [m[c * 4] for c in range(8)]
    assert len(set(labels)) == 7
    pair = [c for c in range(8) if labels.count(labels[c]) == 2]
    assert len(pair) == 2 and (pair[1] - pair[0]) % 8 in (1, 7)
    assert q == pytest.approx(23 / 32, abs=1e-15)
    # 30 triangles: past the resolution limit (k > s(s-1) + 2) merging
    # adjacent cliques raises Q above one community per clique
    rp, cl, w = ring_of_cliques(30, 3, gnp)
    o = orc.Oracle(rp, cl, w, 1)
    q, _ = o.run(1e-6)
    m = o.original_to_community()
    assert all(len(set(m[c * 3:(c + 1) * 3])) == 1 for c in range(30))
    assert len(set(m.tolist())) < 30
    assert q > 30 * (3 / 120 - (8 / 240) ** 2)


def test_duplicate_edge_mtx(orc, lvb, tmp_path):
    """A repeated entry is kept twice, as the reference's reader appends every
    line (utils.cu:50-59): it counts twice in k, in T and in e_own."""
    p = tmp_path / "dup.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 3\n2 1 1\n2 1 1\n3 2 1\n")
    rp, cl, w, _ = orc.read_mtx(str(p))
    assert list(rp) == [0, 2, 5, 6] and list(cl) == [1, 1, 0, 0, 2, 1]
    r = lvb.read_mtx(str(p))
    assert np.array_equal(r.rowptr, rp) and np.array_equal(r.col, cl) and np.array_equal(r.w, w)
    # partition {0, 1}, {2}: T = 6, e_own = 4, S = (2 + 3, 1)
    q = orc.modularity_f64(rp, cl, w, np.array([0, 0, 2], np.int32))
    assert q == pytest.approx(4 / 6 - (25 + 1) / 36, abs=1e-15)
    o = orc.Oracle(rp, cl, w, 1)
    o.set_communities(np.array([0, 0, 2], np.int32))
    assert o.modularity() == q


def test_scale_rule(orc):
    rc, s, ex = orc.choose_scale(np.array([1.0, 2.0, 3.0], np.float32))
    assert (rc, s, ex) == (0, 0, True)
    rc, s, ex = orc.choose_scale(np.array([0.5, 0.75, 1.25], np.float32))
    assert (rc, s, ex) == (0, 2, True)
    w = np.float32(0.5) + np.arange(1000, dtype=np.float32) * np.float32(2.0 ** -24)
    rc, s, ex = orc.choose_scale(w)
    assert (rc, s) == (0, 24)
    assert orc.choose_scale(np.array([1.0, -1.0], np.float32))[0] == 2
    assert orc.choose_scale(np.array([1.0, np.nan], np.float32))[0] == 2
    assert orc.choose_scale(np.array([1.0, np.inf], np.float32))[0] == 2
    # weights too fine for the grid get rounded (exact flag off)
    rc, s, ex = orc.choose_scale(np.array([2.0 ** 40, 2.0 ** -30], np.float32))
    assert rc == 0 and not ex and s == 61 - 40 - 1


def test_thread_count_does_not_change_results(orc, lvb):
    g = lvb.gen_rmat(12, seed=3)
    res = []
    for nt in (1, 3, 8):
        o = orc.Oracle(g.rowptr, g.col, g.w, nt)
        q, st = o.run(1e-6)
        res.append((q, st["sweeps"], o.original_to_community().tobytes()))
    assert res[0] == res[1] == res[2]


def test_planted_partition_recovered(orc, lvb):
    for seed in range(5):
        g = lvb.gen_planted(10000, 64, 16.0, 2.0, seed)
        o = orc.Oracle(g.rowptr, g.col, g.w)
        q, st = o.run(0.01)
        o2c = o.original_to_community()
        blocks = (np.arange(10000, dtype=np.int64) * 64) // 10000
        # each planted block has its own majority community, which holds
        # almost all of its vertices
        major = [np.bincount(o2c[blocks == b]).argmax() for b in range(64)]
        assert len(set(major)) == 64
        agree = sum(int((o2c[blocks == b] == major[b]).sum()) for b in range(64))
        assert agree >= 0.995 * 10000
        assert orc.modularity_f64(g.rowptr, g.col, g.w, o2c) == pytest.approx(q, abs=1e-9)


def test_aggregation_preserves_totals(orc, lvb):
    g = lvb.gen_rmat(11, seed=5)
    o = orc.Oracle(g.rowptr, g.col, g.w)
    o.optimise_modularity(1e-6)
    comm = o.communities()
    _, T = o.scale()
    q_before = o.modularity()
    S = o.community_weights()
    o.aggregate_communities()
    rp, cl, wf = o.csr()
    assert int(wf.sum()) == T
    # aggregated graph with identity communities has the same modularity
    assert o.modularity() == q_before
    # new vertex weights = old Sigma_tot of the non-empty communities, in id order
    nonempty = np.unique(comm)
    assert np.array_equal(o.vertex_weights(), S[nonempty])
    # symmetric
    V = len(rp) - 1
    row = np.repeat(np.arange(V), np.diff(rp))
    A = {(int(a), int(b)): int(x) for a, b, x in zip(row, cl, wf)}
    assert all(A[(b, a)] == x for (a, b), x in A.items())


def test_read_mtx_conventions(orc, tmp_path):
    p = tmp_path / "g.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n% comment\n"
                 "4 4 5\n2 1 1.5\n3 1 0.25\n3 3 2\n4 2 1\n4 3 0.5\n")
    rp, cl, w, m = orc.read_mtx(str(p))
    assert list(rp) == [0, 2, 4, 7, 9]
    assert list(cl) == [1, 2, 0, 3, 0, 2, 3, 1, 2]
    assert list(w) == [1.5, 0.25, 1.5, 1.0, 0.25, 2.0, 0.5, 1.0, 0.5]
    # M = (sum of 2w off-diagonal + w self-loop) / 2
    assert m == pytest.approx((2 * (1.5 + 0.25 + 1 + 0.5) + 2) / 2)


# ---------------------------------------------------------------------------
# golden vectors from the reference's own code (tests/golden/make_golden.py)
# ---------------------------------------------------------------------------
def _goldens():
    idx = os.path.join(GOLDEN_DIR, "index.json")
    if not os.path.exists(idx):
        return []
    with open(idx) as f:
        return json.load(f)["cases"]


def _load_graph(case, orc):
    return orc.read_mtx(os.path.join(GOLDEN_DIR, case["mtx"]))


@pytest.mark.parametrize("case", _goldens(), ids=lambda c: c["name"])
def test_oracle_matches_reference_sweeps(case, orc):
    """Each sweep of the reference's optimiseModularity equals the oracle's."""
    rp, cl, w, _ = _load_graph(case, orc)
    ref = np.fromfile(os.path.join(GOLDEN_DIR, case["sweeps"]), dtype=np.int32)
    V, n = int(ref[0]), int(ref[1])
    ref = ref[2:].reshape(n, V)
    o = orc.Oracle(rp, cl, w, 1)
    for s in range(n):
        o.sweep()
        assert np.array_equal(o.communities(), ref[s]), f"sweep {s + 1} differs"


@pytest.mark.parametrize("case", _goldens(), ids=lambda c: c["name"])
def test_oracle_matches_reference_aggregation(case, orc):
    """aggregateCommunities of the reference == oracle aggregation (rows
    compared as sorted (neighbour, weight) sets; exact sums)."""
    rp, cl, w, _ = _load_graph(case, orc)
    comm = np.fromfile(os.path.join(GOLDEN_DIR, case["agg_in"]), dtype=np.int32)
    raw = np.fromfile(os.path.join(GOLDEN_DIR, case["agg_out"]), dtype=np.int32)
    V2, E2, V0 = int(raw[0]), int(raw[1]), int(raw[2])
    o = 3
    rrp = raw[o:o + V2 + 1]; o += V2 + 1
    rcl = raw[o:o + E2]; o += E2
    rw = raw[o:o + E2].view(np.float32); o += E2
    ro2c = raw[o:o + V0]; o += V0
    rcw = raw[o:o + V2].view(np.float32)
    orac = orc.Oracle(rp, cl, w, 1)
    orac.set_communities(comm)
    orac.aggregate_communities()
    prp, pcl, pwf = orac.csr()
    scale, _ = orac.scale()
    assert orac.V == V2 and orac.E == E2
    for v in range(V2):
        a = sorted(zip(rcl[rrp[v]:rrp[v + 1]].tolist(), rw[rrp[v]:rrp[v + 1]].tolist()))
        b = sorted(zip(pcl[prp[v]:prp[v + 1]].tolist(), (pwf[prp[v]:prp[v + 1]] / 2.0 ** scale).tolist()))
        assert a == b, f"row {v}"
    # the harness set originalToCommunity = comm first, so the reference maps
    # every original vertex to the new id of its community
    newid = np.searchsorted(np.unique(comm), comm)
    assert np.array_equal(newid, ro2c)
    assert np.array_equal(orac.vertex_weights() / 2.0 ** scale, rcw.astype(np.float64))


@pytest.mark.parametrize("case", _goldens(), ids=lambda c: c["name"])
def test_reference_stock_build_does_not_move(case):
    """Evidence of the reference's defect on B200: with its stock launch shape
    the final store of computeMove races (modularity_optimisation.cu:192-196)
    and the old community wins, so (almost) no vertex ever moves."""
    ref = np.fromfile(os.path.join(GOLDEN_DIR, case["sweeps_stock"]), dtype=np.int32)
    V, n = int(ref[0]), int(ref[1])
    moved = (ref[2:].reshape(n, V) != np.arange(V)).sum(axis=1)
    assert moved.max() <= max(16, V // 100)


@pytest.mark.parametrize("case", _goldens(), ids=lambda c: c["name"])
def test_reference_final_modularity(case, orc):
    """The reference binary's printed Q equals the FP64 modularity of its own
    printed map: pins the loader conventions (M, self-loops, vertex count)
    and the Q formula.  (Its partition is the trivial one on B200, see
    test_reference_stock_build_does_not_move.)"""
    rp, cl, w, _ = _load_graph(case, orc)
    with open(os.path.join(GOLDEN_DIR, case["cli"])) as f:
        lines = f.read().split("\n")
    q_ref = float(lines[0])
    nc = int(lines[2])
    o2c = np.empty(len(rp) - 1, np.int32)
    for line in lines[3:3 + nc]:
        parts = [int(x) for x in line.split()]
        for m in parts[1:]:
            o2c[m - 1] = parts[0] - 1
    q_map = orc.modularity_f64(rp, cl, w, o2c)
    assert q_map == pytest.approx(q_ref, abs=2e-6)
    # the oracle evaluates the same partition to the same value
    o = orc.Oracle(rp, cl, w, 1)
    o.set_communities(o2c)
    assert o.modularity() == pytest.approx(q_map, abs=1e-12)
