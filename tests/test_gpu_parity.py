"""GPU engine vs the CPU oracle through the C ABI: every sweep's community
vector, every aggregated CSR and every final partition must be identical
(integer decisions, exact sums); modularity values must be bit-identical
doubles because both sides form them from the same exact integer totals."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu


def hub_graph(seed=0):
    """Background random graph plus hubs of degree 500 / 2000 / 6000 / 20000,
    so that every work class (including the global-table path) runs."""
    rng = np.random.default_rng(seed)
    V = 40000
    m = 60000
    u = rng.integers(0, V, m)
    v = rng.integers(0, V, m)
    hubs = [(5, 500), (17, 2000), (123, 6000), (999, 20000)]
    for h, d in hubs:
        nb = rng.choice(V, d, replace=False)
        u = np.concatenate([u, np.full(d, h)])
        v = np.concatenate([v, nb])
    keep = u != v
    a, b = np.minimum(u[keep], v[keep]), np.maximum(u[keep], v[keep])
    key = np.unique(a.astype(np.int64) * V + b)
    a, b = key // V, key % V
    w = (rng.integers(1, 8, len(a)) * 0.25).astype(np.float32)
    src = np.concatenate([a, b]); dst = np.concatenate([b, a]); ww = np.concatenate([w, w])
    o = np.lexsort((dst, src))
    rowptr = np.concatenate([[0], np.cumsum(np.bincount(src, minlength=V))]).astype(np.int32)
    return rowptr, dst[o].astype(np.int32), ww[o].astype(np.float32)


def megahub_graph(seed=5):
    """Random background plus a hub adjacent to 1.6M vertices and a hub of
    degree 300000: in the first sweep their staged pairs exceed one shared
    table and are decided as hundreds of key-space partitions."""
    rng = np.random.default_rng(seed)
    V = 1_700_000
    m = 1_000_000
    u = rng.integers(0, V, m)
    v = rng.integers(0, V, m)
    for h, d in [(7, 1_600_000), (70001, 300_000)]:
        nb = rng.choice(V, d, replace=False)
        u = np.concatenate([u, np.full(d, h)])
        v = np.concatenate([v, nb])
    keep = u != v
    a, b = np.minimum(u[keep], v[keep]), np.maximum(u[keep], v[keep])
    key = np.unique(a.astype(np.int64) * V + b)
    a, b = key // V, key % V
    w = (rng.integers(1, 8, len(a)) * 0.25).astype(np.float32)
    src = np.concatenate([a, b]); dst = np.concatenate([b, a]); ww = np.concatenate([w, w])
    o = np.lexsort((dst, src))
    rowptr = np.concatenate([[0], np.cumsum(np.bincount(src, minlength=V))]).astype(np.int32)
    return rowptr, dst[o].astype(np.int32), ww[o].astype(np.float32)


def cases(lvb):
    out = {}
    g = lvb.gen_planted(10000, 64, 16.0, 2.0, 0)
    out["planted10k_s0"] = (g.rowptr, g.col, g.w, 0.01)
    g = lvb.gen_planted(10000, 64, 16.0, 2.0, 3, "uniform")
    out["planted10k_uniform"] = (g.rowptr, g.col, g.w, 0.01)
    g = lvb.gen_rmat(12, seed=2)
    out["rmat12"] = (g.rowptr, g.col, g.w, 1e-6)
    g = lvb.gen_rmat(14, seed=1, weights="unit")
    out["rmat14_unit"] = (g.rowptr, g.col, g.w, 1e-6)
    g = lvb.gen_rmat(15, seed=4)
    out["rmat15"] = (g.rowptr, g.col, g.w, 1e-6)
    rp, cl, w = hub_graph()
    out["hubs"] = (rp, cl, w, 1e-6)
    return out


@pytest.fixture(scope="module")
def graphs(lvb):
    return cases(lvb)


NAMES = ["planted10k_s0", "planted10k_uniform", "rmat12", "rmat14_unit", "rmat15", "hubs"]


def canon(rp, cl, wf):
    rows = []
    for v in range(len(rp) - 1):
        a, b = int(rp[v]), int(rp[v + 1])
        o = np.lexsort((wf[a:b], cl[a:b]))
        rows.append((cl[a:b][o].tolist(), wf[a:b][o].tolist()))
    return rows


@pytest.mark.parametrize("name", NAMES)
def test_sweeps_match_oracle(lvb, orc, graphs, name):
    rp, cl, w, _ = graphs[name]
    g = lvb.Graph(rp, cl, w)
    e = lvb.Louvain(g, verify=True)
    o = orc.Oracle(rp, cl, w)
    assert e.scale()[:2] == o.scale()
    assert e.calculate_modularity() == o.modularity()
    for s in range(40):
        m1 = e.sweep()
        m2 = o.sweep()
        assert m1 == m2, f"sweep {s}: moves {m1} vs {m2}"
        assert np.array_equal(e.communities(), o.communities()), f"sweep {s}"
        assert e.calculate_modularity() == o.modularity()
        if m1 == 0:
            break
    e.close()


@pytest.mark.parametrize("name", NAMES)
def test_levels_and_aggregation_match_oracle(lvb, orc, graphs, name):
    rp, cl, w, gain = graphs[name]
    e = lvb.Louvain(lvb.Graph(rp, cl, w), verify=True)
    o = orc.Oracle(rp, cl, w)
    for level in range(12):
        c1 = e.optimise_modularity(gain)
        c2, _ = o.optimise_modularity(gain)
        assert c1 == c2
        assert np.array_equal(e.communities(), o.communities())
        assert np.array_equal(e.original_to_community()[0], o.original_to_community())
        if not c1:
            break
        e.aggregate_communities()
        o.aggregate_communities()
        V1, E1, _ = e.level_info()
        assert (V1, E1) == (o.V, o.E), f"level {level}"
        assert canon(*e.csr()) == canon(*o.csr())
    assert e.calculate_modularity() == o.modularity()


@pytest.mark.parametrize("name", NAMES)
def test_full_run_matches_oracle(lvb, orc, graphs, name):
    rp, cl, w, gain = graphs[name]
    e = lvb.Louvain(lvb.Graph(rp, cl, w))
    q1 = e.run(gain)
    o2c1, nc1 = e.original_to_community()
    o = orc.Oracle(rp, cl, w)
    q2, st = o.run(gain)
    assert q1 == q2
    assert nc1 == o.V
    assert np.array_equal(o2c1, o.original_to_community())
    # FP64 recomputation from the map on the original float weights
    assert abs(orc.modularity_f64(rp, cl, w, o2c1) - q1) < 1e-9
    s = e.stats()
    assert s["sweeps"] == st["sweeps"] and s["levels"] == st["levels"]
    # a second run on the same handle is bit-identical
    e.reset()
    assert e.run(gain) == q1
    assert np.array_equal(e.original_to_community()[0], o2c1)
    e.close()
    # aggregated levels read as uint64 sums instead of their 32-bit copy
    with lvb.Louvain(lvb.Graph(rp, cl, w), wide_weights=True) as ew:
        assert ew.run(gain) == q1
        assert np.array_equal(ew.original_to_community()[0], o2c1)


def test_megahub_matches_oracle(lvb, orc):
    rp, cl, w = megahub_graph()
    e = lvb.Louvain(lvb.Graph(rp, cl, w), verify=True)
    o = orc.Oracle(rp, cl, w)
    for s in range(6):
        m1, m2 = e.sweep(), o.sweep()
        assert m1 == m2, f"sweep {s}: moves {m1} vs {m2}"
        assert np.array_equal(e.communities(), o.communities()), f"sweep {s}"
        assert e.calculate_modularity() == o.modularity()
        if m1 == 0:
            break
    e.close()
    e = lvb.Louvain(lvb.Graph(rp, cl, w))
    q1 = e.run(1e-6)
    q2, _ = o.__class__(rp, cl, w).run(1e-6)
    assert q1 == q2
    e.close()


def test_giant_paths_match_oracle(lvb, orc):
    """Giants (degree > 8192) whose neighbours fall into few communities
    (staged pairs merged in one shared table) and into as many communities as
    neighbours (staged pairs split into key-space partitions), with the
    communities changed between sweeps."""
    rng = np.random.default_rng(11)
    V = 60000
    u = rng.integers(0, V, 120000)
    v = rng.integers(0, V, 120000)
    for h, d in [(0, 30000), (1, 10000), (2, 25000)]:
        nb = rng.choice(V, d, replace=False)
        u = np.concatenate([u, np.full(d, h)])
        v = np.concatenate([v, nb])
    keep = u != v
    a, b = np.minimum(u[keep], v[keep]), np.maximum(u[keep], v[keep])
    key = np.unique(a.astype(np.int64) * V + b)
    a, b = key // V, key % V
    w = (rng.integers(1, 8, len(a)) * 0.25).astype(np.float32)
    src = np.concatenate([a, b]); dst = np.concatenate([b, a]); ww = np.concatenate([w, w])
    o_ = np.lexsort((dst, src))
    rp = np.concatenate([[0], np.cumsum(np.bincount(src, minlength=V))]).astype(np.int32)
    cl, w = dst[o_].astype(np.int32), ww[o_].astype(np.float32)
    e = lvb.Louvain(lvb.Graph(rp, cl, w), verify=True)
    o = orc.Oracle(rp, cl, w)

    def sweeps(k, tag):
        for s in range(k):
            m1, m2 = e.sweep(), o.sweep()
            assert m1 == m2, f"{tag} sweep {s}"
            assert np.array_equal(e.communities(), o.communities()), f"{tag} sweep {s}"
            assert e.calculate_modularity() == o.modularity()

    blocks = (np.arange(V) // 1000).astype(np.int32)
    e.set_communities(blocks); o.set_communities(blocks)
    sweeps(3, "blocks")
    single = np.arange(V, dtype=np.int32)
    e.set_communities(single); o.set_communities(single)
    sweeps(3, "singletons")
    e.close()


@pytest.mark.parametrize("name", ["planted10k_uniform", "rmat15", "hubs"])
def test_sweep_graph_matches_host_loop(lvb, orc, graphs, name):
    """A level's sweep loop run as one CUDA graph (device-side continuation
    test) gives the same sweeps, moves, levels, modularity and map as the
    loop with one host round trip per sweep, and the same as the oracle."""
    rp, cl, w, gain = graphs[name]
    out = []
    for graph_loop in (True, False):
        e = lvb.Louvain(lvb.Graph(rp, cl, w), sweep_graph=graph_loop)
        q = e.run(gain)
        s = e.stats()
        out.append((q, s["sweeps"], s["moves"], s["levels"], s["edge_sweeps"],
                    e.original_to_community()[0].tobytes()))
        e.close()
    assert out[0] == out[1]
    q2, st = orc.Oracle(rp, cl, w).run(gain)
    assert out[0][0] == q2 and out[0][1] == st["sweeps"]


def test_handles_reuse_pooled_memory(lvb, orc, graphs):
    """Handles created after others were destroyed (memory reused from the
    library's device pool) and after the pool was trimmed give the same
    results."""
    rp, cl, w, gain = graphs["rmat14_unit"]
    qs = []
    for trim in (False, False, True, False):
        e = lvb.Louvain(lvb.Graph(rp, cl, w))
        qs.append((e.run(gain), e.original_to_community()[0].tobytes()))
        e.close()
        if trim:
            assert lvb.lib().lv_trim_device_memory(0) == lvb.LV_OK
    assert all(q == qs[0] for q in qs)
    assert lvb.lib().lv_trim_device_memory(-1) == lvb.LV_ERR_INVALID


def test_aggregation_from_given_communities(lvb, orc, graphs):
    rng = np.random.default_rng(7)
    for name in ("rmat12", "hubs", "planted10k_uniform"):
        rp, cl, w, _ = graphs[name]
        V = len(rp) - 1
        for ncomm in (3, V // 50, V // 2):
            comm = rng.integers(0, max(ncomm, 1), V).astype(np.int32)
            e = lvb.Louvain(lvb.Graph(rp, cl, w))
            o = orc.Oracle(rp, cl, w)
            e.set_communities(comm)
            o.set_communities(comm)
            assert e.calculate_modularity() == o.modularity()
            e.aggregate_communities()
            o.aggregate_communities()
            assert e.level_info()[:2] == (o.V, o.E)
            assert canon(*e.csr()) == canon(*o.csr())


def test_edge_cases(lvb, orc, gnp):
    cases = {
        "no_edges": (4, []),
        "single_edge": (2, [(0, 1, 1.0)]),
        "self_loops_only": (3, [(0, 0, 1.0), (1, 1, 2.0)]),
        "star": (200, [(0, i, 1.0) for i in range(1, 200)]),
        "duplicates": (4, [(0, 1, 1.0), (1, 0, 2.0), (1, 2, 1.0), (2, 3, 0.5), (3, 2, 0.5)]),
        "zero_weight": (4, [(0, 1, 0.0), (1, 2, 1.0), (2, 3, 1.0)]),
        "isolated": (6, [(0, 1, 1.0), (1, 2, 1.0), (4, 4, 1.0)]),
    }
    for name, (V, edges) in cases.items():
        rp, cl, w = gnp.csr_from_edges(V, edges)
        e = lvb.Louvain(lvb.Graph(rp, cl, w))
        o = orc.Oracle(rp, cl, w, 1)
        q1 = e.run(1e-6)
        q2, _ = o.run(1e-6)
        assert (q1 == q2) or (np.isnan(q1) and np.isnan(q2)), name
        assert np.array_equal(e.original_to_community()[0], o.original_to_community()), name


def test_invalid_inputs(lvb, gnp):
    rp, cl, w = gnp.csr_from_edges(3, [(0, 1, 1.0), (1, 2, 1.0)])
    bad = w.copy()
    bad[0] = -1.0
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.Louvain(lvb.Graph(rp, cl, bad))
    assert ex.value.status == lvb.LV_ERR_WEIGHT
    bad = w.copy()
    bad[1] = np.nan
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.Louvain(lvb.Graph(rp, cl, bad))
    assert ex.value.status == lvb.LV_ERR_WEIGHT
    badc = cl.copy()
    badc[0] = 7
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.Louvain(lvb.Graph(rp, badc, w))
    assert ex.value.status == lvb.LV_ERR_INVALID
    badr = rp.copy()
    badr[1] = 5
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.Louvain(lvb.Graph(badr, cl, w))
    assert ex.value.status == lvb.LV_ERR_INVALID
    e = lvb.Louvain(lvb.Graph(rp, cl, w))
    with pytest.raises(lvb.LouvainError):
        e.set_communities(np.array([0, 1, 9], np.int32))


def test_device_generator_matches_host(lvb):
    for sc in (10, 14):
        dg = lvb.gen_rmat_device(sc, seed=3)
        hg = lvb.gen_rmat(sc, seed=3)
        assert (dg.V, dg.E) == (hg.V, hg.E)
        e = lvb.Louvain(device_csr=(dg.rowptr, dg.col, dg.w, dg.V, dg.E))
        rp, cl, wf = e.csr()
        s, T, exact = e.scale()
        assert exact and s == 24
        assert np.array_equal(rp, hg.rowptr) and np.array_equal(cl, hg.col)
        assert np.array_equal(wf, (hg.w.astype(np.float64) * 2.0 ** s).astype(np.int64))
        e.close()
        dg.free()


def test_cli_output(lvb, orc, tmp_path):
    g = lvb.gen_planted(2000, 16, 12.0, 2.0, 1)
    p = str(tmp_path / "g.mtx")
    lvb.write_mtx(p, g)
    r = subprocess.run([lvb.CLI_PATH, "-f", p, "-g", "0.01", "-v"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    gr = lvb.read_mtx(p)
    e = lvb.Louvain(gr)
    q = e.run(0.01)
    assert lines[0] == "%f" % q
    algo, total = (float(x) for x in lines[1].split())
    assert 0 <= algo <= total
    o2c, nc = e.original_to_community()
    assert int(lines[2]) == nc
    got = np.empty(gr.V, np.int32)
    for line in lines[3:3 + nc]:
        parts = [int(x) for x in line.split()]
        assert parts[0] >= 1
        for m in parts[1:]:
            got[m - 1] = parts[0] - 1
    assert np.array_equal(got, o2c)
    r2 = subprocess.run([lvb.CLI_PATH, "-f", p, "-g", "0.01"], capture_output=True, text=True)
    assert r2.stdout.split("\n")[0] == lines[0] and len(r2.stdout.split("\n")) == 3


def test_cli_cache_follows_source(lvb, tmp_path):
    """gpulouvain -c reuses <file>.lvcsr only while the text file's size and
    modification time match the ones recorded in the cache: a file replaced
    by another graph with an older modification time is parsed again."""
    p = str(tmp_path / "g.mtx")
    first = lvb.gen_planted(1500, 12, 12.0, 2.0, 1)
    lvb.write_mtx(p, first)
    r1 = subprocess.run([lvb.CLI_PATH, "-f", p, "-g", "0.01", "-c"], capture_output=True, text=True)
    assert r1.returncode == 0, r1.stderr
    assert os.path.exists(p + ".lvcsr")
    r1b = subprocess.run([lvb.CLI_PATH, "-f", p, "-g", "0.01", "-c"], capture_output=True, text=True)
    assert r1b.stdout.split("\n")[0] == r1.stdout.split("\n")[0]
    second = lvb.gen_planted(1800, 9, 14.0, 1.0, 2)
    lvb.write_mtx(p, second)
    old = os.stat(p + ".lvcsr").st_mtime - 3600
    os.utime(p, (old, old))        # older than the cache, as after cp -p / tar / rsync -t
    r2 = subprocess.run([lvb.CLI_PATH, "-f", p, "-g", "0.01", "-c"], capture_output=True, text=True)
    r3 = subprocess.run([lvb.CLI_PATH, "-f", p, "-g", "0.01"], capture_output=True, text=True)
    assert r2.returncode == 0 and r3.returncode == 0
    assert r2.stdout.split("\n")[0] == r3.stdout.split("\n")[0]
    e = lvb.Louvain(lvb.read_mtx(p))
    assert r3.stdout.split("\n")[0] == "%f" % e.run(0.01)
    e.close()


# ---------------------------------------------------------------------------
# golden vectors produced by the reference's own code
# ---------------------------------------------------------------------------
def _goldens():
    import json
    idx = os.path.join(GOLDEN_DIR, "index.json")
    if not os.path.exists(idx):
        return []
    with open(idx) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _goldens(), ids=lambda c: c["name"])
def test_engine_matches_reference_goldens(lvb, case):
    g = lvb.read_mtx(os.path.join(GOLDEN_DIR, case["mtx"]))
    ref = np.fromfile(os.path.join(GOLDEN_DIR, case["sweeps"]), dtype=np.int32)
    V, n = int(ref[0]), int(ref[1])
    ref = ref[2:].reshape(n, V)
    e = lvb.Louvain(g)
    for s in range(n):
        e.sweep()
        assert np.array_equal(e.communities(), ref[s]), f"sweep {s + 1}"
    # aggregation of the given community vector: bit-exact rows
    comm = np.fromfile(os.path.join(GOLDEN_DIR, case["agg_in"]), dtype=np.int32)
    raw = np.fromfile(os.path.join(GOLDEN_DIR, case["agg_out"]), dtype=np.int32)
    V2, E2, V0 = int(raw[0]), int(raw[1]), int(raw[2])
    rrp = raw[3:3 + V2 + 1]
    rcl = raw[4 + V2:4 + V2 + E2]
    rw = raw[4 + V2 + E2:4 + V2 + 2 * E2].view(np.float32)
    e2 = lvb.Louvain(g)
    e2.set_communities(comm)
    e2.aggregate_communities()
    prp, pcl, pwf = e2.csr()
    s, _, _ = e2.scale()
    assert e2.level_info()[:2] == (V2, E2)
    for v in range(V2):
        a = sorted(zip(rcl[rrp[v]:rrp[v + 1]].tolist(), rw[rrp[v]:rrp[v + 1]].tolist()))
        b = sorted(zip(pcl[prp[v]:prp[v + 1]].tolist(), (pwf[prp[v]:prp[v + 1]] / 2.0 ** s).tolist()))
        assert a == b


@pytest.mark.parametrize("name", ["rmat15", "hubs"])
def test_work_mapping_knobs_do_not_change_results(lvb, graphs, name):
    """The autotuner's knobs (giant threshold, warp overflow limit, 64-bit
    sums) move work between kernels; every setting gives the same sweeps."""
    rp, cl, w, gain = graphs[name]
    runs = []
    for kw in ({}, {"giant_degree": 1024}, {"giant_degree": 65536}, {"warp_limit": 32},
               {"warp_limit": 384}, {"giant_degree": 1024, "warp_limit": 32, "wide_weights": True}):
        with lvb.Louvain(lvb.Graph(rp, cl, w), **kw) as e:
            q = e.run(gain)
            runs.append((kw, q, e.original_to_community()[0], e.stats()["sweeps"]))
    for kw, q, m, sw in runs[1:]:
        assert q == runs[0][1], kw
        assert np.array_equal(m, runs[0][2]), kw
        assert sw == runs[0][3], kw


def test_work_mapping_knobs_are_checked(lvb):
    g = lvb.gen_planted(500, 8, 10.0, 2.0, 1)
    for kw in ({"giant_degree": 1000}, {"giant_degree": 70000}, {"warp_limit": 16}, {"warp_limit": 400}):
        with pytest.raises(lvb.LouvainError) as ex:
            lvb.Louvain(g, **kw)
        assert ex.value.status == lvb.LV_ERR_INVALID
