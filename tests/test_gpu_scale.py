"""Parity at the configurations the benchmark metric is quoted on.

R-MAT scale 20 (seed 1, 2^20 vertices, edge factor 16, a=.57 b=.19 c=.19,
float32 weights uniform in [0.5, 1.5), gain threshold 1e-6), run by the engine
through the C ABI and by the CPU oracle: every level-0 sweep's community
vector and move count, every level's partition and aggregated CSR, and the
complete run's map, modularity bits, level, sweep and edge-sweep counts must
be identical.  The R-MAT-24 headline graph is checked the same way (first
sweep, complete run) by bench.py on every benchmark run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAIN = 1e-6


@pytest.fixture(scope="module")
def rmat20(lvb):
    g = lvb.gen_rmat(20, 16, 1)
    assert g.V == 1 << 20 and g.E == 31404496
    return g


def _canon(rp, cl, wf):
    """Rows sorted by (column, weight): a layout-independent form of a CSR."""
    rp = np.asarray(rp, np.int64)
    V = len(rp) - 1
    row = np.repeat(np.arange(V, dtype=np.int64), np.diff(rp))
    o = np.lexsort((np.asarray(wf), np.asarray(cl), row))
    return rp, np.asarray(cl)[o], np.asarray(wf)[o]


def test_rmat20_level0_sweeps_match_oracle(lvb, orc, rmat20):
    g = rmat20
    e = lvb.Louvain(g)
    o = orc.Oracle(g.rowptr, g.col, g.w)
    assert e.calculate_modularity() == o.modularity()
    q_before = o.modularity()
    for s in range(64):
        m1, m2 = e.sweep(), o.sweep()
        assert m1 == m2, f"sweep {s}: moves {m1} vs {m2}"
        assert np.array_equal(e.communities(), o.communities()), f"sweep {s}"
        q = o.modularity()
        assert e.calculate_modularity() == q, f"sweep {s}"
        if m1 == 0 or q - q_before < GAIN:
            break
        q_before = q
    assert s >= 3
    e.close()
    o.close()


def test_rmat20_levels_and_aggregation_match_oracle(lvb, orc, rmat20):
    g = rmat20
    e = lvb.Louvain(g)
    o = orc.Oracle(g.rowptr, g.col, g.w)
    for level in range(12):
        c1 = e.optimise_modularity(GAIN)
        c2, _ = o.optimise_modularity(GAIN)
        assert c1 == c2, f"level {level}"
        assert np.array_equal(e.communities(), o.communities()), f"level {level}"
        assert np.array_equal(e.original_to_community()[0], o.original_to_community()), f"level {level}"
        if not c1:
            break
        e.aggregate_communities()
        o.aggregate_communities()
        V1, E1, _ = e.level_info()
        assert (V1, E1) == (o.V, o.E), f"level {level}"
        a, b = _canon(*e.csr()), _canon(*o.csr())
        for x, y in zip(a, b):
            assert np.array_equal(x, y), f"level {level} aggregated CSR"
    assert level >= 2
    assert e.calculate_modularity() == o.modularity()
    e.close()
    o.close()


def test_rmat20_full_run_matches_oracle(lvb, orc, rmat20):
    g = rmat20
    with lvb.Louvain(g) as e:
        q1 = e.run(GAIN)
        o2c, nc = e.original_to_community()
        st = e.stats()
    o = orc.Oracle(g.rowptr, g.col, g.w)
    q2, info = o.run(GAIN)
    assert q1 == q2
    assert nc == o.V
    assert np.array_equal(o2c, o.original_to_community())
    assert (st["levels"], st["sweeps"], st["edge_sweeps"]) == (info["levels"], info["sweeps"],
                                                               info["edge_sweeps"])
    # the map's modularity recomputed in FP64 from the float weights
    assert abs(orc.modularity_f64(g.rowptr, g.col, g.w, o2c) - q1) < 1e-9
    o.close()


def test_rmat20_device_resident_and_graph_loop_match_host_loop(lvb, rmat20):
    """The device-generated copy of the graph, run on the default path (sweep
    loops as CUDA graphs), equals the host-loop run on host input."""
    g = rmat20
    with lvb.Louvain(g, sweep_graph=False) as e:
        q_host = e.run(GAIN)
        m_host = e.original_to_community()[0]
    dg = lvb.gen_rmat_device(20, 16, 1)
    try:
        with lvb.Louvain(device_csr=(dg.rowptr, dg.col, dg.w, dg.V, dg.E)) as e:
            q_dev = e.run(GAIN)
            m_dev = e.original_to_community()[0]
    finally:
        dg.free()
    assert q_dev == q_host
    assert np.array_equal(m_dev, m_host)


def test_rmat20_weight_widths_agree(lvb, rmat20):
    """Aggregated levels read as 32-bit values (the default when every merged
    sum fits) and as uint64 sums give identical runs."""
    g = rmat20
    out = []
    for wide in (False, True):
        with lvb.Louvain(g, wide_weights=wide) as e:
            q = e.run(GAIN)
            out.append((q, e.original_to_community()[0], e.stats()["sweeps"]))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
