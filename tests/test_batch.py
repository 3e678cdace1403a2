"""Batches of independent graphs (lv_batch_*, Batch, run_batch_sharded).

GPU tests: every graph of a batch, run in one persistent launch, must give
exactly what the CPU oracle's level loop (orc_run) gives for that graph alone:
the same original->community map, the same FP64 modularity bits, and the same
level, sweep and edge-sweep counts.  The batch mixes planted-partition and
R-MAT graphs with the edge cases of the single-graph tests, a hub whose
evaluation needs a graph's global table, and a community whose merged row
needs it during aggregation.

CPU tests: the shard assignment and the sharded runner's gather over two gloo
ranks, with the oracle standing in for each rank's GPU run."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _edges_graph(lvb, gnp, V, edges):
    rp, cl, w = gnp.csr_from_edges(V, edges)
    return lvb.Graph(rp, cl, w)


def _star_pairs(lvb, gnp, leaves, pairs):
    """A star (hub 0 with `leaves` leaves) plus `pairs` disjoint weighted edges:
    the hub's row needs more than the CTA's shared table, and so does the
    star community's merged row after level 0 (its bound is 2 * leaves and
    more than 1024 communities survive)."""
    V = 1 + leaves + 2 * pairs
    edges = [(0, i, 1.0) for i in range(1, leaves + 1)]
    base = leaves + 1
    edges += [(base + 2 * i, base + 2 * i + 1, 3.0) for i in range(pairs)]
    return _edges_graph(lvb, gnp, V, edges)


def _mixed_batch(lvb, gnp):
    rng = np.random.default_rng(11)
    gs = []
    for i in range(24):
        V = int(np.exp(rng.uniform(np.log(100), np.log(4000))))
        gs.append(lvb.gen_planted(V, int(rng.integers(4, 65)), float(rng.uniform(8, 24)),
                                  float(rng.uniform(1, 4)), seed=100 + i,
                                  weights="uniform" if i % 3 == 0 else "unit"))
    for s in (7, 8, 9, 10, 11):
        gs.append(lvb.gen_rmat(s, seed=s))
    gs.append(_star_pairs(lvb, gnp, 1500, 1200))
    gs.append(_edges_graph(lvb, gnp, 40, [(i, j, 1.0) for i in range(40) for j in range(i)]))
    gs.append(_edges_graph(lvb, gnp, 4, []))                                    # no edges
    gs.append(lvb.Graph(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)))  # V = 0
    gs.append(_edges_graph(lvb, gnp, 2, [(0, 1, 1.0)]))
    gs.append(_edges_graph(lvb, gnp, 3, [(0, 0, 1.0), (1, 1, 2.0)]))         # self-loops only
    gs.append(_edges_graph(lvb, gnp, 4, [(0, 1, 0.0), (1, 2, 1.0), (2, 3, 1.0)]))  # zero weight
    gs.append(_edges_graph(lvb, gnp, 6, [(0, 1, 1.0), (1, 2, 1.0), (4, 4, 1.0)]))  # isolated
    gs.append(_edges_graph(lvb, gnp, 300, [(0, i, 1.0) for i in range(1, 300)]))  # star
    return gs


def _oracle_run(orc, g, min_gain, max_sweeps=0):
    o = orc.Oracle(g.rowptr, g.col, g.w, 1)
    q, info = o.run(min_gain, max_sweeps)
    res = dict(info, modularity=q, communities=o.original_to_community(), num_communities=o.V)
    o.close()
    return res


def _same_q(a, b):
    return a == b or (np.isnan(a) and np.isnan(b))


def _check_against_oracle(lvb, orc, graphs, min_gain, max_sweeps=0):
    with lvb.Batch(graphs, max_sweeps=max_sweeps) as b:
        b.run(min_gain)
        r = b.results()
        st = b.graph_stats()
        parts = b.split(r["communities"])
        assert (r["status"] == lvb.LV_OK).all()
        for i, g in enumerate(graphs):
            o = _oracle_run(orc, g, min_gain, max_sweeps)
            assert np.array_equal(parts[i], o["communities"]), i
            assert _same_q(r["modularity"][i], o["modularity"]), (i, r["modularity"][i], o["modularity"])
            assert r["num_communities"][i] == o["num_communities"], i
            assert st["levels"][i] == o["levels"], i
            assert st["sweeps"][i] == o["sweeps"], i
            assert st["edge_sweeps"][i] == o["edge_sweeps"], i
        return r


@pytest.mark.gpu
@pytest.mark.parametrize("min_gain", [1e-6, 0.01])
def test_batch_matches_oracle(lvb, orc, gnp, min_gain):
    _check_against_oracle(lvb, orc, _mixed_batch(lvb, gnp), min_gain)


def _upper_bound_batch(lvb):
    """Graphs at the batched workload's bounds: 50,000 vertices, 4 to 256
    blocks, expected intra-block degree 8 to 24 and inter-block degree 1 to
    4, unit weights (one grid-weight variant), plus the smallest graphs."""
    specs = [(50000, 256, 24.0, 4.0, "unit"), (50000, 4, 24.0, 4.0, "unit"), (50000, 256, 8.0, 1.0, "unit"),
             (50000, 128, 16.0, 4.0, "uniform"), (49999, 255, 23.5, 3.9, "unit"), (25000, 256, 24.0, 4.0, "unit"),
             (12000, 64, 20.0, 3.0, "unit"), (100, 4, 24.0, 4.0, "unit"), (100, 100, 8.0, 1.0, "unit"),
             (101, 4, 8.0, 1.0, "unit")]
    return [lvb.gen_planted(V, B, di, do, seed=900 + i, weights=wt) for i, (V, B, di, do, wt) in enumerate(specs)]


@pytest.mark.gpu
def test_batch_upper_bounds_match_oracle(lvb, orc):
    graphs = _upper_bound_batch(lvb)
    assert max(g.V for g in graphs) == 50000
    _check_against_oracle(lvb, orc, graphs, 1e-6)


@pytest.mark.gpu
def test_batch_max_sweeps_matches_oracle(lvb, orc, gnp):
    graphs = _mixed_batch(lvb, gnp)[:12]
    _check_against_oracle(lvb, orc, graphs, 1e-6, max_sweeps=1)


@pytest.mark.gpu
def test_batch_matches_engine_and_repeats(lvb, gnp):
    graphs = [lvb.gen_planted(5000, 32, 16.0, 2.0, seed=3), lvb.gen_rmat(12, seed=4),
              _star_pairs(lvb, gnp, 2500, 1500)]
    with lvb.Batch(graphs) as b:
        b.run(1e-6)
        r1 = b.results()
        b.run(1e-6)                      # each run starts afresh
        r2 = b.results()
        for k in r1:
            assert np.array_equal(r1[k], r2[k], equal_nan=(k == "modularity")), k
        parts = b.split(r1["communities"])
        assert b.stats()["edge_sweeps"] == int(b.graph_stats()["edge_sweeps"].sum())
    for i, g in enumerate(graphs):
        e = lvb.Louvain(g)
        q = e.run(1e-6)
        m, nc = e.original_to_community()
        e.close()
        assert q == r1["modularity"][i]
        assert nc == r1["num_communities"][i]
        assert np.array_equal(m, parts[i])


@pytest.mark.gpu
def test_batch_device_csr(lvb):
    import torch
    graphs = [lvb.gen_planted(3000, 16, 12.0, 2.0, seed=s) for s in range(4)]
    rp, cl, w, gptr = lvb.concat_graphs(graphs)
    with lvb.Batch(graphs) as b:
        b.run(1e-6)
        ref = b.results()
    d = [torch.from_numpy(x).cuda() for x in (rp, cl, w)]
    with lvb.Batch(graph_ptr=gptr, device_csr=tuple(t.data_ptr() for t in d),
                   num_vertices=len(rp) - 1, num_entries=len(cl)) as b:
        b.run(1e-6)
        got = b.results()
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_batch_per_graph_errors(lvb):
    good = lvb.gen_planted(1000, 8, 12.0, 2.0, seed=1)
    bad = lvb.gen_planted(500, 4, 12.0, 2.0, seed=2)
    rp, cl, w, gptr = lvb.concat_graphs([good, bad, good])
    cl = cl.copy()
    cl[int(rp[gptr[1]])] = 0            # a row of graph 1 reaches into graph 0
    with lvb.Batch(rowptr=rp, col=cl, w=w, graph_ptr=gptr) as b:
        assert b.run(1e-6, check=False) == lvb.LV_ERR_DEVICE
        r = b.results()
        assert list(r["status"]) == [lvb.LV_OK, lvb.LV_ERR_INVALID, lvb.LV_OK]
        parts = b.split(r["communities"])
        assert (parts[1] == -1).all()
        assert np.array_equal(parts[0], parts[2])
        assert r["modularity"][0] == r["modularity"][2]
    # whole-CSR errors fail the creation
    w2 = w.copy()
    w2[3] = -1.0
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.Batch(rowptr=rp, col=cl, w=w2, graph_ptr=gptr)
    assert ex.value.status == lvb.LV_ERR_WEIGHT
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.Batch(rowptr=rp, col=cl, w=w, graph_ptr=np.array([0, 5, 3, len(rp) - 1], np.int32))
    assert ex.value.status == lvb.LV_ERR_INVALID


# ---------------------------------------------------------------------------
# CPU: shard assignment and the sharded runner over two gloo ranks
# ---------------------------------------------------------------------------
def test_concat_graphs_roundtrip(lvb):
    graphs = [lvb.gen_planted(300 + 50 * i, 4, 8.0, 2.0, seed=i) for i in range(5)]
    rp, cl, w, gptr = lvb.concat_graphs(graphs)
    assert gptr[0] == 0 and gptr[-1] == len(rp) - 1 and rp[-1] == len(cl)
    for i, g in enumerate(graphs):
        v0, v1 = gptr[i], gptr[i + 1]
        e0, e1 = rp[v0], rp[v1]
        assert np.array_equal(rp[v0:v1 + 1] - e0, g.rowptr)
        assert np.array_equal(cl[e0:e1] - v0, g.col)
        assert np.array_equal(w[e0:e1], g.w)


def test_assign_shards(lvb):
    rng = np.random.default_rng(5)
    entries = rng.integers(0, 10000, 257)
    for world in (1, 2, 3, 8):
        sh = lvb.assign_shards(entries, world)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(entries)))
        loads = [int(entries[s].sum()) for s in map(np.array, sh)]
        # greedy largest-first: no rank exceeds another by more than the largest graph
        assert max(loads) - min(loads) <= int(entries.max())
    assert lvb.assign_shards([5, 5, 5], 2) == [[0, 2], [1]]


def _oracle_runner(graphs, min_gain, device, max_sweeps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    out = []
    for g in graphs:
        o = oracle.Oracle(g.rowptr, g.col, g.w, 1)
        q, info = o.run(min_gain, max_sweeps)
        out.append(dict(info, modularity=q, communities=o.original_to_community(),
                        num_communities=o.V, status=0, latency_ms=0.0))
        o.close()
    return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _shard_worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist
    from conftest import load_pkg
    lvb = load_pkg()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    graphs = [lvb.gen_planted(200 + 97 * i, 4 + i % 5, 10.0, 2.0, seed=i) for i in range(9)]
    res = lvb.run_batch_sharded(graphs, 1e-6, runner=_oracle_runner)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, [(r["modularity"], r["communities"].tolist(), r["levels"]) for r in res]))


def test_run_batch_sharded_two_ranks(lvb):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(180)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got[0] == got[1]
    graphs = [lvb.gen_planted(200 + 97 * i, 4 + i % 5, 10.0, 2.0, seed=i) for i in range(9)]
    ref = _oracle_runner(graphs, 1e-6, 0, 0)
    assert [(r["modularity"], r["communities"].tolist(), r["levels"]) for r in ref] == got[0]
