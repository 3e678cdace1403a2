"""CPU tests of the autotuner's search and cache (gpu-louvain_b200/autotune.py).

The timed runs and the graph key need a GPU; here they are replaced by a
table of run times per knob setting, so what is tested is the tuner's own
logic: the order of the search, the keep-only-if-faster rule, the check that
no knob changes the modularity, and the cache file."""
import importlib
import json
import os
import threading

import pytest


@pytest.fixture()
def at(lvb, monkeypatch):
    mod = importlib.import_module(lvb.__name__ + ".autotune")
    calls = []
    times = {}

    def fake_key(_lvb, graph=None, device_csr=None, device=0):
        return "FakeGPU|V=10|E=20|classes=" + str(graph)

    def fake_run(_lvb, graph, device_csr, device, min_gain, knobs):
        calls.append(dict(knobs))
        ms, q = times.get((knobs["giant_degree"], knobs["warp_limit"]), (100.0, 0.5))
        return ms, q

    monkeypatch.setattr(mod, "graph_key", fake_key)
    monkeypatch.setattr(mod, "_run_ms", fake_run)
    return mod, times, calls


def test_search_order_and_keep_rule(at):
    mod, times, calls = at
    # giant 16384 is 5 % faster (kept), 32768 only 1 % faster than that (not kept);
    # then warp limit 288 is 3 % faster at giant 16384 (kept)
    times[(16384, 352)] = (95.0, 0.5)
    times[(32768, 352)] = (94.2, 0.5)
    times[(16384, 288)] = (92.0, 0.5)
    out = mod.tune("g1", min_gain_frac=0.02)
    assert out["giant_degree"] == 16384 and out["warp_limit"] == 288
    assert out["ms"] == 92.0 and out["default_ms"] == 100.0 and out["cached"] is False
    # default first, then every other giant degree at the default warp limit,
    # then every other warp limit at the chosen giant degree
    assert calls[0] == mod.DEFAULT
    gd_pass = [c for c in calls[1:1 + len(mod.GIANT_DEGREES) - 1]]
    assert [c["giant_degree"] for c in gd_pass] == [g for g in mod.GIANT_DEGREES if g != 8192]
    assert all(c["warp_limit"] == 352 for c in gd_pass)
    wl_pass = calls[len(mod.GIANT_DEGREES):]
    assert [c["warp_limit"] for c in wl_pass] == [w for w in mod.WARP_LIMITS if w != 352]
    assert all(c["giant_degree"] == 16384 for c in wl_pass)
    assert len(out["trials"]) == len(calls)


def test_default_kept_without_a_clear_gain(at):
    mod, times, _ = at
    times[(4096, 352)] = (99.0, 0.5)   # 1 %: within the noise margin
    out = mod.tune("g2", min_gain_frac=0.02)
    assert (out["giant_degree"], out["warp_limit"]) == (8192, 352)


def test_knob_that_changes_the_result_is_an_error(at):
    mod, times, _ = at
    times[(2048, 352)] = (90.0, 0.5000001)
    with pytest.raises(RuntimeError, match="changed the result"):
        mod.tune("g3")


def test_cache_round_trip(at, tmp_path):
    mod, times, calls = at
    cache = str(tmp_path / "tune.json")
    times[(65536, 352)] = (80.0, 0.5)
    first = mod.tune("g4", cache=cache)
    n = len(calls)
    second = mod.tune("g4", cache=cache)
    assert len(calls) == n                       # answered from the cache
    assert second["cached"] is True
    assert {k: second[k] for k in ("giant_degree", "warp_limit", "ms")} == \
           {k: first[k] for k in ("giant_degree", "warp_limit", "ms")}
    other = mod.tune("g5", cache=cache)          # another graph: tuned and added
    assert other["cached"] is False
    with open(cache) as f:
        store = json.load(f)
    assert len(store) == 2
    assert os.listdir(tmp_path) == ["tune.json"]  # no temporary file left


def test_unreadable_cache_is_ignored(at, tmp_path):
    mod, _, calls = at
    cache = tmp_path / "tune.json"
    cache.write_text("{not json")
    out = mod.tune("g6", cache=str(cache))
    assert out["cached"] is False and calls
    assert json.loads(cache.read_text())[out["key"]]["giant_degree"] == out["giant_degree"]


def test_concurrent_cache_writers(at, tmp_path):
    """Writers that replace the cache at the same time (one process per GPU)
    each use their own temporary file: every write completes and the file is
    always one writer's whole store."""
    mod, _, _ = at
    cache = str(tmp_path / "tune.json")
    errors = []

    def writer(i):
        try:
            for j in range(50):
                mod._write_cache(cache, {f"rank{i}": j})
        except Exception as ex:   # pragma: no cover - reported below
            errors.append(ex)

    ts = [threading.Thread(target=writer, args=(i,)) for i in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors
    with open(cache) as f:
        store = json.load(f)
    assert len(store) == 1 and list(store.values())[0] == 49
    assert os.listdir(tmp_path) == ["tune.json"]
