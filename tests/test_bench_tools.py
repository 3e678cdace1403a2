"""CPU tests of bench.py's profiling helpers: the split of an ncu launch list
into the engine's kernel classes (`--ncu-classes`) and the lookup of the
committed per-class DRAM traffic."""
import csv
import importlib.util
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


HEADER = ["ID", "Process ID", "Process Name", "Host Name", "Kernel Name", "Context", "Stream", "Block Size",
          "Grid Size", "Device", "CC", "Section Name", "Metric Name", "Metric Unit", "Metric Value"]


def write_list(path, kernels):
    """kernels: [(demangled name, time in us, DRAM bytes)] in launch order."""
    with open(path, "w", newline="") as f:
        f.write("==PROF== Connected to process 1 (python)\n")
        w = csv.writer(f, quoting=csv.QUOTE_ALL)
        w.writerow(HEADER)
        for i, (name, us, nbytes) in enumerate(kernels):
            base = [str(i), "1", "python", "host", name, "1", "7", "(256, 1, 1)", "(148, 1, 1)", "0", "10.0",
                    "Command line profiler metrics"]
            w.writerow(base + ["dram__bytes_read.sum", "byte", str(nbytes // 2)])
            w.writerow(base + ["dram__bytes_write.sum", "byte", str(nbytes - nbytes // 2)])
            w.writerow(base + ["gpu__time_duration.sum", "usecond", f"{us:.3f}"])


def k(name):
    return f"void lv::<unnamed>::{name}(lv::GraphView<T1>, lv::StateView, const int *, int)"


def one_sweep():
    """One sweep as the engine issues it: each bucket's move kernels, its
    corrections, its commit; buckets 4-6 on the warp kernel; bucket 6 with
    its queues and the giants."""
    return [
        (k("move_group_narrow_kernel<(int)4, (int)8, float>"), 10.0, 1000),
        (k("corr_group_kernel<(int)4, float>"), 2.0, 100),
        (k("commit_kernel"), 1.0, 10),
        (k("move_group_narrow_kernel<(int)32, (int)64, float>"), 20.0, 2000),
        (k("corr_group_kernel<(int)32, float>"), 2.0, 100),
        (k("commit_kernel"), 1.0, 10),
        (k("move_warp_narrow_kernel<float>"), 30.0, 3000),
        (k("corr_group_kernel<(int)32, float>"), 2.0, 100),
        (k("commit_kernel"), 1.0, 10),
        (k("move_warp_narrow_kernel<float>"), 40.0, 4000),
        (k("corr_cta_kernel<(int)128, float>"), 2.0, 100),
        (k("commit_kernel"), 1.0, 10),
        (k("move_warp_narrow_kernel<float>"), 50.0, 5000),
        (k("move_fallback_kernel<float, (int)1024, (int)16384, (bool)1>"), 60.0, 6000),
        (k("move_rowq_narrow_kernel<float, (int)256, (int)2048>"), 70.0, 7000),
        (k("giant_stage_narrow_kernel<float>"), 80.0, 8000),
        (k("giant_regroup_kernel"), 5.0, 500),
        (k("giant_merge_kernel<(int)1024, (int)16384>"), 6.0, 600),
        (k("move_fallback_kernel<float, (int)1024, (int)16384, (bool)1>"), 90.0, 9000),
        (k("corr_cta_kernel<(int)256, float>"), 2.0, 100),
        (k("corr_cta_kernel<(int)512, float>"), 2.0, 100),
        (k("commit_kernel"), 1.0, 10),
        ("void <unnamed>::s2_kernel(const unsigned long long *, int, unsigned long long *)", 3.0, 300),
    ]


def test_ncu_class_split(tmp_path):
    b = load_bench()
    path = str(tmp_path / "launches.csv")
    setup = [("<unnamed>::rmat_draw_kernel(lvrng::RmatParams, long, unsigned long long *)", 100.0, 10 ** 6)]
    write_list(path, setup + one_sweep() + one_sweep())
    d = b.ncu_class_split(path)
    assert d["launches"] == 1 + 2 * len(one_sweep())
    c = d["classes"]
    # buckets 0 and 3 by their group width, 4 and 5 by their corrections
    assert c["b0_deg4"]["class_launches"] == 2 and c["b0_deg4"]["kernel_launches"] == 2
    assert c["b0_deg4"]["dram_bytes_per_launch"] == pytest.approx(1000)
    assert c["b3_deg32"]["dram_bytes_per_launch"] == pytest.approx(2000)
    assert c["b4_deg84"]["dram_bytes_per_launch"] == pytest.approx(3000)
    assert c["b5_deg319"]["dram_bytes_per_launch"] == pytest.approx(4000)
    assert c["b5_deg319"]["ms_per_launch"] == pytest.approx(0.040)
    # bucket 6: the warp kernel and its queues, then the giants from their
    # staging kernel on (corrections and commits belong to neither)
    assert c["b6_deg8192"]["kernel_launches"] == 2 * 3
    assert c["b6_deg8192"]["dram_bytes_per_launch"] == pytest.approx(5000 + 6000 + 7000)
    assert c["b6_giants"]["kernel_launches"] == 2 * 4
    assert c["b6_giants"]["dram_bytes_per_launch"] == pytest.approx(8000 + 500 + 600 + 9000)
    assert c["b1_deg8"]["class_launches"] == 0


def test_committed_traffic_is_keyed_by_threshold():
    """The committed traffic file holds the dominant class for the default
    giant threshold and for the one the tuner picks on some boxes."""
    b = load_bench()
    t = b.ncu_traffic("rmat24", "b6_deg8192")
    assert t and t["dram_bytes_per_launch"] > 0 and os.path.exists(os.path.join(ROOT, t["source"]))
    t16 = b.ncu_traffic("rmat24_g16384", "b6_deg8192")
    assert t16 and t16["dram_bytes_per_launch"] > t["dram_bytes_per_launch"]
    assert b.ncu_traffic("rmat24_g999", "b6_deg8192") is None
    with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
        d = json.load(f)
    for key in ("rmat24", "rmat24_g16384"):
        assert d[key]["b6_deg8192"]["class_launches"] == 34


class _FakeEngine:
    """Stands in for the Louvain handle: the counters run_lfr reads, with the
    learned mode taking fewer, cheaper sweeps."""

    def __init__(self, graph, device=0, **kw):
        self.learned = bool(kw.get("active_set"))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def set_active_model(self, model, thr):
        pass

    def reset(self):
        pass

    def clear_stats(self):
        pass

    def run(self, min_gain):
        return 0.5 if not self.learned else 0.4999

    def stats(self):
        f = 0.5 if self.learned else 1.0
        return {"levels": 2 * 2, "sweeps": 2 * (30 if self.learned else 20), "move_ms": 2 * 60.0 * f,
                "modularity_ms": 2.0, "aggregate_ms": 8.0, "setup_ms": 0.4, "kernel_launches": 1600}

    def active_stats(self):
        return {"evaluated": 2 * 1000, "full_sweeps": 2 * 10, "active_sweeps": 2 * 18, "last_recall": 0.97,
                "fell_back": False}

    def original_to_community(self):
        import numpy as np
        return np.zeros(4, np.int32), 1


class _FakePkg:
    Louvain = _FakeEngine

    @staticmethod
    def load_active_model(path=None):
        import numpy as np
        return np.zeros(113, np.uint16), -2.7

    @staticmethod
    def gen_lfr(V, mu, seed=0, **kw):
        class G:
            pass
        g = G()
        g.V, g.E = V, 20 * V
        return g, None


def test_learned_summary_schema(monkeypatch):
    """The default bench line's `learned` block (built from run_lfr's records)
    carries per graph the speed-up, modularity difference, recall, sweep
    counts and move-phase times."""
    import types
    import torch
    b = load_bench()
    monkeypatch.setattr(b, "load_pkg", lambda: _FakePkg)
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)

    class _Clock:
        def __init__(self, gpu):
            pass

        def start(self):
            pass

        def stop(self):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}

    monkeypatch.setattr(b, "ClockSampler", _Clock)
    args = types.SimpleNamespace(active_model=None, lfr_vertices=1000, steps=3, warmup=3)
    s = b.learned_summary(args, b.Ranks())
    assert s["target"] == "speed-up >= 1.5 at |dQ| <= 1e-3"
    assert len(s["per_graph"]) == 3
    for r in s["per_graph"]:
        assert r["speedup"] > 0 and abs(r["dq"]) < 1e-3
        assert r["sweeps"] == {"plain": 20, "learned": 30, "learned_full": 10, "learned_active": 18}
        assert r["move_ms"] == {"plain": 60.0, "learned": 30.0}
        assert r["recall"] == 0.97 and r["fell_back"] is False
    assert set(s["settings"]) == {"full_every", "active_start", "min_recall"}
