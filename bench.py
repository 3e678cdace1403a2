#!/usr/bin/env python
"""Louvain benchmark: R-MAT scale 24 (plain method) on one B200 per rank.

One step = one complete Louvain run (all levels, gain threshold 1e-6) from
singleton communities on the seeded R-MAT-24 graph (a=.57 b=.19 c=.19,
edge factor 16, float32 weights uniform in [0.5, 1.5)).

  value : edge-sweeps/s with the graph resident in HBM (lv_create_device once,
          lv_reset + lv_run per step, default options: each level's sweep loop
          runs as one CUDA graph), timed with CUDA events between barriers,
          max over ranks; whole-job value = sum of all ranks' edge-sweeps.
  e2e   : the same metric through the public C ABI with host buffers: each
          step creates the engine from pinned host CSR (host->device copies
          inside lv_create), runs, and reads the original->community map back;
          every step's create / run / map / destroy times are listed.
  roofline: the dominant kernel class (most device time), its algorithmic
          bytes (12 per CSR entry: column, weight and community gather; 20 per
          vertex) over its event-timed duration, against the measured HBM copy
          bandwidth; taken from one extra untimed run with per-class CUDA
          events.  traffic: DRAM bytes per launch of that class measured with
          ncu on this graph (profiles/ncu_traffic.json).
  cpu_baseline + parity: the CPU oracle (OpenMP, the same exact rule) on the
          box's host cores runs the first level-0 sweep and then one complete
          Louvain run of the same graph; its first-sweep community vector,
          final map, modularity bits, levels, sweeps and edge-sweeps are
          compared with the GPU's, and the complete run's edge-sweeps/s is the
          baseline.

--impl reference: the reference has no CPU implementation of the path, so
the reference arm times the CPU restatement of its rule (the oracle, all host
threads) on the same graph, built by the oracle's own generator (the product
library is not loaded).  One step is one level of a Louvain run (the level's
sweeps until the gain threshold, then the aggregation); consecutive steps
continue the run, and a finished run starts again from singletons, so every
4 steps cover one complete run of R-MAT-24 (4 levels).

Multi-GPU: the path does not shard (one graph per GPU); --gpus N runs N
independent replicas under torchrun (weak scaling, no collective on the
data path; the only collectives are the timing barrier and max/sum).

Other workloads (not the default line):
  --workload batch : 4096 seeded planted-partition graphs (V log-uniform in
          [100, 50000], 4-256 blocks, intra degree 8-24, inter 1-4) run by
          lv_batch_run in one persistent launch; value = graphs/s, with
          per-graph latency p50/p99, edge-sweeps/s, the single-graph engine
          run graph by graph on a sample (sequential launches) and the CPU
          oracle on the same sample.  Under torchrun the graphs are sharded
          over the ranks by entry count.
  --workload lfr   : held-out LFR-like graphs (4M vertices, mu 0.2/0.35/0.5):
          the learned active-set mode against plain sweeps; value = plain
          time / learned time, with the modularity difference per graph.
  --profile-only   : one profiled run of the R-MAT graph (per-class CUDA
          events, host loop per sweep) and its class split; for ncu launch
          lists of exactly one run.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "Louvain wall-time + edge-sweeps/s at RMAT-24; learned vs plain at ΔQ≤1e-3"
UNIT = "edge-sweeps/s"
SEED = 1
EDGE_FACTOR = 16
MIN_GAIN = 1e-6
FALLBACK_HBM_GBS = 6650.0
# move-phase profile slots: the update buckets (degree ranges) 0..6
CLASS_NAMES = ["b0_deg4", "b1_deg8", "b2_deg16", "b3_deg32", "b4_deg84", "b5_deg319",
               "b6_deg8192", "b6_giants", "unused8"]


def load_pkg():
    import importlib.util
    if "gpu_louvain_b200" in sys.modules:
        return sys.modules["gpu_louvain_b200"]
    d = os.path.join(ROOT, "gpu-louvain_b200")
    spec = importlib.util.spec_from_file_location("gpu_louvain_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gpu_louvain_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# rank plumbing (torch.distributed; gloo on CPU for tests, nccl on GPUs)
# ---------------------------------------------------------------------------
class Ranks:
    def __init__(self, backend=None):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group(backend or "nccl", timeout=datetime.timedelta(seconds=600))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def reduce(self, x: float, op: str) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


def combine(ranks: Ranks, local_units: float, local_seconds: float):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    units = ranks.reduce(local_units, "sum")
    secs = ranks.reduce(local_seconds, "max")
    return units, secs, (units / secs if secs > 0 else 0.0)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_index_for(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(workload: str, cls_name: str):
    """DRAM bytes per launch of a kernel class on a workload, from the
    committed ncu summary (None when that pair was not captured)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d[workload][cls_name]
    except Exception:
        return None


def ncu_class_split(csv_path: str) -> dict:
    """Per-class device time and DRAM bytes of one --profile-only run, from
    an ncu CSV of its launches (``--metrics gpu__time_duration.sum,
    dram__bytes_read.sum,dram__bytes_write.sum --csv``, every launch).

    Launches are attributed the way the engine issues a sweep: each degree
    bucket's move kernels, then its correction kernels, then commit_kernel;
    a bucket is named by its move kernel (move_group_*<G,...>: G = 4/8/16/32
    -> buckets 0-3) or, for the warp buckets, by its correction kernel
    (corr_group_kernel<32> -> bucket 4, corr_cta_kernel<128> -> bucket 5,
    corr_cta_kernel<256|512> -> bucket 6).  In bucket 6 the giant kernels
    (giant_stage_*, giant_merge_* and the large queue after them) form the
    b6_giants class, as the engine's class events bracket them."""
    import csv
    import re
    with open(csv_path) as f:
        rows = list(csv.reader(f))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r and "Metric Name" in r)
    hdr = rows[hi]
    c_id, c_name = hdr.index("ID"), hdr.index("Kernel Name")
    c_metric, c_value = hdr.index("Metric Name"), hdr.index("Metric Value")
    c_unit = hdr.index("Metric Unit") if "Metric Unit" in hdr else None
    scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "nsecond": 1e-9, "usecond": 1e-6,
             "msecond": 1e-3, "second": 1.0, "ns": 1e-9, "us": 1e-6, "ms": 1e-3}
    launches = {}
    order = []
    for r in rows[hi + 1:]:
        if len(r) <= max(c_id, c_name, c_metric, c_value):
            continue
        lid = int(r[c_id])
        if lid not in launches:
            launches[lid] = {"name": r[c_name], "s": 0.0, "bytes": 0.0}
            order.append(lid)
        v = float(r[c_value].replace(",", ""))
        u = r[c_unit] if c_unit is not None else ""
        v *= scale.get(u, 1.0)
        m = r[c_metric]
        if m.startswith("gpu__time_duration"):
            launches[lid]["s"] += v
        elif m.startswith("dram__bytes"):
            launches[lid]["bytes"] += v

    def short(n):
        # names as ncu prints them by default or with --kernel-name-base
        # demangled (template arguments then carry casts such as "(int)4")
        n = re.sub(r"\((int|bool|unsigned int)\)", "", n)
        n = re.sub(r"\(.*", "", n)
        return n.replace("void ", "").replace("lv::<unnamed>::", "").replace("<unnamed>::", "").strip()

    out = {c: {"class_launches": 0, "kernel_launches": 0, "ms": 0.0, "dram_bytes": 0.0}
           for c in CLASS_NAMES[:8]}
    seg = []

    def close(seg):
        names = [short(launches[i]["name"]) for i in seg]
        moves = [i for i, n in zip(seg, names) if not n.startswith(("corr_", "commit_kernel"))]
        corr = [n for n in names if n.startswith("corr_")]
        grp = [re.match(r"move_group\w*<(\d+),", n) for n in names]
        grp = [int(m.group(1)) for m in grp if m]
        if grp:
            b = {4: 0, 8: 1, 16: 2, 32: 3}.get(grp[0])
        elif any(n.startswith("corr_group_kernel<32") for n in corr):
            b = 4
        elif any(n.startswith("corr_cta_kernel<128") for n in corr):
            b = 5
        elif corr:
            b = 6
        else:
            return
        if b is None:
            return
        parts = {CLASS_NAMES[b]: []}
        if b == 6:
            parts["b6_giants"] = []
            cur = CLASS_NAMES[6]
            for i in moves:
                if short(launches[i]["name"]).startswith("giant_stage"):
                    cur = "b6_giants"
                parts[cur].append(i)
        else:
            parts[CLASS_NAMES[b]] = moves
        for c, ids in parts.items():
            if not ids:
                continue
            o = out[c]
            o["class_launches"] += 1
            o["kernel_launches"] += len(ids)
            o["ms"] += 1e3 * sum(launches[i]["s"] for i in ids)
            o["dram_bytes"] += sum(launches[i]["bytes"] for i in ids)

    in_sweep = False
    for lid in order:
        n = short(launches[lid]["name"])
        if n.startswith(("move_", "giant_", "corr_")):
            in_sweep = True
        if in_sweep:
            seg.append(lid)
        if n.startswith("commit_kernel"):
            close(seg)
            seg, in_sweep = [], False
    for c, o in out.items():
        k = max(o["class_launches"], 1)
        o["dram_bytes_per_launch"] = o["dram_bytes"] / k
        o["ms_per_launch"] = o["ms"] / k
        o["ms"] = round(o["ms"], 3)
    return {"csv": os.path.basename(csv_path), "launches": len(order),
            "total_ms": round(1e3 * sum(l["s"] for l in launches.values()), 3),
            "total_dram_bytes": sum(l["bytes"] for l in launches.values()), "classes": out}


def rmat_config(scale: int, V: int, E: int, world: int) -> dict:
    """The workload description shared by both arms (identical dicts)."""
    return {"workload": f"rmat{scale}_plain", "scale": scale, "edge_factor": EDGE_FACTOR,
            "a_b_c": [0.57, 0.19, 0.19], "seed": SEED, "V": V, "E_csr": E,
            "weights": "fp32 uniform [0.5,1.5) (exact on the 2^-24 grid)",
            "min_gain": MIN_GAIN, "parallelism": f"replicas{world}",
            "l2": "inputs %s than L2 (CSR %.2f GB vs 126 MB L2)" % (
                "larger" if 8 * E + 4 * V > 126e6 else "smaller", (8 * E + 4 * V) / 1e9)}


# ---------------------------------------------------------------------------
# CPU baseline and full-scale parity (the oracle, OpenMP)
# ---------------------------------------------------------------------------
def cpu_check(rowptr, col, w, gpu: dict):
    """The oracle on the host cores: the first level-0 sweep (its community
    vector against the GPU's), then one complete Louvain run from singletons
    (map, modularity bits, levels, sweeps, edge-sweeps against the GPU's run;
    its edge-sweeps/s is the CPU baseline)."""
    import numpy as np
    orc = load_oracle()
    nt = host_threads()
    o = orc.Oracle(rowptr, col, w, nt)
    t0 = time.perf_counter()
    m1 = o.sweep()
    t_sweep = time.perf_counter() - t0
    c1 = o.communities()
    o.close()
    o = orc.Oracle(rowptr, col, w, nt)
    t0 = time.perf_counter()
    q, st = o.run(MIN_GAIN)
    t_run = time.perf_counter() - t0
    o2c = o.original_to_community()
    nc = o.V
    o.close()
    parity = {
        "first_sweep": {"moves_gpu": gpu["first_sweep_moves"], "moves_cpu": int(m1),
                        "communities_equal": bool(np.array_equal(c1, gpu["first_sweep_communities"]))},
        "full_run": {"map_equal": bool(np.array_equal(o2c, gpu["map"])),
                     "modularity_gpu": gpu["modularity"], "modularity_cpu": q,
                     "modularity_bits_equal": q == gpu["modularity"],
                     "communities": [gpu["communities"], int(nc)],
                     "levels": [gpu["levels"], st["levels"]], "sweeps": [gpu["sweeps"], st["sweeps"]],
                     "edge_sweeps": [gpu["edge_sweeps"], st["edge_sweeps"]]},
    }
    fr = parity["full_run"]
    parity["ok"] = bool(parity["first_sweep"]["communities_equal"] and fr["map_equal"]
                        and fr["modularity_bits_equal"] and all(a == b for a, b in
                        (fr["communities"], fr["levels"], fr["sweeps"], fr["edge_sweeps"])))
    cpu = {"value": st["edge_sweeps"] / t_run, "unit": UNIT, "cores": nt, "kind": "port",
           "sample": f"one complete Louvain run of the same graph by the oracle (OpenMP, exact rule): "
                     f"{st['levels']} levels, {st['sweeps']} sweeps, {st['edge_sweeps']} edge-sweeps in "
                     f"{t_run:.2f} s (first level-0 sweep alone {t_sweep:.2f} s)",
           "run_s": t_run}
    return cpu, parity


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def class_table_of(cs):
    return {CLASS_NAMES[c]: {"launches": cs["launches"][c], "ms": round(cs["ms"][c], 3),
                             "GB/s": round(cs["bytes"][c] / (cs["ms"][c] * 1e-3) / 1e9, 1)
                             if cs["ms"][c] > 0 else None}
            for c in range(len(CLASS_NAMES))}


def profiled_run(lvb, dg, dev, wide_weights=False, knobs=None):
    """One untimed run with per-class CUDA events (host loop per sweep)."""
    prof = lvb.Louvain(device_csr=(dg.rowptr, dg.col, dg.w, dg.V, dg.E), device=dev, profile=True,
                       wide_weights=wide_weights, **(knobs or {}))
    prof.run(MIN_GAIN)
    cs = prof.class_stats()
    pst = prof.stats()
    o2c = prof.original_to_community()[0]
    prof.close()
    return cs, pst, o2c


def run_profile_only(args, ranks: Ranks):
    import torch
    lvb = load_pkg()
    dev = ranks.local
    torch.cuda.set_device(dev)
    dg = lvb.gen_rmat_device(args.scale, EDGE_FACTOR, SEED, device=dev)
    knobs = {k: v for k, v in (("giant_degree", args.giant_degree), ("warp_limit", args.warp_limit)) if v}
    cs, pst, _ = profiled_run(lvb, dg, dev, args.wide_weights, knobs)
    dg.free()
    return {"profile_only": True, "wide_weights": args.wide_weights, "knobs": knobs,
            "config": rmat_config(args.scale, dg.V, dg.E, ranks.world),
            "phases_ms": {k: round(pst[k], 3) for k in ("move_ms", "modularity_ms", "aggregate_ms", "setup_ms")},
            "classes": class_table_of(cs), "sweeps": pst["sweeps"], "levels": pst["levels"]}


def run_ours(args, ranks: Ranks):
    import numpy as np
    import torch
    lvb = load_pkg()
    dev = ranks.local
    torch.cuda.set_device(dev)
    scale = args.scale
    dg = lvb.gen_rmat_device(scale, EDGE_FACTOR, SEED, device=dev)
    V, E = dg.V, dg.E
    # --- autotuning of the work-mapping knobs (untimed; results identical) ---
    tuning, knobs = None, {}
    if not args.no_tune:
        t0 = time.perf_counter()
        tuning = lvb.tune(device_csr=(dg.rowptr, dg.col, dg.w, V, E), device=dev, min_gain=MIN_GAIN,
                          cache=os.path.join(ROOT, "_build", "tune_cache.json") if args.tune_cache else None)
        tuning["tuning_s"] = round(time.perf_counter() - t0, 1)
        knobs = {"giant_degree": tuning["giant_degree"], "warp_limit": tuning["warp_limit"]}
    # --- value: resident inputs ---
    # timed runs use the default path (each level's sweep loop as one CUDA
    # graph); the per-class split comes from a separate profiled run below
    eng = lvb.Louvain(device_csr=(dg.rowptr, dg.col, dg.w, V, E), device=dev, trace=args.trace, **knobs)
    for _ in range(args.warmup):
        eng.reset()
        eng.run(MIN_GAIN)
    eng.reset()
    eng.clear_stats()
    sampler = ClockSampler(gpu_index_for(dev))
    ranks.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    qs = []
    for k in range(args.steps):
        if k:
            eng.reset()
        qs.append(eng.run(MIN_GAIN))
    ev1.record()
    torch.cuda.synchronize()
    ranks.barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    st = eng.stats()
    o2c, ncomm = eng.original_to_community()
    units, secs, value = combine(ranks, float(st["edge_sweeps"]), ms / 1e3)
    eng.close()
    # the first level-0 sweep's community vector (checked against the oracle)
    e1 = lvb.Louvain(device_csr=(dg.rowptr, dg.col, dg.w, V, E), device=dev, **knobs)
    first_moves = e1.sweep()
    first_comm = e1.communities()
    e1.close()
    # one untimed profiled run (per-class CUDA events, one host round trip per
    # sweep) for the roofline and the class / phase split
    cs, pst, o2c_prof = profiled_run(lvb, dg, dev, knobs=knobs)
    assert np.array_equal(o2c_prof, o2c), "profiled run differs"
    # roofline of the dominant kernel class
    dom = max(range(len(CLASS_NAMES)), key=lambda c: cs["ms"][c])
    peak, peak_kind = measured_peak()
    achieved = cs["bytes"][dom] / (cs["ms"][dom] * 1e-3) / 1e9 if cs["ms"][dom] > 0 else 0.0
    per_launch_bytes = cs["bytes"][dom] / max(cs["launches"][dom], 1)
    per_launch_stored = cs["stored_bytes"][dom] / max(cs["launches"][dom], 1)
    sweep_gbs = pst["move_bytes"] / (pst["move_ms"] * 1e-3) / 1e9 if pst["move_ms"] > 0 else 0.0
    # --- e2e: host buffers through the C ABI ---
    def dev_tensor(ptr, n, dtype):
        class W:
            __cuda_array_interface__ = {"shape": (n,), "typestr": dtype, "data": (ptr, False), "version": 3}
        return torch.as_tensor(W(), device=f"cuda:{dev}")
    h_rp = torch.empty(V + 1, dtype=torch.int32, pin_memory=True)
    h_cl = torch.empty(E, dtype=torch.int32, pin_memory=True)
    h_w = torch.empty(E, dtype=torch.float32, pin_memory=True)
    h_rp.copy_(dev_tensor(dg.rowptr, V + 1, "<i4"))
    h_cl.copy_(dev_tensor(dg.col, E, "<i4"))
    h_w.copy_(dev_tensor(dg.w, E, "<f4"))
    torch.cuda.synchronize()
    dg.free()
    host_graph = lvb.Graph(h_rp.numpy(), h_cl.numpy(), h_w.numpy())
    out_map = torch.empty(V, dtype=torch.int32, pin_memory=True).numpy()
    e2e_steps = max(1, args.steps)
    step_parts = []

    def e2e_step():
        t_a = time.perf_counter()
        with lvb.Louvain(host_graph, device=dev, **knobs) as e:
            t_b = time.perf_counter()
            e.run(MIN_GAIN)
            t_c = time.perf_counter()
            e.original_to_community(out=out_map)
            units = e.stats()["edge_sweeps"]
            t_d = time.perf_counter()
        t_e = time.perf_counter()
        step_parts.append({"create": t_b - t_a, "run": t_c - t_b, "map": t_d - t_c, "close": t_e - t_d,
                           "step": t_e - t_a})
        return units

    # hand back what the resident runs left in the library's memory pool, so
    # that the warm-up step maps exactly the blocks the timed steps reuse
    lvb.lib().lv_trim_device_memory(dev)
    for _ in range(2):   # warm-up (allocator, module load, the first handle's buffers)
        e2e_step()
    step_parts.clear()
    ranks.barrier()
    torch.cuda.synchronize()
    # the interpreter's cyclic garbage collector stays out of the timed steps
    # (disabled, not run first: a full collection here leaves the GPU idle
    # long enough for its clocks to drop before the first timed step)
    import gc
    gc.disable()
    t0 = time.perf_counter()
    e2e_units = 0
    for _ in range(e2e_steps):
        e2e_units += e2e_step()
    torch.cuda.synchronize()
    gc.enable()
    t_e2e = time.perf_counter() - t0
    ranks.barrier()
    _, _, e2e_value = combine(ranks, float(e2e_units), t_e2e)
    assert np.array_equal(out_map, o2c), "e2e partition differs from the resident run"
    step_ms = [round(1e3 * p["step"], 1) for p in step_parts]
    # --- CPU baseline and full-scale parity on rank 0 at N=1 ---
    cpu = parity = None
    levels_run = st["levels"] // args.steps
    sweeps_run = st["sweeps"] // args.steps
    es_run = st["edge_sweeps"] // args.steps
    if ranks.world == 1 and ranks.rank == 0 and not args.no_cpu_baseline:
        cpu, parity = cpu_check(host_graph.rowptr, host_graph.col, host_graph.w, {
            "first_sweep_moves": int(first_moves), "first_sweep_communities": first_comm, "map": o2c,
            "modularity": qs[-1], "communities": int(ncomm), "levels": levels_run, "sweeps": sweeps_run,
            "edge_sweeps": es_run})
    ms_per_step = secs * 1e3 / args.steps
    # the class sizes depend on giant_degree: the traffic of a tuned setting
    # is looked up under its own key
    gd = int(knobs.get("giant_degree", 8192) or 8192)
    traffic = ncu_traffic(f"rmat{scale}" if gd == 8192 else f"rmat{scale}_g{gd}", CLASS_NAMES[dom])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded R-MAT generated on device)",
        "config": rmat_config(scale, V, E, ranks.world),
        "wall_time_s": ms_per_step / 1e3,
        "modularity": qs[-1], "communities": ncomm, "levels": levels_run,
        "sweeps": sweeps_run, "edge_sweeps_per_run": es_run,
        "phases_ms_per_run": {k: round(st[k] / args.steps, 3)
                              for k in ("move_ms", "modularity_ms", "aggregate_ms", "setup_ms")},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 4 * (V + 1) + 8 * E,
                "d2h_bytes_per_step": 4 * V, "seconds_per_step": t_e2e / e2e_steps,
                "ms_per_step_parts": {k: round(1e3 * statistics.mean(p[k] for p in step_parts), 1)
                                      for k in ("create", "run", "map", "close")},
                "step_ms": step_ms,
                "step_parts_ms": [{k: round(1e3 * p[k], 1) for k in ("create", "run", "map", "close")}
                                  for p in step_parts],
                "value_median_step": (e2e_units / e2e_steps) / (statistics.median(step_ms) / 1e3)
                if step_ms else None},
        "gpu_launches": st["kernel_launches"],
        "roofline": {"bound": "hbm", "kernel": CLASS_NAMES[dom], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "bytes_per_launch": per_launch_bytes,
                     "bytes_rule": "12 per CSR entry + 20 per vertex of the class, per launch",
                     "stored_bytes_per_launch": per_launch_stored,
                     "traffic": traffic["dram_bytes_per_launch"] if traffic else None,
                     "traffic_source": traffic["source"] if traffic else None,
                     "sweep_achieved": sweep_gbs, "sweep_frac": sweep_gbs / peak},
        "profiled_run": {"note": "one untimed run with per-class CUDA events (host loop per sweep); "
                                 "classes, phases and roofline come from it",
                         "phases_ms": {k: round(pst[k], 3)
                                       for k in ("move_ms", "modularity_ms", "aggregate_ms", "setup_ms")}},
        "classes": class_table_of(cs),
        "clocks": clocks,
        "cpu_baseline": cpu,
        "parity": parity,
        "tuning": ({k: tuning[k] for k in ("giant_degree", "warp_limit", "ms", "default_ms", "cached",
                                           "tuning_s", "trials")} if tuning else None),
    }
    return line


# ---------------------------------------------------------------------------
# batched workload: thousands of independent planted-partition graphs
# ---------------------------------------------------------------------------
BATCH_SEED = 5
BATCH_UNIT = "graphs/s"


def batch_graph_params(i: int):
    """Seeded parameters of graph i of the batched workload: V log-uniform in
    [100, 50000], blocks uniform in [4, 256] (at most V), expected intra-block
    degree uniform in [8, 24] and inter-block degree in [1, 4]."""
    import numpy as np
    r = np.random.default_rng([BATCH_SEED, i])
    V = int(round(float(np.exp(r.uniform(np.log(100.0), np.log(50000.0))))))
    blocks = min(int(r.integers(4, 257)), V)
    return V, blocks, float(r.uniform(8.0, 24.0)), float(r.uniform(1.0, 4.0))


def batch_seed(i: int) -> int:
    return BATCH_SEED * 1000003 + i


def batch_graphs(lvb, indices):
    """Graph objects of the given batch indices (samples)."""
    out = []
    for i in indices:
        V, blocks, d_in, d_out = batch_graph_params(i)
        out.append(lvb.gen_planted(V, blocks, d_in, d_out, seed=batch_seed(i)))
    return out


def batch_csr(lvb, indices):
    """Block-diagonal CSR of the given batch indices, generated by all host
    threads: (rowptr, col, w, graph_ptr)."""
    params = []
    for i in indices:
        V, blocks, d_in, d_out = batch_graph_params(i)
        params.append((V, blocks, d_in, d_out, batch_seed(i)))
    return lvb.gen_planted_batch(params)


def batch_shard(lvb, n_graphs: int, ranks: Ranks):
    """This rank's graph indices: largest expected entry counts first, each to
    the least-loaded rank (lvb.assign_shards)."""
    est = [p[0] * (p[2] + p[3]) for p in map(batch_graph_params, range(n_graphs))]
    return lvb.assign_shards(est, ranks.world)[ranks.rank]


def run_batch(args, ranks: Ranks):
    import numpy as np
    import torch
    lvb = load_pkg()
    dev = ranks.local
    torch.cuda.set_device(dev)
    mine = batch_shard(lvb, args.batch_graphs, ranks)
    t_gen = time.perf_counter()
    rp, cl, w, gptr = batch_csr(lvb, mine)
    t_gen = time.perf_counter() - t_gen
    V, E, G = len(rp) - 1, len(cl), len(mine)
    h_rp = torch.from_numpy(rp).pin_memory().numpy()
    h_cl = torch.from_numpy(cl).pin_memory().numpy()
    h_w = torch.from_numpy(w).pin_memory().numpy()
    # --- value: resident batch, one lv_batch_run per step ---
    b = lvb.Batch(rowptr=h_rp, col=h_cl, w=h_w, graph_ptr=gptr, device=dev)
    for _ in range(args.warmup):
        b.run(MIN_GAIN)
    sampler = ClockSampler(gpu_index_for(dev))
    ranks.barrier()
    torch.cuda.synchronize()
    sampler.start()
    dev_ms, es_tot, vs_tot = 0.0, 0, 0
    for _ in range(args.steps):
        b.run(MIN_GAIN)
        st = b.stats()
        dev_ms += st["device_ms"]
        es_tot += st["edge_sweeps"]
        vs_tot += st["vertex_sweeps"]
    torch.cuda.synchronize()
    ranks.barrier()
    clocks = sampler.stop()
    res = b.results()
    gst = b.graph_stats()
    ctas = b.stats()["ctas"]
    b.close()
    assert (res["status"] == lvb.LV_OK).all()
    units, secs, value = combine(ranks, float(G * args.steps), dev_ms / 1e3)
    es_units, _, es_value = combine(ranks, float(es_tot), dev_ms / 1e3)
    lat = gst["latency_ms"]
    # roofline of the batch kernel: the sweep bytes 12 E + 20 V per sweep (the
    # kernel also runs a modularity pass per sweep and the aggregation)
    peak, peak_kind = measured_peak()
    sweep_bytes = 12.0 * es_tot + 20.0 * vs_tot
    achieved = sweep_bytes / (dev_ms * 1e-3) / 1e9 if dev_ms > 0 else 0.0
    # --- e2e: host buffers through the C ABI, create + run + results + destroy ---
    out_comm = torch.empty(V, dtype=torch.int32, pin_memory=True).numpy()

    def e2e_step():
        with lvb.Batch(rowptr=h_rp, col=h_cl, w=h_w, graph_ptr=gptr, device=dev) as bb:
            bb.run(MIN_GAIN)
            r = bb.results()
            out_comm[:] = r["communities"]

    e2e_step()
    ranks.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t_e2e = time.perf_counter() - t0
    ranks.barrier()
    _, _, e2e_value = combine(ranks, float(G * args.steps), t_e2e)
    assert np.array_equal(out_comm, res["communities"]), "e2e partition differs from the resident run"
    # --- sequential launches of the single-graph engine on a sample ---
    n_seq = min(args.batch_seq_sample, G)
    pick = sorted(set(int(x) for x in np.linspace(0, G - 1, n_seq))) if G else []
    parts = [gptr[i:i + 2] for i in range(G)]
    sample = dict(zip(pick, batch_graphs(lvb, [mine[i] for i in pick])))
    t0 = time.perf_counter()
    for i in pick:
        with lvb.Louvain(sample[i], device=dev) as e:
            q = e.run(MIN_GAIN)
            m, _ = e.original_to_community()
        assert q == res["modularity"][i] and np.array_equal(m, res["communities"][parts[i][0]:parts[i][1]])
    t_seq = time.perf_counter() - t0
    seq_lat = (t_seq / len(pick)) if pick else 0.0
    # --- CPU baseline: the oracle on the same sample, rank 0 at N=1 ---
    cpu = None
    if ranks.world == 1 and ranks.rank == 0 and not args.no_cpu_baseline:
        orc = load_oracle()
        nt = host_threads()
        t0 = time.perf_counter()
        for i in pick:
            o = orc.Oracle(sample[i].rowptr, sample[i].col, sample[i].w, nt)
            o.run(MIN_GAIN)
            o.close()
        dt = time.perf_counter() - t0
        cpu = {"value": len(pick) / dt, "unit": BATCH_UNIT, "cores": nt, "kind": "port",
               "sample": f"oracle (OpenMP, exact rule) full runs of {len(pick)} graphs spread over "
                         f"the batch, {dt:.2f} s"}
    return {
        "metric": "batched Louvain graphs/s (planted-partition batch)", "value": value,
        "unit": BATCH_UNIT, "n_gpus": ranks.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded planted-partition graphs generated on the host)",
        "config": {"workload": f"batch{args.batch_graphs}_planted", "graphs": args.batch_graphs,
                   "graphs_this_rank": G, "V_total": V, "E_csr_total": E,
                   "V": "log-uniform [100, 50000]", "blocks": "uniform [4, 256]",
                   "d_in": "uniform [8, 24]", "d_out": "uniform [1, 4]", "weights": "unit",
                   "min_gain": MIN_GAIN, "parallelism": f"shards{ranks.world}",
                   "l2": "inputs larger than L2 (CSR %.2f GB vs 126 MB L2)" % ((8 * E + 4 * V) / 1e9),
                   "ctas": ctas, "generation_s": round(t_gen, 1)},
        "edge_sweeps_per_s": es_value, "edge_sweeps_per_run": es_tot // max(args.steps, 1),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "note": "device time from a graph's start to its end "
                                                        "inside the persistent launch"},
        "sequential": {"graphs_per_s": (1.0 / seq_lat) if seq_lat else None, "sample": len(pick),
                       "mean_latency_ms": seq_lat * 1e3,
                       "note": "lv_create + lv_run + map per graph (host buffers), graphs spread "
                               "over the batch; results identical to the batch"},
        "e2e": {"value": e2e_value, "unit": BATCH_UNIT, "h2d_bytes_per_step": 4 * (V + 1) + 8 * E,
                "d2h_bytes_per_step": 4 * V + 16 * G, "seconds_per_step": t_e2e / args.steps},
        "gpu_launches": 1,
        "roofline": {"bound": "hbm", "kernel": "batch_kernel", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "bytes_per_launch": sweep_bytes / max(args.steps, 1), "traffic": None},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }


def batch_summary(args, ranks: Ranks):
    """Compact driver-visible summary of the batched workload (the 4096-graph
    batch in one persistent launch, device-timed, 1 warm-up + 2 timed runs)."""
    import numpy as np
    import torch
    lvb = load_pkg()
    dev = ranks.local
    torch.cuda.set_device(dev)
    t_gen = time.perf_counter()
    rp, cl, w, gptr = batch_csr(lvb, range(args.batch_graphs))
    t_gen = time.perf_counter() - t_gen
    G = args.batch_graphs
    with lvb.Batch(rowptr=rp, col=cl, w=w, graph_ptr=gptr, device=dev) as b:
        b.run(MIN_GAIN)
        dev_ms, es = 0.0, 0
        lat = []
        for _ in range(2):
            b.run(MIN_GAIN)
            st = b.stats()
            dev_ms += st["device_ms"]
            es += st["edge_sweeps"]
            lat.append(b.graph_stats()["latency_ms"])
        ok = bool((b.results()["status"] == lvb.LV_OK).all())
        gs = b.graph_stats()
    # the graphs that bound the launch: the slowest five with their sizes
    slow = np.argsort(-gs["latency_ms"])[:5]
    vcount = np.diff(gptr)
    ecount = np.diff(rp[gptr])
    slowest = [{"graph": int(i), "V": int(vcount[i]), "E_csr": int(ecount[i]), "levels": int(gs["levels"][i]),
                "sweeps": int(gs["sweeps"][i]), "ms": round(float(gs["latency_ms"][i]), 2)} for i in slow]
    lat = np.concatenate(lat)
    # the launch against its load: the summed per-graph latencies spread over
    # the CTAs (the launch time with perfect balancing) and the longest graph
    ctas = int(st.get("ctas", 0) or 0)
    busy = float(lat.sum()) / 2 / ctas if ctas else None
    return {"workload": f"batch{G}_planted", "graphs_per_s": 2 * G / (dev_ms * 1e-3),
            "ms_per_launch": dev_ms / 2, "edge_sweeps_per_s": es / (dev_ms * 1e-3),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "ctas": ctas, "balanced_ms_per_launch": busy,
            "all_ok": ok, "V_total": len(rp) - 1, "E_csr_total": len(cl), "generation_s": round(t_gen, 1),
            "slowest": slowest,
            "note": "lv_batch_run, one persistent launch per run, device time (1 warm-up + 2 timed runs); "
                    "bench.py --workload batch gives the full line"}


def learned_summary(args, ranks: Ranks):
    """Compact driver-visible summary of the learned active-set form against
    the plain method on the held-out 4M-vertex LFR-like graphs."""
    import copy
    a = copy.copy(args)
    a.steps, a.warmup = 2, 1
    line = run_lfr(a, ranks)
    return {"workload": line["config"]["workload"], "speedup": line["value"],
            "max_abs_dq": line["max_abs_dq"], "target": "speed-up >= 1.5 at |dQ| <= 1e-3",
            "per_graph": [{"mu": r["mu"], "plain_ms": round(r["plain_ms"], 2), "learned_ms": round(r["learned_ms"], 2),
                           "speedup": round(r["speedup"], 3), "dq": r["dq"],
                           "recall": r["learned"]["recall"], "fell_back": r["learned"]["fell_back"],
                           "sweeps": {"plain": r["plain"]["sweeps"], "learned": r["learned"]["sweeps"],
                                      "learned_full": r["learned"]["full_sweeps"],
                                      "learned_active": r["learned"]["active_sweeps"]},
                           "move_ms": {"plain": r["plain"]["device_ms_per_run"]["move_ms"],
                                       "learned": r["learned"]["device_ms_per_run"]["move_ms"]}}
                          for r in line["per_graph"]],
            "settings": {k: line["config"][k] for k in ("full_every", "active_start", "min_recall")},
            "note": "plain vs learned on the same handle options, best of 2 timed runs each; "
                    "bench.py --workload lfr gives the full line"}


def run_reference(args, ranks: Ranks):
    """The reference arm: CPU restatement of the reference's rule (the
    oracle, all host threads), rank 0 only.  One step = one level of a Louvain
    run of the same R-MAT graph (sweeps until the gain threshold, then the
    aggregation); steps continue the run and a finished run restarts from
    singletons, so the timed steps cover complete runs."""
    if ranks.rank != 0:
        return None
    orc = load_oracle()
    nt = host_threads()
    t_gen = time.perf_counter()
    rp, cl, w = orc.gen_rmat(args.scale, EDGE_FACTOR, SEED, nthreads=nt)
    t_gen = time.perf_counter() - t_gen
    V, E = len(rp) - 1, len(cl)
    state = {"o": None, "runs": 0, "levels": 0, "q": None}

    def step():
        if state["o"] is None:
            state["o"] = orc.Oracle(rp, cl, w, nt)
        o = state["o"]
        e_level = o.E
        changed, sw = o.optimise_modularity(MIN_GAIN)
        state["levels"] += 1
        if changed:
            o.aggregate_communities()
        else:
            state["q"] = o.modularity()
            o.close()
            state["o"] = None
            state["runs"] += 1
        return sw * e_level

    for _ in range(args.warmup):
        step()
    runs0, levels0 = state["runs"], state["levels"]
    units = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        units += step()
    dt = time.perf_counter() - t0
    value = units / dt
    sample = (f"levels {levels0 + 1}..{levels0 + args.steps} of consecutive complete Louvain runs of "
              f"R-MAT-{args.scale} (E={E}; each run: every level's sweeps then its aggregation, restarting "
              f"from singletons) by the CPU restatement of the reference rule, {nt} threads; "
              f"{state['runs'] - runs0} runs completed inside the timed steps; graph built by the oracle's "
              f"own generator in {t_gen:.1f} s")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded R-MAT generated on the host by the oracle)",
        "config": rmat_config(args.scale, V, E, ranks.world),
        "impl": "reference",
        "final_modularity": state["q"],
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# learned active set: held-out LFR-like graphs, learned vs plain sweeps
# ---------------------------------------------------------------------------
LFR_EVAL_SEED = 9001
LFR_EVAL_MU = (0.2, 0.35, 0.5)


def run_lfr(args, ranks: Ranks):
    import numpy as np
    import torch
    lvb = load_pkg()
    dev = ranks.local
    torch.cuda.set_device(dev)
    model, thr = lvb.load_active_model(args.active_model)
    import json as _json
    with open(args.active_model or os.path.join(ROOT, "gpu-louvain_b200", "active_set_lfr.json")) as f:
        meta = _json.load(f)
    K = int(meta.get("full_every", 4))
    start = float(meta.get("active_start", 0.0))
    min_recall = float(meta.get("min_recall", 0.0))
    lfr = meta["training"]["lfr"]
    per_mu = []
    t_plain = t_learned = 0.0
    sampler = ClockSampler(gpu_index_for(dev))
    for mu in LFR_EVAL_MU:
        g, _ = lvb.gen_lfr(args.lfr_vertices, mu, seed=LFR_EVAL_SEED + ranks.rank, **lfr)
        res = {}
        for mode in ("plain", "learned"):
            kw = ({"active_set": True, "active_full_every": K, "active_start": start,
                   "active_min_recall": min_recall} if mode == "learned" else {})
            with lvb.Louvain(g, device=dev, **kw) as e:
                if mode == "learned":
                    e.set_active_model(model, thr)
                for _ in range(args.warmup):
                    e.reset()
                    e.run(MIN_GAIN)
                e.clear_stats()
                ranks.barrier()
                if mu == LFR_EVAL_MU[0] and mode == "plain":
                    sampler.start()
                ts = []
                for _ in range(args.steps):
                    e.reset()
                    t0 = time.perf_counter()
                    q = e.run(MIN_GAIN)
                    ts.append(time.perf_counter() - t0)
                st = e.stats()
                a = e.active_stats()
                m, nc = e.original_to_community()
            # device time per run by phase (the engine's coarse CUDA-event
            # counters): in learned mode move_ms also holds the active sweeps
            per_run = {k: round(st[k] / args.steps, 3)
                       for k in ("move_ms", "modularity_ms", "aggregate_ms", "setup_ms")}
            res[mode] = {"s": min(ts), "q": q, "communities": int(nc),
                         "levels": st["levels"] // args.steps, "sweeps": st["sweeps"] // args.steps,
                         "device_ms_per_run": per_run,
                         "kernel_launches_per_run": st["kernel_launches"] // args.steps,
                         "active_sweeps": a["active_sweeps"] // args.steps if mode == "learned" else None,
                         "evaluated_per_run": a["evaluated"] // args.steps if mode == "learned" else None,
                         "full_sweeps": a["full_sweeps"] // args.steps if mode == "learned" else None,
                         "recall": a["last_recall"] if mode == "learned" else None,
                         "fell_back": a["fell_back"] if mode == "learned" else None}
        t_plain += res["plain"]["s"]
        t_learned += res["learned"]["s"]
        per_mu.append({"mu": mu, "V": g.V, "E_csr": g.E, "plain_ms": res["plain"]["s"] * 1e3,
                       "learned_ms": res["learned"]["s"] * 1e3,
                       "speedup": res["plain"]["s"] / res["learned"]["s"],
                       "q_plain": res["plain"]["q"], "q_learned": res["learned"]["q"],
                       "dq": res["learned"]["q"] - res["plain"]["q"],
                       "plain": res["plain"], "learned": res["learned"]})
    clocks = sampler.stop()
    _, secs, _ = combine(ranks, 1.0, t_learned)
    speed = t_plain / t_learned
    return {
        "metric": "learned active-set vs plain Louvain on held-out LFR-like graphs (speed-up at |dQ|<=1e-3)",
        "value": speed, "unit": "x (plain time / learned time)", "n_gpus": ranks.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_learned * 1e3 / len(LFR_EVAL_MU),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (bf16 predictor)",
        "data": "synthetic (seeded LFR-like graphs generated on the host; held-out seeds)",
        "config": {"workload": f"lfr{args.lfr_vertices}_learned_vs_plain", "vertices": args.lfr_vertices,
                   "mu": list(LFR_EVAL_MU), "seed": LFR_EVAL_SEED, "lfr": lfr, "min_gain": MIN_GAIN,
                   "full_every": K, "active_start": start, "min_recall": min_recall,
                   "logit_threshold": thr, "model": os.path.basename(
                       args.active_model or "active_set_lfr.json"), "parallelism": f"replicas{ranks.world}"},
        "max_abs_dq": max(abs(r["dq"]) for r in per_mu),
        "per_graph": per_mu,
        "e2e": None,
        "gpu_launches": None,
        "clocks": clocks,
        "cpu_baseline": None,
    }


def run_reference_batch(args, ranks: Ranks):
    """Reference arm of the batched workload: the CPU restatement of the rule
    (the oracle, all host threads), rank 0 only, one step = full runs of a
    bounded sample of graphs spread over the batch."""
    if ranks.rank != 0:
        return None
    import numpy as np
    lvb = load_pkg()
    orc = load_oracle()
    nt = host_threads()
    n = min(args.batch_seq_sample, args.batch_graphs)
    pick = sorted(set(int(x) for x in np.linspace(0, args.batch_graphs - 1, n)))
    graphs = batch_graphs(lvb, pick)

    def step():
        for g in graphs:
            o = orc.Oracle(g.rowptr, g.col, g.w, nt)
            o.run(MIN_GAIN)
            o.close()
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = len(graphs) * args.steps / dt
    sample = (f"full runs of {len(graphs)} graphs spread over the batch by the CPU restatement of the "
              f"reference rule, {nt} threads")
    return {
        "metric": "batched Louvain graphs/s (planted-partition batch)", "value": value,
        "unit": BATCH_UNIT, "n_gpus": ranks.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded planted-partition graphs)",
        "config": {"workload": f"batch{args.batch_graphs}_planted", "graphs": args.batch_graphs,
                   "min_gain": MIN_GAIN, "parallelism": "cpu"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": BATCH_UNIT, "cores": nt, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": BATCH_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--trace", action="store_true", help="per-level / per-sweep lines on stderr")
    ap.add_argument("--workload", default="rmat", choices=["rmat", "batch", "lfr"],
                    help="rmat: one R-MAT graph per GPU (default); batch: thousands of planted-"
                         "partition graphs per launch, sharded over the GPUs; lfr: learned "
                         "active-set vs plain sweeps on held-out LFR-like graphs")
    ap.add_argument("--lfr-vertices", type=int, default=4000000)
    ap.add_argument("--active-model", default=None, help="predictor JSON (default: the packaged one)")
    ap.add_argument("--batch-graphs", type=int, default=4096)
    ap.add_argument("--batch-seq-sample", type=int, default=64,
                    help="graphs run one by one through the single-graph engine for comparison")
    ap.add_argument("--profile-only", action="store_true",
                    help="one profiled run of the R-MAT graph and its class split (for ncu launch lists)")
    ap.add_argument("--no-tune", action="store_true",
                    help="default workload: run with the default work-mapping knobs (no autotuning)")
    ap.add_argument("--tune-cache", action="store_true",
                    help="keep the autotuner's choice in _build/tune_cache.json between runs")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the learned and batched summaries added to the line")
    ap.add_argument("--wide-weights", action="store_true",
                    help="with --profile-only: 64-bit table sums and weights at every level (lv_opts.wide_weights)")
    ap.add_argument("--giant-degree", type=int, default=0,
                    help="with --profile-only: lv_opts.giant_degree (0 = library default)")
    ap.add_argument("--warp-limit", type=int, default=0,
                    help="with --profile-only: lv_opts.warp_limit (0 = library default)")
    ap.add_argument("--ncu-classes", default=None, metavar="CSV",
                    help="no GPU work: split an ncu CSV of a --profile-only run (time and DRAM "
                         "bytes per launch) into the engine's kernel classes and print it")
    args = ap.parse_args()
    if args.ncu_classes:
        print(json.dumps(ncu_class_split(args.ncu_classes)))
        return
    if args.impl == "reference":
        ranks = Ranks(backend="gloo")
        line = run_reference_batch(args, ranks) if args.workload == "batch" else run_reference(args, ranks)
    else:
        ranks = Ranks()
        line = (run_batch(args, ranks) if args.workload == "batch"
                else run_lfr(args, ranks) if args.workload == "lfr"
                else run_profile_only(args, ranks) if args.profile_only else run_ours(args, ranks))
        if (args.workload == "rmat" and not args.profile_only and not args.no_extras and ranks.world == 1
                and line is not None):
            # the metric also names the learned form and the batched form:
            # compact summaries of both ride on the default line
            for key, fn in (("learned", learned_summary), ("batch", batch_summary)):
                try:
                    line[key] = fn(args, ranks)
                except Exception as ex:   # the headline line is printed regardless
                    line[key] = {"error": f"{type(ex).__name__}: {ex}"}
    if ranks.rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
