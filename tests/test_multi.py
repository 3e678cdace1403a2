"""Replica ranks of bench.py on CPU (gloo, world size 2): whole-job value is
all ranks' units over the slowest rank's time; the reference arm runs on
rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks(backend="gloo")
    units, secs, value = bench.combine(r, 100.0 * (rank + 1), 2.0 + rank)
    r.barrier()
    r.close()
    q.put((rank, units, secs, value))


def test_combine_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, units, secs, value in res:
        assert units == 300.0 and secs == 3.0 and value == pytest.approx(100.0)


def test_single_rank_combine():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks()
    assert bench.combine(r, 50.0, 2.0) == (50.0, 2.0, 25.0)


def _run_bench(args, env_extra=None, timeout=300):
    import json
    import subprocess
    env = dict(os.environ)
    env.update(env_extra or {})
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                       timeout=timeout, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    return [json.loads(ln) for ln in lines]


def test_reference_arm_line_on_cpu():
    """`bench.py --impl reference` needs no GPU: the oracle runs complete
    Louvain runs level by level on the host cores and prints one line with the
    reference-arm keys."""
    (line,) = _run_bench(["--impl", "reference", "--scale", "12", "--steps", "4", "--warmup", "3"])
    assert line["impl"] == "reference"
    assert line["unit"] == "edge-sweeps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 4 and line["warmup"] == 3
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"].startswith("rmat")


def _ref_rank(rank, world, port, q):
    import subprocess
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--scale", "10",
                        "--steps", "2", "--warmup", "3", "--gpus", str(world)], capture_output=True, text=True,
                       timeout=300, env=env, cwd=ROOT)
    q.put((rank, p.returncode, p.stdout))


def test_reference_arm_rank0_only():
    """Under two ranks only rank 0 runs and prints the reference line; the
    other rank exits 0 without output."""
    import json
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_ref_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(320)
    res = dict((r, (rc, out)) for r, rc, out in (q.get(timeout=10) for _ in range(2)))
    assert res[0][0] == 0 and res[1][0] == 0
    lines0 = [ln for ln in res[0][1].splitlines() if ln.startswith("{")]
    assert len(lines0) == 1 and json.loads(lines0[0])["impl"] == "reference"
    assert not [ln for ln in res[1][1].splitlines() if ln.startswith("{")]
