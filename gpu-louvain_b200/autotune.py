"""Autotuner for the engine's work-mapping knobs.

The update rule's seven degree buckets are part of the rule and never
change; what is tuned is how a bucket's vertices are mapped onto the GPU,
which never changes a result:

  giant_degree : vertices of degree above it are decided by the staged-chunk
                 path (many CTAs per vertex) instead of one warp each;
  warp_limit   : distinct neighbour communities after which a warp hands its
                 vertex to a fallback CTA (the warp's shared table holds
                 warp_limit + 128 claims).

The tuner times complete Louvain runs of the caller's graph on the caller's
GPU (device time of every phase, one warm-up and one timed run per setting),
first over giant_degree at the default warp_limit, then over warp_limit at
the best giant_degree, and keeps a setting only when it beats the incumbent
by more than `min_gain_frac`.  The choice is cached in a JSON file keyed by
the GPU and the graph's level-0 work classes (vertex and entry counts per
class), so a second call on the same graph and GPU costs nothing.
"""
from __future__ import annotations

import json
import os

GIANT_DEGREES = (2048, 4096, 8192, 16384, 32768, 65536)
WARP_LIMITS = (128, 224, 288, 352, 384)
DEFAULT = {"giant_degree": 8192, "warp_limit": 352}


def _pkg():
    import sys
    return sys.modules[__name__.rsplit(".", 1)[0]]


def graph_key(lvb, graph=None, device_csr=None, device: int = 0) -> str:
    """Cache key: GPU name plus the level-0 work classes of the graph."""
    kw = {"device_csr": device_csr} if device_csr is not None else {}
    with lvb.Louvain(graph, device=device, **kw) as e:
        v, n = e.level_classes()
    return "%s|V=%s|E=%s|classes=%s" % (lvb.device_name(device), int(sum(v)), int(sum(n)),
                                       ",".join("%d:%d" % (a, b) for a, b in zip(v.tolist(), n.tolist())))


def _run_ms(lvb, graph, device_csr, device, min_gain, knobs) -> tuple[float, float]:
    kw = {"device_csr": device_csr} if device_csr is not None else {}
    with lvb.Louvain(graph, device=device, **kw, **knobs) as e:
        e.run(min_gain)               # warm-up (module load, pool, tables)
        e.reset()
        e.clear_stats()
        q = e.run(min_gain)
        st = e.stats()
    return st["move_ms"] + st["modularity_ms"] + st["aggregate_ms"] + st["setup_ms"], q


def tune(graph=None, *, device_csr=None, device: int = 0, min_gain: float = 1e-6, cache: str | None = None,
         min_gain_frac: float = 0.02, giant_degrees=GIANT_DEGREES, warp_limits=WARP_LIMITS) -> dict:
    """The fastest knob setting for this graph on this GPU:
    {"giant_degree", "warp_limit", "ms", "default_ms", "trials", "cached"}.
    Pass the returned giant_degree / warp_limit to Louvain(...)."""
    lvb = _pkg()
    key = graph_key(lvb, graph, device_csr, device)
    store = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                store = json.load(f)
        except (OSError, ValueError):
            store = {}
    if key in store:
        out = dict(store[key])
        out["cached"] = True
        return out
    trials = []

    def measure(knobs):
        ms, q = _run_ms(lvb, graph, device_csr, device, min_gain, knobs)
        trials.append({"giant_degree": knobs["giant_degree"], "warp_limit": knobs["warp_limit"], "ms": round(ms, 3),
                       "modularity": q})
        return ms

    best = dict(DEFAULT)
    best_ms = default_ms = measure(best)
    # every setting is timed once: the warp-limit pass skips the setting the
    # giant-degree pass already timed (the chosen giant degree at the
    # default warp limit), also after another warp limit has been kept
    seen = {(best["giant_degree"], best["warp_limit"])}
    for gd in giant_degrees:
        if (gd, best["warp_limit"]) in seen:
            continue
        k = {"giant_degree": gd, "warp_limit": best["warp_limit"]}
        seen.add((gd, k["warp_limit"]))
        ms = measure(k)
        if ms < best_ms * (1.0 - min_gain_frac):
            best, best_ms = k, ms
    for wl in warp_limits:
        if (best["giant_degree"], wl) in seen:
            continue
        k = {"giant_degree": best["giant_degree"], "warp_limit": wl}
        seen.add((k["giant_degree"], wl))
        ms = measure(k)
        if ms < best_ms * (1.0 - min_gain_frac):
            best, best_ms = k, ms
    qs = {t["modularity"] for t in trials}
    if len(qs) != 1:
        raise RuntimeError("work-mapping knobs changed the result: %s" % sorted(qs))
    out = {"giant_degree": best["giant_degree"], "warp_limit": best["warp_limit"], "ms": round(best_ms, 3),
           "default_ms": round(default_ms, 3), "trials": trials, "key": key, "cached": False}
    if cache:
        store[key] = {k: v for k, v in out.items() if k != "cached"}
        _write_cache(cache, store)
    return out


def _write_cache(cache: str, store: dict) -> None:
    """Replace the cache file atomically.  Each writer uses its own temporary
    file in the cache's directory, so ranks that tune at the same time (one
    process per GPU) never rename each other's half-written file; the last
    complete write wins."""
    import tempfile
    d = os.path.dirname(os.path.abspath(cache))
    fd, tmp = tempfile.mkstemp(prefix=os.path.basename(cache) + ".", suffix=".tmp", dir=d)
    try:
        with os.fdopen(fd, "w") as f:
            json.dump(store, f, indent=1)
        os.replace(tmp, cache)
    except BaseException:
        try:
            os.unlink(tmp)
        except OSError:
            pass
        raise
