#!/usr/bin/env python
"""Train the learned active-set predictor on LFR-like graphs.

Move traces come from plain Louvain runs on seeded LFR-like graphs (power-law
degrees with exponent 2.5, mean 20, max 2000; power-law community sizes with
exponent 1.5 in [50, 5000]; mixing parameter mu uniform in [0.1, 0.5]).  Each
run records, for a sample of vertices before every sweep, the predictor's
five features and whether the vertex then moved (lv_opts.trace_sample).  The
MLP is trained on the GPU with the library's own kernels (lv_active_train);
the logit threshold is the largest one whose recall of movers on held-out
graphs reaches --target-recall.  The result is a JSON file with the bf16
parameters, the threshold and the training record.

    python gpu-louvain_b200/train_active_set.py --seeds 64 --vertices 1000000 \\
        --out gpu-louvain_b200/active_set_lfr.json
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LFR = {"tau1": 2.5, "mean_degree": 20.0, "kmax": 2000, "tau2": 1.5, "cmin": 50, "cmax": 5000}
TRAIN_SEED0 = 1000      # graph seeds TRAIN_SEED0 + i; held-out evaluation uses other seeds


def load_pkg():
    if "gpu_louvain_b200" in sys.modules:
        return sys.modules["gpu_louvain_b200"]
    spec = importlib.util.spec_from_file_location("gpu_louvain_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gpu_louvain_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def graph_mu(i: int) -> float:
    r = np.random.default_rng([TRAIN_SEED0, i])
    return float(r.uniform(0.1, 0.5))


def collect(lvb, seeds, V, sample, device, min_gain):
    xs, ys = [], []
    for i in seeds:
        g, _ = lvb.gen_lfr(V, graph_mu(i), seed=TRAIN_SEED0 + i, **LFR)
        with lvb.Louvain(g, device=device, trace_sample=sample) as e:
            e.run(min_gain)
            x, y = e.traces()
        xs.append(x)
        ys.append(y)
    return np.concatenate(xs), np.concatenate(ys)


def pick_threshold(logits, y, target):
    """Largest logit threshold t with recall(logit > t) >= target."""
    pos = np.sort(logits[y == 1])
    if len(pos) == 0:
        return 0.0
    k = int(np.floor((1.0 - target) * len(pos)))
    t = float(pos[k]) if k < len(pos) else float(pos[-1])
    return float(np.nextafter(np.float32(t), np.float32(-np.inf)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=64, help="training graphs")
    ap.add_argument("--holdout", type=int, default=4, help="graphs for the threshold")
    ap.add_argument("--vertices", type=int, default=1000000)
    ap.add_argument("--sample", type=float, default=0.05, help="trace fraction per sweep")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--target-recall", type=float, default=0.99)
    ap.add_argument("--full-every", type=int, default=4, help="recommended lv_opts.active_full_every")
    ap.add_argument("--active-start", type=float, default=0.2, help="recommended lv_opts.active_start")
    ap.add_argument("--min-recall", type=float, default=0.5, help="recommended lv_opts.active_min_recall")
    ap.add_argument("--min-gain", type=float, default=1e-6)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--out", default=os.path.join(HERE, "active_set_lfr.json"))
    a = ap.parse_args()
    lvb = load_pkg()
    t0 = time.time()
    x, y = collect(lvb, range(a.seeds), a.vertices, a.sample, a.device, a.min_gain)
    xv, yv = collect(lvb, range(a.seeds, a.seeds + a.holdout), a.vertices, a.sample, a.device, a.min_gain)
    t_collect = time.time() - t0
    t0 = time.time()
    model, loss = lvb.active_train(x, y, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, device=a.device)
    t_train = time.time() - t0
    lv = lvb.active_predict(model, xv, device=a.device)
    thr = pick_threshold(lv, yv, a.target_recall)
    prop = lv > thr
    alt = {}
    for tr in (0.9, 0.95, 0.97, 0.99):
        t = pick_threshold(lv, yv, tr)
        p = lv > t
        alt[str(tr)] = {"logit_threshold": t, "proposed_fraction": float(p.mean()),
                        "recall": float((p & (yv == 1)).sum() / max(1, (yv == 1).sum()))}
    rec = float((prop & (yv == 1)).sum() / max(1, (yv == 1).sum()))
    out = {
        "model_bf16": [int(v) for v in model],
        "logit_threshold": thr,
        "full_every": a.full_every,
        "active_start": a.active_start,
        "min_recall": a.min_recall,
        "thresholds_by_recall": alt,
        "features": ["log2(1+degree)/16", "own-community weight fraction", "relative best gain",
                     "moved in previous sweep", "fraction of neighbours that moved in previous sweep"],
        "hidden": lvb.ACTIVE_HIDDEN,
        "training": {"graphs": a.seeds, "holdout_graphs": a.holdout, "vertices": a.vertices,
                     "graph_seeds": [TRAIN_SEED0, TRAIN_SEED0 + a.seeds + a.holdout - 1],
                     "lfr": LFR, "mu": "uniform [0.1, 0.5] per graph", "trace_sample": a.sample,
                     "rows": int(len(y)), "positive_rate": float(y.mean()), "epochs": a.epochs,
                     "batch": a.batch, "lr": a.lr, "seed": a.seed, "epoch_loss": [float(v) for v in loss],
                     "holdout_rows": int(len(yv)), "holdout_recall": rec,
                     "holdout_proposed_fraction": float(prop.mean()), "target_recall": a.target_recall,
                     "collect_s": round(t_collect, 1), "train_s": round(t_train, 1)},
    }
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({k: v for k, v in out.items() if k != "model_bf16"}))


if __name__ == "__main__":
    main()
