"""Generate golden vectors from the reference's own CUDA code.

Runs where oracle/_ref/gpulouvain_ref and oracle/_ref/ref_harness were built
(`make -C oracle ref`, compiled from the reference sources) and a GPU is
present.  For each small graph it records:
  <name>.mtx            the input (symmetric Matrix Market)
  <name>.sweeps_stock.bin  the community vector after each of the first N
                        sweeps of the stock reference (optimiseModularity
                        called with a gain threshold that admits exactly one
                        sweep per call).  On B200 these show (almost) no moves:
                        computeMove's final store races between lane 0 (the
                        move) and the other lanes (the old community),
                        modularity_optimisation.cu:192-196.
  <name>.sweeps1.bin    the same sweeps with the reference's own move kernels
                        launched at one thread per vertex (no racing lanes),
                        orchestrated like optimiseModularity
  <name>.agg_in.bin     a community vector (the oracle's level-0 result)
  <name>.agg_out.bin    the reference's aggregateCommunities of that vector
  <name>.cli.txt        stdout of `gpulouvain -f <name>.mtx -g <gain> -v`
Usage: python tests/golden/make_golden.py [out_dir]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import graphs_np  # noqa: E402
import oracle  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "gpulouvain_ref")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
NSWEEPS = 10


def write_mtx(path, rowptr, col, w):
    V = len(rowptr) - 1
    row = np.repeat(np.arange(V), np.diff(rowptr))
    m = row >= col
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{V} {V} {int(m.sum())}\n")
        for a, b, x in zip(row[m], col[m], w[m]):
            f.write(f"{a + 1} {b + 1} {float(x):.9g}\n")


def quarter_weights(rowptr, col, seed):
    """Replace weights by multiples of 1/4 in [0.5, 1.5] (symmetric), so that
    FP32 sums in the reference are exact."""
    V = len(rowptr) - 1
    row = np.repeat(np.arange(V), np.diff(rowptr)).astype(np.int64)
    a, b = np.minimum(row, col), np.maximum(row, col)
    h = graphs_np.draw(graphs_np.stream_key(seed, 77), (a.astype(np.uint64) << np.uint64(32)) | b.astype(np.uint64))
    return (2 + (h % np.uint64(5)).astype(np.int64)).astype(np.float32) / np.float32(4)


def cases():
    out = []
    rp, cl, w = graphs_np.rmat(12, seed=2, weights="unit")
    out.append(("rmat12_unit", rp, cl, w, 1e-6))
    rp, cl, w = graphs_np.planted(10000, 64, 16.0, 2.0, 0)
    out.append(("planted10k_s0", rp, cl, w, 0.01))
    rp, cl, w = graphs_np.planted(2000, 16, 12.0, 2.0, 1)
    out.append(("planted2k_s1", rp, cl, w, 0.01))
    rp, cl, w = graphs_np.planted(3000, 24, 10.0, 3.0, 2)
    out.append(("planted3k_quarter", rp, cl, quarter_weights(rp, cl, 2), 0.001))
    rp, cl, w = graphs_np.planted(5000, 40, 6.0, 4.0, 3)
    out.append(("planted5k_weak", rp, cl, w, 0.001))
    return out


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    index = []
    for name, rp, cl, w, gain in cases():
        mtx = os.path.join(out_dir, name + ".mtx")
        write_mtx(mtx, rp, cl, w)
        # the reference reads the file back: use its CSR (file order) everywhere
        frp, fcl, fw, _ = oracle.read_mtx(mtx)
        subprocess.run([HARNESS, "sweeps", mtx, str(NSWEEPS),
                        os.path.join(out_dir, name + ".sweeps_stock.bin")], check=True)
        subprocess.run([HARNESS, "sweeps1", mtx, str(NSWEEPS), os.path.join(out_dir, name + ".sweeps1.bin")],
                       check=True)
        o = oracle.Oracle(frp, fcl, fw)
        o.optimise_modularity(gain)
        o.communities().astype(np.int32).tofile(os.path.join(out_dir, name + ".agg_in.bin"))
        subprocess.run([HARNESS, "aggregate", mtx, os.path.join(out_dir, name + ".agg_in.bin"),
                        os.path.join(out_dir, name + ".agg_out.bin")], check=True)
        r = subprocess.run([REF_BIN, "-f", mtx, "-g", str(gain), "-v"], check=True, capture_output=True,
                           text=True)
        with open(os.path.join(out_dir, name + ".cli.txt"), "w") as f:
            f.write(r.stdout)
        index.append({"name": name, "mtx": name + ".mtx", "sweeps": name + ".sweeps1.bin",
                      "sweeps_stock": name + ".sweeps_stock.bin",
                      "agg_in": name + ".agg_in.bin", "agg_out": name + ".agg_out.bin",
                      "cli": name + ".cli.txt", "min_gain": gain})
    with open(os.path.join(out_dir, "index.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": index}, f, indent=1)


if __name__ == "__main__":
    main()
