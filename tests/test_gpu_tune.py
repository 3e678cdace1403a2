"""The autotuner: it only moves work between kernels, so every trial must
give the same partition (it checks the modularity bits of every trial), the
chosen knobs must be valid, the choice must be cached, and a tuned run must
still equal the oracle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_chooses_valid_cached_knobs(lvb, orc, tmp_path):
    g = lvb.gen_rmat(15, seed=4)
    cache = str(tmp_path / "tune.json")
    t = lvb.tune(g, cache=cache, giant_degrees=(2048, 8192, 65536), warp_limits=(128, 352))
    assert not t["cached"]
    assert 1024 <= t["giant_degree"] <= 65536 and 32 <= t["warp_limit"] <= 384
    assert len(t["trials"]) == 4 and len({x["modularity"] for x in t["trials"]}) == 1
    assert os.path.exists(cache)
    t2 = lvb.tune(g, cache=cache)
    assert t2["cached"] and (t2["giant_degree"], t2["warp_limit"]) == (t["giant_degree"], t["warp_limit"])
    with lvb.Louvain(g, giant_degree=t["giant_degree"], warp_limit=t["warp_limit"]) as e:
        q = e.run(1e-6)
        m = e.original_to_community()[0]
    o = orc.Oracle(g.rowptr, g.col, g.w)
    q_ref, _ = o.run(1e-6)
    assert q == q_ref
    assert np.array_equal(m, o.original_to_community())
