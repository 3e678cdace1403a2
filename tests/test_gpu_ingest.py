"""CSR built on the device from a Matrix Market file (lv_read_mtx_device,
lv_csr_from_entries_device) must equal the host build (lv_read_mtx) entry
for entry: same rows, same order within rows (file order), same weights,
same FP32 M, for the reference's golden inputs, files with self-loops,
repeated and unordered entries, pattern files, and out-of-range entries."""
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu


def _host(ptr, n, dtype):
    import torch

    class W:
        __cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str, "data": (ptr, False),
                                    "version": 3}
    if n == 0:
        return np.zeros(0, dtype)
    return torch.as_tensor(W(), device="cuda").cpu().numpy().copy()


def _check_same(lvb, path):
    h = lvb.read_mtx(path)
    d = lvb.read_mtx_device(path)
    try:
        assert (d.V, d.E) == (h.V, h.E)
        assert np.array_equal(_host(d.rowptr, d.V + 1, np.int32), h.rowptr)
        assert np.array_equal(_host(d.col, d.E, np.int32), h.col)
        assert np.array_equal(_host(d.w, d.E, np.float32).view(np.uint32), h.w.view(np.uint32))
        assert d.m_ref == h.m_ref
    finally:
        d.free()


@pytest.mark.parametrize("name", ["planted2k_s1", "planted3k_quarter", "rmat12_unit"])
def test_device_csr_matches_host_on_goldens(lvb, name):
    _check_same(lvb, os.path.join(GOLDEN_DIR, name + ".mtx"))


def test_device_csr_matches_host_on_irregular_files(lvb, tmp_path):
    rng = np.random.default_rng(4)
    V, n = 5000, 60000
    a = rng.integers(1, V + 1, n)
    b = rng.integers(1, V + 1, n)
    b[:500] = a[:500]                         # self-loops
    a[600:700], b[600:700] = a[700:800], b[700:800]   # repeated entries
    w = rng.integers(1, 100, n) / 8.0
    lines = ["%%MatrixMarket matrix coordinate real symmetric", "% comment", "", f"{V} {V} {n}"]
    lines += [f"{x} {y} {z}" for x, y, z in zip(a, b, w)]
    p = tmp_path / "irr.mtx"
    p.write_text("\n".join(lines) + "\n")
    _check_same(lvb, str(p))
    lines = ["%%MatrixMarket matrix coordinate pattern symmetric", f"{V} {V} {n}"]
    lines += [f"{x} {y}" for x, y in zip(a, b)]
    q = tmp_path / "pat.mtx"
    q.write_text("\n".join(lines) + "\n")
    _check_same(lvb, str(q))
    # one vertex, no entries
    r = tmp_path / "empty.mtx"
    r.write_text("%%MatrixMarket matrix coordinate real symmetric\n1 1 0\n")
    _check_same(lvb, str(r))


def test_device_csr_from_entries_rejects_bad_ids(lvb):
    with pytest.raises(lvb.LouvainError) as ex:
        lvb.csr_from_entries_device(4, [0, 1, 4], [1, 2, 0], [1.0, 1.0, 1.0])
    assert ex.value.status == lvb.LV_ERR_INVALID


def test_engine_on_device_built_csr(lvb):
    g = lvb.gen_rmat(14, seed=3)
    rng = np.random.default_rng(0)
    order = rng.permutation(g.E)
    src = np.repeat(np.arange(g.V, dtype=np.int32), np.diff(g.rowptr))
    keep = src[order] <= g.col[order]       # each undirected edge once, in shuffled order
    a, b, w = src[order][keep], g.col[order][keep], g.w[order][keep]
    d = lvb.csr_from_entries_device(g.V, a, b, w)
    try:
        with lvb.Louvain(device_csr=(d.rowptr, d.col, d.w, d.V, d.E)) as e:
            q_dev = e.run(1e-6)
            m_dev = e.original_to_community()[0]
        rp = _host(d.rowptr, d.V + 1, np.int32)
        cl = _host(d.col, d.E, np.int32)
        ww = _host(d.w, d.E, np.float32)
    finally:
        d.free()
    with lvb.Louvain(lvb.Graph(rp, cl, ww)) as e:
        assert e.run(1e-6) == q_dev
        assert np.array_equal(e.original_to_community()[0], m_dev)
