"""lv_modularity_noalloc: the modularity of a given partition for callers that
cannot allocate device memory (their device memory is owned by another
allocator, or they cannot take the synchronisation of cudaMalloc/cudaFree).

It is called through the C ABI and must return exactly what the handle-based
entry points (lv_create_device + lv_set_communities + lv_modularity) return,
on two calls in a row and after a call on a different partition (the
library's scratch array keeps the previous call's contents), on the default
stream and on a caller's stream, without changing the device's free memory."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lvb, d_rp, d_cl, d_w, V, E, d_comm, stream=None):
    q = C.c_double()
    err = C.create_string_buffer(256)
    rc = lvb.lib().lv_modularity_noalloc(C.c_void_p(d_rp), C.c_void_p(d_cl), C.c_void_p(d_w), V, E,
                                         C.c_void_p(d_comm), C.c_void_p(stream) if stream else None,
                                         C.byref(q), err, 256)
    return rc, q.value, err.value.decode()


def test_noalloc_modularity_matches_handle_path(lvb):
    import torch
    rng = np.random.default_rng(3)
    graphs = [lvb.gen_planted(6000, 48, 16.0, 2.0, 5, "uniform"), lvb.gen_rmat(13, seed=9)]
    side = torch.cuda.Stream()
    for g in graphs:
        rp, cl, w = g.rowptr, g.col, g.w
        V, E = len(rp) - 1, len(cl)
        d_rp = torch.from_numpy(np.ascontiguousarray(rp)).cuda()
        d_cl = torch.from_numpy(np.ascontiguousarray(cl)).cuda()
        d_w = torch.from_numpy(np.ascontiguousarray(w)).cuda()
        dev_csr = (d_rp.data_ptr(), d_cl.data_ptr(), d_w.data_ptr(), V, E)
        # partitions: the final communities of a full run, a random one and singletons
        e = lvb.Louvain(device_csr=dev_csr)
        e.run(1e-6)
        found, _ = e.original_to_community()
        e.close()
        parts = [found.astype(np.int32), rng.integers(0, 50, V).astype(np.int32),
                 np.arange(V, dtype=np.int32)]
        ref = lvb.Louvain(device_csr=dev_csr)
        q_refs = []
        for comm in parts:
            ref.set_communities(comm)
            q_refs.append(ref.calculate_modularity())
        ref.close()
        d_parts = [torch.from_numpy(c).cuda() for c in parts]
        torch.cuda.synchronize()
        rc, _, msg = _noalloc(lvb, *dev_csr, d_parts[0].data_ptr())   # first call on this device
        assert rc == lvb.LV_OK, msg
        free0 = torch.cuda.mem_get_info()[0]
        for comm, q_ref in zip(d_parts, q_refs):
            for stream in (None, side.cuda_stream):
                rc, q, msg = _noalloc(lvb, *dev_csr, comm.data_ptr(), stream)
                assert rc == lvb.LV_OK, msg
                assert q == q_ref          # exact: same fixed-point sums and FP64 formula
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0   # nothing was allocated


def test_noalloc_rejects_bad_sizes(lvb):
    import torch
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    V = (1 << 20) + 1
    rc, _, msg = _noalloc(lvb, d.data_ptr(), d.data_ptr(), d.data_ptr(), V, 0, d.data_ptr())
    assert rc == lvb.LV_ERR_TOO_LARGE
    assert "LV_NOALLOC_MAX_VERTICES" in msg
    # entries without vertices: malformed, as for lv_create_device
    rc, _, msg = _noalloc(lvb, d.data_ptr(), d.data_ptr(), d.data_ptr(), 0, 4, d.data_ptr())
    assert rc == lvb.LV_ERR_INVALID, msg
