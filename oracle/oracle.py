"""ctypes binding of the CPU oracle (liblouvain_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() (as the
checker) and bench.py's CPU baseline.  The product never imports it.
The oracle restates the reference's rule in exact arithmetic; see
louvain_oracle.h for the reference file:line map.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblouvain_oracle.so")
_lib = None
P32 = C.POINTER(C.c_int32)
P64 = C.POINTER(C.c_int64)
PU64 = C.POINTER(C.c_uint64)
PF = C.POINTER(C.c_float)


def build() -> None:
    r = subprocess.run(["make", "-C", _HERE, "liblouvain_oracle.so"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed: " + r.stderr[-2000:])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int32, C.c_int64, P32, P32, PF, C.c_int, C.POINTER(C.c_int)]
        L.orc_destroy.argtypes = [C.c_void_p]
        for n, r in [("orc_num_vertices", C.c_int32), ("orc_num_edges", C.c_int64),
                     ("orc_scale", C.c_int), ("orc_total_weight", C.c_uint64), ("orc_level", C.c_int)]:
            getattr(L, n).restype = r
            getattr(L, n).argtypes = [C.c_void_p]
        L.orc_sweep.restype = C.c_int64
        L.orc_sweep.argtypes = [C.c_void_p]
        L.orc_modularity.restype = C.c_double
        L.orc_modularity.argtypes = [C.c_void_p]
        L.orc_modularity_parts.argtypes = [C.c_void_p, PU64, PU64, PU64]
        L.orc_q_from_parts.restype = C.c_double
        L.orc_q_from_parts.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_optimise_level.argtypes = [C.c_void_p, C.c_float, C.c_int, P32]
        L.orc_aggregate.argtypes = [C.c_void_p]
        L.orc_run.argtypes = [C.c_void_p, C.c_float, C.c_int, C.POINTER(C.c_double), P32, P64, P64]
        L.orc_get_communities.argtypes = [C.c_void_p, P32]
        L.orc_set_communities.argtypes = [C.c_void_p, P32]
        L.orc_get_original_to_community.argtypes = [C.c_void_p, P32]
        L.orc_get_csr.argtypes = [C.c_void_p, P64, P32, P64]
        L.orc_get_vertex_weights.argtypes = [C.c_void_p, PU64]
        L.orc_get_community_weights.argtypes = [C.c_void_p, PU64]
        L.orc_choose_scale.argtypes = [PF, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_read_mtx.argtypes = [C.c_char_p, P32, P64, C.POINTER(P32), C.POINTER(P32),
                                   C.POINTER(PF), PF]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_gen_rmat.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int, P32, P64, C.POINTER(P32), C.POINTER(P32),
                                   C.POINTER(PF)]
        L.orc_modularity_f64.restype = C.c_double
        L.orc_modularity_f64.argtypes = [C.c_int32, P32, P32, PF, P32]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def choose_scale(w: np.ndarray):
    w = np.ascontiguousarray(w, dtype=np.float32)
    s, ex = C.c_int(), C.c_int()
    rc = lib().orc_choose_scale(_p(w, C.c_float), len(w), C.byref(s), C.byref(ex))
    return rc, s.value, bool(ex.value)


def read_mtx(path: str):
    L = lib()
    V, E = C.c_int32(), C.c_int64()
    rp, cl, w = P32(), P32(), PF()
    m = C.c_float()
    rc = L.orc_read_mtx(path.encode(), C.byref(V), C.byref(E), C.byref(rp), C.byref(cl), C.byref(w),
                        C.byref(m))
    if rc:
        raise RuntimeError(f"orc_read_mtx failed: {rc}")
    out = []
    for ptr, n, dt in ((rp, V.value + 1, np.int32), (cl, E.value, np.int32), (w, E.value, np.float32)):
        arr = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
        L.orc_free(C.cast(ptr, C.c_void_p))
        out.append(arr)
    return out[0], out[1], out[2], m.value


def _take(ptr, n, dt):
    """Copy a malloc'd oracle array into numpy and free it."""
    arr = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
    lib().orc_free(C.cast(ptr, C.c_void_p))
    return arr


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 1, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, weights: str = "uniform", nthreads: int = 0):
    """Seeded R-MAT graph as (rowptr, col, w): the same CSR as the engine's
    generators for the same arguments, built without the product library."""
    V, E = C.c_int32(), C.c_int64()
    rp, cl, w = P32(), P32(), PF()
    rc = lib().orc_gen_rmat(scale, edge_factor, seed, a, b, c, 1 if weights == "unit" else 0,
                            nthreads if nthreads > 0 else (os.cpu_count() or 1), C.byref(V), C.byref(E),
                            C.byref(rp), C.byref(cl), C.byref(w))
    if rc:
        raise RuntimeError(f"orc_gen_rmat failed: {rc}")
    return (_take(rp, V.value + 1, np.int32), _take(cl, E.value, np.int32), _take(w, E.value, np.float32))


def modularity_f64(rowptr, col, w, comm) -> float:
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    comm = np.ascontiguousarray(comm, np.int32)
    return lib().orc_modularity_f64(len(rowptr) - 1, _p(rowptr, C.c_int32), _p(col, C.c_int32),
                                    _p(w, C.c_float), _p(comm, C.c_int32))


class Oracle:
    """The oracle's Louvain state for one graph (mirrors the engine API)."""

    def __init__(self, rowptr, col, w, nthreads: int = 0):
        self._rp = np.ascontiguousarray(rowptr, np.int32)
        self._cl = np.ascontiguousarray(col, np.int32)
        self._w = np.ascontiguousarray(w, np.float32)
        if nthreads <= 0:
            nthreads = os.cpu_count() or 1
        err = C.c_int()
        h = lib().orc_create(len(self._rp) - 1, len(self._cl), _p(self._rp, C.c_int32),
                             _p(self._cl, C.c_int32), _p(self._w, C.c_float), nthreads, C.byref(err))
        if not h:
            raise RuntimeError(f"orc_create failed: {err.value}")
        self._h = C.c_void_p(h)
        self.V0 = len(self._rp) - 1

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def V(self):
        return lib().orc_num_vertices(self._h)

    @property
    def E(self):
        return lib().orc_num_edges(self._h)

    @property
    def level(self):
        return lib().orc_level(self._h)

    def scale(self):
        L = lib()
        return L.orc_scale(self._h), L.orc_total_weight(self._h)

    def sweep(self) -> int:
        return lib().orc_sweep(self._h)

    def modularity(self) -> float:
        return lib().orc_modularity(self._h)

    def modularity_parts(self):
        e, hi, lo = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().orc_modularity_parts(self._h, C.byref(e), C.byref(hi), C.byref(lo))
        return e.value, (hi.value << 64) | lo.value

    def optimise_modularity(self, min_gain: float, max_sweeps: int = 0):
        sw = C.c_int32()
        ch = lib().orc_optimise_level(self._h, min_gain, max_sweeps, C.byref(sw))
        if ch < 0:
            raise RuntimeError("oracle optimise failed")
        return bool(ch), sw.value

    def aggregate_communities(self):
        rc = lib().orc_aggregate(self._h)
        if rc:
            raise RuntimeError(f"oracle aggregate failed: {rc}")

    def run(self, min_gain: float, max_sweeps: int = 0):
        q = C.c_double()
        lv, sw, es = C.c_int32(), C.c_int64(), C.c_int64()
        rc = lib().orc_run(self._h, min_gain, max_sweeps, C.byref(q), C.byref(lv), C.byref(sw),
                           C.byref(es))
        if rc:
            raise RuntimeError(f"oracle run failed: {rc}")
        return q.value, {"levels": lv.value, "sweeps": sw.value, "edge_sweeps": es.value}

    def communities(self):
        out = np.empty(self.V, np.int32)
        lib().orc_get_communities(self._h, _p(out, C.c_int32))
        return out

    def set_communities(self, comm):
        c = np.ascontiguousarray(comm, np.int32)
        if lib().orc_set_communities(self._h, _p(c, C.c_int32)):
            raise ValueError("bad community vector")

    def original_to_community(self):
        out = np.empty(self.V0, np.int32)
        lib().orc_get_original_to_community(self._h, _p(out, C.c_int32))
        return out

    def csr(self):
        V, E = self.V, self.E
        rp = np.empty(V + 1, np.int64)
        cl = np.empty(E, np.int32)
        wf = np.empty(E, np.int64)
        lib().orc_get_csr(self._h, _p(rp, C.c_int64), _p(cl, C.c_int32), _p(wf, C.c_int64))
        return rp, cl, wf

    def vertex_weights(self):
        out = np.empty(self.V, np.uint64)
        lib().orc_get_vertex_weights(self._h, _p(out, C.c_uint64))
        return out

    def community_weights(self):
        out = np.empty(self.V, np.uint64)
        lib().orc_get_community_weights(self._h, _p(out, C.c_uint64))
        return out
