"""gpu-louvain_b200 -- Python host mirror of the B200 Louvain engine.

The engine is the C-ABI library ``lib/liblouvain_b200.so`` (CUDA kernels for
sm_100a, see ``include/louvain_b200.h``).  This module binds it with ctypes and
mirrors the reference's operator surface for the level loop:

    Louvain.optimise_modularity(min_gain)  <- optimiseModularity
                                             (modularity_optimisation.cuh:28)
    Louvain.aggregate_communities()        <- aggregateCommunities
                                             (community_aggregation.cuh:11)
    Louvain.calculate_modularity()         <- calculateModularity
                                             (modularity_optimisation.cuh:30)
    Louvain.run(min_gain)                  <- the level loop of main()
                                             (gpulouvain.cu:30-37)
    read_mtx(path)                         <- readInputData (utils.cu:9-62)
    print_communities(...)                 <- printOriginalToCommunity
                                             (modularity_optimisation.cu:403-418)

Errors raise LouvainError carrying the lv_status code (the reference exits
the process instead, utils.cuh:92-98).  There is no CPU fallback: when the
library or a CUDA device is missing the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# LV_LIB may point at another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("LV_LIB") or os.path.join(_HERE, "lib", "liblouvain_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "gpulouvain")

LV_OK = 0
LV_ERR_INVALID = 1
LV_ERR_WEIGHT = 2
LV_ERR_TOO_LARGE = 3
LV_ERR_NOMEM = 4
LV_ERR_CUDA = 5
LV_ERR_DEVICE = 6
LV_ERR_IO = 7
LV_ERR_NO_DEVICE = 8

NUM_CLASSES = 9
# move-phase profile slots: the update buckets (degree ranges) 0..6
CLASS_NAMES = ["b0_deg4", "b1_deg8", "b2_deg16", "b3_deg32", "b4_deg84", "b5_deg319",
               "b6_deg8192", "b6_giants", "unused8"]


class LouvainError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"lv_status {status}: {msg}")


class _Opts(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("device", C.c_int32), ("max_sweeps", C.c_int32),
                ("profile", C.c_int32), ("verify", C.c_int32), ("trace", C.c_int32),
                ("sweep_graph", C.c_int32), ("active_set", C.c_int32), ("active_full_every", C.c_int32),
                ("active_min_recall", C.c_float), ("trace_sample", C.c_float), ("active_start", C.c_float),
                ("wide_weights", C.c_int32), ("giant_degree", C.c_int32), ("warp_limit", C.c_int32),
                ("reserved", C.c_int32 * 1)]


class _Stats(C.Structure):
    _fields_ = [("levels", C.c_int32), ("final_vertices", C.c_int32), ("sweeps", C.c_int64),
                ("edge_sweeps", C.c_int64), ("moves", C.c_int64), ("move_ms", C.c_double),
                ("modularity_ms", C.c_double), ("aggregate_ms", C.c_double),
                ("setup_ms", C.c_double), ("move_bytes", C.c_double),
                ("kernel_launches", C.c_int64)]


class _ClassStats(C.Structure):
    _fields_ = [("launches", C.c_int64 * NUM_CLASSES), ("vertices", C.c_int64 * NUM_CLASSES),
                ("edges", C.c_int64 * NUM_CLASSES), ("ms", C.c_double * NUM_CLASSES),
                ("bytes", C.c_double * NUM_CLASSES), ("stored_bytes", C.c_double * NUM_CLASSES)]


EXPORTED = [
    "lv_default_opts", "lv_status_string", "lv_version", "lv_create", "lv_create_device",
    "lv_reset", "lv_destroy", "lv_last_error", "lv_optimise_level", "lv_aggregate",
    "lv_modularity", "lv_run", "lv_sweep", "lv_get_original_to_community", "lv_get_communities",
    "lv_set_communities", "lv_get_level_info", "lv_get_csr", "lv_get_scale", "lv_get_stats",
    "lv_get_class_stats", "lv_clear_stats", "lv_read_mtx", "lv_write_mtx", "lv_free_host",
    "lv_print_communities", "lv_gen_rmat", "lv_gen_planted", "lv_gen_rmat_device",
    "lv_free_device", "lv_modularity_noalloc", "lv_trim_device_memory",
    "lv_batch_create", "lv_batch_create_device", "lv_batch_run", "lv_batch_get_results",
    "lv_batch_get_graph_stats", "lv_batch_get_stats", "lv_batch_last_error", "lv_batch_destroy",
    "lv_gen_lfr", "lv_set_active_model", "lv_get_traces", "lv_get_active_stats", "lv_active_train",
    "lv_active_predict", "lv_write_csr", "lv_read_csr", "lv_write_csr_stamped", "lv_read_csr_stamp", "lv_gen_planted_batch", "lv_read_mtx_device",
    "lv_csr_from_entries_device", "lv_read_mtx_entries", "lv_get_level_classes", "lv_get_device_name",
    "lv_read_active_model",
]

_lib = None

P32 = C.POINTER(C.c_int32)
P64 = C.POINTER(C.c_int64)
PF = C.POINTER(C.c_float)


def build(verbose: bool = False) -> None:
    """Compile the CUDA library and CLI in-tree (nvcc, sm_100a)."""
    r = subprocess.run(["make", "-C", _HERE, "-j8"], capture_output=True, text=True)
    if verbose or r.returncode != 0:
        print(r.stdout[-4000:], r.stderr[-4000:])
    if r.returncode != 0:
        raise RuntimeError("building liblouvain_b200.so failed")


def lib() -> C.CDLL:
    """Load the engine library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build the CUDA extension first")
    L = C.CDLL(LIB_PATH)
    L.lv_status_string.restype = C.c_char_p
    L.lv_version.restype = C.c_char_p
    L.lv_last_error.restype = C.c_char_p
    L.lv_last_error.argtypes = [C.c_void_p]
    L.lv_default_opts.argtypes = [C.POINTER(_Opts)]
    L.lv_create.argtypes = [P32, P32, PF, C.c_int32, C.c_int64, C.POINTER(_Opts), C.POINTER(C.c_void_p)]
    L.lv_create_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64,
                                   C.POINTER(_Opts), C.POINTER(C.c_void_p)]
    for name in ["lv_reset", "lv_destroy", "lv_aggregate", "lv_clear_stats"]:
        getattr(L, name).argtypes = [C.c_void_p]
    L.lv_optimise_level.argtypes = [C.c_void_p, C.c_float, P32]
    L.lv_modularity.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.lv_run.argtypes = [C.c_void_p, C.c_float, C.POINTER(C.c_double)]
    L.lv_sweep.argtypes = [C.c_void_p, P64]
    L.lv_get_original_to_community.argtypes = [C.c_void_p, P32, P32]
    L.lv_get_communities.argtypes = [C.c_void_p, P32]
    L.lv_set_communities.argtypes = [C.c_void_p, P32]
    L.lv_get_level_info.argtypes = [C.c_void_p, P32, P64, P32]
    L.lv_get_csr.argtypes = [C.c_void_p, P32, P32, P64]
    L.lv_get_scale.argtypes = [C.c_void_p, P32, C.POINTER(C.c_uint64), P32]
    L.lv_get_stats.argtypes = [C.c_void_p, C.POINTER(_Stats)]
    L.lv_get_class_stats.argtypes = [C.c_void_p, C.POINTER(_ClassStats)]
    L.lv_read_mtx.argtypes = [C.c_char_p, P32, P64, C.POINTER(P32), C.POINTER(P32), C.POINTER(PF), PF]
    L.lv_write_mtx.argtypes = [C.c_char_p, C.c_int32, C.c_int64, P32, P32, PF]
    L.lv_write_csr.argtypes = [C.c_char_p, C.c_int32, C.c_int64, P32, P32, PF, C.c_float]
    L.lv_read_csr.argtypes = [C.c_char_p, P32, P64, C.POINTER(P32), C.POINTER(P32), C.POINTER(PF), PF]
    L.lv_write_csr_stamped.argtypes = [C.c_char_p, C.c_int32, C.c_int64, P32, P32, PF, C.c_float, C.c_int64,
                                       C.c_int64]
    L.lv_read_csr_stamp.argtypes = [C.c_char_p, P64, P64]
    L.lv_get_level_classes.argtypes = [C.c_void_p, P32, P64]
    L.lv_read_mtx_entries.argtypes = [C.c_char_p, P32, P64, C.POINTER(P32), C.POINTER(P32), C.POINTER(PF)]
    L.lv_get_device_name.argtypes = [C.c_int32, C.c_char_p, C.c_int32]
    L.lv_read_mtx_device.argtypes = [C.c_char_p, C.c_int32, P32, P64, C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), PF]
    L.lv_csr_from_entries_device.argtypes = [C.c_int32, C.c_int32, C.c_int64, P32, P32, PF, P64,
                                             C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                             C.POINTER(C.c_void_p)]
    L.lv_gen_planted_batch.argtypes = [C.c_int32, P32, P32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_uint64), C.c_int32, P32, P64, C.POINTER(P32),
                                       C.POINTER(P32), C.POINTER(PF), C.POINTER(P32)]
    L.lv_free_host.argtypes = [C.c_void_p]
    L.lv_print_communities.argtypes = [C.c_char_p, P32, C.c_int32, C.c_int32]
    L.lv_gen_rmat.argtypes = [C.c_int32, C.c_int32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                              C.c_int32, P32, P64, C.POINTER(P32), C.POINTER(P32), C.POINTER(PF)]
    L.lv_gen_planted.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_uint64, C.c_int32,
                                 P64, C.POINTER(P32), C.POINTER(P32), C.POINTER(PF)]
    L.lv_gen_rmat_device.argtypes = [C.c_int32, C.c_int32, C.c_uint64, C.c_double, C.c_double,
                                     C.c_double, C.c_int32, C.c_int32, P32, P64,
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_void_p)]
    L.lv_free_device.argtypes = [C.c_void_p]
    L.lv_gen_lfr.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_int32,
                             C.c_int32, C.c_double, C.c_uint64, P64, C.POINTER(P32), C.POINTER(P32),
                             C.POINTER(PF), C.POINTER(P32)]
    L.lv_trim_device_memory.argtypes = [C.c_int32]
    L.lv_modularity_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64,
                                        C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_char_p,
                                        C.c_int32]
    L.lv_batch_create.argtypes = [P32, P32, PF, C.c_int32, C.c_int64, P32, C.c_int32,
                                  C.POINTER(_Opts), C.POINTER(C.c_void_p)]
    L.lv_batch_create_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64,
                                         P32, C.c_int32, C.POINTER(_Opts), C.POINTER(C.c_void_p)]
    L.lv_batch_run.argtypes = [C.c_void_p, C.c_float]
    L.lv_batch_get_results.argtypes = [C.c_void_p, P32, C.POINTER(C.c_double), P32, P32]
    L.lv_batch_get_graph_stats.argtypes = [C.c_void_p, P32, P64, P64, C.POINTER(C.c_double)]
    L.lv_batch_get_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double), P64, P64, P32]
    L.lv_batch_last_error.restype = C.c_char_p
    L.lv_batch_last_error.argtypes = [C.c_void_p]
    L.lv_batch_destroy.argtypes = [C.c_void_p]
    PU16 = C.POINTER(C.c_uint16)
    PU8 = C.POINTER(C.c_uint8)
    L.lv_set_active_model.argtypes = [C.c_void_p, PU16, C.c_int32, C.c_float]
    L.lv_read_active_model.argtypes = [C.c_char_p, PU16, C.c_int32, P32, PF, C.POINTER(_Opts)]
    L.lv_get_traces.argtypes = [C.c_void_p, PF, PU8, C.c_int64, P64]
    L.lv_get_active_stats.argtypes = [C.c_void_p, P64, P64, P64, C.POINTER(C.c_double), P32]
    L.lv_active_train.argtypes = [PF, PU8, C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_float,
                                  C.c_uint64, C.c_int32, PU16, PF]
    L.lv_active_predict.argtypes = [PU16, PF, C.c_int64, C.c_int32, PF]
    _lib = L
    return L


def status_string(code: int) -> str:
    return lib().lv_status_string(code).decode()


def _check(code: int, handle=None) -> None:
    if code != LV_OK:
        msg = status_string(code)
        if handle:
            detail = lib().lv_last_error(handle)
            if detail:
                msg += f" ({detail.decode()})"
        raise LouvainError(code, msg)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))


def _take_host(ptr, n: int, dtype) -> np.ndarray:
    """Copy a malloc'd C array into numpy and free it."""
    L = lib()
    buf = np.empty(n if n > 0 else 0, dtype=dtype)
    if n > 0:
        C.memmove(buf.ctypes.data, ptr, n * buf.itemsize)
    L.lv_free_host(C.cast(ptr, C.c_void_p))
    return buf


class Graph:
    """A CSR graph on the host: rowptr int32[V+1], col int32[E], w float32[E]."""

    def __init__(self, rowptr, col, w, m_ref: float | None = None):
        self.rowptr = _i32(rowptr)
        self.col = _i32(col)
        self.w = np.ascontiguousarray(w, dtype=np.float32)
        self.m_ref = m_ref

    @property
    def V(self) -> int:
        return int(self.rowptr.shape[0] - 1)

    @property
    def E(self) -> int:
        return int(self.col.shape[0])

    def edges(self):
        """Undirected edge list (u > v, plus self-loops) with weights."""
        row = np.repeat(np.arange(self.V, dtype=np.int32), np.diff(self.rowptr))
        m = row >= self.col
        return row[m], self.col[m], self.w[m]


def read_mtx(path: str) -> Graph:
    L = lib()
    V = C.c_int32()
    E = C.c_int64()
    rp, cl, w = P32(), P32(), PF()
    m = C.c_float()
    _check(L.lv_read_mtx(path.encode(), C.byref(V), C.byref(E), C.byref(rp), C.byref(cl), C.byref(w),
                         C.byref(m)))
    return Graph(_take_host(rp, V.value + 1, np.int32), _take_host(cl, E.value, np.int32),
                 _take_host(w, E.value, np.float32), m_ref=m.value)


def write_csr(path: str, g: Graph) -> None:
    """Binary CSR cache file (lv_write_csr)."""
    _check(lib().lv_write_csr(path.encode(), g.V, g.E, _ptr(g.rowptr, C.c_int32), _ptr(g.col, C.c_int32),
                              _ptr(g.w, C.c_float), g.m_ref if g.m_ref is not None else 0.0))


def read_csr(path: str) -> Graph:
    """Graph from a binary CSR cache file (lv_read_csr)."""
    L = lib()
    V = C.c_int32()
    E = C.c_int64()
    rp, cl, w = P32(), P32(), PF()
    m = C.c_float()
    _check(L.lv_read_csr(path.encode(), C.byref(V), C.byref(E), C.byref(rp), C.byref(cl), C.byref(w),
                         C.byref(m)))
    return Graph(_take_host(rp, V.value + 1, np.int32), _take_host(cl, E.value, np.int32),
                 _take_host(w, E.value, np.float32), m_ref=m.value)


def write_mtx(path: str, g: Graph) -> None:
    u, v, w = g.edges()
    u, v, w = _i32(u), _i32(v), np.ascontiguousarray(w, dtype=np.float32)
    _check(lib().lv_write_mtx(path.encode(), g.V, len(u), _ptr(u, C.c_int32), _ptr(v, C.c_int32),
                              _ptr(w, C.c_float)))


def _weight_mode(weights: str) -> int:
    """Generator weight mode: "unit" (every weight 1) or "uniform" (uniform in
    [0.5, 1.5) on a 2^-24 grid)."""
    modes = {"unit": 0, "uniform": 1}
    if weights not in modes:
        raise ValueError(f"weights must be 'unit' or 'uniform', not {weights!r}")
    return modes[weights]


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 1, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, weights: str = "uniform") -> Graph:
    L = lib()
    V = C.c_int32()
    E = C.c_int64()
    rp, cl, w = P32(), P32(), PF()
    _check(L.lv_gen_rmat(scale, edge_factor, seed, a, b, c, _weight_mode(weights),
                         C.byref(V), C.byref(E), C.byref(rp), C.byref(cl), C.byref(w)))
    return Graph(_take_host(rp, V.value + 1, np.int32), _take_host(cl, E.value, np.int32),
                 _take_host(w, E.value, np.float32))


def gen_planted(V: int = 10000, blocks: int = 64, d_in: float = 16.0, d_out: float = 2.0,
                seed: int = 0, weights: str = "unit") -> Graph:
    L = lib()
    E = C.c_int64()
    rp, cl, w = P32(), P32(), PF()
    _check(L.lv_gen_planted(V, blocks, d_in, d_out, seed, _weight_mode(weights),
                            C.byref(E), C.byref(rp), C.byref(cl), C.byref(w)))
    return Graph(_take_host(rp, V + 1, np.int32), _take_host(cl, E.value, np.int32),
                 _take_host(w, E.value, np.float32))


def gen_planted_batch(params, weights: str = "unit"):
    """Block-diagonal CSR (rowptr, col, w, graph_ptr) of planted-partition
    graphs, one per (V, blocks, d_in, d_out, seed) in params, generated by all
    host threads; graph i equals gen_planted(*params[i]) offset by
    graph_ptr[i]."""
    G = len(params)
    Vs = np.array([p[0] for p in params], np.int32)
    Bs = np.array([p[1] for p in params], np.int32)
    di = np.array([p[2] for p in params], np.float64)
    do = np.array([p[3] for p in params], np.float64)
    sd = np.array([p[4] for p in params], np.uint64)
    Vt, Et = C.c_int32(), C.c_int64()
    rp, cl, w, gp = P32(), P32(), PF(), P32()
    _check(lib().lv_gen_planted_batch(G, _ptr(Vs, C.c_int32), _ptr(Bs, C.c_int32), _ptr(di, C.c_double),
                                      _ptr(do, C.c_double), _ptr(sd, C.c_uint64),
                                      _weight_mode(weights), C.byref(Vt), C.byref(Et), C.byref(rp),
                                      C.byref(cl), C.byref(w), C.byref(gp)))
    return (_take_host(rp, Vt.value + 1, np.int32), _take_host(cl, Et.value, np.int32),
            _take_host(w, Et.value, np.float32), _take_host(gp, G + 1, np.int32))


def gen_lfr(V: int = 1000000, mu: float = 0.3, seed: int = 0, tau1: float = 2.5,
            mean_degree: float = 20.0, kmax: int = 2000, tau2: float = 1.5, cmin: int = 50,
            cmax: int = 5000):
    """LFR-like graph (lv_gen_lfr): returns (Graph, planted community array)."""
    L = lib()
    E = C.c_int64()
    rp, cl, w, cm = P32(), P32(), PF(), P32()
    _check(L.lv_gen_lfr(V, tau1, mean_degree, kmax, tau2, cmin, cmax, mu, seed, C.byref(E), C.byref(rp),
                        C.byref(cl), C.byref(w), C.byref(cm)))
    g = Graph(_take_host(rp, V + 1, np.int32), _take_host(cl, E.value, np.int32),
              _take_host(w, E.value, np.float32))
    return g, _take_host(cm, V, np.int32)


class DeviceGraph:
    """A CSR graph drawn on the device (owned device buffers)."""

    def __init__(self, V, E, rowptr, col, w, device):
        self.V, self.E = V, E
        self.rowptr, self.col, self.w = rowptr, col, w
        self.device = device

    def free(self) -> None:
        L = lib()
        for p in (self.rowptr, self.col, self.w):
            if p:
                L.lv_free_device(C.c_void_p(p))
        self.rowptr = self.col = self.w = 0


def gen_rmat_device(scale: int, edge_factor: int = 16, seed: int = 1, a: float = 0.57,
                    b: float = 0.19, c: float = 0.19, weights: str = "uniform",
                    device: int = 0) -> DeviceGraph:
    L = lib()
    V = C.c_int32()
    E = C.c_int64()
    rp, cl, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(L.lv_gen_rmat_device(scale, edge_factor, seed, a, b, c, _weight_mode(weights),
                                device, C.byref(V), C.byref(E), C.byref(rp), C.byref(cl), C.byref(w)))
    return DeviceGraph(V.value, E.value, rp.value, cl.value, w.value, device)


def device_name(device: int = 0) -> str:
    buf = C.create_string_buffer(256)
    _check(lib().lv_get_device_name(device, buf, 256))
    return buf.value.decode()


def read_mtx_device(path: str, device: int = 0) -> DeviceGraph:
    """Matrix Market file -> CSR built on the device (lv_read_mtx_device);
    the same CSR as read_mtx.  m_ref is set on the returned object."""
    L = lib()
    V, E = C.c_int32(), C.c_int64()
    rp, cl, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    m = C.c_float()
    _check(L.lv_read_mtx_device(path.encode(), device, C.byref(V), C.byref(E), C.byref(rp), C.byref(cl),
                                C.byref(w), C.byref(m)))
    g = DeviceGraph(V.value, E.value, rp.value, cl.value, w.value, device)
    g.m_ref = m.value
    return g


def csr_from_entries_device(V: int, v1, v2, w, device: int = 0) -> DeviceGraph:
    """CSR on the device from 0-based entries in file order
    (lv_csr_from_entries_device)."""
    a, b = _i32(v1), _i32(v2)
    ww = np.ascontiguousarray(w, dtype=np.float32)
    E = C.c_int64()
    rp, cl, dw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(lib().lv_csr_from_entries_device(device, V, len(a), _ptr(a, C.c_int32), _ptr(b, C.c_int32),
                                            _ptr(ww, C.c_float), C.byref(E), C.byref(rp), C.byref(cl),
                                            C.byref(dw)))
    return DeviceGraph(V, E.value, rp.value, cl.value, dw.value, device)


def print_communities(orig2comm: np.ndarray, num_communities: int, path: str | None = None) -> None:
    o = _i32(orig2comm)
    _check(lib().lv_print_communities(path.encode() if path else None, _ptr(o, C.c_int32), len(o),
                                      num_communities))


class Louvain:
    """One engine handle: a graph resident on one GPU plus its Louvain state."""

    def __init__(self, graph: Graph | None = None, *, device: int = 0, max_sweeps: int = 0,
                 profile: bool = False, verify: bool = False, trace: bool = False,
                 device_csr: tuple | None = None, sweep_graph: bool = True,
                 active_set: bool = False, active_full_every: int = 0, active_min_recall: float = 0.0,
                 trace_sample: float = 0.0, active_start: float = 0.0, wide_weights: bool = False,
                 giant_degree: int = 0, warp_limit: int = 0):
        L = lib()
        opts = _Opts()
        L.lv_default_opts(C.byref(opts))
        opts.device = device
        opts.max_sweeps = max_sweeps
        opts.profile = 1 if profile else 0
        opts.verify = 1 if verify else 0
        opts.trace = 1 if trace else 0
        opts.sweep_graph = 1 if sweep_graph else 0
        opts.active_set = 1 if active_set else 0
        opts.active_full_every = active_full_every
        opts.active_min_recall = active_min_recall
        opts.trace_sample = trace_sample
        opts.active_start = active_start
        opts.wide_weights = 1 if wide_weights else 0
        opts.giant_degree = giant_degree
        opts.warp_limit = warp_limit
        h = C.c_void_p()
        if device_csr is not None:
            rp, cl, w, V, E = device_csr
            _check(L.lv_create_device(C.c_void_p(rp), C.c_void_p(cl), C.c_void_p(w), V, E,
                                      C.byref(opts), C.byref(h)))
            self.V0 = V
        else:
            g = graph
            self._keep = g
            _check(L.lv_create(_ptr(g.rowptr, C.c_int32), _ptr(g.col, C.c_int32),
                               _ptr(g.w, C.c_float), g.V, g.E, C.byref(opts), C.byref(h)))
            self.V0 = g.V
        self._h = h

    # -- lifecycle --
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().lv_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, code: int) -> None:
        _check(code, self._h)

    def reset(self) -> None:
        self._c(lib().lv_reset(self._h))

    # -- reference operators --
    def optimise_modularity(self, min_gain: float) -> bool:
        ch = C.c_int32()
        self._c(lib().lv_optimise_level(self._h, min_gain, C.byref(ch)))
        return bool(ch.value)

    def aggregate_communities(self) -> None:
        self._c(lib().lv_aggregate(self._h))

    def calculate_modularity(self) -> float:
        q = C.c_double()
        self._c(lib().lv_modularity(self._h, C.byref(q)))
        return q.value

    def run(self, min_gain: float) -> float:
        q = C.c_double()
        self._c(lib().lv_run(self._h, min_gain, C.byref(q)))
        return q.value

    def sweep(self) -> int:
        m = C.c_int64()
        self._c(lib().lv_sweep(self._h, C.byref(m)))
        return m.value

    # -- state access --
    def level_info(self):
        V, E, lvl = C.c_int32(), C.c_int64(), C.c_int32()
        self._c(lib().lv_get_level_info(self._h, C.byref(V), C.byref(E), C.byref(lvl)))
        return V.value, E.value, lvl.value

    def original_to_community(self, out: np.ndarray | None = None):
        """(map, number of communities); out (int32, V0 entries, contiguous),
        e.g. a pinned buffer, receives the map instead of a new array."""
        if out is None:
            out = np.empty(self.V0, np.int32)
        elif out.dtype != np.int32 or out.shape != (self.V0,) or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous int32 array of V0 entries")
        nc = C.c_int32()
        self._c(lib().lv_get_original_to_community(self._h, _ptr(out, C.c_int32), C.byref(nc)))
        return out, nc.value

    def communities(self) -> np.ndarray:
        V, _, _ = self.level_info()
        out = np.empty(V, np.int32)
        self._c(lib().lv_get_communities(self._h, _ptr(out, C.c_int32)))
        return out

    def set_communities(self, comm) -> None:
        c = _i32(comm)
        self._c(lib().lv_set_communities(self._h, _ptr(c, C.c_int32)))

    def csr(self):
        """(rowptr int32, col int32, wfix int64) of the current level."""
        V, E, _ = self.level_info()
        rp = np.empty(V + 1, np.int32)
        cl = np.empty(E, np.int32)
        wf = np.empty(E, np.int64)
        self._c(lib().lv_get_csr(self._h, _ptr(rp, C.c_int32), _ptr(cl, C.c_int32), _ptr(wf, C.c_int64)))
        return rp, cl, wf

    def scale(self):
        s, t, ex = C.c_int32(), C.c_uint64(), C.c_int32()
        self._c(lib().lv_get_scale(self._h, C.byref(s), C.byref(t), C.byref(ex)))
        return s.value, t.value, bool(ex.value)

    def stats(self) -> dict:
        st = _Stats()
        self._c(lib().lv_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _Stats._fields_}

    def level_classes(self):
        """(vertices, entries) per work class of the current level."""
        v = np.zeros(NUM_CLASSES, np.int32)
        e = np.zeros(NUM_CLASSES, np.int64)
        self._c(lib().lv_get_level_classes(self._h, _ptr(v, C.c_int32), _ptr(e, C.c_int64)))
        return v, e

    def class_stats(self) -> dict:
        st = _ClassStats()
        self._c(lib().lv_get_class_stats(self._h, C.byref(st)))
        return {k: list(getattr(st, k)) for k, _ in _ClassStats._fields_}

    def clear_stats(self) -> None:
        self._c(lib().lv_clear_stats(self._h))

    def set_active_model(self, model, logit_threshold: float) -> None:
        """Predictor for active_set=True: ACTIVE_MODEL_SIZE bf16 bit patterns."""
        m = np.ascontiguousarray(model, dtype=np.uint16)
        self._c(lib().lv_set_active_model(self._h, _ptr(m, C.c_uint16), len(m), logit_threshold))

    def traces(self):
        """(features [n, ACTIVE_FEATURES] float32, labels [n] uint8) recorded with trace_sample > 0.

        The device appends the sampled rows in whatever order its threads get
        to them; the rows are returned sorted (by label, then feature bits),
        so that the same run gives the same arrays and a model trained on
        them is reproducible across processes."""
        n = C.c_int64()
        self._c(lib().lv_get_traces(self._h, None, None, 0, C.byref(n)))
        x = np.empty((n.value, ACTIVE_FEATURES), np.float32)
        y = np.empty(n.value, np.uint8)
        self._c(lib().lv_get_traces(self._h, _ptr(x, C.c_float), _ptr(y, C.c_uint8), n.value, C.byref(n)))
        if len(y) > 1:
            bits = x.view(np.uint32)
            order = np.lexsort(tuple(bits[:, j] for j in range(ACTIVE_FEATURES - 1, -1, -1)) + (y,))
            x, y = np.ascontiguousarray(x[order]), np.ascontiguousarray(y[order])
        return x, y

    def active_stats(self) -> dict:
        ev, fs, as_, fb = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        rc = C.c_double()
        self._c(lib().lv_get_active_stats(self._h, C.byref(ev), C.byref(fs), C.byref(as_), C.byref(rc),
                                          C.byref(fb)))
        return {"evaluated": ev.value, "full_sweeps": fs.value, "active_sweeps": as_.value,
                "last_recall": rc.value, "fell_back": bool(fb.value)}


# ---------------------------------------------------------------------------
# learned active-set predictor (lv_active_*)
# ---------------------------------------------------------------------------
ACTIVE_FEATURES = 5
ACTIVE_HIDDEN = 16
ACTIVE_MODEL_SIZE = ACTIVE_HIDDEN * ACTIVE_FEATURES + 2 * ACTIVE_HIDDEN + 1


def active_train(x, y, *, epochs: int = 4, batch: int = 8192, lr: float = 1e-2, pos_weight: float = 1.0,
                 seed: int = 0, device: int = 0):
    """Train the move predictor on traces; returns (bf16 model as uint16, per-epoch loss)."""
    xx = np.ascontiguousarray(x, dtype=np.float32)
    yy = np.ascontiguousarray(y, dtype=np.uint8)
    model = np.empty(ACTIVE_MODEL_SIZE, np.uint16)
    loss = np.empty(epochs, np.float32)
    _check(lib().lv_active_train(_ptr(xx, C.c_float), _ptr(yy, C.c_uint8), len(yy), epochs, batch, lr,
                                 pos_weight, seed, device, _ptr(model, C.c_uint16), _ptr(loss, C.c_float)))
    return model, loss


def active_predict(model, x, device: int = 0) -> np.ndarray:
    """Logits of the predictor (the engine's inference kernel) for features x [n, ACTIVE_FEATURES]."""
    m = np.ascontiguousarray(model, dtype=np.uint16)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(len(xx), np.float32)
    _check(lib().lv_active_predict(_ptr(m, C.c_uint16), _ptr(xx, C.c_float), len(xx), device,
                                   _ptr(out, C.c_float)))
    return out


def read_active_model(path: str | None = None):
    """The predictor file read by the library (lv_read_active_model, as the
    CLI's --mode learned reads it): (model uint16[ACTIVE_MODEL_SIZE], logit
    threshold, {"full_every", "active_start", "min_recall"} as they land in
    lv_opts)."""
    L = lib()
    path = path or os.path.join(_HERE, "active_set_lfr.json")
    m = np.zeros(ACTIVE_MODEL_SIZE, np.uint16)
    n, thr = C.c_int32(), C.c_float()
    opts = _Opts()
    L.lv_default_opts(C.byref(opts))
    _check(L.lv_read_active_model(path.encode(), _ptr(m, C.c_uint16), len(m), C.byref(n), C.byref(thr),
                                  C.byref(opts)))
    return m[:n.value], thr.value, {"full_every": opts.active_full_every, "active_start": opts.active_start,
                                    "min_recall": opts.active_min_recall, "active_set": opts.active_set}


def load_active_model(path: str | None = None):
    """(model uint16[ACTIVE_MODEL_SIZE], logit threshold) from a JSON file written by
    train_active_set.py (default: the packaged LFR model)."""
    import json
    path = path or os.path.join(_HERE, "active_set_lfr.json")
    with open(path) as f:
        d = json.load(f)
    return np.array(d["model_bf16"], dtype=np.uint16), float(d["logit_threshold"])


# ---------------------------------------------------------------------------
# batches of independent graphs (lv_batch_*)
# ---------------------------------------------------------------------------
def concat_graphs(graphs):
    """Block-diagonal CSR of a list of Graphs: (rowptr, col, w, graph_ptr)."""
    vs = np.array([g.V for g in graphs], dtype=np.int64)
    es = np.array([g.E for g in graphs], dtype=np.int64)
    gptr = np.zeros(len(graphs) + 1, dtype=np.int64)
    np.cumsum(vs, out=gptr[1:])
    eptr = np.zeros(len(graphs) + 1, dtype=np.int64)
    np.cumsum(es, out=eptr[1:])
    if gptr[-1] >= 2**31 - len(graphs) - 1 or eptr[-1] >= 2**31:
        raise ValueError("batch exceeds int32 vertex ids or entry offsets")
    rowptr = np.empty(int(gptr[-1]) + 1, dtype=np.int32)
    col = np.empty(int(eptr[-1]), dtype=np.int32)
    w = np.empty(int(eptr[-1]), dtype=np.float32)
    rowptr[0] = 0
    for i, g in enumerate(graphs):
        v0, v1, e0, e1 = int(gptr[i]), int(gptr[i + 1]), int(eptr[i]), int(eptr[i + 1])
        rowptr[v0 + 1:v1 + 1] = g.rowptr[1:] + e0
        col[e0:e1] = g.col + v0
        w[e0:e1] = g.w
    return rowptr, col, w, gptr.astype(np.int32)


class Batch:
    """Many independent graphs, each run through the level loop of lv_run in
    one persistent launch (lv_batch_run).  Build it from a list of Graphs or
    from a block-diagonal CSR plus graph_ptr (vertex offsets of the graphs);
    device_csr=(rowptr, col, w) device pointers borrows a resident CSR."""

    def __init__(self, graphs=None, *, rowptr=None, col=None, w=None, graph_ptr=None,
                 device: int = 0, max_sweeps: int = 0, device_csr: tuple | None = None,
                 num_vertices: int | None = None, num_entries: int | None = None):
        L = lib()
        opts = _Opts()
        L.lv_default_opts(C.byref(opts))
        opts.device = device
        opts.max_sweeps = max_sweeps
        if graphs is not None:
            rowptr, col, w, graph_ptr = concat_graphs(graphs)
        self.graph_ptr = _i32(graph_ptr)
        self.G = len(self.graph_ptr) - 1
        self._b = C.c_void_p()
        if device_csr is not None:
            d_rp, d_cl, d_w = device_csr
            self.V, self.E = int(num_vertices), int(num_entries)
            rc = L.lv_batch_create_device(C.c_void_p(d_rp), C.c_void_p(d_cl), C.c_void_p(d_w), self.V,
                                          self.E, _ptr(self.graph_ptr, C.c_int32), self.G,
                                          C.byref(opts), C.byref(self._b))
        else:
            rp, cl = _i32(rowptr), _i32(col)
            ww = np.ascontiguousarray(w, dtype=np.float32)
            self.V, self.E = len(rp) - 1, len(cl)
            rc = L.lv_batch_create(_ptr(rp, C.c_int32), _ptr(cl, C.c_int32), _ptr(ww, C.c_float),
                                   self.V, self.E, _ptr(self.graph_ptr, C.c_int32), self.G,
                                   C.byref(opts), C.byref(self._b))
        if rc != LV_OK:
            raise LouvainError(rc, status_string(rc))

    def _c(self, code: int) -> None:
        if code != LV_OK:
            detail = lib().lv_batch_last_error(self._b)
            raise LouvainError(code, status_string(code) + (f" ({detail.decode()})" if detail else ""))

    def close(self) -> None:
        if self._b:
            lib().lv_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, min_gain: float, check: bool = True) -> int:
        """Run every graph; returns the lv_status (raises unless check=False)."""
        rc = lib().lv_batch_run(self._b, min_gain)
        if check:
            self._c(rc)
        return rc

    def results(self) -> dict:
        comm = np.empty(self.V, np.int32)
        q = np.empty(self.G, np.float64)
        nc = np.empty(self.G, np.int32)
        st = np.empty(self.G, np.int32)
        self._c(lib().lv_batch_get_results(self._b, _ptr(comm, C.c_int32), _ptr(q, C.c_double),
                                           _ptr(nc, C.c_int32), _ptr(st, C.c_int32)))
        return {"communities": comm, "modularity": q, "num_communities": nc, "status": st}

    def graph_stats(self) -> dict:
        lv = np.empty(self.G, np.int32)
        sw = np.empty(self.G, np.int64)
        es = np.empty(self.G, np.int64)
        lat = np.empty(self.G, np.float64)
        self._c(lib().lv_batch_get_graph_stats(self._b, _ptr(lv, C.c_int32), _ptr(sw, C.c_int64),
                                               _ptr(es, C.c_int64), _ptr(lat, C.c_double)))
        return {"levels": lv, "sweeps": sw, "edge_sweeps": es, "latency_ms": lat}

    def stats(self) -> dict:
        ms, es, vs, ctas = C.c_double(), C.c_int64(), C.c_int64(), C.c_int32()
        self._c(lib().lv_batch_get_stats(self._b, C.byref(ms), C.byref(es), C.byref(vs), C.byref(ctas)))
        return {"device_ms": ms.value, "edge_sweeps": es.value, "vertex_sweeps": vs.value,
                "ctas": ctas.value}

    def split(self, communities: np.ndarray) -> list:
        """Per-graph views of a communities array."""
        return [communities[self.graph_ptr[g]:self.graph_ptr[g + 1]] for g in range(self.G)]


def assign_shards(entries, world: int) -> list:
    """Graphs of a batch over `world` GPUs: largest first, each to the GPU with
    the fewest entries so far (ties to the lower rank).  Returns one list of
    graph indices per rank, each in increasing order."""
    order = sorted(range(len(entries)), key=lambda g: (-int(entries[g]), g))
    load = [0] * world
    out = [[] for _ in range(world)]
    for g in order:
        r = min(range(world), key=lambda i: (load[i], i))
        out[r].append(g)
        load[r] += int(entries[g])
    return [sorted(x) for x in out]


def _run_local(graphs, min_gain, device, max_sweeps):
    b = Batch(graphs, device=device, max_sweeps=max_sweeps)
    try:
        b.run(min_gain, check=False)
        r = b.results()
        gs = b.graph_stats()
        parts = b.split(r["communities"])
        return [{"communities": parts[i].copy(), "modularity": float(r["modularity"][i]),
                 "num_communities": int(r["num_communities"][i]), "status": int(r["status"][i]),
                 "levels": int(gs["levels"][i]), "sweeps": int(gs["sweeps"][i]),
                 "edge_sweeps": int(gs["edge_sweeps"][i]), "latency_ms": float(gs["latency_ms"][i])}
                for i in range(len(graphs))]
    finally:
        b.close()


def run_batch_sharded(graphs, min_gain: float, *, max_sweeps: int = 0, device: int | None = None,
                      runner=None) -> list:
    """Run a batch of graphs over all ranks of the default torch.distributed
    process group: each rank runs its shard (assign_shards, by entry count) as
    one lv_batch on its GPU, and every rank gets all graphs' results in input
    order.  Graphs are independent, so the only exchange is the final gather of
    results.  runner(graphs, min_gain, device, max_sweeps) -> list of per-graph
    dicts replaces the local lv_batch run (for tests)."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    if device is None:
        device = int(os.environ.get("LOCAL_RANK", "0"))
    mine = assign_shards([g.E for g in graphs], world)[rank]
    res = (runner or _run_local)([graphs[i] for i in mine], min_gain, device, max_sweeps)
    local = list(zip(mine, res))
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    else:
        gathered = [local]
    out = [None] * len(graphs)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out


def tune(graph=None, **kw) -> dict:
    """Choose the work-mapping knobs for a graph on this GPU (autotune.tune)."""
    import importlib
    return importlib.import_module(__name__ + ".autotune").tune(graph, **kw)
