"""lpa_b200 -- synchronous label propagation over CGR-compressed graphs on B200.

Python mirror of the library's C ABI (include/lpa_capi.h), used by the tests,
the benchmark and scripting.  The compute path is the native library
``liblpa_b200.so`` (hand-written sm_100a kernels); importing this module never
falls back to a CPU implementation -- if the library is missing, every call
raises.

Reference counterparts (paths inside the reference project):
  * ``LabelPropagator`` mirrors ``LabelPropagator<V,E>`` / ``NovaPlusPropagator``
    (include/label_propagator.h:11-38, baselines/novaplus/novaplus_propogator.cuh:
    24-199): ``run(niter) -> (lp_ms, total_ms)`` and ``get_labels()``.
  * ``HostGraph`` covers ``File`` and ``CgrCompressor`` (include/file.h:28-76,
    include/compressor.h:23-138).
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import time
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "liblpa_b200.so"
METHOD_PATH = _PKG / "bin" / "method"

_lib = None


class Status(enum.IntEnum):
    OK = 0
    CUDA = 1
    OOM = 2
    BAD_STREAM = 3
    TIMEOUT = 4
    INVALID_ARG = 5
    IO = 6
    NO_DEVICE = 7
    CAPACITY = 8


class Variant(enum.IntEnum):
    WARP = 0
    PACKED = 1
    BLOCK = 2
    TWO_PASS = 3


class Dispatch(enum.IntEnum):
    FIXED = 0
    LEARNED = 1
    FORCE = 2


class LpaError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = Status(status) if status in Status._value2member_map_ else status
        msg = f"{what}: {lib().lpa_status_str(status).decode()}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class Tune(C.Structure):
    """Work shapes of the two-pass count pass (lpa_tune)."""
    _fields_ = [
        ("group_positions", C.c_uint32),
        ("warp_positions", C.c_uint32),
        ("warp_max_degree", C.c_uint32),
        ("warp_claim", C.c_uint32),
        ("bulk_stage", C.c_uint32),
        ("gather_cache", C.c_uint32),
        ("stage_stream", C.c_uint32),
    ]

    def as_tuple(self):
        return (self.group_positions, self.warp_positions, self.warp_max_degree, self.warp_claim, self.bulk_stage,
                self.gather_cache, self.stage_stream)


class GraphDesc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_compressed", C.c_uint64),
        ("words", C.POINTER(C.c_uint32)),
        ("num_words", C.c_uint64),
        ("offsets", C.POINTER(C.c_uint64)),
        ("vertices", C.POINTER(C.c_uint32)),
        ("small_graph", C.POINTER(C.c_uint32)),
        ("num_small_arcs", C.c_uint64),
        ("small_offset", C.POINTER(C.c_uint32)),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("cms_threshold", C.c_uint32),
        ("cms_seed", C.c_uint64),
        ("dispatch", C.c_int),
        ("force_variant", C.c_int),
        ("stream", C.c_void_p),
        ("record_timings", C.c_int),
        ("verbose", C.c_int),
        ("batch_mode", C.c_int),
        ("queue_wait_limit", C.c_uint64),
        ("stream_budget", C.c_uint64),
    ]


class BatchMode(enum.IntEnum):
    LOCKSTEP = 0  # the batch concatenated into one graph, run by one handle
    QUEUE = 1  # one persistent launch fed by a device work queue


class Info(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_compressed", C.c_uint64),
        ("num_arcs", C.c_uint64),
        ("num_small_arcs", C.c_uint64),
        ("stream_bits", C.c_uint64),
        ("num_segments", C.c_uint64),
        ("max_degree", C.c_uint64),
        ("bytes_algorithmic", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64),
        ("last_changed", C.c_uint64),
        ("last_iter_ms", C.c_double),
        ("variant_ms", C.c_double * 4),
        ("variant_segments", C.c_uint64 * 4),
        ("variant_arcs", C.c_uint64 * 4),
        ("mlp_loss", C.c_double),
        ("mlp_updates", C.c_uint64),
        ("dispatch_reverts", C.c_uint64),
        ("learned_active", C.c_int),
        ("launches", C.c_uint64),
        ("decode_ms", C.c_double),
        ("iterate_ms", C.c_double),
        ("count_ms", C.c_double),
        ("packed_ms", C.c_double),
        ("stream_ranges", C.c_uint64),
        ("stream_bytes", C.c_uint64),
    ]


def _sig(lib_, name, argtypes, restype=C.c_int):
    f = getattr(lib_, name)
    f.argtypes = argtypes
    f.restype = restype


def lib():
    """Loads liblpa_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lpa_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    PP = C.POINTER(C.c_void_p)
    u32p, u64p, u8p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint8)
    _sig(L, "lpa_status_str", [C.c_int], C.c_char_p)
    _sig(L, "lpa_version", [], C.c_char_p)
    _sig(L, "lpa_opts_default", [C.POINTER(Opts)], None)
    _sig(L, "lpa_create", [C.POINTER(GraphDesc), C.POINTER(Opts), PP])
    _sig(L, "lpa_destroy", [P])
    _sig(L, "lpa_get_info", [P, C.POINTER(Info)])
    _sig(L, "lpa_last_error", [P], C.c_char_p)
    _sig(L, "lpa_init_labels", [P])
    _sig(L, "lpa_set_labels", [P, u32p, C.c_size_t])
    _sig(L, "lpa_iterate", [P, u64p])
    _sig(L, "lpa_run", [P, C.c_int, C.c_int, C.POINTER(C.c_int)])
    _sig(L, "lpa_get_changed_history", [P, u64p, C.c_size_t])
    _sig(L, "lpa_get_labels", [P, u32p, C.c_size_t])
    _sig(L, "lpa_get_stats", [P, C.POINTER(Stats)])
    _sig(L, "lpa_decode_csr", [P, u64p, u32p])
    _sig(L, "lpa_get_degrees", [P, u32p, C.c_size_t])
    _sig(L, "lpa_set_dispatch", [P, C.c_int, C.c_int])
    _sig(L, "lpa_set_plan", [P, C.POINTER(C.c_uint8), C.c_size_t])
    _sig(L, "lpa_get_tune", [P, C.POINTER(Tune)])
    _sig(L, "lpa_set_tune", [P, C.POINTER(Tune)])
    _sig(L, "lpa_autotune", [P, C.c_char_p, C.c_int, C.POINTER(Tune)])
    _sig(L, "lpa_get_segments", [P, u32p, u32p, u8p, u8p, C.c_size_t])
    _sig(L, "lpa_hg_generate_road", [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_int, C.c_uint64, PP])
    _sig(L, "lpa_hg_generate_rmat", [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                     C.c_int, C.c_uint64, PP])
    _sig(L, "lpa_hg_generate_copy", [C.c_uint64, C.c_uint32, C.c_double, C.c_int, C.c_double, C.c_uint64, PP])
    _sig(L, "lpa_hg_from_csr", [C.c_uint64, u64p, u32p, PP])
    _sig(L, "lpa_hg_read_edge_list", [C.c_char_p, C.c_int, PP])
    _sig(L, "lpa_hg_write_edge_list", [P, C.c_char_p, C.c_int])
    _sig(L, "lpa_hg_compress", [P, C.c_int, C.c_int, C.c_int])
    _sig(L, "lpa_hg_compress_gpu", [P, C.c_int, C.c_int, C.c_int])
    _sig(L, "lpa_hg_load_cgr", [C.c_char_p, C.c_int, PP])
    _sig(L, "lpa_hg_write_cgr", [P, C.c_char_p])
    _sig(L, "lpa_hg_write_csr", [P, C.c_char_p])
    _sig(L, "lpa_hg_csr", [P, u64p, C.POINTER(u64p), C.POINTER(u32p)])
    _sig(L, "lpa_hg_desc", [P, C.POINTER(GraphDesc)])
    _sig(L, "lpa_hg_free", [P])
    _sig(L, "lpa_hg_concat", [C.POINTER(GraphDesc), C.c_size_t, PP])
    fp = C.POINTER(C.c_float)
    _sig(L, "lpa_mlp_gradient", [C.c_int, fp, fp, u8p, fp, C.c_size_t, fp, fp])
    _sig(L, "lpa_mlp_predict", [C.c_int, fp, fp, C.c_size_t, fp])
    _sig(L, "lpa_get_mlp", [P, fp, C.c_size_t])
    _sig(L, "lpa_get_learned_plan", [P, u8p, fp, C.c_size_t])
    _sig(L, "lpa_get_segment_cycles", [P, u64p, C.c_size_t])
    _sig(L, "lpa_get_mlp_plan", [P, u8p, C.c_size_t])
    _sig(L, "lpa_get_capable", [P, u8p, C.c_size_t])
    _sig(L, "lpa_batch_create", [C.POINTER(GraphDesc), C.c_size_t, C.POINTER(Opts), PP])
    _sig(L, "lpa_batch_run", [P, C.c_int, C.c_int, u32p])
    _sig(L, "lpa_batch_get_labels", [P, C.c_size_t, u32p, C.c_size_t])
    _sig(L, "lpa_batch_destroy", [P])
    _sig(L, "lpa_batch_handle", [P], C.c_void_p)
    _lib = L
    return L


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def _check(st: int, what: str, handle=None):
    if st != 0:
        detail = ""
        if handle is not None:
            detail = lib().lpa_last_error(handle).decode(errors="replace")
        raise LpaError(st, what, detail)


def _view(ptr, count: int, dtype) -> np.ndarray:
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(int(count),)).copy()


class HostGraph:
    """A host graph: CSR by vertex id and/or its CGR-compressed form.

    Covers the reference's File (ingest, caching files) and CgrCompressor
    (include/file.h:28-76, include/compressor.h:23-138).  Compression is the
    fast bit-identical parallel encoder.
    """

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def __del__(self):
        try:
            if self._h:
                lib().lpa_hg_free(self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    @staticmethod
    def _make(fn, *args) -> "HostGraph":
        out = C.c_void_p()
        _check(fn(*args, C.byref(out)), fn.__name__)
        return HostGraph(out.value)

    @classmethod
    def road(cls, width, height, keep_p=0.7, extra_p=0.02, max_dist=3, seed=1):
        return cls._make(lib().lpa_hg_generate_road, width, height, keep_p, extra_p, max_dist, seed)

    @classmethod
    def rmat(cls, scale, edge_factor=16.0, a=0.57, b=0.19, c=0.19, seed=1, bfs_relabel=True, n_limit=0):
        return cls._make(lib().lpa_hg_generate_rmat, scale, edge_factor, a, b, c, seed, int(bfs_relabel),
                         n_limit)

    @classmethod
    def copy_model(cls, n, out_degree=30, copy_p=0.6, copy_offset=8, zipf_s=1.1, seed=1):
        return cls._make(lib().lpa_hg_generate_copy, n, out_degree, copy_p, copy_offset, zipf_s, seed)

    @classmethod
    def from_csr(cls, row: np.ndarray, clm: np.ndarray):
        row = np.ascontiguousarray(row, dtype=np.uint64)
        clm = np.ascontiguousarray(clm, dtype=np.uint32)
        return cls._make(lib().lpa_hg_from_csr, len(row) - 1, _ptr(row, C.c_uint64), _ptr(clm, C.c_uint32))

    @classmethod
    def concat(cls, graphs):
        """Compressed graphs as one (lpa_hg_concat): graph k's ids shifted by the
        vertex counts before it, bitstreams joined bit for bit."""
        descs = [g.desc() if isinstance(g, HostGraph) else g for g in graphs]
        arr = (GraphDesc * len(descs))()
        for i, d in enumerate(descs):
            C.memmove(C.byref(arr, i * C.sizeof(GraphDesc)), C.byref(d), C.sizeof(GraphDesc))
        out = C.c_void_p()
        _check(lib().lpa_hg_concat(arr, len(descs), C.byref(out)), "lpa_hg_concat")
        return HostGraph(out.value)

    @classmethod
    def read_edge_list(cls, path, one_way: bool):
        return cls._make(lib().lpa_hg_read_edge_list, str(path).encode(), int(one_way))

    @classmethod
    def load_cgr(cls, base, small_thresh: int):
        return cls._make(lib().lpa_hg_load_cgr, str(base).encode(), small_thresh)

    def write_edge_list(self, path, both_arcs: bool):
        _check(lib().lpa_hg_write_edge_list(self._h, str(path).encode(), int(both_arcs)), "write_edge_list")

    def compress(self, small_thresh=0, large_thresh=128, threads=0, device=None):
        """CGR-compress the CSR on the host (threads) or, with device, on that GPU."""
        if device is None:
            _check(lib().lpa_hg_compress(self._h, small_thresh, large_thresh, threads), "compress")
        else:
            _check(lib().lpa_hg_compress_gpu(self._h, small_thresh, large_thresh, int(device)), "compress_gpu")
        return self

    def write_cgr(self, base):
        _check(lib().lpa_hg_write_cgr(self._h, str(base).encode()), "write_cgr")

    def write_csr(self, base):
        _check(lib().lpa_hg_write_csr(self._h, str(base).encode()), "write_csr")

    def csr(self):
        n = C.c_uint64()
        row = C.POINTER(C.c_uint64)()
        clm = C.POINTER(C.c_uint32)()
        _check(lib().lpa_hg_csr(self._h, C.byref(n), C.byref(row), C.byref(clm)), "csr")
        r = _view(row, n.value + 1, np.uint64)
        return r, _view(clm, int(r[-1]) if len(r) else 0, np.uint32)

    def num_arcs(self) -> int:
        """Stored arcs of the CSR (no copy)."""
        n = C.c_uint64()
        row = C.POINTER(C.c_uint64)()
        clm = C.POINTER(C.c_uint32)()
        _check(lib().lpa_hg_csr(self._h, C.byref(n), C.byref(row), C.byref(clm)), "csr")
        return int(row[n.value])

    def desc(self) -> GraphDesc:
        d = GraphDesc()
        _check(lib().lpa_hg_desc(self._h, C.byref(d)), "desc")
        d._owner = self  # keep the arrays alive
        return d

    def arrays(self) -> dict:
        """Copies of the compressed arrays (words, offsets, vertices, small CSR)."""
        d = self.desc()
        n, n_c = d.num_vertices, d.num_compressed
        return {
            "n": int(n),
            "n_c": int(n_c),
            "words": _view(d.words, d.num_words, np.uint32),
            "offsets": _view(d.offsets, n_c + 1, np.uint64),
            "vertices": _view(d.vertices, n, np.uint32),
            "small_graph": _view(d.small_graph, d.num_small_arcs, np.uint32),
            "small_offset": _view(d.small_offset, n - n_c + 1, np.uint32) if n > n_c else
            np.zeros(1, np.uint32),
        }


def desc_from_arrays(arr: dict) -> GraphDesc:
    """A GraphDesc over numpy arrays (kept alive by the returned object)."""
    keep = {k: np.ascontiguousarray(v) for k, v in arr.items() if isinstance(v, np.ndarray)}
    d = GraphDesc()
    d.num_vertices = arr["n"]
    d.num_compressed = arr["n_c"]
    d.words = _ptr(keep["words"], C.c_uint32)
    d.num_words = len(keep["words"])
    d.offsets = _ptr(keep["offsets"], C.c_uint64)
    d.vertices = _ptr(keep["vertices"], C.c_uint32)
    d.small_graph = _ptr(keep["small_graph"], C.c_uint32)
    d.num_small_arcs = len(keep["small_graph"])
    d.small_offset = _ptr(keep["small_offset"], C.c_uint32) if arr["n"] > arr["n_c"] else None
    d._keep = keep
    return d


def default_opts(**kw) -> Opts:
    o = Opts()
    lib().lpa_opts_default(C.byref(o))
    for k, v in kw.items():
        if k == "dispatch":
            v = int(v)
        setattr(o, k, v)
    return o


class Propagator:
    """One device-resident graph and its label buffers (C ABI lpa_handle)."""

    def __init__(self, graph, **opts):
        desc = graph.desc() if isinstance(graph, HostGraph) else graph
        self._desc = desc
        o = default_opts(**opts)
        out = C.c_void_p()
        st = lib().lpa_create(C.byref(desc), C.byref(o), C.byref(out))
        _check(st, "lpa_create")
        self._h = out
        self.info = self.get_info()
        self.n = int(self.info.num_vertices)

    def close(self):
        if getattr(self, "_owner", None) is not None:  # a batch's handle: the batch frees it
            self._h = None
            self._owner = None
        if getattr(self, "_h", None):
            lib().lpa_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, st, what):
        _check(st, what, self._h)

    def get_info(self) -> Info:
        i = Info()
        self._chk(lib().lpa_get_info(self._h, C.byref(i)), "lpa_get_info")
        return i

    def init_labels(self):
        self._chk(lib().lpa_init_labels(self._h), "lpa_init_labels")

    def set_labels(self, labels: np.ndarray):
        a = np.ascontiguousarray(labels, dtype=np.uint32)
        self._chk(lib().lpa_set_labels(self._h, _ptr(a, C.c_uint32), len(a)), "lpa_set_labels")

    def iterate(self) -> int:
        c = C.c_uint64()
        self._chk(lib().lpa_iterate(self._h, C.byref(c)), "lpa_iterate")
        return int(c.value)

    def run(self, max_iter: int, early_exit: bool = False) -> int:
        done = C.c_int()
        self._chk(lib().lpa_run(self._h, max_iter, int(early_exit), C.byref(done)), "lpa_run")
        return int(done.value)

    def changed_history(self, count: int) -> np.ndarray:
        out = np.zeros(count, np.uint64)
        self._chk(lib().lpa_get_changed_history(self._h, _ptr(out, C.c_uint64), count), "history")
        return out

    def labels(self) -> np.ndarray:
        out = np.empty(self.n, np.uint32)
        self._chk(lib().lpa_get_labels(self._h, _ptr(out, C.c_uint32), self.n), "lpa_get_labels")
        return out

    def degrees(self) -> np.ndarray:
        out = np.empty(self.n, np.uint32)
        self._chk(lib().lpa_get_degrees(self._h, _ptr(out, C.c_uint32), self.n), "lpa_get_degrees")
        return out

    def decode_csr(self):
        row = np.empty(self.n + 1, np.uint64)
        clm = np.empty(max(1, int(self.info.num_arcs)), np.uint32)
        self._chk(lib().lpa_decode_csr(self._h, _ptr(row, C.c_uint64), _ptr(clm, C.c_uint32)), "lpa_decode_csr")
        return row, clm[: int(self.info.num_arcs)]

    def stats(self) -> Stats:
        s = Stats()
        self._chk(lib().lpa_get_stats(self._h, C.byref(s)), "lpa_get_stats")
        return s

    def set_dispatch(self, dispatch, force_variant=Variant.BLOCK):
        self._chk(lib().lpa_set_dispatch(self._h, int(dispatch), int(force_variant)), "lpa_set_dispatch")

    def mlp_params(self) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, np.float32)
        self._chk(lib().lpa_get_mlp(self._h, _ptr(out, C.c_float), MLP_PARAMS), "lpa_get_mlp")
        return out

    def set_plan(self, plan):
        a = np.ascontiguousarray(plan, dtype=np.uint8)
        self._chk(lib().lpa_set_plan(self._h, _ptr(a, C.c_uint8), len(a)), "lpa_set_plan")

    def get_tune(self) -> Tune:
        t = Tune()
        self._chk(lib().lpa_get_tune(self._h, C.byref(t)), "lpa_get_tune")
        return t

    def set_tune(self, group_positions, warp_positions, warp_max_degree, warp_claim, bulk_stage=0, gather_cache=0,
                 stage_stream=0):
        t = Tune(group_positions, warp_positions, warp_max_degree, warp_claim, bulk_stage, gather_cache, stage_stream)
        self._chk(lib().lpa_set_tune(self._h, C.byref(t)), "lpa_set_tune")

    def autotune(self, cache_path=None, repeats=2) -> Tune:
        t = Tune()
        path = None if cache_path is None else str(cache_path).encode()
        self._chk(lib().lpa_autotune(self._h, path, int(repeats), C.byref(t)), "lpa_autotune")
        return t

    def learned_plan(self):
        k = int(self.get_info().num_segments)
        plan = np.zeros(k, np.uint8)
        pred = np.zeros((k, 4), np.float32)
        self._chk(lib().lpa_get_learned_plan(self._h, _ptr(plan, C.c_uint8), _ptr(pred, C.c_float), k),
                  "lpa_get_learned_plan")
        return plan, pred

    def mlp_plan(self) -> np.ndarray:
        """The cost model's own plan (before the learner's trials)."""
        k = int(self.get_info().num_segments)
        plan = np.zeros(k, np.uint8)
        self._chk(lib().lpa_get_mlp_plan(self._h, _ptr(plan, C.c_uint8), k), "lpa_get_mlp_plan")
        return plan

    def current_plan(self) -> np.ndarray:
        """The variant of every segment as the next iteration will run it."""
        return self.segments()[3]

    def capable(self) -> np.ndarray:
        """Per segment, a bit mask of the variants that can run it."""
        k = int(self.get_info().num_segments)
        m = np.zeros(k, np.uint8)
        self._chk(lib().lpa_get_capable(self._h, _ptr(m, C.c_uint8), k), "lpa_get_capable")
        return m

    def segment_cycles(self) -> np.ndarray:
        k = int(self.get_info().num_segments)
        out = np.zeros(k, np.uint64)
        self._chk(lib().lpa_get_segment_cycles(self._h, _ptr(out, C.c_uint64), k), "lpa_get_segment_cycles")
        return out

    def segments(self):
        k = int(self.get_info().num_segments)
        b = np.empty(k, np.uint32)
        e = np.empty(k, np.uint32)
        bk = np.empty(k, np.uint8)
        v = np.empty(k, np.uint8)
        self._chk(lib().lpa_get_segments(self._h, _ptr(b, C.c_uint32), _ptr(e, C.c_uint32), _ptr(bk, C.c_uint8),
                                         _ptr(v, C.c_uint8), k), "lpa_get_segments")
        return b, e, bk, v


MLP_PARAMS = 1412


def mlp_gradient(params, x, variant, target, device=0):
    """Gradient of the dispatch cost model, computed by the library's GPU kernel."""
    P = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(x, np.float32)
    V = np.ascontiguousarray(variant, np.uint8)
    T = np.ascontiguousarray(target, np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = C.c_float()
    _check(lib().lpa_mlp_gradient(device, _ptr(P, C.c_float), _ptr(X, C.c_float), _ptr(V, C.c_uint8),
                                  _ptr(T, C.c_float), len(T), _ptr(g, C.c_float), C.byref(loss)), "lpa_mlp_gradient")
    return g, float(loss.value)


def mlp_predict(params, x, device=0):
    P = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(x, np.float32)
    out = np.zeros((len(X), 4), np.float32)
    _check(lib().lpa_mlp_predict(device, _ptr(P, C.c_float), _ptr(X, C.c_float), len(X), _ptr(out, C.c_float)),
           "lpa_mlp_predict")
    return out


class Batch:
    """Many graphs propagated together, each with its own convergence test
    (lpa_batch_*).  ``batch_mode`` (BatchMode) picks lockstep, the default, or
    the persistent queue."""

    def __init__(self, graphs, **opts):
        if "batch_mode" in opts:
            opts["batch_mode"] = int(opts["batch_mode"])
        descs = [g.desc() if isinstance(g, HostGraph) else g for g in graphs]
        arr = (GraphDesc * len(descs))()
        for i, d in enumerate(descs):
            C.memmove(C.byref(arr, i * C.sizeof(GraphDesc)), C.byref(d), C.sizeof(GraphDesc))
        self._keep = (graphs, descs, arr)
        self.n = [int(d.num_vertices) for d in descs]
        o = default_opts(**opts)
        out = C.c_void_p()
        _check(lib().lpa_batch_create(arr, len(descs), C.byref(o), C.byref(out)), "lpa_batch_create")
        self._h = out

    def run(self, max_iter: int, early_exit: bool = True) -> np.ndarray:
        iters = np.zeros(len(self.n), np.uint32)
        _check(lib().lpa_batch_run(self._h, max_iter, int(early_exit), _ptr(iters, C.c_uint32)), "lpa_batch_run")
        return iters

    def labels(self, i: int) -> np.ndarray:
        out = np.empty(self.n[i], np.uint32)
        _check(lib().lpa_batch_get_labels(self._h, i, _ptr(out, C.c_uint32), self.n[i]), "lpa_batch_get_labels")
        return out

    def handle(self):
        """The lockstep batch's concatenated graph as a Propagator that the batch
        owns (autotune, set_dispatch, stats, info); None in queue mode."""
        h = lib().lpa_batch_handle(self._h)
        if not h:
            return None
        p = Propagator.__new__(Propagator)
        p._desc = None
        p._h = C.c_void_p(h)
        p._owner = self
        p.info = p.get_info()
        p.n = int(p.info.num_vertices)
        return p

    def close(self):
        if getattr(self, "_h", None):
            lib().lpa_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class LabelPropagator:
    """Mirror of the reference's propagator interface
    (include/label_propagator.h:11-38; baselines/novaplus/novaplus_propogator.cuh:100-129):
    ``run(niter)`` returns ``(lp_ms, preprocess_plus_lp_ms)`` and ``get_labels()``
    returns the labels by vertex id."""

    def __init__(self, graph, **opts):
        self._graph = graph
        self._opts = opts
        self._p = None

    def run(self, niter: int):
        t0 = time.perf_counter()
        if self._p is None:
            self._p = Propagator(self._graph, **self._opts)
        self._p.init_labels()
        t1 = time.perf_counter()
        self._p.run(niter)
        t2 = time.perf_counter()
        return (t2 - t1) * 1e3, (t2 - t0) * 1e3

    def get_labels(self) -> np.ndarray:
        return self._p.labels()
