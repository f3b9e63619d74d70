"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over oracle/liboracle.so, the plain-C restatement of the
reference's CGR decode (include/graph_utils.cuh:19-180) and of the synchronous
label-propagation update rule (see oracle/oracle.h for every reference citation).
Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the product (lpa_b200) never does.

Also reads the reference's on-disk files with numpy (src/file.cpp:197-262 word
packing, .offset text) so fixtures produced by the reference compressor can be
checked without the product library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "cgr_ref"

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        u32p, u64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
        L.orc_decode_vertex.argtypes = [u32p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, u32p, C.c_uint64]
        L.orc_decode_vertex.restype = C.c_int64
        L.orc_vertex_degree.argtypes = [u32p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32]
        L.orc_vertex_degree.restype = C.c_int64
        L.orc_decode_csr.argtypes = [u32p, C.c_uint64, u64p, C.c_uint64, u32p, C.c_uint64, u32p, u32p, u64p, u32p]
        L.orc_decode_csr.restype = C.c_int64
        L.orc_cms_index.argtypes = [C.c_int, C.c_uint32, C.c_uint32]
        L.orc_cms_index.restype = C.c_uint32
        L.orc_cms_seeds.argtypes = [C.c_uint64, u32p]
        L.orc_cms_seeds.restype = None
        L.orc_lp_iterate_csr.argtypes = [u64p, u32p, C.c_uint64, u32p, u32p, C.c_uint64, C.c_uint64, C.c_int]
        L.orc_lp_iterate_csr.restype = C.c_uint64
        L.orc_lp_iterate_cgr.argtypes = [u32p, C.c_uint64, u64p, C.c_uint64, u32p, C.c_uint64, u32p, u32p, u32p,
                                         u32p, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64, C.c_uint64]
        L.orc_lp_iterate_cgr.restype = C.c_uint64
        L.orc_range_arcs.argtypes = [u32p, C.c_uint64, u64p, C.c_uint64, u32p, u32p, C.c_uint64, C.c_uint64]
        L.orc_range_arcs.restype = C.c_uint64
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


# --------------------------------------------------------------- file reading --
def read_reference_files(base) -> dict:
    """The reference's compressed files as arrays (File::load_compress_graph,
    src/file.cpp:197-262, with 64-bit offsets) plus .row/.clm when present."""
    base = str(base)
    raw = np.fromfile(base + ".graph", dtype=np.uint8)
    pad = (-len(raw)) % 4
    words = np.frombuffer(np.concatenate([raw, np.zeros(pad + 16, np.uint8)]).tobytes(), dtype=">u4")
    words = words.astype(np.uint32)
    txt = Path(base + ".offset").read_text().split()
    cnt = int(txt[0])
    offsets = np.zeros(cnt + 1, np.uint64)
    offsets[1:] = np.array([int(x) for x in txt[1:1 + cnt]], dtype=np.uint64)
    vertices = np.fromfile(base + ".vertices.bin", dtype=np.uint32)
    n = len(vertices)
    if os.path.exists(base + ".graph.small.bin"):
        small_graph = np.fromfile(base + ".graph.small.bin", dtype=np.uint32)
        small_offset = np.fromfile(base + ".offset.small.bin", dtype=np.uint32)
    else:
        small_graph = np.zeros(0, np.uint32)
        small_offset = np.zeros(n - cnt + 1, np.uint32)
    out = {"n": n, "n_c": cnt, "words": words, "offsets": offsets, "vertices": vertices,
           "small_graph": small_graph, "small_offset": small_offset}
    if os.path.exists(base + ".row"):
        out["row"] = np.fromfile(base + ".row", dtype=np.uint32).astype(np.uint64)
        out["clm"] = np.fromfile(base + ".clm", dtype=np.uint32)
    return out


# ------------------------------------------------------------------- decode --
def decode_vertex(arr: dict, p: int) -> np.ndarray:
    w = _u32(arr["words"])
    off = arr["offsets"]
    cap = 1 << 20
    out = np.zeros(cap, np.uint32)
    r = lib().orc_decode_vertex(_p(w, C.c_uint32), len(w), int(off[p]), int(off[p + 1]),
                                int(arr["vertices"][p]), _p(out, C.c_uint32), cap)
    if r < 0:
        raise ValueError(f"malformed stream at position {p} ({r})")
    return out[:r].copy()


def decode_csr(arr: dict):
    """(row, clm) by vertex id, lists sorted ascending (the reference .clm order)."""
    w, off, vert = _u32(arr["words"]), _u64(arr["offsets"]), _u32(arr["vertices"])
    sg, so = _u32(arr["small_graph"]), _u32(arr["small_offset"])
    n, n_c = int(arr["n"]), int(arr["n_c"])
    row = np.zeros(n + 1, np.uint64)
    m = lib().orc_decode_csr(_p(w, C.c_uint32), len(w), _p(off, C.c_uint64), n_c, _p(vert, C.c_uint32), n,
                             _p(sg, C.c_uint32), _p(so, C.c_uint32), _p(row, C.c_uint64), None)
    if m < 0:
        raise ValueError("malformed stream")
    clm = np.zeros(max(1, m), np.uint32)
    m2 = lib().orc_decode_csr(_p(w, C.c_uint32), len(w), _p(off, C.c_uint64), n_c, _p(vert, C.c_uint32), n,
                              _p(sg, C.c_uint32), _p(so, C.c_uint32), _p(row, C.c_uint64), _p(clm, C.c_uint32))
    if m2 != m:
        raise ValueError("malformed stream")
    return row, clm[:m]


# ------------------------------------------------------------------------ LP --
def cms_seeds(seed: int) -> np.ndarray:
    out = np.zeros(4, np.uint32)
    lib().orc_cms_seeds(seed, _p(out, C.c_uint32))
    return out


def cms_index(r: int, key: int, seed_r: int) -> int:
    return int(lib().orc_cms_index(r, key, seed_r))


def lp_iterate_csr(row, clm, labels, cms_thr=0, cms_seed=1, threads=0):
    row, clm, lab = _u64(row), _u32(clm), _u32(labels)
    out = np.empty_like(lab)
    ch = lib().orc_lp_iterate_csr(_p(row, C.c_uint64), _p(clm, C.c_uint32), len(lab), _p(lab, C.c_uint32),
                                  _p(out, C.c_uint32), cms_thr, cms_seed, threads)
    return out, int(ch)


def lp_iterate_cgr(arr: dict, labels, cms_thr=0, cms_seed=1, threads=0, pos_begin=0, pos_end=None):
    w, off, vert = _u32(arr["words"]), _u64(arr["offsets"]), _u32(arr["vertices"])
    sg, so = _u32(arr["small_graph"]), _u32(arr["small_offset"])
    lab = _u32(labels)
    out = lab.copy()
    n = int(arr["n"])
    pos_end = n if pos_end is None else pos_end
    ch = lib().orc_lp_iterate_cgr(_p(w, C.c_uint32), len(w), _p(off, C.c_uint64), int(arr["n_c"]),
                                  _p(vert, C.c_uint32), n, _p(sg, C.c_uint32), _p(so, C.c_uint32),
                                  _p(lab, C.c_uint32), _p(out, C.c_uint32), cms_thr, cms_seed, threads,
                                  pos_begin, pos_end)
    if ch == (1 << 64) - 1:
        raise ValueError("malformed stream")
    return out, int(ch)


def range_arcs(arr: dict, pos_begin: int, pos_end: int) -> int:
    w, off, vert, so = _u32(arr["words"]), _u64(arr["offsets"]), _u32(arr["vertices"]), _u32(arr["small_offset"])
    r = lib().orc_range_arcs(_p(w, C.c_uint32), len(w), _p(off, C.c_uint64), int(arr["n_c"]), _p(vert, C.c_uint32),
                             _p(so, C.c_uint32), pos_begin, pos_end)
    if r == (1 << 64) - 1:
        raise ValueError("malformed stream")
    return int(r)


def lp_run(row, clm, iters, cms_thr=0, cms_seed=1, labels=None, early_exit=False):
    """Labels after each iteration (list), starting from labels (default identity)."""
    n = len(row) - 1
    lab = np.arange(n, dtype=np.uint32) if labels is None else _u32(labels)
    hist, changed = [], []
    for _ in range(iters):
        lab, ch = lp_iterate_csr(row, clm, lab, cms_thr, cms_seed)
        hist.append(lab)
        changed.append(ch)
        if early_exit and ch == 0:
            break
    return hist, changed


# ------------------------------------------------- pure-python restatement --
def lp_iterate_py(row, clm, labels, cms_thr=0, cms_seed=1):
    """A second, independent restatement (pure Python loops; small graphs only)
    used to cross-check the C oracle's update rule."""
    n = len(row) - 1
    seeds = [int(s) for s in cms_seeds(cms_seed)]
    out = list(int(x) for x in labels)
    changed = 0
    for v in range(n):
        nb = clm[int(row[v]):int(row[v + 1])]
        if len(nb) == 0:
            continue
        labs = [int(labels[u]) for u in nb]
        if cms_thr and len(labs) >= cms_thr:
            table = [[0] * 1024 for _ in range(4)]
            for l in labs:
                for r in range(4):
                    table[r][cms_index(r, l, seeds[r])] += 1
            best = min(((-min(table[r][cms_index(r, l, seeds[r])] for r in range(4)), l) for l in set(labs)))
            nl = best[1]
        else:
            counts = {}
            for l in labs:
                counts[l] = counts.get(l, 0) + 1
            nl = min(counts, key=lambda l: (-counts[l], l))
        changed += nl != int(labels[v])
        out[v] = nl
    return np.array(out, np.uint32), changed
