"""lpa_iterate_noalloc: one iteration over caller-owned device buffers with no
allocation inside the library.

It serves callers that cannot allocate device memory: a spent memory budget,
buffers owned by the caller's own pool, or a context where allocation is not
allowed. Its output must equal the regular entry point's (lpa_create +
lpa_iterate) exactly -- labels and changed counts are integers -- on two
calls in a row. The second call also shows that the leftover contents of the
shared scratch array do not leak into a new call.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import lpa_b200 as L

pytestmark = pytest.mark.gpu


def _device_desc(torch, arr):
    """A GraphDesc whose pointers are CUDA tensors (kept alive by the caller)."""
    dev = "cuda:0"
    keep = {
        "words": torch.from_numpy(arr["words"].view(np.int32)).to(dev),
        "offsets": torch.from_numpy(arr["offsets"].view(np.int64)).to(dev),
        "vertices": torch.from_numpy(arr["vertices"].view(np.int32)).to(dev),
        "small_graph": torch.from_numpy(np.ascontiguousarray(arr["small_graph"]).view(np.int32)).to(dev),
        "small_offset": torch.from_numpy(np.ascontiguousarray(arr["small_offset"]).view(np.int32)).to(dev),
    }
    d = L.GraphDesc()
    d.num_vertices = arr["n"]
    d.num_compressed = arr["n_c"]
    d.words = C.cast(C.c_void_p(keep["words"].data_ptr()), C.POINTER(C.c_uint32))
    d.num_words = len(arr["words"])
    d.offsets = C.cast(C.c_void_p(keep["offsets"].data_ptr()), C.POINTER(C.c_uint64))
    d.vertices = C.cast(C.c_void_p(keep["vertices"].data_ptr()), C.POINTER(C.c_uint32))
    d.small_graph = C.cast(C.c_void_p(keep["small_graph"].data_ptr()), C.POINTER(C.c_uint32))
    d.num_small_arcs = len(arr["small_graph"])
    d.small_offset = (C.cast(C.c_void_p(keep["small_offset"].data_ptr()), C.POINTER(C.c_uint32))
                      if arr["n"] > arr["n_c"] else None)
    return d, keep


def _call(desc, lab_in, lab_out, cms_thr=0):
    lib = L.lib()
    fn = lib.lpa_iterate_noalloc
    fn.argtypes = [C.POINTER(L.GraphDesc), C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                   C.POINTER(C.c_uint64)]
    fn.restype = C.c_int
    changed = C.c_uint64()
    st = fn(C.byref(desc), C.c_void_p(lab_in.data_ptr()), C.c_void_p(lab_out.data_ptr()), cms_thr, None,
            C.byref(changed))
    return st, int(changed.value)


@pytest.mark.parametrize("make", [
    lambda: L.HostGraph.road(160, 120, seed=2).compress(0, 128),
    lambda: L.HostGraph.rmat(12, 8, seed=4, n_limit=4000).compress(16, 128),
], ids=["road", "rmat"])
def test_noalloc_matches_regular_entry_point_twice(make):
    torch = pytest.importorskip("torch")
    g = make()
    row, _ = g.csr()
    assert int(np.diff(row.astype(np.int64)).max()) <= 1023  # within this path's exact-count limit
    arr = g.arrays()
    n = arr["n"]
    desc, keep = _device_desc(torch, arr)
    a = torch.arange(n, dtype=torch.int32, device="cuda:0")
    b = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    c = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    with L.Propagator(g) as p:
        st, ch1 = _call(desc, a, b)
        assert st == 0, L.lib().lpa_status_str(st)
        ref1 = p.iterate()
        assert np.array_equal(b.cpu().numpy().view(np.uint32), p.labels())
        assert ch1 == ref1
        st, ch2 = _call(desc, b, c)
        assert st == 0, L.lib().lpa_status_str(st)
        ref2 = p.iterate()
        assert np.array_equal(c.cpu().numpy().view(np.uint32), p.labels())
        assert ch2 == ref2
    torch.cuda.synchronize()
    del keep


def test_noalloc_rejects_beyond_its_limits():
    torch = pytest.importorskip("torch")
    # one vertex of degree 1500: above the exact per-warp limit of this path
    n = 1600
    adj = [set() for _ in range(n)]
    for v in range(1, 1501):
        adj[0].add(v)
        adj[v].add(0)
    row = np.zeros(n + 1, np.uint64)
    for v in range(n):
        row[v + 1] = row[v] + len(adj[v])
    clm = np.concatenate([np.array(sorted(s), np.uint32) for s in adj])
    g = L.HostGraph.from_csr(row, clm).compress(0, 128)
    desc, keep = _device_desc(torch, g.arrays())
    a = torch.arange(n, dtype=torch.int32, device="cuda:0")
    b = torch.empty(n, dtype=torch.int32, device="cuda:0")
    st, _ = _call(desc, a, b)
    assert st == L.Status.CAPACITY
    del keep


def _dense_random_graph(n, per_vertex, seed):
    """Undirected random graph: every vertex draws per_vertex partners."""
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(n, dtype=np.int64), per_vertex)
    dst = rng.integers(0, n, size=src.size)
    keep = src != dst
    a = np.concatenate([src[keep], dst[keep]])
    b = np.concatenate([dst[keep], src[keep]])
    key = np.unique(a * n + b)
    a, b = key // n, key % n
    row = np.zeros(n + 1, np.uint64)
    np.add.at(row, a + 1, 1)
    row = np.cumsum(row).astype(np.uint64)
    return row, b.astype(np.uint32)


def test_noalloc_refuses_ids_beyond_its_array():
    """4.9M decoded ids (degrees <= 1023) exceed the 16 MiB array: CAPACITY."""
    torch = pytest.importorskip("torch")
    n = 8192
    row, clm = _dense_random_graph(n, 300, seed=3)
    assert int(np.diff(row.astype(np.int64)).max()) <= 1023 and len(clm) > (16 << 20) // 4
    g = L.HostGraph.from_csr(row, clm).compress(0, 128)
    desc, keep = _device_desc(torch, g.arrays())
    a = torch.arange(n, dtype=torch.int32, device="cuda:0")
    b = torch.empty(n, dtype=torch.int32, device="cuda:0")
    st, _ = _call(desc, a, b)
    assert st == L.Status.CAPACITY
    del keep


def test_noalloc_refuses_a_vertex_at_the_sketch_threshold():
    torch = pytest.importorskip("torch")
    g = L.HostGraph.road(64, 48, seed=5).compress(0, 128)
    row, _ = g.csr()
    dmax = int(np.diff(row.astype(np.int64)).max())
    desc, keep = _device_desc(torch, g.arrays())
    n = g.arrays()["n"]
    a = torch.arange(n, dtype=torch.int32, device="cuda:0")
    b = torch.empty(n, dtype=torch.int32, device="cuda:0")
    st, _ = _call(desc, a, b, cms_thr=dmax)
    assert st == L.Status.CAPACITY
    # one above the largest degree: every vertex is exact, so the call runs
    st, _ = _call(desc, a, b, cms_thr=dmax + 1)
    assert st == 0
    del keep


def test_noalloc_small_csr_only_matches_regular_entry_point():
    """Every vertex below the compression threshold (no compressed position):
    the decode steps are skipped and only the small CSR is counted."""
    torch = pytest.importorskip("torch")
    g = L.HostGraph.road(96, 80, seed=6).compress(32, 128)
    arr = g.arrays()
    assert arr["n_c"] == 0
    n = arr["n"]
    desc, keep = _device_desc(torch, arr)
    a = torch.arange(n, dtype=torch.int32, device="cuda:0")
    b = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    c = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    with L.Propagator(g) as p:
        st, ch1 = _call(desc, a, b)
        assert st == 0
        assert ch1 == p.iterate()
        assert np.array_equal(b.cpu().numpy().view(np.uint32), p.labels())
        st, ch2 = _call(desc, b, c)
        assert st == 0
        assert ch2 == p.iterate()
        assert np.array_equal(c.cpu().numpy().view(np.uint32), p.labels())
    del keep
