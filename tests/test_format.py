"""The native format layer against the reference's own files (CPU only)."""
import filecmp
import os

import numpy as np
import pytest

import lpa_b200 as L
import oracle
from conftest import CASES, golden_base, golden_meta

EXTS = [".graph", ".offset", ".vertices.bin", ".graph.small.bin", ".offset.small.bin"]


@pytest.mark.parametrize("case", CASES)
def test_encoder_bit_identical_to_reference(case, tmp_path):
    """The fast parallel encoder writes byte-identical .graph/.offset/.vertices.bin/
    small-CSR files to the reference CgrCompressor (src/compressor.cpp)."""
    base = golden_base(case)
    meta = golden_meta(case)
    ref = oracle.read_reference_files(base)
    g = L.HostGraph.from_csr(ref["row"], ref["clm"])
    g.compress(meta["small_thresh"], meta["large_thresh"], threads=4)
    out = str(tmp_path / "g")
    g.write_cgr(out)
    g.write_csr(out)
    for ext in EXTS + [".row", ".clm"]:
        assert os.path.exists(base + ext) == os.path.exists(out + ext), ext
        if os.path.exists(base + ext):
            assert filecmp.cmp(base + ext, out + ext, shallow=False), ext


@pytest.mark.parametrize("case", CASES)
def test_loader_reads_reference_files(case):
    base = golden_base(case)
    meta = golden_meta(case)
    ref = oracle.read_reference_files(base)
    a = L.HostGraph.load_cgr(base, meta["small_thresh"]).arrays()
    assert a["n"] == ref["n"] and a["n_c"] == ref["n_c"]
    assert np.array_equal(a["offsets"], ref["offsets"])
    assert np.array_equal(a["vertices"], ref["vertices"])
    nw = (int(ref["offsets"][-1]) + 31) // 32
    assert np.array_equal(a["words"][:nw], ref["words"][:nw])
    assert not a["words"][nw:].any()
    if ref["n"] > ref["n_c"]:
        assert np.array_equal(a["small_offset"], ref["small_offset"])
        assert np.array_equal(a["small_graph"], ref["small_graph"])


@pytest.mark.parametrize("case", ["road_a", "road_b"])
def test_edge_list_ingest(case):
    """read_edge_list follows File::read_from_edge_list (src/file.cpp:115-195)."""
    base = golden_base(case)
    meta = golden_meta(case)
    ref = oracle.read_reference_files(base)
    row, clm = L.HostGraph.read_edge_list(base, bool(meta["one_way"])).csr()
    assert np.array_equal(row, ref["row"])
    assert np.array_equal(clm, ref["clm"])


def test_offsets_beyond_32_bits(tmp_path):
    """Bit offsets above 2^32 (the reference parses them as uint32) load intact."""
    base = str(tmp_path / "big")
    total = (1 << 32) + 4096  # bits
    with open(base + ".graph", "wb") as f:  # sparse file of zero bytes
        f.truncate((total + 7) // 8)
    cuts = [0, (1 << 32) - 8, (1 << 32) + 8, total]
    with open(base + ".offset", "w") as f:
        f.write(f"{len(cuts) - 1}\n" + "".join(f"{c}\n" for c in cuts[1:]))
    np.arange(3, dtype=np.uint32).tofile(base + ".vertices.bin")
    a = L.HostGraph.load_cgr(base, 0).arrays()
    assert [int(x) for x in a["offsets"]] == cuts


def test_loader_rejects_missing_and_truncated(tmp_path):
    with pytest.raises(L.LpaError):
        L.HostGraph.load_cgr(str(tmp_path / "nothing"), 0)
    base = golden_base("road_a")
    bad = str(tmp_path / "t")
    for ext in [".graph", ".vertices.bin"]:
        with open(base + ext, "rb") as s, open(bad + ext, "wb") as d:
            d.write(s.read())
    lines = open(base + ".offset").read().split("\n")
    open(bad + ".offset", "w").write("\n".join(lines[: len(lines) // 2]))
    with pytest.raises(L.LpaError) as e:
        L.HostGraph.load_cgr(bad, 0)
    assert e.value.status == L.Status.IO


def test_encoder_rejects_threshold_order():
    g = L.HostGraph.road(10, 10)
    with pytest.raises(L.LpaError) as e:
        g.compress(200, 128)
    assert e.value.status == L.Status.INVALID_ARG


def test_generators_deterministic_and_clean():
    for make in (lambda: L.HostGraph.road(30, 20, seed=5), lambda: L.HostGraph.rmat(9, 8, seed=2),
                 lambda: L.HostGraph.copy_model(800, 12, seed=3)):
        r1, c1 = make().csr()
        r2, c2 = make().csr()
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2)
        for v in range(len(r1) - 1):
            nb = c1[r1[v]:r1[v + 1]]
            assert np.all(np.diff(nb.astype(np.int64)) > 0)  # sorted, no duplicates
            assert v not in set(nb.tolist())  # no loops


def test_road_generator_shape():
    row, clm = L.HostGraph.road(362, 362, seed=1).csr()
    n = len(row) - 1
    assert n == 131044
    deg = np.diff(row)
    assert 2.5 < deg.mean() < 3.2  # 4 * 0.7 kept grid arcs plus extras
    # symmetric
    src = np.repeat(np.arange(n), deg.astype(np.int64))
    fwd = set(zip(src.tolist(), clm.tolist()))
    assert all((v, u) in fwd for (u, v) in list(fwd)[:5000])


@pytest.mark.skipif(not oracle.REF_BIN.exists(), reason="the reference compressor was not built here")
def test_encoder_matches_reference_on_the_benchmark_family(tmp_path):
    """The benchmark's graph family at a size the reference compressor handles
    in seconds: R-MAT scale 18, edge factor 16, symmetrised, BFS order,
    threshold 32 (7.6M arcs, hubs with intervals).  The reference's own
    CgrCompressor (built from its sources into oracle/_ref) and this library
    write byte-identical files from the same edge list (which, like the
    reference's ingest, ends at the largest id that has an edge)."""
    import subprocess

    el = str(tmp_path / "e.txt")
    L.HostGraph.rmat(18, 16.0, seed=1).write_edge_list(el, False)
    subprocess.run([str(oracle.REF_BIN), el, "1", "32"], check=True, capture_output=True)
    g = L.HostGraph.read_edge_list(el, True)
    g.compress(32, 128)
    out = str(tmp_path / "ours")
    g.write_cgr(out)
    for ext in EXTS:
        assert os.path.exists(el + ext) == os.path.exists(out + ext), ext
        if os.path.exists(el + ext):
            assert filecmp.cmp(el + ext, out + ext, shallow=False), ext
