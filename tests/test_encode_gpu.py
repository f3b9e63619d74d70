"""The GPU-side CGR encoder against the host encoder (itself byte-identical to
the reference's CgrCompressor on the golden fixtures): every array equal, on
the fixtures and on generated graphs with and without long intervals."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle
from conftest import CASES, golden_base, golden_meta

pytestmark = pytest.mark.gpu

KEYS = ("words", "offsets", "vertices", "small_graph", "small_offset")


def _same(a, b):
    for k in ("n", "n_c"):
        assert a[k] == b[k], k
    for k in KEYS:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.shape == y.shape and np.array_equal(x, y), k


def _both(row, clm, small):
    host = L.HostGraph.from_csr(row, clm).compress(small, 128).arrays()
    gpu = L.HostGraph.from_csr(row, clm).compress(small, 128, device=0).arrays()
    return host, gpu


@pytest.mark.parametrize("case", CASES)
def test_fixtures_match_host_encoder(case):
    ref = oracle.read_reference_files(golden_base(case))
    host, gpu = _both(ref["row"], ref["clm"], golden_meta(case)["small_thresh"])
    _same(host, gpu)


@pytest.mark.parametrize("make,small", [
    (lambda: L.HostGraph.rmat(14, 16, seed=5), 0),
    (lambda: L.HostGraph.rmat(14, 16, seed=5), 32),
    (lambda: L.HostGraph.road(80, 70, seed=9), 0),
    (lambda: L.HostGraph.copy_model(30000, 30, seed=4), 16),  # long intervals, many segments
], ids=["rmat_t0", "rmat_t32", "road_t0", "copy_t16"])
def test_generated_graphs_match_host_encoder(make, small):
    row, clm = make().csr()
    host, gpu = _both(row, clm, small)
    _same(host, gpu)
