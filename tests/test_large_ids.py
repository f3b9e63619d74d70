"""Vertex ids at and above 2^27 through the two-pass and fused kernels.

The pre-pass stages a decoded id with its lane in the id's top five bits
only when every id fits in 27 bits (n <= 2^27); a larger graph runs the form
that keeps the lane in a separate byte.  This graph puts an R-MAT scale-12
graph (sketch at degree >= 64) at ids 2^27 - 2048 .. 2^27 + 2047 of a
2^27 + 2112-vertex graph whose other vertices are isolated, and checks the
labels and changed counts after every iteration against the CPU oracle.
"""
import numpy as np
import pytest

import lpa_b200 as L
import oracle

pytestmark = pytest.mark.gpu

ITERS = 3


@pytest.fixture(scope="module")
def big():
    sub = L.HostGraph.rmat(12, 16.0, seed=3)
    srow, sclm = sub.csr()
    base = (1 << 27) - 2048
    m = len(srow) - 1
    n = base + m + 64
    deg = np.zeros(n, np.uint64)
    deg[base:base + m] = np.diff(srow.astype(np.uint64))
    row = np.zeros(n + 1, np.uint64)
    np.cumsum(deg, out=row[1:])
    clm = (sclm.astype(np.uint64) + base).astype(np.uint32)
    g = L.HostGraph.from_csr(row, clm)
    g.compress(32, 128)
    hist, changed = oracle.lp_run(row, clm, ITERS, 64, 1)
    return g, n, hist, changed


@pytest.mark.parametrize("plan", ["two_pass", "fixed"])
def test_ids_above_2_27_every_iteration(big, plan):
    g, n, hist, changed = big
    opts = dict(cms_threshold=64, cms_seed=1)
    if plan == "two_pass":
        opts.update(dispatch=L.Dispatch.FORCE, force_variant=int(L.Variant.TWO_PASS))
    with L.Propagator(g, device=0, **opts) as p:
        assert int(p.get_info().num_vertices) == n > (1 << 27)
        for it in range(ITERS):
            ch = p.iterate()
            lab = p.labels()
            bad = np.flatnonzero(lab != hist[it])
            assert bad.size == 0, f"iteration {it + 1}: {bad.size} labels differ, first at vertex {bad[:5]}"
            assert ch == changed[it], f"iteration {it + 1}: changed {ch} vs {changed[it]}"
