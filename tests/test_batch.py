"""Batched graphs in one persistent launch: per-graph labels and iteration
counts equal running each graph alone (and the oracle)."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle

pytestmark = pytest.mark.gpu


def _graphs():
    """Uneven sizes: road grids and R-MAT graphs, log-spaced vertex counts."""
    out = []
    rng = np.random.default_rng(5)
    for i in range(12):
        n = int(np.exp(rng.uniform(np.log(200), np.log(60000))))
        if i % 2 == 0:
            side = max(4, int(np.sqrt(n)))
            g = L.HostGraph.road(side, side, seed=1 + i)
            g.compress(0 if i % 4 == 0 else 16, 128)
        else:
            scale = max(8, int(np.ceil(np.log2(n))))
            g = L.HostGraph.rmat(scale, 8, seed=1 + i, n_limit=n)
            g.compress(16, 128)
        out.append(g)
    return out


@pytest.mark.parametrize("cms_thr", [0, 64])
def test_batch_matches_single_runs(cms_thr):
    graphs = _graphs()
    with L.Batch(graphs, cms_threshold=cms_thr) as b:
        iters = b.run(30, early_exit=True)
        for i, g in enumerate(graphs):
            row, clm = g.csr()
            hist, changed = oracle.lp_run(row, clm, 30, cms_thr=cms_thr, early_exit=True)
            assert iters[i] == len(hist), f"graph {i}: {iters[i]} iterations vs {len(hist)}"
            assert np.array_equal(b.labels(i), hist[-1]), f"graph {i}"
            with L.Propagator(g, cms_threshold=cms_thr) as p:
                assert p.run(30, early_exit=True) == len(hist)
                assert np.array_equal(p.labels(), hist[-1])


def test_batch_fixed_iterations_and_rerun():
    graphs = _graphs()[:6]
    with L.Batch(graphs) as b:
        for max_iter in (1, 5):
            iters = b.run(max_iter, early_exit=False)
            assert (iters == max_iter).all()
            for i, g in enumerate(graphs):
                row, clm = g.csr()
                hist, _ = oracle.lp_run(row, clm, max_iter)
                assert np.array_equal(b.labels(i), hist[-1])
