"""Batched graphs: per-graph labels and iteration counts equal running each
graph alone (and the oracle), in both batch modes -- the lockstep
concatenated graph and the persistent queue."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle

pytestmark = pytest.mark.gpu

MODES = [L.BatchMode.LOCKSTEP, L.BatchMode.QUEUE]


def _graphs():
    """Uneven sizes: road grids and R-MAT graphs, log-spaced vertex counts,
    plus a graph without arcs and one whose vertices are all in the small CSR."""
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
    empty = L.HostGraph.from_csr(np.zeros(40, np.uint64), np.zeros(0, np.uint32))
    empty.compress(0, 128)
    out.insert(3, empty)
    small = L.HostGraph.rmat(10, 4, seed=77)
    small.compress(1 << 20, 1 << 20)  # every vertex below the threshold: no bitstream
    out.insert(7, small)
    return out


def _alone(g, max_iter, cms_thr, early_exit):
    row, clm = g.csr()
    hist, _ = oracle.lp_run(row, clm, max_iter, cms_thr=cms_thr, early_exit=early_exit)
    return hist


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("cms_thr", [0, 64])
def test_batch_matches_single_runs(mode, cms_thr):
    graphs = _graphs()
    with L.Batch(graphs, cms_threshold=cms_thr, batch_mode=mode) as b:
        assert (b.handle() is None) == (mode == L.BatchMode.QUEUE)
        iters = b.run(30, early_exit=True)
        for i, g in enumerate(graphs):
            hist = _alone(g, 30, cms_thr, True)
            if mode == L.BatchMode.LOCKSTEP or len(g.csr()[1]):
                # the queue counts a graph without arcs as one iteration in every case
                assert iters[i] == len(hist), f"graph {i}: {iters[i]} iterations vs {len(hist)}"
            assert np.array_equal(b.labels(i), hist[-1]), f"graph {i}"
            with L.Propagator(g, cms_threshold=cms_thr) as p:
                assert p.run(30, early_exit=True) == len(hist)
                assert np.array_equal(p.labels(), hist[-1])


@pytest.mark.parametrize("mode", MODES)
def test_batch_fixed_iterations_and_rerun(mode):
    graphs = _graphs()[:6]
    with L.Batch(graphs, batch_mode=mode) as b:
        for max_iter in (1, 5):
            iters = b.run(max_iter, early_exit=False)
            for i, g in enumerate(graphs):
                if mode == L.BatchMode.LOCKSTEP or len(g.csr()[1]):
                    assert iters[i] == max_iter
                hist = _alone(g, max_iter, 0, False)
                assert np.array_equal(b.labels(i), hist[-1])
        assert (b.run(0) == 0).all()


@pytest.mark.parametrize("dispatch,force", [(L.Dispatch.LEARNED, L.Variant.BLOCK),
                                            (L.Dispatch.FORCE, L.Variant.TWO_PASS),
                                            (L.Dispatch.FORCE, L.Variant.BLOCK)])
def test_lockstep_any_dispatch(dispatch, force):
    """The concatenated graph runs every plan; the sketch counts each graph's
    labels relative to its own ids (cms 24 puts R-MAT hubs on it)."""
    graphs = _graphs()
    with L.Batch(graphs, cms_threshold=24, dispatch=dispatch, force_variant=force,
                 batch_mode=L.BatchMode.LOCKSTEP) as b:
        for _ in range(2):  # the learner changes the plan between runs
            iters = b.run(30, early_exit=True)
            for i, g in enumerate(graphs):
                hist = _alone(g, 30, 24, True)
                assert iters[i] == len(hist), f"graph {i}"
                assert np.array_equal(b.labels(i), hist[-1]), f"graph {i}"


def test_lockstep_autotune_through_handle(tmp_path):
    graphs = _graphs()[:8]
    with L.Batch(graphs, batch_mode=L.BatchMode.LOCKSTEP) as b:
        h = b.handle()
        assert h.n == sum(int(g.csr()[0].shape[0]) - 1 for g in graphs)
        h.autotune(str(tmp_path / "tune.txt"), repeats=1)
        iters = b.run(30, early_exit=True)
        for i, g in enumerate(graphs):
            hist = _alone(g, 30, 0, True)
            assert iters[i] == len(hist)
            assert np.array_equal(b.labels(i), hist[-1])
        assert h.stats().launches > 0


def test_lockstep_rejects_foreign_ids():
    """A graph whose arcs leave its own vertices is refused, as when run alone,
    though the concatenation holds the ids it names."""
    a = L.HostGraph.road(8, 8, seed=1)
    a.compress(0, 128)
    b = L.HostGraph.rmat(8, 4, seed=3)
    b.compress(1 << 20, 1 << 20)  # all in the small CSR
    arr = b.arrays()
    arr["small_graph"] = arr["small_graph"].copy()
    arr["small_graph"][0] = arr["n"]  # the first id of the next graph in the batch
    bad = L.desc_from_arrays(arr)
    with pytest.raises(L.LpaError):
        L.Propagator(bad)
    for mode in MODES:
        with pytest.raises(L.LpaError):
            L.Batch([bad, a], batch_mode=mode)


def test_queue_wait_that_runs_out_returns_timeout():
    """The persistent queue's wait for an item is bounded.  With a bound of one
    try, the many blocks that find no item while the graphs still run give up
    at once: the kernel sets the timeout error and returns (it does not trap),
    the run reports LPA_ERR_TIMEOUT, and the context stays usable."""
    graphs = _graphs()[:4]
    with L.Batch(graphs, batch_mode=L.BatchMode.QUEUE, queue_wait_limit=1) as b:
        with pytest.raises(L.LpaError) as e:
            b.run(30, early_exit=True)
        assert e.value.status == L.Status.TIMEOUT
    # the device still works: the same batch with the default bound
    with L.Batch(graphs, batch_mode=L.BatchMode.QUEUE) as b:
        iters = b.run(30, early_exit=True)
        for i, g in enumerate(graphs):
            assert np.array_equal(b.labels(i), _alone(g, 30, 0, True)[-1])
