"""Out-of-core streaming (lpa_opts.stream_budget): the bitstream stays in host
memory and every iteration processes the compressed positions range by range,
each range's stream copied to the device on a second stream while the previous
range is processed (the reference streams CSR batches this way,
include/outofcore.cuh:10-96).  With the budget forced well below the graph's
size, labels and changed counts must equal the oracle's after every iteration
(integer work: bit-exact), for the fixed plan, the two-pass kernels and the
learned dispatch; the decoded adjacency must equal the resident handle's."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle

pytestmark = pytest.mark.gpu


def _check(p, arr, cms, iters):
    lab = np.arange(arr["n"], dtype=np.uint32)
    for it in range(iters):
        ch = p.iterate()
        lab, och = oracle.lp_iterate_cgr(arr, lab, cms, 1, 0)
        got = p.labels()
        bad = np.flatnonzero(got != lab)
        assert bad.size == 0, f"iteration {it + 1}: {bad.size} labels differ, first at {bad[:5]}"
        assert ch == och, f"iteration {it + 1}: changed {ch} vs {och}"


PLANS = {
    "fixed": {},
    "two_pass": dict(dispatch=L.Dispatch.FORCE, force_variant=int(L.Variant.TWO_PASS)),
    "warp": dict(dispatch=L.Dispatch.FORCE, force_variant=int(L.Variant.WARP)),
    "learned": dict(dispatch=L.Dispatch.LEARNED),
}


@pytest.mark.parametrize("plan", sorted(PLANS))
def test_rmat_streamed_every_iteration(plan):
    """R-MAT scale 16 (hubs near degree 10k, sketch at 64): a 2 MB budget cuts
    the 1.7 MB stream and its 6 MB of labels into several ranges."""
    g = L.HostGraph.rmat(16, 16, seed=1).compress(32, 128)
    arr = g.arrays()
    with L.Propagator(g, cms_threshold=64, stream_budget=2 << 20, **PLANS[plan]) as p:
        _check(p, arr, 64, 8)
        st = p.stats()
        assert st.stream_ranges >= 3
        assert st.stream_bytes >= 8 * 4 * (len(arr["words"]) - 8)  # every iteration read the stream again


def test_copy_model_streamed_two_pass_and_run():
    """Long intervals (copy model); the host loop of lpa_run with early exit
    stops where the oracle does."""
    g = L.HostGraph.copy_model(200_000, 30, seed=1).compress(16, 128)
    arr = g.arrays()
    opts = dict(stream_budget=4 << 20, dispatch=L.Dispatch.FORCE, force_variant=int(L.Variant.TWO_PASS))
    with L.Propagator(g, **opts) as p:
        _check(p, arr, 0, 5)
        assert p.stats().stream_ranges >= 4
    row, clm = g.csr()
    hist, changed = oracle.lp_run(row, clm, 40, early_exit=True)
    with L.Propagator(g, **opts) as p:
        done = p.run(40, early_exit=True)
        assert done == len(hist)
        assert np.array_equal(p.labels(), hist[-1])
        assert list(p.changed_history(done)) == changed


def test_streamed_decode_matches_resident():
    g = L.HostGraph.rmat(14, 16, seed=2).compress(16, 128)
    with L.Propagator(g) as p:
        row, clm = p.decode_csr()
    with L.Propagator(g, stream_budget=1 << 20) as p:
        assert p.stats().stream_ranges >= 2
        row2, clm2 = p.decode_csr()
    assert np.array_equal(row, row2)
    assert np.array_equal(clm, clm2)


def test_vertex_beyond_the_budget_is_refused():
    """One hub (degree 9674: about 18 KB of stream, 39 KB of labels) fits
    neither a 64 KB budget's 16 KB stream buffers nor its 32 KB scratch:
    LPA_ERR_CAPACITY at create, not a fault."""
    g = L.HostGraph.rmat(16, 16, seed=1).compress(32, 128)
    with pytest.raises(L.LpaError) as e:
        L.Propagator(g, stream_budget=64 << 10)
    assert e.value.status == L.Status.CAPACITY


@pytest.mark.parametrize("stage", [1, 2])
def test_streamed_two_pass_with_staged_stream_spans(stage):
    """The pre-pass's stream staging (L2 prefetch, or bulk copies into shared
    memory) reading from a streamed range's buffer: same labels."""
    g = L.HostGraph.rmat(16, 16, seed=1).compress(32, 128)
    arr = g.arrays()
    opts = dict(cms_threshold=64, stream_budget=2 << 20, dispatch=L.Dispatch.FORCE,
                force_variant=int(L.Variant.TWO_PASS))
    with L.Propagator(g, **opts) as p:
        p.set_tune(32, 4, 511, 2, 1, 0, stage)
        _check(p, arr, 64, 5)
