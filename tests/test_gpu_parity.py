"""GPU parity: the sm_100a path against the CPU oracle, through the C ABI.

Decode parity is bit-exact against the reference compressor's own .row/.clm;
label parity is bit-exact against the oracle after every iteration (integer
work: no tolerance).
"""
import numpy as np
import pytest

import lpa_b200 as L
import oracle
from conftest import CASES, golden_base, golden_meta

pytestmark = pytest.mark.gpu

VARIANTS = [None, L.Variant.WARP, L.Variant.PACKED, L.Variant.BLOCK, L.Variant.TWO_PASS]


def _load(case):
    base = golden_base(case)
    meta = golden_meta(case)
    return L.HostGraph.load_cgr(base, meta["small_thresh"]), oracle.read_reference_files(base)


def _sorted_rows(row, clm):
    out = clm.copy()
    for v in range(len(row) - 1):
        out[row[v]:row[v + 1]].sort()
    return out


def _check_iterations(p, row, clm, iters, cms_thr, seed=1):
    hist, changed = oracle.lp_run(row, clm, iters, cms_thr, seed)
    for it in range(iters):
        ch = p.iterate()
        lab = p.labels()
        bad = np.flatnonzero(lab != hist[it])
        assert bad.size == 0, f"iteration {it + 1}: {bad.size} labels differ, first at vertex {bad[:5]}"
        assert ch == changed[it], f"iteration {it + 1}: changed {ch} vs {changed[it]}"


@pytest.mark.parametrize("case", CASES)
def test_decode_csr_matches_reference(case):
    g, ref = _load(case)
    with L.Propagator(g) as p:
        row, clm = p.decode_csr()
        assert np.array_equal(row, ref["row"])
        assert np.array_equal(_sorted_rows(row, clm), ref["clm"])
        deg = p.degrees()
        assert np.array_equal(deg.astype(np.uint64), np.diff(ref["row"])[ref["vertices"]])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("variant", VARIANTS, ids=lambda v: "fixed" if v is None else v.name.lower())
@pytest.mark.parametrize("cms_thr", [0, 8])
def test_labels_every_iteration(case, variant, cms_thr):
    g, ref = _load(case)
    opts = dict(cms_threshold=cms_thr, cms_seed=1)
    if variant is not None:
        opts.update(dispatch=L.Dispatch.FORCE, force_variant=int(variant))
    with L.Propagator(g, **opts) as p:
        _check_iterations(p, ref["row"], ref["clm"], 8, cms_thr)


@pytest.mark.parametrize("case", ["road_a", "rmat_t16", "stress"])
def test_graph_loop_early_exit(case):
    """The CUDA-graph loop (conditional WHILE node) stops where the oracle does."""
    g, ref = _load(case)
    hist, changed = oracle.lp_run(ref["row"], ref["clm"], 60, 0, 1, early_exit=True)
    with L.Propagator(g) as p:
        done = p.run(60, early_exit=True)
        assert done == len(hist)
        assert np.array_equal(p.labels(), hist[-1])
        assert list(p.changed_history(done)) == changed
        # a second run continues from there: it stops at once after a fixed point;
        # synchronous LP can also settle into a period-2 oscillation that never stops
        more, more_changed = oracle.lp_run(ref["row"], ref["clm"], 10, 0, 1, labels=hist[-1], early_exit=True)
        assert p.run(10, early_exit=True) == len(more)
        assert np.array_equal(p.labels(), more[-1])
        assert list(p.changed_history(len(more))) == more_changed


def test_run_without_early_exit_matches_iterate():
    g, ref = _load("rmat_t32")
    hist, changed = oracle.lp_run(ref["row"], ref["clm"], 7, 0, 1)
    with L.Propagator(g) as p:
        assert p.run(7) == 7
        assert np.array_equal(p.labels(), hist[-1])
        assert list(p.changed_history(7)) == changed


def test_config_a_full_every_iteration():
    """Road 362x362, p=0.7, 2% extras, seed 1, threshold 0: 20 iterations."""
    g = L.HostGraph.road(362, 362, seed=1)
    row, clm = g.csr()
    g.compress(0, 128)
    with L.Propagator(g) as p:
        _check_iterations(p, row, clm, 20, 0)


@pytest.mark.parametrize("variant", [None, L.Variant.TWO_PASS], ids=["fused", "two_pass"])
def test_config_b_full_early_exit(variant):
    """Road 1404x1404 (each edge once, symmetrised), threshold 0, <= 30 iterations
    with early exit; fused and two-pass give the same labels."""
    g = L.HostGraph.road(1404, 1404, seed=1)
    row, clm = g.csr()
    g.compress(0, 128)
    hist, changed = oracle.lp_run(row, clm, 30, 0, 1, early_exit=True)
    opts = {} if variant is None else dict(dispatch=L.Dispatch.FORCE, force_variant=int(variant))
    with L.Propagator(g, **opts) as p:
        done = p.run(30, early_exit=True)
        assert done == len(hist)
        assert np.array_equal(p.labels(), hist[-1])
        assert list(p.changed_history(done)) == changed


@pytest.mark.parametrize("cms_thr", [1024, 64])
def test_rmat_sketch_every_iteration(cms_thr):
    """R-MAT scale 16 (edge factor 16, BFS order), threshold 32, sketch above cms_thr."""
    g = L.HostGraph.rmat(16, 16, seed=1)
    row, clm = g.csr()
    g.compress(32, 128)
    with L.Propagator(g, cms_threshold=cms_thr, cms_seed=1) as p:
        _check_iterations(p, row, clm, 6, cms_thr)


def test_exact_hub_uses_global_table():
    """An exact-count vertex above the shared-memory table (degree 12000)."""
    n = 20000
    hub = np.arange(1, 12001, dtype=np.uint32)
    rows = [hub] + [np.array([0], np.uint32)] * 12000 + [np.zeros(0, np.uint32)] * (n - 12001)
    rng = np.random.default_rng(3)
    # a second layer so the hub sees several labels
    extra = {}
    for v in range(12001, n):
        extra[v] = int(rng.integers(1, 12001))
    adj = [set(r.tolist()) for r in rows]
    for v, u in extra.items():
        adj[v].add(u)
        adj[u].add(v)
    row = np.zeros(n + 1, np.uint64)
    for v in range(n):
        row[v + 1] = row[v] + len(adj[v])
    clm = np.concatenate([np.array(sorted(a), np.uint32) for a in adj])
    g = L.HostGraph.from_csr(row, clm).compress(0, 128)
    for variant in (None, L.Variant.TWO_PASS):
        opts = {} if variant is None else dict(dispatch=L.Dispatch.FORCE, force_variant=int(variant))
        with L.Propagator(g, **opts) as p:
            _check_iterations(p, row, clm, 4, 0)


def test_set_labels_and_history():
    g, ref = _load("rmat_t16")
    rng = np.random.default_rng(9)
    start = rng.integers(0, 50, ref["n"]).astype(np.uint32)
    a, ca = oracle.lp_iterate_csr(ref["row"], ref["clm"], start)
    with L.Propagator(g) as p:
        p.set_labels(start)
        assert p.iterate() == ca
        assert np.array_equal(p.labels(), a)


def test_damaged_stream_is_reported():
    """Zeroed stream words are caught by the decoder's bounds checks and reported
    as BAD_STREAM (no trap, no out-of-range read: every read stays inside the
    padded stream and every id is checked against n)."""
    g, ref = _load("road_a")
    arr = g.arrays()
    words = arr["words"].copy()
    words[len(words) // 3: len(words) // 3 + 40] = 0
    arr["words"] = words
    with pytest.raises(L.LpaError) as e:
        L.Propagator(L.desc_from_arrays(arr))
    assert e.value.status == L.Status.BAD_STREAM


def test_dispatch_switch_keeps_labels_identical():
    g, ref = _load("stress")
    hist, _ = oracle.lp_run(ref["row"], ref["clm"], 6)
    with L.Propagator(g) as p:
        for it, v in enumerate([L.Variant.WARP, L.Variant.BLOCK, L.Variant.TWO_PASS, L.Variant.PACKED,
                                L.Variant.WARP, L.Variant.BLOCK]):
            p.set_dispatch(L.Dispatch.FORCE, v)
            p.iterate()
            assert np.array_equal(p.labels(), hist[it])


@pytest.mark.parametrize("case", ["rmat_t16", "stress"])
def test_explicit_plan_mixes_variants_exactly(case):
    """lpa_set_plan: a random mix of the variants each segment can run gives
    the oracle's labels after every iteration; a plan with a variant a segment
    cannot run is refused and leaves the plan in place."""
    g, ref = _load(case)
    with L.Propagator(g, cms_threshold=8) as p:
        _, _, bucket, fixed = p.segments()
        rng = np.random.default_rng(7)
        # the fixed plan's variant, or the block or two-pass variant (both run
        # every segment)
        choice = rng.integers(0, 3, size=len(fixed))
        plan = np.where(choice == 0, fixed, np.where(choice == 1, int(L.Variant.TWO_PASS), int(L.Variant.BLOCK)))
        p.set_plan(plan.astype(np.uint8))
        _check_iterations(p, ref["row"], ref["clm"], 4, 8)
        if (bucket >= 1).any():  # several vertices per warp: not for sketch or degree > 32
            bad = np.full(len(fixed), int(L.Variant.PACKED), np.uint8)
            with pytest.raises(L.LpaError) as e:
                p.set_plan(bad)
            assert e.value.status == L.Status.INVALID_ARG
            assert np.array_equal(p.segments()[3], plan)
