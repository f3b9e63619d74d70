"""The autotuner and its knobs: the count pass's work shapes change speed,
never labels; tuning leaves the labels where they were; results are cached."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle
from conftest import golden_base, golden_meta

pytestmark = pytest.mark.gpu


def _load(case):
    base = golden_base(case)
    return L.HostGraph.load_cgr(base, golden_meta(case)["small_thresh"]), oracle.read_reference_files(base)


def _two_pass(p):
    plan = p.segments()[3].copy()
    plan[:] = int(L.Variant.TWO_PASS)
    p.set_plan(plan)


@pytest.mark.parametrize("knobs", [(1, 1, 32, 1, 0, 0, 0), (7, 3, 100, 8, 1, 1, 1), (32, 32, 511, 5, 0, 2, 2),
                                   (32, 4, 511, 2, 1, 0, 2), (32, 4, 511, 2, 0, 1, 2), (16, 8, 255, 2, 0, 0, 1)])
@pytest.mark.parametrize("case", ["rmat_t16", "stress", "copy_t16"])
def test_knobs_keep_labels_exact(knobs, case):
    """bulk_stage = 1 stages the several-vertices items by bulk copies;
    gather_cache picks the pre-pass's label read path (hot ids / L2 / L1);
    stage_stream moves each decode group's stream span ahead of its decode
    (1 a bulk prefetch into L2, 2 double-buffered bulk copies into shared
    memory); the stress graph has long intervals and many segments per vertex."""
    g, ref = _load(case)
    hist, changed = oracle.lp_run(ref["row"], ref["clm"], 4, 64)
    with L.Propagator(g, cms_threshold=64) as p:
        _two_pass(p)
        p.set_tune(*knobs)
        assert p.get_tune().as_tuple() == knobs
        for it in range(4):
            assert p.iterate() == changed[it]
            assert np.array_equal(p.labels(), hist[it]), f"iteration {it + 1}"


def test_out_of_range_knobs_are_refused():
    g, _ = _load("road_a")
    with L.Propagator(g) as p:
        before = p.get_tune().as_tuple()
        for bad in [(0, 4, 511, 2), (33, 4, 511, 2), (32, 4, 31, 2), (32, 4, 512, 2), (32, 4, 511, 9),
                    (32, 4, 511, 2, 2), (32, 4, 511, 2, 0, 3), (32, 4, 511, 2, 0, 0, 3)]:
            with pytest.raises(L.LpaError) as e:
                p.set_tune(*bad)
            assert e.value.status == L.Status.INVALID_ARG
        assert p.get_tune().as_tuple() == before


def test_autotune_leaves_labels_and_caches(tmp_path):
    g, ref = _load("stress")
    hist, _ = oracle.lp_run(ref["row"], ref["clm"], 5, 8)
    cache = tmp_path / "tune.txt"
    with L.Propagator(g, cms_threshold=8) as p:
        _two_pass(p)
        p.iterate()
        p.iterate()
        lab = p.labels()
        t = p.autotune(cache, repeats=1)
        assert np.array_equal(p.labels(), lab)
        assert p.stats().iterations == 2
        assert cache.read_text().count("\n") == 1
        for it in range(2, 5):
            p.iterate()
            assert np.array_equal(p.labels(), hist[it]), f"iteration {it + 1}"
        # a second handle on the same GPU, graph and plan takes the cached result
        with L.Propagator(g, cms_threshold=8) as q:
            _two_pass(q)
            assert q.autotune(cache).as_tuple() == t.as_tuple()
        assert cache.read_text().count("\n") == 1


@pytest.mark.parametrize("case,thr", [("road_a", 0), ("copy_t16", 0), ("stress_t8", 8)])
def test_bulk_staged_groups_exact(case, thr):
    """Several-vertices items staged by one bulk copy each (16-byte-aligned
    ranges around arbitrary scratch offsets) give the oracle's labels."""
    g, ref = _load(case)
    hist, changed = oracle.lp_run(ref["row"], ref["clm"], 3, thr)
    with L.Propagator(g, cms_threshold=thr) as p:
        _two_pass(p)
        t = p.get_tune().as_tuple()
        p.set_tune(*t[:4], 1)
        for it in range(3):
            assert p.iterate() == changed[it]
            assert np.array_equal(p.labels(), hist[it]), f"iteration {it + 1}"
