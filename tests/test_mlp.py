"""The dispatch cost model: gradients against the CPU oracle, and learned
dispatch against the fixed heuristic."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle
from oracle import mlp as M


def test_oracle_gradient_matches_finite_differences():
    """The numpy oracle itself, checked by central differences (float64)."""
    rng = np.random.default_rng(0)
    P = rng.normal(0, 0.3, M.N_PARAMS)
    X = rng.uniform(0, 1, (16, 6))
    V = rng.integers(0, 4, 16)
    T = rng.uniform(0, 1, 16)
    g, _ = M.gradient(P, X, V, T)
    eps = 1e-6
    for i in rng.choice(M.N_PARAMS, 40, replace=False):
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        num = (M.gradient(Pp, X, V, T)[1] - M.gradient(Pm, X, V, T)[1]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-5 * max(1.0, abs(g[i]))


@pytest.mark.gpu
def test_gpu_gradient_matches_oracle():
    """The library's backward kernel against the CPU oracle (fp32 vs fp64:
    relative tolerance 2e-3 on the gradient vector, 1e-4 on the loss)."""
    rng = np.random.default_rng(1)
    P = rng.normal(0, 0.3, M.N_PARAMS).astype(np.float32)
    X = rng.uniform(0, 1, (3000, 6)).astype(np.float32)
    V = rng.integers(0, 4, 3000).astype(np.uint8)
    T = rng.uniform(0, 1, 3000).astype(np.float32)
    g_gpu, loss_gpu = L.mlp_gradient(P, X, V, T)
    g_cpu, loss_cpu = M.gradient(P, X, V, T)
    assert abs(loss_gpu - loss_cpu) <= 1e-4 * loss_cpu
    err = np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu)
    assert err < 2e-3, err
    y_gpu = L.mlp_predict(P, X[:100])
    y_cpu, _ = M.forward(P, X[:100])
    assert np.allclose(y_gpu, y_cpu, rtol=1e-4, atol=1e-5)


@pytest.mark.gpu
def test_learned_dispatch_labels_identical_and_judged():
    """Learned dispatch never changes labels; after exploring it is judged
    against the fixed heuristic and keeps whichever plan was faster."""
    g = L.HostGraph.rmat(18, 16, seed=3)
    row, clm = g.csr()
    g.compress(32, 128)
    hist, _ = oracle.lp_run(row, clm, 10, cms_thr=1024)
    with L.Propagator(g, cms_threshold=1024, dispatch=L.Dispatch.LEARNED) as p:
        for it in range(10):
            p.iterate()
            assert np.array_equal(p.labels(), hist[it]), f"iteration {it + 1}"
        st = p.stats()
        assert st.mlp_updates > 0
        plan, pred = p.learned_plan()
        assert len(plan) == p.get_info().num_segments
        assert np.isfinite(pred).all()
        # the judge's verdict decides what runs: the learned plan while it is
        # the faster, else the fixed plan with the revert counted
        if st.learned_active:
            assert np.array_equal(p.current_plan(), plan)
        else:
            assert st.dispatch_reverts >= 1


def _plan_ms(p, plan, iters=10, reps=3):
    """Least mean device time of iterations 1..iters from the initial labels."""
    p.set_plan(plan)
    best = None
    for _ in range(reps):
        p.init_labels()
        t = 0.0
        for _ in range(iters):
            p.iterate()
            t += p.stats().last_iter_ms
        best = t / iters if best is None else min(best, t / iters)
    return best


@pytest.mark.gpu
def test_mlp_plan_beats_every_single_variant_plan_on_a_mixed_graph():
    """What the trained network gains: on a graph whose parts want different
    kernels -- a road grid (tiny degrees: the lane-per-vertex kernel) joined
    with an R-MAT graph (power-law degrees: the two-pass kernels) -- the
    cost model's own plan, chosen per segment, is at least as fast as the
    best plan that puts every segment on one variant (where it can run), and
    faster than the fixed degree buckets.  Its labels equal the oracle's."""
    road = L.HostGraph.road(1404, 1404, seed=1).compress(0, 128)
    rmat = L.HostGraph.rmat(18, 16, seed=1).compress(32, 128)
    g = L.HostGraph.concat([road, rmat])
    with L.Propagator(g, dispatch=L.Dispatch.FIXED, record_timings=1) as p:
        fixed = p.current_plan().copy()
        cap = p.capable()
        p.set_dispatch(L.Dispatch.LEARNED)
        p.init_labels()
        for _ in range(8):  # fixed, 4 explorations, trials: the learner settles
            p.iterate()
        mlp = p.mlp_plan()
        assert (((cap >> mlp) & 1) == 1).all()
        t_mlp = _plan_ms(p, mlp)
        static = {}
        for v in L.Variant:
            plan = fixed.copy()
            plan[((cap >> int(v)) & 1) == 1] = int(v)
            static[v.name] = _plan_ms(p, plan)
        t_fixed = _plan_ms(p, fixed)
        best = min(static.values())
        assert t_mlp <= best, f"cost model's plan {t_mlp:.4f} ms vs single-variant plans {static}"
        assert t_mlp < t_fixed, f"cost model's plan {t_mlp:.4f} ms vs fixed plan {t_fixed:.4f} ms"
        # the plan is per segment: it mixes variants on this graph
        assert len(np.unique(mlp)) >= 2
        # and it computes the same labels
        arr = g.arrays()
        lab = np.arange(arr["n"], dtype=np.uint32)
        p.set_plan(mlp)
        p.init_labels()
        for it in range(3):
            ch = p.iterate()
            lab, och = oracle.lp_iterate_cgr(arr, lab)
            assert np.array_equal(p.labels(), lab) and ch == och, f"iteration {it + 1}"
