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
        assert st.learned_active in (0, 1)
