"""Compressed graphs joined into one (lpa_hg_concat), the layout of a
lockstep batch: each graph's arcs decode shifted by its id base, and exact
label propagation on the joined graph is each graph's own, shifted."""
import numpy as np
import pytest

import lpa_b200 as L
import oracle


def _graphs():
    out = []
    for i, (kind, size, thr) in enumerate([("road", 30, 0), ("rmat", 11, 16), ("empty", 17, 0), ("road", 9, 16),
                                           ("small", 9, 1 << 20), ("rmat", 9, 0), ("road", 4, 0)]):
        if kind == "road":
            g = L.HostGraph.road(size, size + 3, seed=10 + i)
        elif kind == "empty":
            g = L.HostGraph.from_csr(np.zeros(size + 1, np.uint64), np.zeros(0, np.uint32))
        else:
            g = L.HostGraph.rmat(size, 6, seed=10 + i)
        g.compress(thr, max(thr, 128))
        out.append(g)
    return out


def test_concat_decodes_each_graph_shifted():
    graphs = _graphs()
    u = L.HostGraph.concat(graphs)
    arr = u.arrays()
    row, clm = oracle.decode_csr(arr)
    base = 0
    bits = 0
    for g in graphs:
        grow, gclm = g.csr()
        n = len(grow) - 1
        sub_row = row[base:base + n + 1] - row[base]
        assert np.array_equal(sub_row, grow)
        assert np.array_equal(clm[row[base]:row[base + n]], gclm + base)
        a = g.arrays()
        bits += int(a["offsets"][-1]) if a["n_c"] else 0
        base += n
    assert arr["n"] == base and len(row) == base + 1
    assert int(arr["offsets"][-1]) == bits  # joined bit for bit: every offset exact
    assert arr["n_c"] == sum(g.arrays()["n_c"] for g in graphs)


def test_concat_exact_propagation_is_shift_invariant():
    graphs = _graphs()
    u = L.HostGraph.concat(graphs)
    row, clm = oracle.decode_csr(u.arrays())
    joined, _ = oracle.lp_run(row, clm, 6)
    base = 0
    for g in graphs:
        grow, gclm = g.csr()
        n = len(grow) - 1
        alone, _ = oracle.lp_run(grow, gclm, 6)
        for it in range(6):
            assert np.array_equal(joined[it][base:base + n] - base, alone[it])
        base += n


def test_concat_rejects_bad_input():
    with pytest.raises(L.LpaError):
        L.HostGraph.concat([])
    a = L.HostGraph.road(6, 6, seed=1).compress(0, 128).arrays()
    a["offsets"] = a["offsets"].copy()
    a["offsets"][-1] = 32 * len(a["words"]) + 1  # past the words
    with pytest.raises(L.LpaError):
        L.HostGraph.concat([L.desc_from_arrays(a)])
