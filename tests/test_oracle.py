"""The CPU oracle against the reference's own outputs (CPU only)."""
import numpy as np
import pytest

import oracle
from conftest import CASES, golden_base


@pytest.mark.parametrize("case", CASES)
def test_oracle_decode_matches_reference_csr(case):
    """Decoding the reference compressor's .graph/.offset reproduces its .row/.clm."""
    arr = oracle.read_reference_files(golden_base(case))
    row, clm = oracle.decode_csr(arr)
    assert np.array_equal(row, arr["row"])
    assert np.array_equal(clm, arr["clm"])


@pytest.mark.parametrize("case", ["road_a", "stress", "rmat_t32"])
def test_oracle_rejects_damaged_stream(case):
    arr = oracle.read_reference_files(golden_base(case))
    off = arr["offsets"].copy()
    # move one vertex boundary by a bit: that vertex no longer ends where it should
    k = len(off) // 2
    off[k] += 1
    bad = dict(arr, offsets=off)
    with pytest.raises(ValueError):
        oracle.decode_csr(bad)


def _py_lp_check(row, clm, iters, cms_thr):
    lab = np.arange(len(row) - 1, dtype=np.uint32)
    for _ in range(iters):
        a, ca = oracle.lp_iterate_csr(row, clm, lab, cms_thr, 1)
        b, cb = oracle.lp_iterate_py(row, clm, lab, cms_thr, 1)
        assert np.array_equal(a, b)
        assert ca == cb
        lab = a


@pytest.mark.parametrize("case", ["road_a", "rmat_t32", "copy_t16"])
@pytest.mark.parametrize("cms_thr", [0, 8])
def test_oracle_rule_matches_python_restatement(case, cms_thr):
    """Two independent restatements of the update rule agree (C vs pure Python)."""
    arr = oracle.read_reference_files(golden_base(case))
    _py_lp_check(arr["row"], arr["clm"], 3, cms_thr)


def test_oracle_cgr_path_matches_csr_path():
    arr = oracle.read_reference_files(golden_base("rmat_t16"))
    lab = np.arange(arr["n"], dtype=np.uint32)
    for thr in (0, 16):
        a, ca = oracle.lp_iterate_csr(arr["row"], arr["clm"], lab, thr, 7)
        b, cb = oracle.lp_iterate_cgr(arr, lab, thr, 7)
        assert np.array_equal(a, b) and ca == cb
        lab = a


def test_tie_break_and_isolated_vertices():
    # 0:{1,2}  1:{0}  2:{0}  3:{} ; labels 1 and 2 tie for vertex 0 -> smallest (1)
    row = np.array([0, 2, 3, 4, 4], np.uint64)
    clm = np.array([1, 2, 0, 0], np.uint32)
    lab = np.array([9, 5, 3, 7], np.uint32)
    out, ch = oracle.lp_iterate_csr(row, clm, lab)
    assert list(out) == [3, 9, 9, 7]  # vertex 0: labels {5,3} tie -> 3; isolated 3 keeps 7
    assert ch == 3


def _cm_hash_py(r, k):
    """include/cms.cuh:96-132 restated once more in Python (32-bit wrap)."""
    M = 0xFFFFFFFF
    consts = [(16, 0x12ebcb3b, 13, 0xc123ae53, 16), (16, 0x21eb21bb, 13, 0x2cb2ea35, 16),
              (16, 0x8febce61, 13, 0xa2b2be25, 16), (12, 0x13ebdb3a, 12, 0xc123ae53, 14)]
    s1, m1, s2, m2, s3 = consts[r]
    k ^= k >> s1
    k = (k * m1) & M
    k ^= k >> s2
    k = (k * m2) & M
    k ^= k >> s3
    return k


def test_cms_hash_family():
    seeds = oracle.cms_seeds(1)
    rng = np.random.default_rng(0)
    for key in [0, 1, 2, 12345, 0xFFFFFFFE] + [int(x) for x in rng.integers(0, 2**32 - 1, 50)]:
        for r in range(4):
            assert oracle.cms_index(r, key, int(seeds[r])) == _cm_hash_py(r, key ^ int(seeds[r])) % 1024


def test_cms_rule_small_example():
    # vertex 0 has 10 neighbours; with a sketch threshold of 4 it takes the sketch path.
    nb = [1, 1, 1, 2, 2, 3, 4, 5, 6, 7]
    n = 8
    row = np.zeros(n + 1, np.uint64)
    row[1:] = len(nb)
    clm = np.array(nb, np.uint32)
    lab = np.arange(n, dtype=np.uint32)
    out, _ = oracle.lp_iterate_csr(row, clm, lab, cms_thr=4)
    py, _ = oracle.lp_iterate_py(row, clm, lab, cms_thr=4)
    assert out[0] == py[0] == 1
