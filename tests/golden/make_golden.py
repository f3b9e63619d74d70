"""Generates the golden fixtures under tests/golden/<case>/.

Each case is a small seeded graph written as an edge list (g.txt) and run
through the REFERENCE's own CPU ingest + compressor (oracle/_ref/cgr_ref,
built from the reference's unmodified src/compressor.cpp and src/file.cpp by
oracle/Makefile), which writes g.txt.{graph,offset,vertices.bin,row,clm} and,
when small vertices exist, g.txt.{graph.small.bin,offset.small.bin}.  These
reference outputs pin (a) the CPU oracle's decoder (decode == .row/.clm) and
(b) the native encoder (byte-identical files).

Run from the repository root after `python -m lpa_b200.build` and
`make -C oracle ref` (needs the reference sources):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import lpa_b200 as L  # noqa: E402
import oracle  # noqa: E402

HERE = Path(__file__).resolve().parent


def stress_csr():
    """A graph built to exercise every layout path: long intervals, many
    interval segments, many residual segments, the merged final segment,
    huge gaps and first values on both sides of the vertex id."""
    rng = np.random.default_rng(12345)
    n = 6000
    adj = [set() for _ in range(n)]

    def add(u, v):
        if u != v:
            adj[u].add(v)
            adj[v].add(u)

    for v in range(1, 2500):  # vertex 0: one long interval
        add(0, v)
    for v in range(3, 5000, 2):  # vertex 1: many residual segments (gap 1)
        add(1, v)
    x = 100
    while x < 5900:  # vertex 2: many short intervals -> many interval segments
        for k in range(int(rng.integers(4, 7))):
            add(2, x + k)
        x += int(rng.integers(8, 20))
    for v in list(range(4000, 4003)) + list(range(4010, 4013)):  # vertex 3: runs of 3 (residuals)
        add(3, v)
    for v in [5999, 5998, 5000, 4, 5]:  # vertex 4: large gaps
        add(4, v)
    x = 10
    while x < 5990:  # vertex 5: alternating intervals and residuals
        for k in range(4):
            add(5, x + k)
        add(5, x + 6)
        x += int(rng.integers(9, 40))
    for v in range(6, n):  # background: a few random neighbours each
        for u in rng.integers(0, n, size=int(rng.integers(0, 4))):
            add(v, int(u))
    row = np.zeros(n + 1, np.uint64)
    for v in range(n):
        row[v + 1] = row[v] + len(adj[v])
    clm = np.concatenate([np.array(sorted(a), np.uint32) for a in adj])
    return row, clm


CASES = {
    # name: (builder, both_arcs, one_way flag, small-node threshold)
    "road_a": (lambda: L.HostGraph.road(40, 40, seed=1), True, 0, 0),
    "road_b": (lambda: L.HostGraph.road(50, 30, seed=3), False, 1, 0),
    "rmat_t32": (lambda: L.HostGraph.rmat(10, 8, seed=1), True, 0, 32),
    "rmat_t16": (lambda: L.HostGraph.rmat(11, 16, seed=7), True, 0, 16),
    "copy_t16": (lambda: L.HostGraph.copy_model(1500, 30, seed=1), True, 0, 16),
    "stress": (lambda: L.HostGraph.from_csr(*stress_csr()), True, 0, 0),
    "stress_t8": (lambda: L.HostGraph.from_csr(*stress_csr()), True, 0, 8),
}

# edge lists kept as ingest fixtures (one per one_way setting)
KEEP_EDGE_LIST = {"road_a", "road_b"}

OUT_EXT = [".graph", ".offset", ".vertices.bin", ".graph.small.bin", ".offset.small.bin", ".row", ".clm"]


def main():
    if not oracle.REF_BIN.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref"], check=True)
    for name, (build, both, one_way, thr) in CASES.items():
        d = HERE / name
        d.mkdir(exist_ok=True)
        el = d / "g.txt"
        build().write_edge_list(str(el), both)
        for ext in OUT_EXT:
            p = Path(str(el) + ext)
            if p.exists():
                p.unlink()
        r = subprocess.run([str(oracle.REF_BIN), str(el), str(one_way), str(thr)], capture_output=True, text=True)
        if r.returncode != 0:
            raise SystemExit(f"reference compressor failed on {name}:\n{r.stdout}\n{r.stderr}")
        meta = {"one_way": one_way, "small_thresh": thr, "large_thresh": 128,
                "generator": "tests/golden/make_golden.py", "reference": "oracle/_ref/cgr_ref"}
        (d / "meta.json").write_text(json.dumps(meta, indent=1) + "\n")
        if name not in KEEP_EDGE_LIST:  # the .row/.clm outputs hold the same adjacency
            el.unlink()
        sizes = {ext: os.path.getsize(str(el) + ext) for ext in OUT_EXT if os.path.exists(str(el) + ext)}
        print(name, sizes)


if __name__ == "__main__":
    main()
