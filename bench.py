#!/usr/bin/env python
"""Benchmark: one synchronous label-propagation iteration over a CGR graph.

Metric: decoded arcs x iterations per second (every stored arc is decoded and
its label counted once per iteration), with the roofline of one iteration
(its kernels together) against the measured HBM copy bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload rmat-s24]
    python bench.py --impl reference ...   # the CPU path (oracle port), same metric

Multi-GPU: one process per GPU (torchrun); every rank runs an independent
replica of the workload (the path has no exchange step on one graph);
value = the arcs all ranks processed / the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "decoded arcs×iters/sec"
UNIT = "arcs*iters/s"
L2_BYTES = 126 * 1024 * 1024

WORKLOADS = {
    # R-MAT scale 24, edge factor 16 (a,b,c,d = .57,.19,.19,.05), symmetrised,
    # de-duplicated, loops dropped, BFS relabelled; CGR threshold 32; sketch at >= 1024
    "rmat-s24": dict(kind="rmat", scale=24, edge_factor=16.0, seed=1, small_thresh=32, cms=1024, iters=20),
    # road-like grid 1404x1404, p=0.7, 2% extras within distance 3, threshold 0
    "road-1404": dict(kind="road", width=1404, height=1404, seed=1, small_thresh=0, cms=0, iters=30),
    # road-like grid 362x362 (the reference's CPU-runnable case)
    "road-362": dict(kind="road", width=362, height=362, seed=1, small_thresh=0, cms=0, iters=20),
    # smaller R-MAT for quick checks
    "rmat-s20": dict(kind="rmat", scale=20, edge_factor=16.0, seed=1, small_thresh=32, cms=1024, iters=20),
    "rmat-s22": dict(kind="rmat", scale=22, edge_factor=16.0, seed=1, small_thresh=32, cms=1024, iters=20),
    # web-like copy model: 100M vertices, out-degree 30 (prototype copies p=0.6 with
    # offsets in [-8,8], else Zipf(1.1) targets); threshold 16, sketch >= 4096
    "copy-100m": dict(kind="copy", n=100_000_000, out_degree=30, seed=1, small_thresh=16, cms=4096, iters=10,
                      loop="graph"),
    # many uneven graphs in one persistent launch: vertex counts log-uniform in
    # [1k, 256k], even graphs road grids (p=0.7), odd graphs R-MAT (edge factor 8),
    # threshold 16, per-graph early exit (the 4096-graph [1k, 2M] batch scaled down)
    "batch-256": dict(kind="batch", graphs=256, n_lo=1000, n_hi=262144, seed=1, small_thresh=16, cms=0, iters=30),
    # all 4096 graphs, sizes log-uniform in [1k, 128k]
    "batch-4096": dict(kind="batch", graphs=4096, n_lo=1000, n_hi=131072, seed=1, small_thresh=16, cms=0,
                       iters=30),
    # the full batch: 4096 graphs, sizes log-uniform in [1k, 2M] (about 1.1e9 vertices, 1e10 arcs)
    "batch-4096-full": dict(kind="batch", graphs=4096, n_lo=1000, n_hi=2_000_000, seed=1, small_thresh=16, cms=0,
                            iters=30),
}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Maximum of a per-rank scalar over all ranks (the slowest rank's time)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist

        if device is not None and str(device).startswith("cuda"):
            dist.barrier(device_ids=[int(str(device).split(":")[1])])
        else:
            dist.barrier()


def build_graph(w: dict):
    import lpa_b200 as L

    if w["kind"] == "rmat":
        g = L.HostGraph.rmat(w["scale"], w["edge_factor"], seed=w["seed"])
    elif w["kind"] == "copy":
        g = L.HostGraph.copy_model(w["n"], w["out_degree"], seed=w["seed"])
    else:
        g = L.HostGraph.road(w["width"], w["height"], seed=w["seed"])
    g.compress(w["small_thresh"], 128)
    return g


def build_batch(w: dict):
    """The batched workload's graphs (seeded; seed + i for graph i), generated
    and compressed on all host cores (the generators release the GIL)."""
    import concurrent.futures as cf

    import lpa_b200 as L

    rng = np.random.default_rng(w["seed"])
    sizes = [int(np.exp(rng.uniform(np.log(w["n_lo"]), np.log(w["n_hi"])))) for _ in range(w["graphs"])]

    def make(i):
        n = sizes[i]
        if i % 2 == 0:
            side = max(4, int(round(np.sqrt(n))))
            g = L.HostGraph.road(side, side, seed=w["seed"] + i)
        else:
            g = L.HostGraph.rmat(max(8, int(np.ceil(np.log2(n)))), 8.0, seed=w["seed"] + i, n_limit=n)
        g.compress(w["small_thresh"], 128, threads=1)
        return g

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        return list(ex.map(make, range(w["graphs"])))


def verify_batch(bt, graphs, iters, max_check: int = 8) -> dict:
    """Per-graph labels of the batch's last run against the oracle run alone
    on that graph (same iterations, early exit), on a sample: the smallest and
    the largest graph of each kind and graphs spread between them."""
    import oracle

    order = sorted(range(len(graphs)), key=lambda i: int(graphs[i].desc().num_vertices))
    pick = sorted(set(order[:: max(1, len(order) // (max_check - 2))][: max_check - 2] + order[-2:]))
    bad = 0
    for i in pick:
        row, clm = graphs[i].csr()
        hist, _ = oracle.lp_run(row, clm, 30, early_exit=True)
        want = hist[min(int(iters[i]), len(hist)) - 1] if len(hist) else np.arange(len(row) - 1, dtype=np.uint32)
        bad += int(len(hist) != int(iters[i])) + int(np.count_nonzero(bt.labels(i) != want))
    return {"graphs_checked": len(pick), "mismatches": bad,
            "vertices_checked": int(sum(int(graphs[i].desc().num_vertices) for i in pick))}


def graph_meta(g) -> dict:
    """Sizes of a compressed host graph, read without copying its arrays."""
    d = g.desc()
    n, n_c = int(d.num_vertices), int(d.num_compressed)
    return {"n": n, "n_c": n_c, "bits": int(d.offsets[n_c]) if n_c else 0, "m_small": int(d.num_small_arcs)}


def algorithmic_bytes(meta: dict) -> int:
    """One iteration's compulsory bytes of one graph (see lpa_info)."""
    n, n_c = meta["n"], meta["n_c"]
    return ((meta["bits"] + 7) // 8 + 8 * (n_c + 1) + 4 * n_c + 4 * (n - n_c + 1) + 4 * meta["m_small"] + 12 * n)


def run_batch(args, w, rank, world, local):
    """Batched graphs: a step is one persistent launch running every graph to
    convergence (<= iters iterations)."""
    import torch

    import lpa_b200 as L

    device = f"cuda:{local}"
    graphs = build_batch(w)
    arrs = [graph_meta(g) for g in graphs]
    stream = torch.cuda.Stream(device=device)
    mode = L.BatchMode.LOCKSTEP if args.batch_mode == "lockstep" else L.BatchMode.QUEUE
    dispatch = L.Dispatch.LEARNED if args.dispatch == "learned" else L.Dispatch.FIXED
    with L.Batch(graphs, device=local, cms_threshold=w["cms"], stream=stream.cuda_stream, batch_mode=mode,
                 dispatch=dispatch) as bt:
        h = bt.handle()  # lockstep: the concatenated graph's handle
        degs = [g.num_arcs() for g in graphs]  # arcs per graph from the host CSR
        for _ in range(args.warmup):
            iters = bt.run(w["iters"], early_exit=True)
        tune = None
        if h is not None and args.autotune:  # tuned on the labels the last warm-up run left
            tune = list(h.autotune(None, repeats=2).as_tuple())
        barrier(world, device)
        torch.cuda.synchronize()
        launches0 = h.stats().launches if h is not None else 0
        clocks = ClockSampler(local)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total_ms = 0.0
        work = 0
        bytes_done = 0
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            ev0.record(stream)
            iters = bt.run(w["iters"], early_exit=True)
            ev1.record(stream)
            ev1.synchronize()
            total_ms += ev0.elapsed_time(ev1)
            work += sum(int(d) * int(k) for d, k in zip(degs, iters))
            bytes_done += sum(algorithmic_bytes(a) * int(k) for a, k in zip(arrs, iters))
        wall = time.perf_counter() - wall0
        clk = clocks.stop()
        # lockstep: the handle's own count (iteration kernels plus the
        # two tracker launches); queue: the init kernel and k_batch
        launches = (h.stats().launches - launches0) if h is not None else 2 * args.steps
        total_ms = max_over_ranks(total_ms, world, device)
        value = work * world / (total_ms / 1e3)
        # end to end: a run plus every graph's labels back to pinned host memory
        pinned = torch.empty(sum(a["n"] for a in arrs), dtype=torch.int32, pin_memory=True)
        outs, at = [], 0
        for a in arrs:
            outs.append(pinned.narrow(0, at, a["n"]))
            at += a["n"]
        lib = L.lib()
        import ctypes as C

        e0 = time.perf_counter()
        for _ in range(max(1, args.e2e_steps)):
            it_e = bt.run(w["iters"], early_exit=True)
            for gi, o in enumerate(outs):
                assert lib.lpa_batch_get_labels(bt._h, gi, C.cast(C.c_void_p(o.data_ptr()), C.POINTER(C.c_uint32)),
                                                arrs[gi]["n"]) == 0
        e2e_s = max_over_ranks(time.perf_counter() - e0, world, device)
        e2e_work = sum(int(d) * int(k) for d, k in zip(degs, it_e)) * max(1, args.e2e_steps)
        verify = verify_batch(bt, graphs, it_e) if (rank == 0 and not args.no_cpu_baseline) else None
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_done / (total_ms / 1e3) / 1e9
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": {"workload": args.workload, "graphs": len(graphs), "vertices": int(sum(a["n"] for a in arrs)),
                           "arcs": int(sum(degs)), "iterations_per_graph": [int(k) for k in iters][:8] + ["..."],
                           "l2": "inputs larger than L2" if sum(algorithmic_bytes(a) for a in arrs) > 2 * L2_BYTES
                           else "resident", "parallelism": f"replicas x{world}", "batch_mode": args.batch_mode,
                           "dispatch": args.dispatch if h is not None else "fixed", "tune": tune},
                "roofline": {"bound": "hbm", "kernel": "lockstep iteration kernels" if h is not None else "k_batch",
                             "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": peak_kind, "traffic": None},
                "cpu_baseline": None,
                "verify": verify,
                "e2e": {"value": e2e_work * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": int(4 * sum(a["n"] for a in arrs))},
                "gpu_launches": int(launches), "clocks": clk, "wall_s_timed": wall}
        print(json.dumps(line), flush=True)


def shared_graph_arrays(name: str, w: dict, rank: int, world: int, device=None) -> dict:
    """Rank 0 builds the workload; under torchrun the other ranks load rank 0's
    arrays from /dev/shm instead of regenerating them."""
    import lpa_b200 as L

    if world <= 1:
        return build_graph(w).arrays()
    d = Path("/dev/shm") / f"lpa_bench_{name}"
    if rank == 0:
        arr = build_graph(w).arrays()
        d.mkdir(exist_ok=True)
        for k, v in arr.items():
            if isinstance(v, np.ndarray):
                np.save(d / f"{k}.npy", v)
        (d / "meta.json").write_text(json.dumps({"n": arr["n"], "n_c": arr["n_c"]}))
    barrier(world, device)
    if rank != 0:
        meta = json.loads((d / "meta.json").read_text())
        arr = dict(meta)
        for k in ("words", "offsets", "vertices", "small_graph", "small_offset"):
            arr[k] = np.load(d / f"{k}.npy")
    barrier(world, device)
    return arr


class ClockSampler:
    """nvidia-smi samples (SM clock, reasons) while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-i", str(device_index), "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for nm, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def traffic_summary(workload: str):
    """DRAM bytes per iteration (its kernels together) from the committed ncu summaries."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(workload)
        except Exception:
            return None
    return None


def cpu_baseline(arr: dict, w: dict, budget_s: float = 12.0) -> dict:
    """The oracle's OpenMP CPU path (decode + synchronous LP, same rule) on a
    bounded sample of the same workload: a prefix of the positions."""
    import oracle

    threads = os.cpu_count() or 1
    n = arr["n"]
    lab = np.arange(n, dtype=np.uint32)
    p_end = min(n, 1 << 14)
    while True:
        t0 = time.perf_counter()
        oracle.lp_iterate_cgr(arr, lab, w["cms"], 1, threads, 0, p_end)
        dt = time.perf_counter() - t0
        if dt > budget_s / 8 or p_end >= n:
            break
        p_end = min(n, p_end * 4)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        oracle.lp_iterate_cgr(arr, lab, w["cms"], 1, threads, 0, p_end)
        times.append(time.perf_counter() - t0)
    row_arcs = oracle.range_arcs(arr, 0, p_end)
    t = statistics.median(times)
    return {"value": row_arcs / t, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
            "sample": f"positions [0,{p_end}) of {n} ({row_arcs} arcs), median of 3 iterations after 1 warm-up"}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_compressor_sample() -> dict | None:
    """The reference's own CPU compressor (CgrCompressor::compresswithcost,
    built from the reference sources into oracle/_ref/cgr_ref) on a bounded
    sample: R-MAT scale 19, edge factor 16, threshold 32, one thread (the
    reference compressor is single-threaded).  None when it was not built."""
    import re

    import lpa_b200 as L

    exe = ROOT / "oracle" / "_ref" / "cgr_ref"
    if not exe.exists():
        return None
    with tempfile.TemporaryDirectory() as td:
        g = L.HostGraph.rmat(19, 16.0, seed=1)
        arcs = int(len(g.csr()[1]))
        path = str(Path(td) / "rmat19.txt")
        g.write_edge_list(path, False)
        t0 = time.perf_counter()
        r = subprocess.run([str(exe), path, "1", "32"], capture_output=True, text=True)
        wall = time.perf_counter() - t0
        m = re.search(r"without I/O:\s*([0-9.eE+-]+)", r.stdout)
        ours0 = time.perf_counter()
        g.compress(32, 128, threads=1)
        ours = time.perf_counter() - ours0
    if r.returncode != 0 or not m:
        return {"error": f"cgr_ref exited {r.returncode}"}
    sec = float(m.group(1))
    return {"sample": "R-MAT scale 19, edge factor 16, threshold 32 (edge list written as the reference's text)",
            "arcs": arcs, "compresswithcost_s": sec, "with_io_s": wall, "arcs_per_s": arcs / sec,
            "this_library_1_thread_s": ours}


def cpu_baseline_and_verify(p, arr: dict, w: dict) -> dict:
    """The oracle's OpenMP CPU path (decode + synchronous LP, same rule) on the
    whole workload, iterations 1..iters from the initial labels: timed, it is
    the CPU baseline; beside it the GPU runs the same iterations on the plan
    and knobs of the timed region, and its labels and changed count are
    compared with the oracle's after every iteration (outside any timed
    region)."""
    import oracle

    threads = os.cpu_count() or 1
    n = arr["n"]
    iters = w["iters"]
    lab = np.arange(n, dtype=np.uint32)
    p.init_labels()
    times = []
    mismatches = changed_mismatches = 0
    first_bad = None
    for it in range(iters):
        gch = p.iterate()
        glab = p.labels()
        t0 = time.perf_counter()
        nxt, och = oracle.lp_iterate_cgr(arr, lab, w["cms"], 1, threads)
        times.append(time.perf_counter() - t0)
        bad = int(np.count_nonzero(glab != nxt))
        mismatches += bad
        changed_mismatches += int(gch != och)
        if (bad or gch != och) and first_bad is None:
            first_bad = {"iteration": it + 1, "labels": bad, "changed": [int(gch), int(och)]}
        lab = nxt
    arcs = oracle.range_arcs(arr, 0, n)
    t = sum(times)
    cb = {"value": arcs * iters / t, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
          "sample": f"the whole workload ({arcs} arcs), iterations 1..{iters} from the initial labels, "
                    f"{t:.1f} s; the oracle's OpenMP decode + LP loop",
          "reference_compressor": reference_compressor_sample()}
    verify = {"iterations": iters, "mismatches": mismatches, "changed_mismatches": changed_mismatches,
              "first_mismatch": first_bad, "oracle": "oracle.lp_iterate_cgr (CPU restatement of the update rule)"}
    return cb, verify


def dispatch_report(p, fixed_plan, steps: int, timed_region) -> dict:
    """Iterations 1..steps from the initial labels on explicit plans, each timed
    like the main region: the cost model's own plan (before the learner's
    trials), the merged candidate (its plan with every capable segment on the
    two-pass kernels), and every single-variant plan (each segment on that
    variant where it can run, else the fixed plan's choice).  The learner is
    reset by the first explicit plan, so this runs last."""
    import lpa_b200 as L

    cap = p.capable()
    plans = {}
    try:
        mlp = p.mlp_plan()
    except L.LpaError:
        mlp = None
    if mlp is not None:
        plans["mlp_plan"] = mlp
        merged = mlp.copy()
        two = int(L.Variant.TWO_PASS)
        merged[(cap >> two) & 1 == 1] = two
        plans["merged"] = merged
    for v in L.Variant:
        plan = fixed_plan.copy()
        ok = (cap >> int(v)) & 1 == 1
        plan[ok] = int(v)
        plans[f"all_{v.name.lower()}"] = plan
    out = {}
    change_ms = []
    for name, plan in plans.items():
        t0 = time.perf_counter()
        p.set_plan(plan)  # the work lists are rebuilt on the device
        change_ms.append((time.perf_counter() - t0) * 1e3)
        p.init_labels()
        ms, _ = timed_region(steps)
        out[name] = ms / steps
    static = {k: v for k, v in out.items() if k.startswith("all_")}
    best = min(static, key=static.get)
    rep = {"mlp_plan_ms": out.get("mlp_plan"), "merged_ms": out.get("merged"), "best_static_ms": static[best],
           "best_static": best, "static_ms": static, "plan_change_ms": statistics.median(change_ms),
           "mlp_plan_variant_segments": [int((plans["mlp_plan"] == v).sum()) for v in range(4)]
           if "mlp_plan" in plans else None}
    return rep


def run_reference(args, w, rank, world):
    if rank != 0:
        return
    arr = build_graph(w).arrays()
    cb = cpu_baseline(arr, w, budget_s=20.0)
    steps = args.steps
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": 0, "steps": steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload, "n": arr["n"], "small_thresh": w["small_thresh"],
                       "cms_threshold": w["cms"], "parallelism": "cpu-openmp"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat-s24", choices=sorted(WORKLOADS))
    ap.add_argument("--dispatch", default="learned", choices=["fixed", "learned"],
                    help="learned: the MLP plan (judged against the fixed buckets, also measured)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--tune", default="",
                    help="explicit two-pass knobs g,w,d,c,bulk,l2 (lpa_tune), instead of the autotuner")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip tuning the count pass's work shapes (lpa_autotune) after the learner's warm-up")
    ap.add_argument("--batch-mode", default="lockstep", choices=["lockstep", "queue"],
                    help="batched workloads: the concatenated graph in lockstep, or the persistent queue")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--loop", choices=["host", "graph"], default=None,
                    help="host: one lpa_iterate per step; graph: the timed steps in one lpa_run (CUDA-graph loop); "
                         "default per workload (graph for copy-100m)")
    ap.add_argument("--no-dispatch-report", dest="dispatch_report", action="store_false",
                    help="skip timing the cost model's own plan and the single-variant plans after the run")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    w = WORKLOADS[args.workload]
    rank, world, local = dist_env()

    if args.impl == "reference":
        run_reference(args, w, rank, world)
        return

    import torch

    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=torch.device(device))

    if w["kind"] == "batch":
        run_batch(args, w, rank, world, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    import lpa_b200 as L

    arr = shared_graph_arrays(args.workload, w, rank, world, device)
    stream = torch.cuda.Stream(device=device)
    p = L.Propagator(L.desc_from_arrays(arr), device=local, cms_threshold=w["cms"], cms_seed=1,
                     record_timings=1, stream=stream.cuda_stream, dispatch=L.Dispatch.FIXED)
    info = p.get_info()
    fixed_plan = p.current_plan()
    arcs = int(info.num_arcs)
    b_alg = int(info.bytes_algorithmic)
    inputs_bytes = b_alg
    flush = inputs_bytes < 2 * L2_BYTES
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=device) if flush else None

    loop = args.loop or w.get("loop", "host")
    if loop == "graph" and flush:
        raise SystemExit("--loop graph needs inputs larger than L2 (no flush fits inside the graph)")

    def timed_region(steps):
        """K iterations; device time of each from the library's CUDA events,
        or with the CUDA-graph loop one lpa_run call of K iterations (the
        iteration kernels and the device-side loop test in a conditional
        node), timed by CUDA events on the library's stream around it."""
        if loop == "graph":
            p.run(1)  # the graph is (re)built for the current plan outside the timing
            p.init_labels()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            done = p.run(steps, early_exit=False)
            e1.record(stream)
            e1.synchronize()
            assert done == steps
            return e0.elapsed_time(e1), np.full(4, np.nan)
        dev = 0.0
        kern = np.zeros(4)
        for _ in range(steps):
            if flush:
                with torch.cuda.stream(stream):
                    flush_buf.fill_(1)
            p.iterate()
            s = p.stats()
            dev += s.last_iter_ms
            kern += np.array([s.decode_ms, s.count_ms, s.packed_ms, s.iterate_ms])
        return dev, kern

    # fixed degree-bucket plan (the reference's buckets): warm-up, then the
    # timed steps are iterations 1..K of a run from the initial labels (the
    # reference's run(20) protocol), so early, label-diverse iterations count
    p.init_labels()
    for _ in range(args.warmup):
        p.iterate()
    p.init_labels()
    barrier(world, device)
    torch.cuda.synchronize()
    fixed_ms, _ = timed_region(args.steps)
    fixed_ms = max_over_ranks(fixed_ms, world, device)
    learned_info = None
    if args.dispatch == "learned":
        # the cost model explores and trains on warm-up iterations, then its plan is timed
        p.set_dispatch(L.Dispatch.LEARNED)
        tune = None
        if args.tune:  # explicit knobs: no tuning
            p.set_tune(*[int(x) for x in args.tune.split(",")])
            tune = list(p.get_tune().as_tuple())
        p.init_labels()
        for _ in range(max(args.warmup, 8)):
            p.iterate()
        if args.autotune and not args.tune:  # the two-pass knobs, tuned on these mid-run labels
            tune = list(p.autotune(None, repeats=2).as_tuple())
        p.init_labels()
        ls = p.stats()
        learned_info = {"active": int(ls.learned_active), "mlp_updates": int(ls.mlp_updates),
                        "mlp_loss": float(ls.mlp_loss), "reverts": int(ls.dispatch_reverts),
                        "segments_per_variant": [int(x) for x in ls.variant_segments],
                        "arcs_per_variant": [int(x) for x in ls.variant_arcs],
                        "tune": tune if tune is not None else list(p.get_tune().as_tuple()),
                        "autotuned": tune is not None and not args.tune}

    st0 = p.stats()
    barrier(world, device)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    wall0 = time.perf_counter()
    dev_ms, kern_ms = timed_region(args.steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    barrier(world, device)
    st1 = p.stats()
    total_ms = max_over_ranks(dev_ms, world, device)
    value = arcs * args.steps * world / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps

    # roofline of one iteration: its kernels (two-pass decode, two-pass
    # count, persistent iteration kernel) together read the compressed graph
    # and the labels and write the labels once; the algorithmic bytes of the
    # iteration over its device time
    kern_avg = kern_ms / args.steps
    peak, peak_kind = measured_peak_gbs()
    achieved = b_alg / (ms_per_step / 1e3) / 1e9

    # end to end through the C ABI with host buffers (pinned)
    host_in = torch.empty(arr["n"], dtype=torch.int32, pin_memory=True)
    host_out = torch.empty(arr["n"], dtype=torch.int32, pin_memory=True)
    host_in.copy_(torch.from_numpy(p.labels().view(np.int32)))
    import ctypes as C

    lib = L.lib()
    in_ptr = C.cast(C.c_void_p(host_in.data_ptr()), C.POINTER(C.c_uint32))
    out_ptr = C.cast(C.c_void_p(host_out.data_ptr()), C.POINTER(C.c_uint32))
    chg = C.c_uint64()
    barrier(world, device)
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        assert lib.lpa_set_labels(p._h, in_ptr, arr["n"]) == 0
        assert lib.lpa_iterate(p._h, C.byref(chg)) == 0
        assert lib.lpa_get_labels(p._h, out_ptr, arr["n"]) == 0
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - e0, world, device)
    e2e_value = arcs * args.e2e_steps * world / e2e_s

    cb = verify = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, verify = cpu_baseline_and_verify(p, arr, w)
    report = None
    if args.dispatch == "learned" and args.dispatch_report:
        report = dispatch_report(p, fixed_plan, args.steps, timed_region)
        report["learned_ms"] = ms_per_step
        report["fixed_ms"] = fixed_ms / args.steps

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": args.workload, "n": arr["n"], "arcs": arcs, "compressed": arr["n_c"],
                       "stream_bytes": (int(info.stream_bits) + 7) // 8, "small_thresh": w["small_thresh"],
                       "cms_threshold": w["cms"], "dispatch": args.dispatch,
                       "timed_iterations": f"1..{args.steps} from the initial labels",
                       "loop": "CUDA-graph loop (lpa_run)" if loop == "graph" else "host loop (lpa_iterate per step)",
                       "l2": "L2 flushed between iterations" if flush else "inputs larger than L2",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm",
                         "kernel": "iteration (k_decode_two_pass + k_count_two_pass + k_packed + k_iterate)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "bytes_per_launch": b_alg, "ms_per_launch": ms_per_step,
                         "traffic": traffic_summary(args.workload),
                         "kernel_ms": None if loop == "graph" else
                         {"k_decode_two_pass": float(kern_avg[0]), "k_count_two_pass": float(kern_avg[1]),
                          "k_packed": float(kern_avg[2]), "k_iterate": float(kern_avg[3])}},
            "dispatch": {"mode": args.dispatch,
                         "fixed_value": arcs * args.steps * world / (fixed_ms / 1e3),
                         "fixed_ms_per_step": fixed_ms / args.steps,
                         "learned_over_fixed": (fixed_ms / total_ms) if args.dispatch == "learned" else None,
                         "learner": learned_info, "plans": report},
            "cpu_baseline": cb,
            "verify": verify,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 4 * arr["n"],
                    "d2h_bytes_per_step": 4 * arr["n"] + 8},
            "gpu_launches": int(st1.launches - st0.launches),
            "clocks": clk,
            "wall_s_timed": wall,
        }
        print(json.dumps(line), flush=True)
    p.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
