"""Multi-GPU runs are replicas (no data-path exchange): the only cross-rank
steps are the barrier around the timed region, the maximum of the ranks'
device times, and rank 0 sharing the generated graph with the other ranks.
These run here as two gloo processes on the CPU."""
import os
import socket
import uuid

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the slowest rank's time is the job's time
        t = bench.max_over_ranks(10.0 + rank, world, "cpu")
        bench.barrier(world, "cpu")
        w = dict(kind="road", width=24, height=20, seed=3, small_thresh=0, cms=0, iters=5)
        arr = bench.shared_graph_arrays(name, w, rank, world)
        out[rank] = (t, int(arr["n"]), int(arr["n_c"]), int(np.asarray(arr["words"]).sum() % 1000003))
    finally:
        dist.destroy_process_group()


def test_two_replicas_share_graph_and_max_time():
    pytest.importorskip("torch")
    world = 2
    name = f"test_{uuid.uuid4().hex[:8]}"
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), name, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0
    assert res[0][1:] == res[1][1:]  # rank 1 loaded what rank 0 built
    import shutil
    shutil.rmtree(f"/dev/shm/lpa_bench_{name}", ignore_errors=True)
