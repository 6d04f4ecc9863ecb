"""bench.py's multi-GPU plumbing (replicas, max-over-ranks timing) on two
CPU processes with the gloo backend — the host logic that `torchrun bench.py
--gpus N` runs, without a GPU."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local = bench.dist_env()
    dist_mod = bench.init_dist(ws, "gloo")
    try:
        bench.barrier(dist_mod)
        mx = bench.aggregate_max(float(10 * (rank + 1)), dist_mod)
        out.put((rank, ws, mx))
    finally:
        dist_mod.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert res == [(0, 2, 20.0), (1, 2, 20.0)]


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_max(3.5, None) == 3.5
