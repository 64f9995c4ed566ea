"""bench.py's aggregation over ranks (replicas on N GPUs): the whole-job time is the slowest
rank's, the work counts are summed.  Two gloo ranks on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        seconds, counts = bench.reduce_ranks(dist, torch, 1.5 + rank, [10 * (rank + 1), 7], "cpu")
        out[rank] = (seconds, counts)
    finally:
        dist.destroy_process_group()


def test_reduce_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    for r in range(2):
        assert out[r] == (2.5, [30, 14])
