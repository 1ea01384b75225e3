"""The bench's multi-rank plumbing on CPU with gloo, world size 2: each rank times its own
stream of problems (weak scaling, distinct seeds per rank), and the line reports the maximum
time over ranks and the sum of the work. No data-path collective exists to test."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import torch.distributed as dist
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ms, flops = bench.over_ranks(dist, torch, world, torch.device("cpu"), 10.0 + rank, 1e12 * (rank + 1))
        specs = bench.stream_specs(2025 + 7919 * rank, 4)
        out.put((rank, ms, flops, specs))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_sum_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for _, ms, flops, _ in res:
        assert ms == 11.0 and flops == 3e12
    assert res[0][3] != res[1][3]  # each rank its own problems


def test_one_rank_is_identity():
    import torch
    import bench
    assert bench.over_ranks(None, torch, 1, torch.device("cpu"), 5.0, 7.0) == (5.0, 7.0)
