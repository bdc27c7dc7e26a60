"""The multi-process host logic of bench.py with 2 gloo ranks on CPU: each rank searches
its own planes (no exchange on the data path) and the step time is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = bench.rank_seeds(rank)
        t = bench.reduce_max(0.5 + rank, dist)
        out.put((rank, seeds, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, t0), (r1, s1, t1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 1.5
    assert s0[0] == 1 and s1[0] == 2 and sorted(s0) == sorted(s1) == list(range(1, 9))


def test_single_process_identity():
    import bench
    assert bench.reduce_max(3.25) == 3.25
    assert bench.rank_seeds(0) == list(range(1, 9))
