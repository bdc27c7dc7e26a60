"""The multi-process host logic of bench.py with 2 gloo ranks on CPU: each rank takes its
own planes (no exchange on the data path), runs the per-rank bookkeeping of a step (its
plane, the level node lists, the eval count the plan must report) and a search of its own
plane (the CPU oracle standing in for the device), and the step time is the max over ranks.
Rank 0 gathers every rank's result and checks it against the same work done in one process:
the partition covers the seeds without overlap and no rank's result depends on another's."""
import hashlib
import os
import socket

import numpy as np
import torch.multiprocessing as mp

CROP = 96  # the per-rank search runs on a crop of the rank's plane (seconds on CPU)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_work(rank):
    """One rank's step bookkeeping and the digest of its plane's search (size 8, stride 2)."""
    import bench
    from mars_b200 import synthetic
    from oracle import oracle as orc
    seeds = bench.rank_seeds(rank)
    plane = synthetic.gray(bench.W, bench.H, seeds[0])
    nodes = {s: len(bench.level_nodes(s)[0]) for s in bench.SIZES}
    crop = plane[:CROP, :CROP]
    cands, evals = orc.search_grid(crop, 8, 2, orc.make_params(shift=2), nthreads=1)
    return {"rank": rank, "seeds": seeds, "nodes": nodes, "evals_per_step": bench.evals_per_step(),
            "plane": hashlib.sha256(plane.tobytes()).hexdigest(),
            "search": hashlib.sha256(cands.tobytes()).hexdigest(), "search_evals": int(evals.sum())}


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = _rank_work(rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = bench.reduce_max(0.5 + rank, dist)
        out.put((rank, gathered, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_search_and_max():
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, g0, t0), (r1, g1, t1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 1.5  # the step time is the slowest rank's
    assert g0 == g1  # every rank sees the same gathered results
    s0, s1 = g0[0]["seeds"], g0[1]["seeds"]
    assert s0[0] == 1 and s1[0] == 2 and sorted(s0) == sorted(s1) == list(range(1, 9))
    # Each rank's result equals the same work done alone in this process.
    for r in range(2):
        assert g0[r] == _rank_work(r)
    assert g0[0]["plane"] != g0[1]["plane"]
    assert g0[0]["evals_per_step"] == sum(bench.level_evals(s) * n for s, n in g0[0]["nodes"].items())


def test_single_process_identity():
    import bench
    assert bench.reduce_max(3.25) == 3.25
    assert bench.rank_seeds(0) == list(range(1, 9))
    assert bench.evals_per_step() == 11_000_915_968
    assert sum(len(bench.level_nodes(s)[0]) for s in bench.SIZES) == 21_760
    np.testing.assert_array_equal(bench.level_nodes(32)[0][:3], [0, 0, 0])
