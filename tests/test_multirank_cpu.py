"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks.

Under torchrun each rank compresses its own block (independent blocks,
weak scaling, no collective on the data path); the step times are reduced
to their maximum over the ranks, and rank 0 alone reports."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    bench.init_dist(world)
    try:
        # step, e2e and one-call times of this rank
        got = bench.reduce_max([1.0 + rank, 10.0 - rank, 5.0], world)
        w = bench.workload(200, 20_000, bench.rank_seed(rank))
        out.put((rank, got, bench.rank_seed(rank), w.sequences().tobytes()))
    finally:
        bench.finish_dist(world)


def test_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict((r, (got, seed, seqs)) for r, got, seed, seqs in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest rank's times
    for r in range(world):
        assert res[r][0] == [2.0, 10.0, 5.0]
    # every rank has a block of its own
    assert res[0][1] != res[1][1]
    assert res[0][2] != res[1][2]


def test_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max([3, 4.5], 1) == [3.0, 4.5]
    a = np.frombuffer(bench.workload(50, 10_000, bench.rank_seed(0)).sequences().tobytes(), dtype=np.uint8)
    b = np.frombuffer(bench.workload(50, 10_000, bench.rank_seed(0)).sequences().tobytes(), dtype=np.uint8)
    assert np.array_equal(a, b)
