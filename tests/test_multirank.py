"""The N>1 benchmark path on CPU: two gloo ranks combine their replica figures.

Replicas track disjoint seed sets with no data-path collective; only the
timing maxima and work sums are reduced, which this test runs with the
gloo backend on two processes (127.0.0.1 rendezvous).
"""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, str(__import__("pathlib").Path(__file__).resolve().parents[1]))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = [10.0 + rank, 20.0 - rank, 5.0 * (rank + 1)]
        counts = [100 * (rank + 1), 7, 3, 1, 1]
        t, c = bench.combine_ranks(dist, times, counts, "cpu")
        out.put((rank, t, c, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_two_rank_combination():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, c, seed in results:
        assert t == [11.0, 20.0, 10.0]            # max over ranks
        assert c == [300, 14, 6, 2, 2]            # sums over ranks
    assert results[0][3] != results[1][3]         # replicas draw different seeds
