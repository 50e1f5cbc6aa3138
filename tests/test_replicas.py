"""The multi-GPU path without GPUs: two gloo ranks on the CPU run the replica bookkeeping of
bench.py (disjoint photon-id ranges, max over ranks of the timings, exact sum of integer tallies)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from xmcml_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ranges = [replicas.photon_range(rank, world, 1000, step) for step in range(3)]
        t = replicas.max_over_ranks(1.5 + rank, dist)
        rng = np.random.default_rng(rank)
        tallies = {"absorption": rng.integers(0, 2 ** 62, 64, dtype=np.uint64),
                   "det_count": np.full(5, rank + 1, dtype=np.uint64)}
        summed = replicas.sum_tallies(tallies, dist)
        q.put((rank, ranges, t, {k: v.tolist() for k, v in summed.items()},
               {k: v.tolist() for k, v in tallies.items()}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replica_bookkeeping():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    ids = set()
    for rank, ranges, t, summed, mine in res:
        assert t == 2.5  # max over ranks
        for first, n in ranges:
            block = set(range(first, first + n))
            assert not (ids & block)  # disjoint photon ids across ranks and steps
            ids |= block
    assert len(ids) == world * 3 * 1000
    a0, a1 = np.array(res[0][4]["absorption"], dtype=np.uint64), np.array(res[1][4]["absorption"], dtype=np.uint64)
    for rank, _, _, summed, _ in res:
        assert np.array_equal(np.array(summed["absorption"], dtype=np.uint64), a0 + a1)
        assert summed["det_count"] == [3] * 5


@pytest.mark.parametrize("world,n", [(2, 11), (3, 10), (8, 1_000_001)])
def test_split_total_matches_reference_mpi_split(world, n):
    parts = [replicas.split_total(r, world, n) for r in range(world)]
    assert sum(c for _, c in parts) == n
    assert parts[0][0] == 0
    for (f0, c0), (f1, _) in zip(parts, parts[1:]):
        assert f0 + c0 == f1
    assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
