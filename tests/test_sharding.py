"""Multi-rank host logic on CPU: 2 gloo ranks shard a particle list, each "searches" its slice
(a deterministic stand-in computed on the host), and rank 0 gathers identical rows to a single-rank
run; the step time is the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from emclarity_b200 import sharding


@pytest.mark.parametrize("n,world", [(10, 3), (2000, 8), (1, 2), (0, 2), (7, 7)])
def test_shard_range_partitions(n, world):
    seen = []
    for r in range(world):
        b, e = sharding.shard_range(n, r, world)
        seen.extend(range(b, e))
        assert e - b in (n // world, n // world + 1)
    assert seen == list(range(n))


def test_shard_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        sharding.shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_search(begin, end):
    # one result row per particle: (particle id, best orientation, cc, dx, dy, dz)
    ids = np.arange(begin, end)
    return np.stack([ids, ids % 17, 0.1 + ids * 1e-3, ids % 3 - 1, ids % 5 - 2, ids % 7 - 3], axis=1).astype(float)


def _worker(rank, world, port, n, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b, e = sharding.shard_range(n, rank, world)
        rows = _fake_search(b, e)
        allrows = sharding.gather_rows(rows, world)
        t = sharding.max_over_ranks(1.0 + rank, world)
        if rank == 0:
            out.put((allrows, t))
        else:
            assert allrows is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [11, 64])
def test_two_gloo_ranks_gather_matches_single_rank(n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    rows, t = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.array_equal(rows, _fake_search(0, n))
    assert t == 2.0
