"""Host logic of the multi-GPU batched form, on CPU: the cost-balanced partition and
the one all-gather of per-matrix results, run as world_size-2 gloo process groups
(no GPU needed)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from cucholesky import shard


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    sizes = rng.integers(8, 513, 1000).tolist()
    for parts in (1, 2, 3, 8):
        p = shard.partition_by_cost(sizes, parts)
        flat = sorted(i for ix in p for i in ix)
        assert flat == list(range(len(sizes)))
        ld = shard.loads(sizes, p)
        # LPT guarantee: the spread is at most the largest single cost
        assert max(ld) - min(ld) <= max(s ** 3 for s in sizes)
        assert max(ld) <= sum(ld) / parts * 1.01 + max(s ** 3 for s in sizes)


def test_partition_deterministic_and_edge_cases():
    sizes = [5, 5, 5, 9]
    assert shard.partition_by_cost(sizes, 2) == shard.partition_by_cost(sizes, 2)
    assert shard.partition_by_cost([], 3) == [[], [], []]
    assert shard.partition_by_cost([7], 4) == [[0], [], [], []]
    with pytest.raises(ValueError):
        shard.partition_by_cost(sizes, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        part = shard.partition_by_cost(sizes, world)[rank]
        # stand-in results of this rank's plan: info 0 except every 7th matrix
        info = [(i + 1) if i % 7 == 0 else 0 for i in part]
        logdet = [0.5 * i for i in part]
        info_all, logdet_all = shard.gather_results(part, info, logdet, len(sizes))
        q.put((rank, info_all.tolist(), logdet_all.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gather_results_gloo(world):
    import torch.multiprocessing as mp
    sizes = [int(s) for s in np.random.default_rng(1).integers(8, 513, 37)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_info = [(i + 1) if i % 7 == 0 else 0 for i in range(len(sizes))]
    want_ld = [0.5 * i for i in range(len(sizes))]
    for rank, info_all, logdet_all in got:
        assert info_all == want_info
        assert logdet_all == want_ld
