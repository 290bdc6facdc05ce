"""Row-group sharding over ranks (host logic, no GPU): contiguous, complete, byte-balanced ranges that every
rank computes identically, checked across two gloo processes."""
import os

import numpy as np
import pytest

from fastlanes_b200.rowgroups import shard_chunks


def test_shards_tile_and_balance():
    rng = np.random.default_rng(0)
    w = rng.integers(1, 1000, 5000)
    for world in (1, 2, 3, 8):
        sh = shard_chunks(w, world)
        assert sh[0][0] == 0 and sh[-1][1] == w.size
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        loads = [w[b:e].sum() for b, e in sh]
        assert max(loads) - min(loads) <= 2 * w.max()


def test_more_ranks_than_chunks():
    sh = shard_chunks([5, 5], 4)
    assert sh[0][0] == 0 and sh[-1][1] == 2
    assert sum(e - b for b, e in sh) == 2


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = np.random.default_rng(7).integers(1, 10_000, 777)
    b, e = shard_chunks(w, world)[rank]
    mine = torch.tensor([b, e, int(w[b:e].sum())], dtype=torch.int64)
    got = [torch.zeros(3, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(got, mine)
    if rank == 0:
        q.put([t.tolist() for t in got])
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_split():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = q.get(timeout=120)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    (b0, e0, l0), (b1, e1, l1) = res
    assert b0 == 0 and e0 == b1 and e1 == 777
    w = np.random.default_rng(7).integers(1, 10_000, 777)
    assert l0 + l1 == w.sum() and abs(l0 - l1) <= 2 * w.max()
