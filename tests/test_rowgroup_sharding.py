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


def _decode_rank(rank, world, port, q):
    """One rank of the sharded decode: its byte-balanced share of a mixed set's row-group chunks (each chunk in
    the wizard's expression), decoded on the GPU; the decoded chunks go to rank 0 over gloo."""
    import torch
    import torch.distributed as dist

    from fastlanes_b200 import rowgroups as RG
    from fastlanes_b200 import select as SL
    from fastlanes_b200 import workloads as W

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    torch.cuda.set_device(0)  # every rank on the call's one GPU: the ranks never wait on one another's kernels
    rng = np.random.default_rng(21)
    cols = [W.selection_column(rng, int(rng.integers(70, 200)), "cuda", fam)
            for fam in ("for_u32", "for_i64", "delta_i64", "rle", "dict_i32", "dict_rle", "noise")]
    plan = SL.SelectionPlan(cols)
    _, best, _ = plan.wizard()
    chunks = plan.chunks()
    col, first, count = chunks
    width = np.array([cols[c][0].element_size() for c in col])
    b, e = RG.shard_chunks(count * 1024 * width, world)[rank]
    rg = RG.RowGroupSet(cols, chunks, best.cpu().numpy(), "cuda", chunk_range=(b, e))
    rg.decode(graph=False)
    torch.cuda.synchronize()
    # this rank's chunks, flattened in chunk order, as int64 bit patterns
    def as64(t):
        return t.view(torch.int32).to(torch.int64) if t.element_size() == 4 else t.view(torch.int64)

    def chunk(outs, c):
        return outs[col[c]][int(first[c]) * 1024:(int(first[c]) + int(count[c])) * 1024].cpu()

    mine = [as64(chunk(rg.outputs, c)) for c in range(b, e)]
    flat = torch.cat(mine) if mine else torch.zeros(0, dtype=torch.int64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([flat.numel()], dtype=torch.int64))
    top = max(int(s.item()) for s in sizes)  # gloo gathers equal sizes: every share padded to the largest
    padded = torch.zeros(top, dtype=torch.int64)
    padded[: flat.numel()] = flat
    parts = [torch.zeros(top, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(parts, padded)
    if rank == 0:
        whole = torch.cat([p[: int(s.item())] for p, s in zip(parts, sizes)])
        want = torch.cat([as64(chunk([t for t, _ in cols], c)) for c in range(len(col))])
        q.put((int(e - b), len(col), bool(torch.equal(whole, want)), [int(s.item()) for s in sizes]))
    rg.close()
    plan.close()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_decode_their_row_group_shares_and_the_union_is_the_columns():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_decode_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    n0, n_chunks, equal, sizes = q.get(timeout=600)
    for p in ps:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert 0 < n0 < n_chunks and all(s > 0 for s in sizes)
    assert equal
