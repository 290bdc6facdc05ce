"""GPU parity of the batched primitives against the CPU oracle (which is pinned to the reference's golden
vectors by test_oracle_golden.py).  Bit-exact comparisons throughout."""
import re

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

TYPES = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}


def _t(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _np(t):
    return t.cpu().numpy()


def _batch(w, n_vec, rng, bws=None):
    """Random vectors with per-vector bit width and base; returns packed bytes, offsets, bw, base, values."""
    T = TYPES[w]
    bw = rng.integers(0, w + 1, n_vec).astype(np.uint8) if bws is None else np.asarray(bws, np.uint8)
    base = rng.integers(0, np.iinfo(T).max, n_vec, dtype=np.uint64, endpoint=True).astype(T)
    vals, chunks, offs, pos = [], [], [], 0
    for v in range(n_vec):
        b = int(bw[v])
        x = rng.integers(0, np.iinfo(np.uint64).max, 1024, dtype=np.uint64, endpoint=True)
        if b < 64:
            x &= np.uint64((1 << b) - 1)
        x = (x.astype(T) + base[v]).astype(T)
        vals.append(x)
        p = oracle.ffor(x, b, base[v])
        chunks.append(p.view(np.uint8))
        offs.append(pos)
        pos += p.nbytes
    packed = np.concatenate(chunks + [np.zeros(256, np.uint8)])
    return packed, np.array(offs, np.uint64), bw, base, np.concatenate(vals)


@pytest.mark.parametrize("w", [8, 16, 32, 64])
def test_golden_vectors_unpack_unffor(cuda, prim_golden, w):
    from fastlanes_b200 import primitives as P

    T = TYPES[w]
    for kind, base in (("unpack", 0), ("unffor", 10)):
        keys = sorted((int(m.group(1)) for k in prim_golden.files
                       if (m := re.match(rf"{kind}_w{w}_b(\d+)_in$", k))))
        xs = [prim_golden[f"{kind}_w{w}_b{b}_in"] for b in keys]
        chunks, offs, pos = [], [], 0
        for b, x in zip(keys, xs):
            p = oracle.ffor(x, b, base)
            chunks.append(p.view(np.uint8))
            offs.append(pos)
            pos += p.nbytes
        packed = np.concatenate(chunks + [np.zeros(256, np.uint8)])
        bw = np.array(keys, np.uint8)
        bases = np.full(len(keys), base, T)
        for order in (P.TRANSPOSED, P.ORIGINAL):
            if kind == "unpack":
                got = _np(P.unpack(_t(packed, cuda), _t(bw, cuda), _t(np.array(offs, np.uint64), cuda), order, width=w))
            else:
                got = _np(P.unffor(_t(packed, cuda), _t(bw, cuda), _t(bases, cuda), _t(np.array(offs, np.uint64), cuda),
                                   order))
            want = np.concatenate([oracle.untranspose_i(x) if order else x for x in xs])
            assert np.array_equal(got, want), (kind, order)
    assert P.device_status() == 0


@pytest.mark.parametrize("w", [8, 16, 32, 64])
@pytest.mark.parametrize("order", [0, 1])
def test_random_mixed_width_batches(cuda, w, order):
    from fastlanes_b200 import primitives as P

    rng = np.random.default_rng(100 + w)
    packed, offs, bw, base, vals = _batch(w, 700, rng)
    got = _np(P.unffor(_t(packed, cuda), _t(bw, cuda), _t(base, cuda), _t(offs, cuda), order))
    want = oracle.unffor_batch(packed, offs, bw, base, order == 1)
    assert np.array_equal(want.reshape(-1, 1024)[:, :8].shape, (700, 8))
    assert np.array_equal(got, want)
    if order == 0:
        assert np.array_equal(got, vals)
    assert P.device_status() == 0


@pytest.mark.parametrize("w", [16, 32, 64])
def test_unaligned_packed_words_take_the_warp_copy_path(cuda, w):
    from fastlanes_b200 import primitives as P

    rng = np.random.default_rng(7 + w)
    packed, offs, bw, base, vals = _batch(w, 150, rng)
    shifted = np.concatenate([np.zeros(4, np.uint8), packed])  # 4-byte aligned, not 16
    got = _np(P.unffor(_t(shifted, cuda), _t(bw, cuda), _t(base, cuda), _t(offs + np.uint64(4), cuda), 1))
    assert np.array_equal(got, oracle.unffor_batch(packed, offs, bw, base, True))
    assert P.device_status() == 0


@pytest.mark.parametrize("w", [8, 16, 32, 64])
def test_rsum_untranspose_transpose(cuda, w):
    from fastlanes_b200 import primitives as P

    T = TYPES[w]
    rng = np.random.default_rng(200 + w)
    n = 64
    d = rng.integers(0, np.iinfo(np.uint64).max, n * 1024, dtype=np.uint64, endpoint=True).astype(T)
    lb = rng.integers(0, np.iinfo(np.uint64).max, n * (1024 // w), dtype=np.uint64, endpoint=True).astype(T)
    want_t = np.concatenate([oracle.rsum(d[v * 1024:(v + 1) * 1024].copy(), lb[v * (1024 // w):(v + 1) * (1024 // w)].copy())
                             for v in range(n)])
    want_o = np.concatenate([oracle.untranspose_i(want_t[v * 1024:(v + 1) * 1024].copy()) for v in range(n)])
    assert np.array_equal(_np(P.rsum(_t(d, cuda), _t(lb, cuda), 0)), want_t)
    assert np.array_equal(_np(P.rsum(_t(d, cuda), _t(lb, cuda), 1)), want_o)
    assert np.array_equal(_np(P.untranspose_i(_t(want_t, cuda))), want_o)
    assert np.array_equal(_np(P.transpose_i(_t(want_o, cuda))), want_t)
    assert P.device_status() == 0


@pytest.mark.parametrize("w", [16, 32, 64])
@pytest.mark.parametrize("order", [0, 1])
def test_fused_delta_decode(cuda, w, order):
    from fastlanes_b200 import primitives as P

    T = TYPES[w]
    rng = np.random.default_rng(300 + w)
    packed, offs, bw, base, _ = _batch(w, 200, rng)
    lb = rng.integers(0, np.iinfo(np.uint64).max, 200 * (1024 // w), dtype=np.uint64, endpoint=True).astype(T)
    got = _np(P.unffor_rsum(_t(packed, cuda), _t(bw, cuda), _t(base, cuda), _t(lb, cuda), _t(offs, cuda), order))
    want = oracle.delta_batch(packed, offs, bw, base, lb, order == 1)
    assert np.array_equal(got, want)
    assert P.device_status() == 0


@pytest.mark.parametrize("w", [8, 16, 32, 64])
def test_gpu_encoders_match_oracle(cuda, w):
    from fastlanes_b200 import primitives as P

    T = TYPES[w]
    rng = np.random.default_rng(400 + w)
    n = 40
    _, _, bw, base, vals = _batch(w, n, rng)
    gp, goff = P.ffor(_t(vals, cuda), _t(bw, cuda), _t(base, cuda))
    gp, goff = _np(gp), _np(goff)
    for v in range(n):
        want = oracle.ffor(vals[v * 1024:(v + 1) * 1024], int(bw[v]), base[v]).view(np.uint8)
        assert np.array_equal(gp[int(goff[v]):int(goff[v]) + want.size], want), v
    if w >= 16:
        want_d = np.concatenate([oracle.unrsum(vals[v * 1024:(v + 1) * 1024].copy()) for v in range(n)])
        assert np.array_equal(_np(P.unrsum(_t(vals, cuda))), want_d)
        gbw, gbase = P.analyze(_t(vals, cuda))
        for v in range(n):
            b, bs = oracle.analyze(vals[v * 1024:(v + 1) * 1024].copy())
            assert int(_np(gbw)[v]) == b and _np(gbase)[v] == bs
    assert P.device_status() == 0


def test_bit_width_above_type_width_is_reported_not_decoded(cuda):
    from fastlanes_b200 import primitives as P

    rng = np.random.default_rng(5)
    packed, offs, bw, base, _ = _batch(32, 4, rng, bws=[3, 5, 7, 9])
    bw_bad = bw.copy()
    bw_bad[2] = 40
    P.unffor(_t(packed, cuda), _t(bw_bad, cuda), _t(base, cuda), _t(offs, cuda), 0)
    st = P.device_status()
    assert st & 2
    assert P.device_status() == 0


@pytest.mark.parametrize("keep_order", [False, True])
@pytest.mark.parametrize("order", [0, 1])
def test_plan_mixed_batch_shuffled_queue(cuda, keep_order, order):
    """One persistent launch over several columns of different widths with a shuffled work queue."""
    import torch

    from fastlanes_b200 import workloads as W

    rng = np.random.default_rng(900 + order + 2 * keep_order)
    cols, wants = [], []
    for w, n in ((32, 300), (64, 200), (16, 100), (8, 50)):
        packed, offs, bw, base, vals = _batch(w, n, rng)
        c = W.FforColumn(w, _t(packed, cuda), _t(offs, cuda), _t(bw, cuda), _t(base, cuda))
        cols.append(c)
        wants.append(oracle.unffor_batch(packed, offs, bw, base, order == 1))
    items = np.concatenate([(i << 24) | np.arange(c.n_vec, dtype=np.uint32) for i, c in enumerate(cols)])
    items = items[rng.permutation(items.size)].astype(np.uint32)
    queue = torch.from_numpy(items.view(np.int32)).to(cuda)
    outs = [torch.zeros(c.n_vec * 1024, dtype=W._DT[c.width], device=cuda) for c in cols]
    plan = W.Plan(cols, outs, order=order, queue=queue, keep_order=keep_order)
    plan.decode()
    torch.cuda.synchronize()
    for o, want in zip(outs, wants):
        assert np.array_equal(_np(o), want)
    plan.close()
    from fastlanes_b200 import primitives as P

    assert P.device_status() == 0


@pytest.mark.parametrize("w", [16, 32, 64])
def test_delta_with_misaligned_lane_bases(cuda, w):
    """Lane bases that do not start on a 16-byte boundary are copied by the warp, not by a TMA window."""
    import torch

    from fastlanes_b200 import primitives as P

    T = TYPES[w]
    rng = np.random.default_rng(600 + w)
    packed, offs, bw, base, _ = _batch(w, 60, rng)
    lb = rng.integers(0, np.iinfo(np.uint64).max, 60 * (1024 // w), dtype=np.uint64, endpoint=True).astype(T)
    raw = torch.zeros(lb.nbytes + 8, dtype=torch.uint8, device=cuda)
    raw[4:4 + lb.nbytes] = torch.from_numpy(lb.view(np.uint8)).to(cuda)
    lb_view = raw[4:4 + lb.nbytes]
    from fastlanes_b200._lib import lib

    out = torch.empty(60 * 1024, dtype=getattr(torch, f"uint{w}"), device=cuda)
    keep = [_t(packed, cuda), _t(bw, cuda), _t(base, cuda), _t(offs, cuda)]  # alive until the kernel has run
    rc = getattr(lib, f"fls_gpu_unffor_rsum_u{w}")(keep[0].data_ptr(), out.data_ptr(), keep[1].data_ptr(),
                                                   keep[2].data_ptr(), lb_view.data_ptr(), keep[3].data_ptr(), 60, 1,
                                                   torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    assert np.array_equal(_np(out), oracle.delta_batch(packed, offs, bw, base, lb, True))
    assert P.device_status() == 0
