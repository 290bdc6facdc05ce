"""Predicate pushdown on the GPU (filter plans): bitmaps of `column OP constant` evaluated on compressed
reference pages and on our own pages of every integer width, equal to the oracle's restatement of the
reference's predicate primitives (src/primitive/predicate/equal.cpp) on the decoded values; selections
(index lists) and their intersection as the reference's SelectionDS and and_selection_ds_func."""
import numpy as np
import pytest

from oracle import oracle
from oracle import predicate as PR

pytestmark = pytest.mark.gpu

KEYS = [f"i64_{e}" for e in (0, 1, 6, 7, 11, 16, 17, 22, 27)] + [f"i64patch_{e}" for e in (2, 3, 4, 5, 12, 13, 14, 15)] \
    + [f"i64rec_{e}" for e in (8, 9, 16, 17, 22, 27)] + [f"i64dpatch_{e}" for e in (18, 20, 21, 23, 26)]


def _dev_bytes(a, dev, shift=0):
    import torch

    buf = torch.zeros(a.size + 64, dtype=torch.uint8, device=dev)
    buf[shift:shift + a.size] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return buf, buf.data_ptr() + shift


def _in_order(values, order):
    if order == 1:
        return values
    w = values.dtype.itemsize * 8
    u = values.view({64: np.uint64, 32: np.uint32, 16: np.uint16}[w])
    return np.concatenate([oracle.transpose_i(u[v * 1024:(v + 1) * 1024].copy())
                           for v in range(u.size // 1024)]).view(values.dtype)


def _filter(cols, op, value):
    """cols: (page column dict without d_out, n_vec); returns the bitmaps (n_vec, 16) of every column."""
    import torch

    from fastlanes_b200 import pages

    outs = [torch.full((n * 16,), 0x5A5A5A5A5A5A5A5A, dtype=torch.int64, device="cuda") for _, n in cols]
    plan = pages.FilterPlan([dict(c, d_out=o.data_ptr()) for (c, _), o in zip(cols, outs)], op, value)
    plan.decode()
    torch.cuda.synchronize()
    plan.close()
    return [o.cpu().numpy().view(np.uint64).reshape(-1, 16) for o in outs]


@pytest.mark.parametrize("key", KEYS)
def test_filter_reference_pages(cuda, col_golden, key):
    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    if f"{key}_page" not in col_golden.files:
        pytest.skip(f"no fixture {key}")
    page = col_golden[f"{key}_page"]
    dic = col_golden[f"{key}_dict"] if f"{key}_dict" in col_golden.files else np.zeros(0, np.uint8)
    want = np.ascontiguousarray(col_golden[f"{key}_input"]).view(np.int64)
    pbuf, pptr = _dev_bytes(page, cuda, 3)
    col = dict(d_page=pptr, page_size=page.size, data_type=pages.INT64)
    if dic.size:
        dbuf, dptr = _dev_bytes(dic, cuda, 1)
        col.update(d_dict=dptr, dict_size=dic.size)
    n_vec = want.size // 1024
    for order in (1, 0):
        vals = _in_order(want, order)
        for value in (int(want[11]), int(want.min()) - 1, int(want.max()), int(np.median(want))):
            for op in range(6):
                (got,) = _filter([(dict(col, order=order), n_vec)], op, value)
                assert np.array_equal(got, PR.bitmaps(vals, op, value)), (key, order, op, value)
    assert P.device_status() == 0


def _column(rng, kind, dtype, n_vec):
    info = np.iinfo(dtype)
    n = n_vec * 1024
    if kind == "ffor":
        lo = int(info.min) // 4 if info.min < 0 else 1000
        x = (lo + rng.integers(0, 3000, n)).astype(dtype)
        expr = 1
    elif kind == "rle":
        runs = rng.geometric(1 / 8, n)
        x = np.repeat(rng.integers(0, 200, runs.size), runs)[:n].astype(dtype)
        if info.min < 0:
            x = (x.astype(np.int64) - 100).astype(dtype)
        expr = 6
    else:
        x = (np.cumsum(rng.integers(0, 9, n)) + (int(info.min) // 2 if info.min < 0 else 0)).astype(dtype)
        expr = 11
    return x, expr


def test_filter_plan_of_mixed_columns(cuda):
    """One filter plan over FFOR / RLE / DELTA columns of u32, i32, u64 and i64 (our encoder), original and
    transposed order in the same launch; constants drawn from each column."""
    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    rng = np.random.default_rng(5)
    specs = [("ffor", "UINT32"), ("rle", "INT32"), ("delta", "UINT64"), ("ffor", "INT64"), ("rle", "UINT32"),
             ("delta", "INT32"), ("ffor", "INT32"), ("rle", "INT64")]
    keep, cols, vals = [], [], []
    for i, (kind, dt) in enumerate(specs):
        code = getattr(pages, dt)
        x, expr = _column(rng, kind, pages.DTYPE_OF[code], 3 + i)
        page, _ = pages.encode_from_memory(x, code, expr)
        pb, pp = _dev_bytes(page, cuda, i % 7)
        keep.append(pb)
        order = i % 2
        cols.append((dict(d_page=pp, page_size=page.size, data_type=code, order=order), x.size // 1024))
        vals.append(_in_order(x, order))
    for op in range(6):
        for pick in (0, 1):
            # the same constant for every column (as one predicate): a value of column `pick`
            value = int(vals[pick][100])
            got = _filter(cols, op, value)
            for g, v in zip(got, vals):
                assert np.array_equal(g, PR.bitmaps(v, op, value)), (op, value)
    assert P.device_status() == 0


def test_selections_and_their_intersection(cuda, col_golden):
    """Bitmaps -> index lists (SelectionDS::idx_arr / n_selected_values), bitmap AND / OR / ANDNOT, and the
    intersection of index lists, against the oracle (and_selection_ds_func restated)."""
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    page = col_golden["i64_1_page"]
    want = np.ascontiguousarray(col_golden["i64_1_input"]).view(np.int64)
    n_vec = want.size // 1024
    pbuf, pptr = _dev_bytes(page, cuda)
    col = (dict(d_page=pptr, page_size=page.size, data_type=pages.INT64, order=1), n_vec)
    lo, hi = np.percentile(want, [30, 70]).astype(np.int64)
    (b_gt,) = _filter([col], PR.GT, int(lo))
    (b_lt,) = _filter([col], PR.LT, int(hi))
    d_gt, d_lt = torch.from_numpy(b_gt.view(np.int64).ravel()).cuda(), torch.from_numpy(b_lt.view(np.int64).ravel()).cuda()
    idx = [torch.full((n_vec * 1024,), 0x7777, dtype=torch.int16, device=cuda) for _ in range(3)]
    cnt = [torch.zeros(n_vec, dtype=torch.int16, device=cuda) for _ in range(3)]
    pages.bitmap_to_selection(d_gt.data_ptr(), n_vec, idx[0].data_ptr(), cnt[0].data_ptr())
    pages.bitmap_to_selection(d_lt.data_ptr(), n_vec, idx[1].data_ptr(), cnt[1].data_ptr())
    pages.selection_and(idx[0].data_ptr(), cnt[0].data_ptr(), idx[1].data_ptr(), cnt[1].data_ptr(),
                        idx[2].data_ptr(), cnt[2].data_ptr(), n_vec)
    both = torch.empty_like(d_gt)
    pages.bitmap_combine(d_gt.data_ptr(), d_lt.data_ptr(), both.data_ptr(), n_vec, pages.BITMAP_AND)
    torch.cuda.synchronize()
    I = [i.cpu().numpy().view(np.uint16).reshape(n_vec, 1024) for i in idx]
    C = [c.cpu().numpy().view(np.uint16) for c in cnt]
    for v in range(n_vec):
        s_gt, n_gt = PR.selection(b_gt[v])
        s_lt, n_lt = PR.selection(b_lt[v])
        assert C[0][v] == n_gt and np.array_equal(I[0][v, :n_gt], s_gt)
        assert C[1][v] == n_lt and np.array_equal(I[1][v, :n_lt], s_lt)
        s_and = PR.selection_and(s_gt, n_gt, s_lt, n_lt)
        assert C[2][v] == s_and.size and np.array_equal(I[2][v, :s_and.size], s_and)
    assert np.array_equal(both.cpu().numpy().view(np.uint64).reshape(n_vec, 16), b_gt & b_lt)
    for op, f in ((pages.BITMAP_OR, np.bitwise_or), (pages.BITMAP_ANDNOT, lambda a, b: a & ~b)):
        pages.bitmap_combine(d_gt.data_ptr(), d_lt.data_ptr(), both.data_ptr(), n_vec, op)
        assert np.array_equal(both.cpu().numpy().view(np.uint64).reshape(n_vec, 16), f(b_gt, b_lt))
    assert P.device_status() == 0


def test_filter_plan_refuses_bad_requests(cuda, col_golden):
    import torch

    from fastlanes_b200 import _lib, pages

    page = col_golden["i64_1_page"]
    pbuf, pptr = _dev_bytes(page, cuda)
    out = torch.zeros(4096, dtype=torch.int64, device=cuda)
    col = dict(d_page=pptr, page_size=page.size, data_type=pages.INT64, order=1, d_out=out.data_ptr())
    with pytest.raises(_lib.FlsError):
        pages.FilterPlan([col], 6, 0)  # no such operator
    with pytest.raises(_lib.FlsError):
        pages.FilterPlan([dict(col, data_type=1)], PR.EQ, 0)  # DOUBLE
