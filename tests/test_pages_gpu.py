"""GPU decode of reference pages (bytes written by the reference's own encoder) and the fastlanes.h C API."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

INT_IDS = [0, 1, 6, 7, 11, 16, 17, 22]


def _dev_bytes(a, dev, shift=0):
    import torch

    buf = torch.zeros(a.size + 64, dtype=torch.uint8, device=dev)
    buf[shift:shift + a.size] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return buf, buf.data_ptr() + shift


@pytest.mark.parametrize("eid", INT_IDS)
@pytest.mark.parametrize("shift", [0, 1, 4, 8])
def test_reference_int64_pages(cuda, col_golden, eid, shift):
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    page = col_golden[f"i64_{eid}_page"]
    dic = col_golden[f"i64_{eid}_dict"]
    want = col_golden[f"i64_{eid}_input"]
    pbuf, pptr = _dev_bytes(page, cuda, shift)
    dbuf, dptr = _dev_bytes(dic, cuda, (shift * 3) % 8) if dic.size else (None, None)
    for order in (1, 0):
        out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
        pages.decode_pages([dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size,
                                 data_type=pages.INT64, order=order, d_out=out.data_ptr())])
        got = out.cpu().numpy()
        if order == 1:
            assert np.array_equal(got, want), (eid, shift)
        else:
            tw = np.concatenate([oracle.transpose_i(want[v * 1024:(v + 1) * 1024].view(np.uint64).copy())
                                 for v in range(want.size // 1024)]).view(np.int64)
            assert np.array_equal(got, tw), (eid, shift)
    assert P.device_status() == 0


def test_several_pages_one_launch(cuda, col_golden):
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    keep, cols, wants, outs = [], [], [], []
    for eid in INT_IDS:
        page, dic, want = col_golden[f"i64_{eid}_page"], col_golden[f"i64_{eid}_dict"], col_golden[f"i64_{eid}_input"]
        pbuf, pptr = _dev_bytes(page, cuda, eid % 5)
        dbuf, dptr = _dev_bytes(dic, cuda) if dic.size else (None, None)
        out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
        keep += [pbuf, dbuf]
        outs.append(out)
        wants.append(want)
        cols.append(dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size, data_type=pages.INT64,
                         order=1, d_out=out.data_ptr()))
    pages.decode_pages(cols)
    for o, w in zip(outs, wants):
        assert np.array_equal(o.cpu().numpy(), w)
    assert P.device_status() == 0


@pytest.mark.parametrize("eid", [0, 1, 11])
def test_c_api_encode_matches_reference_bytes_and_decodes(cuda, col_golden, eid):
    """encode_from_memory of the reference's INT64 input reproduces the reference's page byte for byte;
    decode_to_memory returns the input."""
    from fastlanes_b200 import pages

    want = col_golden[f"i64_{eid}_input"]
    page, mtd = pages.encode_from_memory(want, pages.INT64, eid)
    assert np.array_equal(page, col_golden[f"i64_{eid}_page"])
    info = pages.page_info(page)
    assert mtd == info["meta_size"]
    assert np.array_equal(pages.decode_to_memory(page, pages.INT64), want)
    assert np.array_equal(pages.decode_to_memory(col_golden[f"i64_{eid}_page"], pages.INT64), want)


@pytest.mark.parametrize("dt", ["UINT32", "INT32", "UINT64"])
@pytest.mark.parametrize("eid", [0, 1, 11])
def test_c_api_round_trip_other_widths(cuda, dt, eid):
    from fastlanes_b200 import pages

    code = getattr(pages, dt)
    T = pages.DTYPE_OF[code]
    rng = np.random.default_rng(eid + 7 * code)
    n = 5 * 1024 + 77  # the tail of n % 1024 values is dropped, as in the reference encoder
    info = np.iinfo(T)
    if eid == 11:
        x = (np.cumsum(rng.integers(0, 50, n)) + int(info.min) // 2).astype(T)
    else:
        x = rng.integers(int(info.min), int(info.max), n, dtype=np.int64 if T != np.uint64 else np.uint64).astype(T)
    page, _ = pages.encode_from_memory(x, code, eid)
    got = pages.decode_to_memory(page, code)
    assert np.array_equal(got, x[:5 * 1024])


def test_c_api_rejects_unknown_expression(cuda):
    from fastlanes_b200 import _lib, pages

    with pytest.raises(_lib.FlsError):
        pages.encode_from_memory(np.arange(2048, dtype=np.int64), pages.INT64, 2)


def test_c_api_rle_matches_reference_bytes(cuda, col_golden):
    from fastlanes_b200 import pages

    want = col_golden["i64_6_input"]
    page, _ = pages.encode_from_memory(want, pages.INT64, 6)
    assert np.array_equal(page, col_golden["i64_6_page"])


@pytest.mark.parametrize("dt", ["UINT32", "INT32", "INT64"])
def test_rle_round_trip_through_the_page_decoder(cuda, dt):
    import torch

    from fastlanes_b200 import pages

    code = getattr(pages, dt)
    T = pages.DTYPE_OF[code]
    rng = np.random.default_rng(code)
    runs = rng.geometric(1 / 8, 20000)
    x = np.repeat(rng.integers(0, 10**6, runs.size), runs)[: 7 * 1024].astype(T)
    page, _ = pages.encode_from_memory(x, code, 6)
    pb, pp = _dev_bytes(page, cuda, 2)
    out = torch.zeros(x.size, dtype=torch.from_numpy(np.zeros(1, T)).dtype, device=cuda)
    pages.decode_pages([dict(d_page=pp, page_size=page.size, data_type=code, order=1, d_out=out.data_ptr())])
    assert np.array_equal(out.cpu().numpy(), x)


def test_page_plan_equals_direct_decode(cuda, col_golden):
    import torch

    from fastlanes_b200 import pages

    keep, cols, wants, outs = [], [], [], []
    for eid in INT_IDS:
        page, dic, want = col_golden[f"i64_{eid}_page"], col_golden[f"i64_{eid}_dict"], col_golden[f"i64_{eid}_input"]
        pbuf, pptr = _dev_bytes(page, cuda, (eid * 7) % 16)
        dbuf, dptr = _dev_bytes(dic, cuda) if dic.size else (None, None)
        out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
        keep += [pbuf, dbuf]
        outs.append(out)
        wants.append(want)
        cols.append(dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size, data_type=pages.INT64,
                         order=1, d_out=out.data_ptr()))
    plan = pages.PagePlan(cols)
    for _ in range(2):
        for o in outs:
            o.zero_()
        plan.decode()
        for o, w in zip(outs, wants):
            assert np.array_equal(o.cpu().numpy(), w)
    plan.close()


@pytest.mark.parametrize("expr", [1, 11, 6])
def test_c_api_decode_pipelines_large_pages(cuda, expr):
    """decode_to_memory of a page spanning several pipeline chunks (u64: chunks of 128, 256, 512, 1024 and then
    2048 vectors, so 3000 vectors make five chunks, the last partial, and from the third on each chunk's copy in
    waits for the copy out of the chunk two places before it), from pinned and from pageable host memory."""
    import torch

    from fastlanes_b200 import pages

    rng = np.random.default_rng(expr)
    if expr == 6:
        runs = rng.geometric(1 / 24, 200000)
        x = np.repeat(rng.integers(-10**12, 10**12, runs.size), runs)[: 3000 * 1024].astype(np.int64)
    elif expr == 11:
        x = (1_600_000_000_000_000_000 + np.cumsum(rng.geometric(0.1, 3000 * 1024))).astype(np.int64)
    else:
        x = rng.integers(-2**40, 2**40, 3000 * 1024).astype(np.int64)
    page, _ = pages.encode_from_memory(x, pages.INT64, expr)
    assert np.array_equal(pages.decode_to_memory(page, pages.INT64), x)
    hp = torch.from_numpy(page).pin_memory()
    ho = torch.zeros(x.size, dtype=torch.int64).pin_memory()
    from fastlanes_b200 import _lib

    _lib.lib.decode_to_memory(hp.data_ptr(), ho.data_ptr(), pages.INT64)
    assert np.array_equal(ho.numpy(), x)


def test_plan_autotune_and_graph_replay(cuda):
    """The autotuner picks a variant per launch segment without changing results; graph replays of a plan with
    a plain and a gather segment equal direct launches."""
    import torch

    from fastlanes_b200 import rowgroups as RG
    from fastlanes_b200 import select as S
    from fastlanes_b200 import workloads as W

    rng = np.random.default_rng(3)
    cols = [W.selection_column(rng, 6, "cuda", f) for f in ("for_i64", "rle", "dict_i32", "delta_i64", "for_u32")]
    plan = S.SelectionPlan(cols, 3)
    _, best, _ = plan.wizard()
    choice = best.cpu().numpy()
    choice[0], choice[2] = 1, 2  # make sure both kernel families are present
    rg = RG.RowGroupSet(cols, plan.chunks(), choice)
    names = rg.autotune(2)
    assert len(names) == 2 and all(names)
    for graph in (False, True, True):
        for o in rg.outputs:
            o.zero_()
        rg.decode(graph=graph)
        torch.cuda.synchronize()
        for o, (t, _) in zip(rg.outputs, cols):
            assert torch.equal(o, t)
    rg.close()
    plan.close()


@pytest.mark.parametrize("eid", [8, 9, 10, 16, 17, 22, 27])
@pytest.mark.parametrize("shift", [0, 3, 8])
def test_reference_rec_pages(cuda, col_golden, eid, shift):
    """Reference pages whose rec buffers (dictionary entries, run values, run codes) hold FFOR blocks with
    exceptions: decoded on the GPU one-shot and through a page plan, equal to the reference's input."""
    import torch

    from fastlanes_b200 import pages

    page, dic, want = (col_golden[f"i64rec_{eid}_{k}"] for k in ("page", "dict", "input"))
    pbuf, pptr = _dev_bytes(page, cuda, shift)
    col = dict(d_page=pptr, page_size=page.size, data_type=pages.INT64, order=1)
    if dic.size:
        dbuf, dptr = _dev_bytes(dic, cuda, 5)
        col.update(d_dict=dptr, dict_size=dic.size)
    out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
    pages.decode_pages([dict(col, d_out=out.data_ptr())])
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    out.zero_()
    plan = pages.PagePlan([dict(col, d_out=out.data_ptr())])
    plan.decode()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    plan.close()
    if not dic.size:
        assert np.array_equal(pages.decode_to_memory(page, pages.INT64), want)


@pytest.mark.parametrize("eid", [2, 3, 4, 5, 12, 13, 14, 15])
@pytest.mark.parametrize("shift", [0, 5])
def test_reference_patched_pages(cuda, col_golden, eid, shift):
    """Patched FFOR / DELTA pages of the reference (S / B / LL patches, rec-compressed exceptions) decode
    bit-exactly one-shot, through a page plan (both orders) and through decode_to_memory."""
    import torch

    from fastlanes_b200 import pages

    page, want = col_golden[f"i64patch_{eid}_page"], col_golden[f"i64patch_{eid}_input"]
    pbuf, pptr = _dev_bytes(page, cuda, shift)
    out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
    pages.decode_pages([dict(d_page=pptr, page_size=page.size, data_type=pages.INT64, order=1, d_out=out.data_ptr())])
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    for order in (0, 1):
        out.zero_()
        plan = pages.PagePlan([dict(d_page=pptr, page_size=page.size, data_type=pages.INT64, order=order,
                                    d_out=out.data_ptr())])
        plan.decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        if order == 0:
            got = np.concatenate([oracle.untranspose_i(got[v * 1024:(v + 1) * 1024].view(np.uint64).copy())
                                  for v in range(want.size // 1024)]).view(np.int64)
        assert np.array_equal(got, want), order
        plan.close()
    assert np.array_equal(pages.decode_to_memory(page, pages.INT64), want)


@pytest.mark.parametrize("eid", [18, 19, 20, 21, 23, 24, 25, 26, "frq_28", "frq_29", "frq_30", "frq_31", "frq_32",
                                 "frq_33", "frq_34", "frq_35", "frq_36", "frq_37", "frq_38"])
@pytest.mark.parametrize("shift", [0, 7])
def test_reference_patched_dict_pages(cuda, col_golden, eid, shift):
    """DICT pages of the reference whose u32 codes are patched FFOR / DELTA streams (pool ids 18-26): the
    patched codes decode into a plan-owned buffer, then a gather launch reads the dictionary; one-shot, through
    a page plan in both orders, and next to other pages in one plan."""
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    key = f"i64{eid}" if isinstance(eid, str) else f"i64dpatch_{eid}"  # DICT_FRQ (ids 28-38): DICT pages
    page, dic, want = (col_golden[f"{key}_{k}"] for k in ("page", "dict", "input"))
    pbuf, pptr = _dev_bytes(page, cuda, shift)
    dbuf, dptr = _dev_bytes(dic, cuda, 3)
    col = dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size, data_type=pages.INT64)
    out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
    pages.decode_pages([dict(col, order=1, d_out=out.data_ptr())])
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    for order in (0, 1):
        out.zero_()
        plan = pages.PagePlan([dict(col, order=order, d_out=out.data_ptr())])
        plan.decode()
        plan.decode()  # replays reuse the plan's code buffer
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        if order == 0:
            got = np.concatenate([oracle.untranspose_i(got[v * 1024:(v + 1) * 1024].view(np.uint64).copy())
                                  for v in range(want.size // 1024)]).view(np.int64)
        assert np.array_equal(got, want), order
        plan.close()
    # with a plain and an RLE page in the same plan
    other = [col_golden["i64_1_page"], col_golden["i64_6_page"]]
    keep, cols, outs = [], [dict(col, order=1, d_out=out.data_ptr())], [out]
    for pg in other:
        b, p = _dev_bytes(pg, cuda, 5)
        o = torch.zeros(3 * 1024, dtype=torch.int64, device=cuda)
        keep.append(b)
        outs.append(o)
        cols.append(dict(d_page=p, page_size=pg.size, data_type=pages.INT64, order=1, d_out=o.data_ptr()))
    out.zero_()
    plan = pages.PagePlan(cols)
    plan.decode_graph()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    assert np.array_equal(outs[1].cpu().numpy(), col_golden["i64_1_input"])
    assert np.array_equal(outs[2].cpu().numpy(), col_golden["i64_6_input"])
    plan.close()
    assert P.device_status() == 0


F64_IDS = [0, 6, 7] + list(range(16, 39))


@pytest.mark.parametrize("eid", F64_IDS)
@pytest.mark.parametrize("shift", [0, 3])
def test_reference_double_pages(cuda, col_golden, eid, shift):
    """Double columns written by the reference (double pool: UNCOMPRESSED, RLE, DICT with every code variant over
    a raw double dictionary, DICT_RLE, DICT_FRQ) decode to the input's exact bit patterns, through the page
    decoder and through a plan."""
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P

    page, dic = col_golden[f"f64_{eid}_page"], col_golden[f"f64_{eid}_dict"]
    want = col_golden[f"f64_{eid}_input"].view(np.uint64)
    pbuf, pptr = _dev_bytes(page, cuda, shift)
    dbuf, dptr = _dev_bytes(dic, cuda, (shift * 5) % 8) if dic.size else (None, 0)
    col = dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size, data_type=pages.DOUBLE, order=1)
    out = torch.zeros(want.size, dtype=torch.float64, device=cuda)
    pages.decode_pages([dict(col, d_out=out.data_ptr())])
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want), (eid, shift)
    out2 = torch.zeros_like(out)
    plan = pages.PagePlan([dict(col, d_out=out2.data_ptr())])
    plan.decode()
    torch.cuda.synchronize()
    plan.close()
    assert np.array_equal(out2.cpu().numpy().view(np.uint64), want), (eid, shift)
    assert P.device_status() == 0


def test_c_api_doubles(cuda, col_golden):
    """decode_to_memory reads the reference's double UNCOMPRESSED and RLE pages; encode_from_memory writes the
    UNCOMPRESSED one byte for byte; ALP (expression 1) is refused: the ALP library is not part of the reference."""
    from fastlanes_b200 import pages

    for eid in (0, 6, 7):
        want = col_golden[f"f64_{eid}_input"]
        got = pages.decode_to_memory(col_golden[f"f64_{eid}_page"], pages.DOUBLE)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), eid
    page, _ = pages.encode_from_memory(col_golden["f64_0_input"], pages.DOUBLE, 0)
    assert np.array_equal(page, col_golden["f64_0_page"])
    # RLE of doubles runs on bit patterns (the fixture has no NaN or signed zero, where the reference's ==
    # would merge or split runs differently): the reference's bytes, and a bit-exact round trip
    page, _ = pages.encode_from_memory(col_golden["f64_6_input"], pages.DOUBLE, 6)
    assert np.array_equal(page, col_golden["f64_6_page"])
    assert np.array_equal(pages.decode_to_memory(page, pages.DOUBLE).view(np.uint64),
                          col_golden["f64_6_input"].view(np.uint64))
    with pytest.raises(Exception):
        pages.encode_from_memory(col_golden["f64_0_input"], pages.DOUBLE, 1)


def test_double_dictionary_too_short_is_refused(cuda, col_golden):
    """A double DICT page whose dictionary holds fewer bytes than entry_c values is a format error."""
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200._lib import FlsError

    page, dic = col_golden["f64_17_page"], col_golden["f64_17_dict"]
    pbuf, pptr = _dev_bytes(page, cuda)
    short = dic[:-8].copy()
    dbuf, dptr = _dev_bytes(short, cuda)
    out = torch.zeros(col_golden["f64_17_input"].size, dtype=torch.float64, device=cuda)
    with pytest.raises(FlsError):
        pages.decode_pages([dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=short.size,
                                 data_type=pages.DOUBLE, order=1, d_out=out.data_ptr())])


@pytest.mark.parametrize("key", ["i64_11", "i64_6", "i64_17", "i64_27", "i64rec_9", "i64rec_16", "i64patch_13",
                                 "i64dpatch_25", "i64frq_33", "f64_22"])
def test_page_vector_ranges(cuda, col_golden, key):
    """Random access by vector: every range decodes to the same values as the whole page, for plain, DELTA,
    RLE, DICT, DICT_RLE, rec-compressed, patched and two-step (patched DICT codes) pages."""
    import torch

    from fastlanes_b200 import pages
    from fastlanes_b200 import primitives as P
    from fastlanes_b200._lib import FlsError

    page = col_golden[f"{key}_page"]
    dic = col_golden[f"{key}_dict"] if f"{key}_dict" in col_golden.files else np.zeros(0, np.uint8)
    want = col_golden[f"{key}_input"].view(np.uint64)
    dt = pages.DOUBLE if key.startswith("f64") else pages.INT64
    pbuf, pptr = _dev_bytes(page, cuda, 3)
    dbuf, dptr = _dev_bytes(dic, cuda, 1) if dic.size else (None, 0)
    n_vec = want.size // 1024
    for first, n in [(0, n_vec), (n_vec - 1, 1), (1, n_vec - 2), (n_vec // 2, 1), (0, 0)]:
        out = torch.full((max(n, 1) * 1024 + 1024,), 7, dtype=torch.int64, device=cuda)
        pages.decode_page_vectors(dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size,
                                       data_type=dt, order=1, d_out=out.data_ptr()), first, n)
        got = out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got[:n * 1024], want[first * 1024:(first + n) * 1024]), (key, first, n)
        assert np.all(got[n * 1024:] == 7)  # nothing written past the range
    with pytest.raises(FlsError):
        pages.decode_page_vectors(dict(d_page=pptr, page_size=page.size, d_dict=dptr, dict_size=dic.size,
                                       data_type=dt, order=1, d_out=out.data_ptr()), n_vec - 1, 2)
    assert P.device_status() == 0
