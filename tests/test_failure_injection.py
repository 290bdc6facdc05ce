"""Failure detection without a GPU fault: a wait that runs out (a staging copy armed on its mbarrier but never
issued), and pages corrupted on the host whose indexes point outside their run values, dictionaries or bytes.
Each case must end with the matching device status bit, every read kept in bounds, the other vectors decoded,
and the context still usable for the next decode."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

TIMEOUT, BAD_INDEX = 1, 4


def _ffor_batch(n, bw_val, seed):
    rng = np.random.default_rng(seed)
    vals = rng.integers(0, 1 << bw_val, (n, 1024), dtype=np.uint64).astype(np.uint32)
    base = rng.integers(0, 1 << 20, n).astype(np.uint32)
    vals += base[:, None]
    packed = np.concatenate([oracle.ffor(v, bw_val, b).view(np.uint8) for v, b in zip(vals, base)])
    offs = np.arange(n, dtype=np.uint64) * (bw_val * 128)
    return vals, base, packed, offs


def test_stalled_copy_times_out_and_the_context_survives(cuda):
    import torch

    from fastlanes_b200 import primitives as P

    n, stall = 256, 37
    vals, base, packed, offs = _ffor_batch(n, 8, 5)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    pk = torch.zeros(packed.size + 256, dtype=torch.uint8, device=cuda)
    pk[: packed.size] = t(packed)
    bw = torch.full((n,), 8, dtype=torch.uint8, device=cuda)
    bs, off = t(base), t(offs)
    assert P.device_status() == 0
    out, rc = P.stalled_unffor(pk, bw, bs, off, stall, 256)
    assert rc == 0
    assert P.device_status() == TIMEOUT
    want = vals  # the packed arrays are transposed-order vectors: a transposed decode returns them as given
    got = out.cpu().numpy().reshape(n, 1024)
    # one vector per warp at this size: only the stalled vector is missing
    others = np.arange(n) != stall
    assert np.array_equal(got[others], want[others])
    assert not got[stall].any()
    # the context is usable: a plain decode of the same batch afterwards is complete and clean
    res = P.unffor(pk, bw, bs, off, P.TRANSPOSED)
    assert np.array_equal(res.cpu().numpy().reshape(n, 1024), want)
    assert P.device_status() == 0


def _page_on_device(page, cuda, shift=0):
    import torch

    from fastlanes_b200 import pages as PG

    sh = PG.placement(page) if shift is None else shift
    buf = torch.zeros(page.size + 64, dtype=torch.uint8, device=cuda)
    buf[sh:sh + page.size] = torch.from_numpy(np.ascontiguousarray(page)).to(cuda)
    return buf, buf.data_ptr() + sh


@pytest.mark.parametrize("key,buf_index,elem,value", [
    ("i64_7", 1, np.uint16, 0xFFFF),      # RLE UNCOMPRESSED: a run index past the vector's run values
    ("i64_16", 0, np.uint32, 0x00FFFFFF),  # DICT UNCOMPRESSED: a code past the dictionary
])
def test_corrupted_integer_index_is_reported_and_contained(cuda, col_golden, key, buf_index, elem, value):
    import torch

    from fastlanes_b200 import pages as PG
    from fastlanes_b200 import primitives as P
    from oracle import pages as OP

    page = col_golden[f"{key}_page"].copy()
    dic = col_golden[f"{key}_dict"]
    want = col_golden[f"{key}_input"].view(np.int64)
    pg = OP.parse_page(page)
    # one index of vector 1 (transposed position 5) set out of range
    pos = pg.off[buf_index] + pg.ep_of(1, buf_index) + 5 * np.dtype(elem).itemsize
    page[pos:pos + np.dtype(elem).itemsize] = np.frombuffer(np.array([value], elem).tobytes(), np.uint8)
    pb, pp = _page_on_device(page, cuda, None)
    db, dp = (_page_on_device(dic, cuda, 0) if dic.size else (None, None))
    out = torch.zeros(want.size, dtype=torch.int64, device=cuda)
    assert P.device_status() == 0
    PG.decode_pages([dict(d_page=pp, page_size=page.size, d_dict=dp, dict_size=dic.size, data_type=PG.INT64, order=1,
                          d_out=out.data_ptr())])
    assert P.device_status() == BAD_INDEX
    got = out.cpu().numpy()
    # the other vectors decode exactly; the corrupted position reads no memory and decodes as 0
    assert np.array_equal(got[:1024], want[:1024]) and np.array_equal(got[2048:], want[2048:])
    # where transposed position 5 lands in original order
    bad = int(np.nonzero(oracle.untranspose_i(np.arange(1024, dtype=np.uint32)) == 5)[0][0])
    assert got[1024 + bad] == 0
    ok = np.ones(1024, bool)
    ok[bad] = False
    assert np.array_equal(got[1024:2048][ok], want[1024:2048][ok])


@pytest.mark.parametrize("eid,buf_index,value", [
    (2, 0, 0x00FFFFFF),   # string DICT UNCOMPRESSED: a code past the dictionary
    (13, 1, 0x0FFFFFFF),  # FSST: a row end past the vector's compressed bytes
])
def test_corrupted_string_index_is_reported_and_contained(cuda, col_golden, eid, buf_index, value):
    import torch

    from fastlanes_b200 import primitives as P
    from fastlanes_b200.strings import StringPlan
    from oracle import pages as OP

    page = col_golden[f"str_{eid}_page"].copy()
    dic = col_golden[f"str_{eid}_dict"]
    pg = OP.parse_page(page)
    pos = pg.off[buf_index] + pg.ep_of(1, buf_index) + 4 * 9
    page[pos:pos + 4] = np.frombuffer(np.array([value], np.uint32).tobytes(), np.uint8)
    pb, pp = _page_on_device(page, cuda, 0)
    db, dp = _page_on_device(dic, cuda, 0)
    assert P.device_status() == 0
    plan = StringPlan(pp, page.size, dp, dic.size)
    n = plan.measure()
    offs = torch.zeros(plan.n_rows + 1, dtype=torch.int32, device=cuda)
    data = torch.zeros(n + 64, dtype=torch.uint8, device=cuda)
    plan.decode_into(offs, data)
    plan.close()
    assert P.device_status() & BAD_INDEX
    o = offs.cpu().numpy().astype(np.int64)
    assert (np.diff(o) >= 0).all() and o[-1] == n  # offsets stay a valid, bounded Arrow layout
