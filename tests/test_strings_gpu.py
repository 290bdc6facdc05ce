"""String pages written by the reference's encoder, decoded on the GPU, against the reference decoder's output
(golden fixtures: tests/golden/columns.npz)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STR_IDS = [0, 2, 3, 8, 13, 14, 15, 16]


def _dev(a, dev, shift=0):
    import torch

    buf = torch.zeros(a.size + 64, dtype=torch.uint8, device=dev)
    if a.size:
        buf[shift:shift + a.size] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return buf, buf.data_ptr() + shift


def _expected(g, eid):
    if f"str_{eid}_decoded_bytes" in g.files:
        return g[f"str_{eid}_decoded_offsets"], g[f"str_{eid}_decoded_bytes"]
    return g[f"str_{eid}_input_offsets"], g[f"str_{eid}_input_bytes"]


@pytest.mark.parametrize("eid", STR_IDS)
@pytest.mark.parametrize("shift", [0, 3])
def test_reference_string_pages(cuda, col_golden, eid, shift):
    from fastlanes_b200 import primitives as P
    from fastlanes_b200.strings import StringPlan

    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    pb, pp = _dev(page, cuda, shift)
    db, dp = _dev(dic, cuda, (shift + 1) % 4) if dic.size else (None, None)
    plan = StringPlan(pp, page.size, dp, dic.size)
    offs, data = plan.decode(cuda)
    want_o, want_b = _expected(col_golden, eid)
    assert plan.n_rows == want_o.size - 1
    assert np.array_equal(offs.cpu().numpy().astype(np.uint64), want_o)
    assert np.array_equal(data.cpu().numpy(), want_b)
    # the plan can decode again (graph-style replay) with the same result
    offs2, data2 = plan.decode(cuda)
    assert np.array_equal(offs2.cpu().numpy(), offs.cpu().numpy()) and np.array_equal(data2.cpu().numpy(), want_b)
    plan.close()
    assert P.device_status() == 0


def test_string_dict_encoder_round_trip(cuda):
    """Our DICT + FSST encoder (true entry lengths) decodes back to dict[codes] on the GPU."""
    from fastlanes_b200 import strings
    from tests.test_encoders import _strings

    rng = np.random.default_rng(4)
    dbytes, doffs = _strings(rng, 700)
    n_dict = doffs.size - 1
    codes = (rng.zipf(1.1, 9 * 1024) % n_dict).astype(np.uint32)
    page, dic = strings.encode_string_dict(dbytes, doffs, codes)
    pb, pp = _dev(page, cuda, 5)
    db, dp = _dev(dic, cuda, 2)
    plan = strings.StringPlan(pp, page.size, dp, dic.size)
    offs, data = plan.decode(cuda)
    plan.close()
    want = [dbytes[int(doffs[c]):int(doffs[c + 1])] for c in codes]
    want_off = np.zeros(codes.size + 1, np.uint64)
    want_off[1:] = np.cumsum([w.size for w in want])
    assert np.array_equal(offs.cpu().numpy().astype(np.uint64), want_off)
    assert np.array_equal(data.cpu().numpy(), np.concatenate(want))
