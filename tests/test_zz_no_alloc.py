"""The allocation-free FSST / BYTE_ARR page decode (fls_gpu_decode_fsst_page_noalloc, through the C ABI).

Callers that cannot allocate device memory (an engine whose buffer manager owns all of HBM, or a path where
cudaMalloc is not allowed) decode with scratch compiled into the library.  Its output must equal the
allocating string plan's, bit for bit, call after call.  This file is collected last on purpose."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, dev, shift=0):
    import torch

    buf = torch.zeros(a.size + 64, dtype=torch.uint8, device=dev)
    if a.size:
        buf[shift:shift + a.size] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return buf, buf.data_ptr() + shift


@pytest.mark.parametrize("eid", [13, 14, 0])
def test_noalloc_decode_equals_plan_decode_two_calls_in_a_row(cuda, col_golden, eid):
    import torch

    from fastlanes_b200 import strings

    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    pb, pp = _dev(page, cuda, 1)
    db, dp = _dev(dic, cuda) if dic.size else (None, None)
    plan = strings.StringPlan(pp, page.size, dp, dic.size)
    want_off, want_data = plan.decode(cuda)
    plan.close()
    want_off, want_data = want_off.cpu().numpy(), want_data.cpu().numpy()
    assert np.array_equal(want_off.astype(np.uint64), col_golden[f"str_{eid}_input_offsets"])

    n_rows = want_off.size - 1
    offsets = torch.zeros(n_rows + 1, dtype=torch.int32, device=cuda)
    data = torch.zeros(want_data.size + 64, dtype=torch.uint8, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    for _ in range(2):
        offsets.fill_(-1)
        data.fill_(0xEE)
        rc = strings.decode_fsst_page_noalloc(pp, page.size, dp, dic.size, offsets, data, status)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        assert np.array_equal(offsets.cpu().numpy(), want_off)
        assert np.array_equal(data[: want_data.size].cpu().numpy(), want_data)


def test_noalloc_rejects_pages_beyond_its_scratch(cuda):
    import torch

    from fastlanes_b200 import strings

    hdr = np.zeros(64, np.uint8)
    hdr[0], hdr[1] = 7, 1  # FSST page header
    hdr[4:6] = np.frombuffer(np.uint16(8193).tobytes(), np.uint8)  # one vector more than the scratch holds
    pb, pp = _dev(hdr, cuda)
    offsets = torch.zeros(16, dtype=torch.int32, device=cuda)
    data = torch.zeros(16, dtype=torch.uint8, device=cuda)
    rc = strings.decode_fsst_page_noalloc(pp, hdr.size, None, 0, offsets, data)
    assert rc == -6  # FLS_ERR_TOO_LARGE
