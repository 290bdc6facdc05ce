"""The allocation-free FSST / BYTE_ARR page decode (fls_gpu_decode_fsst_page_noalloc, through the C ABI).

Some callers of a decoder cannot allocate device memory: an engine whose buffer manager owns all of HBM and
forbids plugins to call cudaMalloc, or a caller on a path where allocating is not allowed.  They decode with
scratch compiled into the library.  Its output must equal the allocating string plan's, bit for bit, call after
call; it must read a page that the caller's own stream is still producing only after that stream has written
it; and its first call in a process must allocate nothing.  This file is collected last, so that a run stopping
at the first failure has run every other test before it."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _dev(a, dev, shift=0):
    import torch

    buf = torch.zeros(a.size + 64, dtype=torch.uint8, device=dev)
    if a.size:
        buf[shift:shift + a.size] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return buf, buf.data_ptr() + shift


def _plan_decode(cuda, pp, page_size, dp, dict_size):
    from fastlanes_b200 import strings

    plan = strings.StringPlan(pp, page_size, dp, dict_size)
    off, data = plan.decode(cuda)
    plan.close()
    return off.cpu().numpy(), data.cpu().numpy()


@pytest.mark.parametrize("eid", [13, 14, 0])
def test_noalloc_decode_equals_plan_decode_two_calls_in_a_row(cuda, col_golden, eid):
    import torch

    from fastlanes_b200 import strings

    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    pb, pp = _dev(page, cuda, 1)
    db, dp = _dev(dic, cuda) if dic.size else (None, None)
    want_off, want_data = _plan_decode(cuda, pp, page.size, dp, dic.size)
    assert np.array_equal(want_off.astype(np.uint64), col_golden[f"str_{eid}_input_offsets"])

    n_rows = want_off.size - 1
    offsets = torch.zeros(n_rows + 1, dtype=torch.int32, device=cuda)
    data = torch.zeros(want_data.size + 64, dtype=torch.uint8, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    for _ in range(2):
        offsets.fill_(-1)
        data.fill_(0xEE)
        status.zero_()
        rc = strings.decode_fsst_page_noalloc(pp, page.size, dp, dic.size, offsets, data, status)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        assert np.array_equal(offsets.cpu().numpy(), want_off)
        assert np.array_equal(data[: want_data.size].cpu().numpy(), want_data)


def test_noalloc_reads_the_page_in_the_callers_stream_order(cuda, col_golden):
    """The page is uploaded on a non-blocking stream behind a delay and the call is queued right after it on
    that stream: the header and table reads must wait for the upload."""
    import torch

    from fastlanes_b200 import strings

    page, dic = col_golden["str_13_page"], col_golden["str_13_dict"]
    ref_b, ref_p = _dev(page, cuda)
    db, dp = _dev(dic, cuda)
    want_off, want_data = _plan_decode(cuda, ref_p, page.size, dp, dic.size)

    host = torch.from_numpy(np.ascontiguousarray(page)).pin_memory()
    buf = torch.zeros(page.size + 64, dtype=torch.uint8, device=cuda)
    offsets = torch.zeros(want_off.size, dtype=torch.int32, device=cuda)
    data = torch.zeros(want_data.size + 64, dtype=torch.uint8, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    torch.cuda.synchronize()
    s = torch.cuda.Stream()  # created non-blocking: no implicit order with the legacy default stream
    with torch.cuda.stream(s):
        torch.cuda._sleep(20_000_000)  # about 10 ms of spinning before the upload lands
        buf[: page.size].copy_(host, non_blocking=True)
    rc = strings.decode_fsst_page_noalloc(buf.data_ptr(), page.size, dp, dic.size, offsets, data, status,
                                          stream=s.cuda_stream)
    s.synchronize()
    assert rc == 0
    assert int(status.item()) == 0
    assert np.array_equal(offsets.cpu().numpy(), want_off)
    assert np.array_equal(data[: want_data.size].cpu().numpy(), want_data)


def test_noalloc_rejects_pages_beyond_its_scratch_and_a_missing_status(cuda):
    import torch

    from fastlanes_b200 import strings

    hdr = np.zeros(64, np.uint8)
    hdr[0], hdr[1] = 7, 1  # FSST page header
    hdr[4:6] = np.frombuffer(np.uint16(8193).tobytes(), np.uint8)  # one vector more than the scratch holds
    pb, pp = _dev(hdr, cuda)
    offsets = torch.zeros(16, dtype=torch.int32, device=cuda)
    data = torch.zeros(16, dtype=torch.uint8, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    assert strings.decode_fsst_page_noalloc(pp, hdr.size, None, 0, offsets, data, status) == -6  # FLS_ERR_TOO_LARGE
    assert strings.decode_fsst_page_noalloc(pp, hdr.size, None, 0, offsets, data, None) == -1  # FLS_ERR_ARG


_CHILD = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from fastlanes_b200 import strings, _lib

g = np.load(sys.argv[2])
dev = torch.device("cuda:0")
page, dic = g["str_13_page"], g["str_13_dict"]
pb = torch.zeros(page.size + 64, dtype=torch.uint8, device=dev)
pb[: page.size] = torch.from_numpy(page).to(dev)
db = torch.zeros(dic.size + 64, dtype=torch.uint8, device=dev)
db[: dic.size] = torch.from_numpy(dic).to(dev)
bad = torch.zeros(64, dtype=torch.uint8, device=dev)
bad[0] = 99  # no string expression: the call stops after reading the header
n_rows = 1024 * int(page[4:6].view(np.uint16)[0])
offsets = torch.zeros(n_rows + 1, dtype=torch.int32, device=dev)
data = torch.zeros(1 << 20, dtype=torch.uint8, device=dev)
status = torch.zeros(1, dtype=torch.int32, device=dev)
torch.cuda.synchronize()
# the library's runtime starts (and, with eager module loading, loads its kernels) on its first CUDA call
rc0 = strings.decode_fsst_page_noalloc(bad.data_ptr(), 64, None, 0, offsets, data, status)
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
rcs = [strings.decode_fsst_page_noalloc(pb.data_ptr(), page.size, db.data_ptr(), dic.size, offsets, data, status)
       for _ in range(2)]
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
# control: an allocating entry point (the library's per-device status word is cudaMalloc'd on first use)
_lib.lib.fls_gpu_status(0)
torch.cuda.synchronize()
free2 = torch.cuda.mem_get_info()[0]
print(json.dumps({"rc0": rc0, "rcs": rcs, "status": int(status.item()), "free0": free0, "free1": free1,
                  "free2": free2}))
"""


def test_noalloc_first_call_in_a_fresh_process_allocates_nothing(cuda):
    """The first call on a device must not reach any cudaMalloc (the library's per-device state is allocated on
    first use, so a path through it would).  A fresh process with eager module loading: the library's kernels
    load on its first CUDA call (a page with an unknown expression), then free device memory must not change
    over two decodes.  A control call of an allocating entry point afterwards shows whether a 4-byte cudaMalloc
    is visible in free memory on this driver."""
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    out = subprocess.run([sys.executable, "-c", _CHILD, ROOT, os.path.join(ROOT, "tests", "golden", "columns.npz")],
                         capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["rc0"] == -4  # FLS_ERR_UNSUPPORTED
    assert r["rcs"] == [0, 0] and r["status"] == 0
    assert r["free1"] == r["free0"], r
    print("control: an allocating call changed free memory by", r["free1"] - r["free2"], "bytes")
