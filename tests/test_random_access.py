"""Random access by vector through the reference's C API (include/fastlanes.h init_random_access / random_access,
declared by the reference and defined nowhere there), on pages written by the reference's encoder."""
import numpy as np
import pytest

from fastlanes_b200 import pages

# pages whose buffers are all per vector: UNCOMPRESSED, FFOR, DELTA, RLE (6, 7) and the patched FFOR / DELTA
# variants without rec buffers
KEYS = ["i64_0", "i64_1", "i64_11", "i64_6", "i64_7", "i64patch_2", "i64patch_4", "i64patch_5", "i64patch_12",
        "i64patch_13", "i64patch_14"]


def _slices(page, v):
    r = pages.random_access_ranges(page, v)
    out = []
    for off, size in r:
        end = min(int(off) + int(size), page.size)  # the last vector's packed range is clipped to the page
        out.append(page[int(off):end])
    return r, out


@pytest.mark.parametrize("key", KEYS)
def test_ranges_tile_every_buffer(col_golden, key):
    page = col_golden[f"{key}_page"]
    info = pages.page_info(page)
    n_vec = info["vec_c"]
    ranges = [pages.random_access_ranges(page, v) for v in range(n_vec)]
    n_buf = ranges[0].shape[0]
    for i in range(n_buf):
        for v in range(n_vec - 1):
            assert ranges[v + 1][i][0] == ranges[v][i][0] + ranges[v][i][1]
        if i + 1 < n_buf:
            assert ranges[-1][i][0] + ranges[-1][i][1] == ranges[0][i + 1][0]
    assert ranges[0][0][0] == 8 + 4 * n_buf + 4 * n_buf * (n_vec - 1)
    with pytest.raises(pages.FlsError):
        pages.random_access_ranges(page, n_vec)


def test_ranges_refuse_pages_with_page_wide_buffers(col_golden):
    # a dictionary (17, 27) or rec-compressed exceptions (3: FFOR S_PATCH_REC, 15: DELTA B_PATCH_REC)
    for key in ("i64_17", "i64_27", "i64patch_3", "i64patch_15"):
        with pytest.raises(pages.FlsError):
            pages.random_access_ranges(col_golden[f"{key}_page"], 0)


@pytest.mark.gpu
@pytest.mark.parametrize("key", KEYS)
def test_random_access_decodes_each_vector(cuda, col_golden, key):
    page, want = col_golden[f"{key}_page"], col_golden[f"{key}_input"].view(np.int64)
    n_vec = pages.page_info(page)["vec_c"]
    for v in range(n_vec):
        r, bufs = _slices(page, v)
        got = pages.random_access(page, v, bufs, r)
        assert np.array_equal(got, want[1024 * v:1024 * (v + 1)]), (key, v)
