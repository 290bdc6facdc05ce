"""A 1 Mi-row string DICT page written by the reference's own encoder (string pool id 3, an FSST-compressed
4096-entry dictionary; tests/golden/str_dict_1m.npz, made by tests/golden/make_str_dict_1m.py): every offset
and every byte the GPU decodes equals the reference decoder's rows."""
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixture():
    spec = importlib.util.spec_from_file_location("make_str_dict_1m", os.path.join(HERE, "golden", "make_str_dict_1m.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod, np.load(os.path.join(HERE, "golden", "str_dict_1m.npz"))


def test_regenerated_codes_are_the_pages_codes():
    """The fixture's rows are regenerated by row_codes() (seeded values through the reference's own numbering);
    the oracle's decode of the page's code stream (DICT FFOR_NO_PATCH: unffor + untranspose per vector) must give
    exactly those codes."""
    from oracle import oracle
    from oracle import pages

    mod, g = _fixture()
    codes = mod.row_codes(g["code_of_value"])
    pg = pages.parse_page(g["page"])
    assert (pg.exp_t, pg.var, pg.vec_c) == (8, 2, codes.size // 1024)
    got = np.concatenate([oracle.untranspose_i(np.ascontiguousarray(pages._stream(pg, v, 0, 32, "ffor", np.uint32)))
                          for v in range(pg.vec_c)])
    assert np.array_equal(got, codes)
    lens = np.diff(g["ref_dict_offsets"]).astype(np.int64)
    assert int(lens[codes].sum()) == int(g["n_decoded_bytes"])


@pytest.mark.gpu
@pytest.mark.parametrize("shift", [0, 5])
def test_million_row_reference_dict_page_every_byte(cuda, shift):
    import torch

    from fastlanes_b200 import strings as S
    from fastlanes_b200 import workloads as W

    mod, g = _fixture()
    page, dic = g["page"], g["dict"]
    pb = torch.zeros(page.size + 64, dtype=torch.uint8, device=cuda)
    pb[shift:shift + page.size] = torch.from_numpy(page).to(cuda)
    db = torch.from_numpy(dic).to(cuda)
    plan = S.StringPlan(pb.data_ptr() + shift, page.size, db.data_ptr(), dic.size)
    n = plan.measure()
    assert n == int(g["n_decoded_bytes"])
    offs = torch.full((plan.n_rows + 1,), -1, dtype=torch.int32, device=cuda)
    data = torch.full((n + 16,), 0xEE, dtype=torch.uint8, device=cuda)
    plan.decode_into(offs, data)
    torch.cuda.synchronize()
    plan.close()
    assert W.dict_rows_match(offs, data[:n], g["ref_dict_bytes"], g["ref_dict_offsets"], mod.row_codes(g["code_of_value"]))
    assert (data[n:] == 0xEE).all()
