"""The whole-buffer parity checker of the string legs (workloads.dict_rows_match), on the CPU: it accepts the
rows the generator meant and refuses a single wrong byte or offset anywhere."""
import numpy as np
import torch

from fastlanes_b200 import workloads as W


def _rows(dbytes, doffs, codes):
    parts = [dbytes[int(doffs[c]):int(doffs[c + 1])] for c in codes]
    offs = np.zeros(codes.size + 1, np.int64)
    offs[1:] = np.cumsum([p.size for p in parts])
    return np.concatenate(parts), offs


def test_dict_rows_match_accepts_exact_rows_and_refuses_any_difference():
    dbytes, doffs = W.string_dictionary(n_dict=300)
    rng = np.random.default_rng(3)
    codes = rng.integers(0, 300, 5000).astype(np.uint32)
    data, offs = _rows(dbytes, doffs, codes)
    d = torch.from_numpy(data.copy())
    o = torch.from_numpy(offs.astype(np.int32))
    assert W.dict_rows_match(o, d, dbytes, doffs, codes, chunk_rows=777)
    for pos in (0, data.size // 2, data.size - 1):
        bad = d.clone()
        bad[pos] ^= 1
        assert not W.dict_rows_match(o, bad, dbytes, doffs, codes, chunk_rows=777)
    bad_o = o.clone()
    bad_o[1234] += 1
    assert not W.dict_rows_match(bad_o, d, dbytes, doffs, codes)
    assert not W.dict_rows_match(o, d[:-1], dbytes, doffs, codes)
