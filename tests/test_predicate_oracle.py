"""Predicate pushdown without a GPU: the oracle's restatement of the reference's predicate primitives
(src/primitive/predicate/equal.cpp) pinned against the reference's own code, and the filter form of the
device decode logic (emulated warp) against the oracle on reference-encoded pages."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from oracle import predicate as PR
from tests.emu import build

REF = oracle.reference
REF_OPS = {PR.EQ: 0, PR.GT: 1, PR.LT: 2}  # eq_vector_constant_func, ge_tvec_cvec (>), lessthan_func (<)


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.skipif(REF is None or not hasattr(REF, "ref_predicate_i64"), reason="reference build absent")
@pytest.mark.parametrize("op", sorted(REF_OPS))
@pytest.mark.parametrize("seed", range(4))
def test_oracle_predicates_match_reference(op, seed):
    rng = np.random.default_rng(seed)
    vec = rng.integers(-50, 50, 1024).astype(np.int64)
    if seed == 3:
        vec = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, 1024, dtype=np.int64)
    for value in [int(vec[7]), -51, 50, 0, int(np.iinfo(np.int64).min)]:
        idx = np.zeros(1024, np.uint16)
        n = REF.ref_predicate_i64(REF_OPS[op], P(vec), ctypes.c_int64(value), P(idx))
        want = idx[:n]
        assert np.array_equal(PR.select_vector(vec, op, value), want)
        got, m = PR.selection(PR.bitmaps(vec, op, value)[0])
        assert m == n and np.array_equal(got, want)


@pytest.mark.skipif(REF is None or not hasattr(REF, "ref_selection_and"), reason="reference build absent")
@pytest.mark.parametrize("seed", range(5))
def test_oracle_selection_and_matches_reference(seed):
    rng = np.random.default_rng(seed)
    a = np.sort(rng.choice(1024, int(rng.integers(0, 1024)), replace=False)).astype(np.uint16)
    b = np.sort(rng.choice(1024, int(rng.integers(0, 1024)), replace=False)).astype(np.uint16)
    out = np.zeros(1024, np.uint16)
    n = REF.ref_selection_and(P(a), a.size, P(b), b.size, P(out))
    assert np.array_equal(PR.selection_and(a, a.size, b, b.size), out[:n])
    assert np.array_equal(np.intersect1d(a, b), out[:n])


@pytest.fixture(scope="module")
def emu():
    return ctypes.CDLL(build.build())


def _emu_bitmaps(emu, page, dic, width, order, signed, op, value, n_vec):
    out = np.zeros(n_vec * 16, np.uint64)
    st = emu.emu_filter_page(P(page), ctypes.c_uint64(page.size), P(dic) if dic is not None and dic.size else None,
                             ctypes.c_uint64(0 if dic is None else dic.size), width, order, 2 if signed else 1,
                             ctypes.c_uint32(op), ctypes.c_uint64(value & (2**64 - 1)), P(out))
    return out.reshape(n_vec, 16), st


def _in_order(values, order):
    if order == 1:
        return values
    u = values.view(np.uint64)
    return np.concatenate([oracle.transpose_i(u[v * 1024:(v + 1) * 1024].copy())
                           for v in range(u.size // 1024)]).view(values.dtype)


@pytest.mark.parametrize("key", ["i64_1", "i64_6", "i64_11", "i64_17", "i64_22", "i64patch_2", "i64patch_13"])
@pytest.mark.parametrize("order", [0, 1])
def test_emulated_filter_reference_pages(emu, col_golden, key, order):
    """FFOR, RLE, DELTA, DICT, DICT_RLE and patched pages: every operator, constants inside and outside the
    values' range, bitmaps in original and transposed order equal to the oracle's on the decoded values."""
    if f"{key}_page" not in col_golden.files:
        pytest.skip(f"no fixture {key}")
    page = np.ascontiguousarray(col_golden[f"{key}_page"])
    dic = np.ascontiguousarray(col_golden[f"{key}_dict"]) if f"{key}_dict" in col_golden.files else None
    want = np.ascontiguousarray(col_golden[f"{key}_input"]).view(np.int64)
    n_vec = want.size // 1024
    vals = _in_order(want, order)
    for value in [int(want[3]), int(want.min()) - 1, int(want.max()), int(np.median(want))]:
        for op in range(6):
            got, st = _emu_bitmaps(emu, page, dic, 64, order, True, op, value, n_vec)
            assert st == 0
            assert np.array_equal(got, PR.bitmaps(vals, op, value)), (op, value)
    # unsigned comparison of the same bits
    value = int(want.view(np.uint64)[5])
    got, st = _emu_bitmaps(emu, page, dic, 64, order, False, PR.LT, value, n_vec)
    assert st == 0 and np.array_equal(got, PR.bitmaps(vals.view(np.uint64), PR.LT, value))
