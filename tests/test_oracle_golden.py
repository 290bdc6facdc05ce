"""The CPU oracle against the reference's own golden vectors (and, where it was built here, the reference
library itself).  Pins the oracle before any GPU result is compared with it."""
import hashlib
import re

import numpy as np
import pytest

from oracle import oracle

TYPES = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}


def _cases(z):
    for k in z.files:
        m = re.match(r"(unpack|unffor)_w(\d+)_b(\d+)_in$", k)
        if m:
            yield m.group(1), int(m.group(2)), int(m.group(3))


def test_every_golden_vector_present(prim_golden):
    cases = list(_cases(prim_golden))
    # 124 vectors per helper: bw 0..W for W = 8, 16, 32, 64
    assert len(cases) == 2 * (9 + 17 + 33 + 65)


def test_pack_ffor_unpack_unffor_golden(prim_golden):
    for kind, w, bw in _cases(prim_golden):
        T = TYPES[w]
        x = prim_golden[f"{kind}_w{w}_b{bw}_in"]
        base = 0 if kind == "unpack" else 10
        packed = oracle.ffor(x, bw, base)
        digest = hashlib.sha256(packed.tobytes()).digest()
        assert digest == prim_golden[f"{kind}_w{w}_b{bw}_packed_sha256"].tobytes(), (kind, w, bw)
        if w <= 16:
            assert np.array_equal(packed, prim_golden[f"{kind}_w{w}_b{bw}_packed"])
        assert np.array_equal(oracle.unffor(packed, bw, base, T), x), (kind, w, bw)


@pytest.mark.parametrize("w", [8, 16, 32, 64])
def test_transpose_rsum_golden(prim_golden, w):
    g = lambda s: prim_golden[f"range_w{w}{s}"]
    assert np.array_equal(oracle.transpose_i(g("")), g("_transposed"))
    assert np.array_equal(oracle.untranspose_i(g("")), g("_untransposed"))
    assert np.array_equal(oracle.untranspose_i(g("_transposed")), g(""))
    assert np.array_equal(oracle.unrsum(g("_transposed")), g("_delta"))
    assert np.array_equal(oracle.rsum(g("_delta"), g("_bases")), g("_rsum"))
    assert np.array_equal(g("_rsum"), g("_transposed"))


@pytest.mark.skipif(oracle.reference is None, reason="reference library not built in this container")
@pytest.mark.parametrize("w", [8, 16, 32, 64])
def test_oracle_matches_reference_random(w):
    import ctypes

    ref = oracle.reference
    T = TYPES[w]
    rng = np.random.default_rng(w)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    for bw in range(w + 1):
        x = rng.integers(0, np.iinfo(np.uint64).max, 1024, dtype=np.uint64, endpoint=True).astype(T)
        base = T(rng.integers(0, np.iinfo(T).max, dtype=np.uint64, endpoint=True))
        if bw < w:
            x = ((x & T((1 << bw) - 1)) + base).astype(T)
        rp = np.zeros(1024, T)
        getattr(ref, f"ref_ffor_u{w}")(P(x), P(rp), ctypes.c_uint8(bw), P(np.array([base], T)))
        assert np.array_equal(rp[: bw * 1024 // w], oracle.ffor(x, bw, base)), bw
        ro = np.zeros(1024, T)
        getattr(ref, f"ref_unffor_u{w}")(P(rp), P(ro), ctypes.c_uint8(bw), P(np.array([base], T)))
        assert np.array_equal(ro, oracle.unffor(rp[: bw * 1024 // w], bw, base, T)), bw
    d = rng.integers(0, 1 << 62, 1024, dtype=np.uint64).astype(T)
    lb = rng.integers(0, 1 << 62, 1024 // w, dtype=np.uint64).astype(T)
    ro = np.zeros(1024, T)
    getattr(ref, f"ref_rsum_u{w}")(P(d), P(ro), P(lb))
    assert np.array_equal(ro, oracle.rsum(d, lb))


def test_fsst_import_and_decode_golden(col_golden):
    """FSST symbol table of a reference FSST column (str expression 13) decodes every row of its page."""
    from oracle import pages

    page = col_golden["str_13_page"]
    dic = col_golden["str_13_dict"]
    used, sym, ln = oracle.fsst_decode_table(dic[8:])
    assert used > 17
    pg = pages.parse_page(page)
    assert pg.arr_c == 2
    exp_bytes = col_golden["str_13_input_bytes"]
    exp_offs = col_golden["str_13_input_offsets"]
    row = 0
    for v in range(pg.vec_c):
        data = pg.vector_slice(v, 0)
        ends_t = np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32)
        ends = oracle.untranspose_i(ends_t.copy())
        start = 0
        for i in range(1024):
            got = oracle.fsst_decode(sym, ln, data[start:ends[i]])
            want = exp_bytes[exp_offs[row]:exp_offs[row + 1]]
            assert np.array_equal(got, want), row
            start = ends[i]
            row += 1


@pytest.mark.parametrize("eid", [0, 1, 6, 7, 11, 16, 17, 22, 27])
def test_page_oracle_decodes_reference_int64_pages(col_golden, eid):
    """The page-framing restatement reproduces the reference decoder on reference-encoded int64 pages."""
    from oracle import pages

    page = col_golden[f"i64_{eid}_page"]
    dic = col_golden[f"i64_{eid}_dict"]
    got = pages.decode_int(page, dic if dic.size else None, np.uint64).view(np.int64)
    assert np.array_equal(got, col_golden[f"i64_{eid}_input"])


@pytest.mark.parametrize("eid", [8, 9, 10, 16, 17, 22, 27])
def test_page_oracle_decodes_reference_rec_pages(col_golden, eid):
    """Reference pages whose rec buffers hold FFOR blocks with exceptions (large dictionaries, many runs)."""
    from oracle import pages

    page = col_golden[f"i64rec_{eid}_page"]
    dic = col_golden[f"i64rec_{eid}_dict"]
    got = pages.decode_int(page, dic if dic.size else None, np.uint64).view(np.int64)
    assert np.array_equal(got, col_golden[f"i64rec_{eid}_input"])
    # the fixtures do exercise FFOR rec blocks
    buf = dic[8:] if eid in (16, 17, 22) else page[pages.parse_page(page).off[0]:]
    assert buf[0] != 255


@pytest.mark.parametrize("eid", [2, 3, 4, 5, 12, 13, 14, 15])
def test_page_oracle_decodes_reference_patched_pages(col_golden, eid):
    """Patched FFOR / DELTA pages of the reference (S / B / LL patches, rec-compressed exceptions)."""
    from oracle import pages

    page = col_golden[f"i64patch_{eid}_page"]
    got = pages.decode_int(page, None, np.uint64).view(np.int64)
    assert np.array_equal(got, col_golden[f"i64patch_{eid}_input"])


@pytest.mark.parametrize("eid", [18, 19, 20, 21, 22, 23, 24, 25, 26])
def test_page_oracle_decodes_reference_patched_dict_pages(col_golden, eid):
    """DICT pages whose u32 codes are patched FFOR / DELTA streams (pool ids 18-26), then gathered."""
    from oracle import pages

    page, dic = col_golden[f"i64dpatch_{eid}_page"], col_golden[f"i64dpatch_{eid}_dict"]
    got = pages.decode_int(page, dic, np.uint64).view(np.int64)
    assert np.array_equal(got, col_golden[f"i64dpatch_{eid}_input"])


@pytest.mark.parametrize("eid", list(range(28, 39)))
def test_page_oracle_decodes_reference_dict_frq_pages(col_golden, eid):
    """DICT_FRQ pages (pool ids 28-38, exp_t 9): DICT pages over a frequency-ordered dictionary."""
    from oracle import pages

    page, dic = col_golden[f"i64frq_{eid}_page"], col_golden[f"i64frq_{eid}_dict"]
    got = pages.decode_int(page, dic, np.uint64).view(np.int64)
    assert np.array_equal(got, col_golden[f"i64frq_{eid}_input"])


@pytest.mark.parametrize("eid", [28, 29])
def test_fsst12_import_and_decode_golden(col_golden, eid):
    """FSST12 columns of the reference (string pool ids 28, 29: end offsets plain or DELTA-coded) decode every
    row of their page through the FSST12 restatement."""
    from oracle import pages

    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    used, sym, ln = oracle.fsst12_decode_table(dic[8:])
    assert used > 24 and used <= dic.size - 8
    assert sym[4095] == 32774747032022883 and ln[4095] == 8  # unused codes decode as "corrupt"
    pg = pages.parse_page(page)
    assert (pg.exp_t, pg.var) == (20, 1 if eid == 28 else 2)
    exp_bytes, exp_offs = col_golden[f"str_{eid}_input_bytes"], col_golden[f"str_{eid}_input_offsets"]
    row = 0
    for v in range(pg.vec_c):
        data = pg.vector_slice(v, 0)
        if eid == 28:
            ends_t = np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32).copy()
        else:
            ends_t = pages._stream(pg, v, 1, 32, "delta", np.uint32)
        ends = oracle.untranspose_i(ends_t)
        start = 0
        for i in range(1024):
            got = oracle.fsst12_decode(sym, ln, data[start:ends[i]])
            assert (ends[i] - start) % 3 != 1  # codes come in 3-byte pairs and 2-byte singles
            assert np.array_equal(got, exp_bytes[exp_offs[row]:exp_offs[row + 1]]), row
            start = ends[i]
            row += 1
    assert row == exp_offs.size - 1


@pytest.mark.parametrize("eid", [0, 6, 7] + list(range(16, 39)))
def test_page_oracle_decodes_reference_double_pages(col_golden, eid):
    """Double columns of the reference (double pool ids 0, 6, 7, 16-38: raw double dictionaries): the page
    restatement reproduces the values' bit patterns, NaNs, infinities and signed zeros included."""
    from oracle import pages

    page, dic = col_golden[f"f64_{eid}_page"], col_golden[f"f64_{eid}_dict"]
    got = pages.decode_int(page, dic if dic.size else None, np.uint64, raw_dict=True)
    assert np.array_equal(got, col_golden[f"f64_{eid}_input"].view(np.uint64))


def test_fsst_column_page_writer_round_trips(col_golden):
    """The engine's FSST column page writer (strings.encode_fsst_page, host only) lays pages out as the
    reference does: same header and buffer structure as the reference's FSST page of the same strings, and
    every row decodes back through the oracle's restatement of the reference decoder."""
    from fastlanes_b200 import strings as S
    from oracle import pages

    byts, offs = col_golden["str_13_input_bytes"], col_golden["str_13_input_offsets"]
    page, dic = S.encode_fsst_page(byts, offs)
    ref = pages.parse_page(col_golden["str_13_page"])
    pg = pages.parse_page(page)
    assert (pg.exp_t, pg.var, pg.vec_c, pg.arr_c) == (ref.exp_t, ref.var, ref.vec_c, ref.arr_c)
    assert dic[0] == col_golden["str_13_dict"][0]
    _, sym, ln = oracle.fsst_decode_table(dic[8:])
    row = 0
    for v in range(pg.vec_c):
        assert pg.vector_slice(v, 1).size == 4096
        data = pg.vector_slice(v, 0)
        ends = oracle.untranspose_i(np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32).copy())
        start = 0
        for i in range(1024):
            assert np.array_equal(oracle.fsst_decode(sym, ln, data[start:ends[i]]), byts[offs[row]:offs[row + 1]])
            start = ends[i]
            row += 1
