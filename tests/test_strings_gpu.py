"""String pages written by the reference's encoder, decoded on the GPU, against the reference decoder's output
(golden fixtures: tests/golden/columns.npz)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STR_IDS = [0, 2, 3, 8, 13, 14, 15, 16]
# the rest of the string pool: BYTE_ARR DELTA (1), DICT with patched codes (4-7, 9-12), DICT_FRQ (17-27), FSST12
# (28, 29)
STR_MORE_IDS = [1, 4, 5, 6, 7, 9, 10, 11, 12] + list(range(17, 28)) + [28, 29]


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


@pytest.mark.parametrize("eid", STR_IDS + STR_MORE_IDS)
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


def _mixed_length_dictionary(rng, n):
    """n entries: 10 % empty, 20 % of 1-3 bytes, 50 % of 4-40, 20 % of 41-300 (every byte value)."""
    kind = rng.choice(4, n, p=[0.1, 0.2, 0.5, 0.2])
    lo = np.array([0, 1, 4, 41])[kind]
    hi = np.array([0, 3, 40, 300])[kind]
    lens = rng.integers(lo, hi + 1)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    return rng.integers(0, 256, int(offs[-1]), dtype=np.uint8), offs


@pytest.mark.parametrize("n_dict", [600, 12000, 20000, 70000])
def test_string_dict_shared_memory_modes(cuda, n_dict):
    """DICT rows of every length class: the decoded dictionary in shared memory for the materialising pass
    (600 entries) or not (the larger ones), its end offsets in shared memory for the lengths pass (up to
    12000) or not (20000: 80 KB of them); 16-bit code rows below 65535 entries, 32-bit ones at 70000.  Batches
    of 32 long rows exceed the per-warp window."""
    from fastlanes_b200 import strings

    rng = np.random.default_rng(n_dict)
    dbytes, doffs = _mixed_length_dictionary(rng, n_dict)
    codes = rng.integers(0, n_dict, 37 * 1024).astype(np.uint32)  # the encoder takes whole vectors
    codes[5 * 1024:6 * 1024] = int(np.argmax(np.diff(doffs)))  # a vector of the longest entry only
    page, dic = strings.encode_string_dict(dbytes, doffs, codes)
    pb, pp = _dev(page, cuda, 1)
    db, dp = _dev(dic, cuda, 0)
    plan = strings.StringPlan(pp, page.size, dp, dic.size)
    offs, data = plan.decode(cuda)
    plan.close()
    lens = np.diff(doffs).astype(np.int64)
    want_off = np.zeros(codes.size + 1, np.int64)
    want_off[1:] = np.cumsum(lens[codes])
    assert np.array_equal(offs.cpu().numpy().astype(np.int64), want_off)
    idx = np.concatenate([np.arange(int(doffs[c]), int(doffs[c + 1])) for c in codes])
    assert np.array_equal(data.cpu().numpy(), dbytes[idx])


def _oracle_fsst12_rows(page, table):
    """Rows of an FSST12 page (plain end offsets) decoded by the oracle's FSST12 restatement."""
    from oracle import oracle, pages

    _, sym, ln = oracle.fsst12_decode_table(table)
    pg = pages.parse_page(page)
    rows = []
    for v in range(pg.vec_c):
        data = pg.vector_slice(v, 0)
        ends = oracle.untranspose_i(np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32).copy())
        start = 0
        for i in range(1024):
            rows.append(oracle.fsst12_decode(sym, ln, data[start:ends[i]]))
            start = ends[i]
    return rows


def test_fsst12_codes_past_the_symbol_count_decode_as_corrupt(cuda, col_golden):
    """A reference FSST12 page read with a table cut to its first 100 symbols: every code past them decodes as
    the 8 bytes "corrupt" (fsst12_import's fill), on the GPU as in the oracle."""
    from fastlanes_b200 import primitives as P
    from fastlanes_b200.strings import StringPlan

    page, dic = col_golden["str_28_page"], col_golden["str_28_dict"].copy()
    hist = np.frombuffer(dic[16:32].tobytes(), np.uint16)
    assert int(hist.sum()) > 100
    dic[16:32] = np.frombuffer(np.array([100, 0, 0, 0, 0, 0, 0, 0], np.uint16).tobytes(), np.uint8)
    rows = _oracle_fsst12_rows(page, dic[8:])
    want_b = np.concatenate(rows)
    assert b"corrupt" in want_b.tobytes()
    want_o = np.zeros(len(rows) + 1, np.uint64)
    want_o[1:] = np.cumsum([r.size for r in rows])
    pb, pp = _dev(page, cuda, 0)
    db, dp = _dev(dic, cuda, 0)
    plan = StringPlan(pp, page.size, dp, dic.size)
    offs, data = plan.decode(cuda)
    plan.close()
    assert np.array_equal(offs.cpu().numpy().astype(np.uint64), want_o)
    assert np.array_equal(data.cpu().numpy(), want_b)
    assert P.device_status() == 0


def test_fsst12_malformed_tables_are_refused(cuda, col_golden):
    """An FSST12 symbol table whose counts exceed 4096 codes, with a symbol longer than 8 bytes, cut short, or
    with another version word is a format error at plan creation (the reference would write past its table)."""
    from fastlanes_b200._lib import FlsError
    from fastlanes_b200.strings import StringPlan

    page, dic = col_golden["str_28_page"], col_golden["str_28_dict"]
    pb, pp = _dev(page, cuda, 0)
    bad = []
    d = dic.copy()
    d[16:32] = np.frombuffer(np.array([4000, 97, 0, 0, 0, 0, 0, 0], np.uint16).tobytes(), np.uint8)
    bad.append(d)
    d = dic.copy()
    d[32] = 9  # the first symbol's length byte
    bad.append(d)
    bad.append(dic[:40].copy())
    d = dic.copy()
    d[12] ^= 1  # the version word's upper half
    bad.append(d)
    for d in bad:
        db, dp = _dev(d, cuda, 0)
        with pytest.raises(FlsError):
            StringPlan(pp, page.size, dp, d.size)


def test_decode_after_measure_and_alone_agree(cuda, col_golden):
    """decode() straight after measure() reuses the measured vector totals; decode() alone recomputes them; both
    give the reference's rows (DICT FFOR page, string pool id 3)."""
    import torch

    from fastlanes_b200.strings import StringPlan

    page, dic = col_golden["str_3_page"], col_golden["str_3_dict"]
    want_o, want_b = _expected(col_golden, 3)
    pb, pp = _dev(page, cuda, 0)
    db, dp = _dev(dic, cuda, 0)
    plan = StringPlan(pp, page.size, dp, dic.size)
    n = plan.measure()
    assert n == want_b.size
    for _ in range(3):  # after measure, then twice without
        offs = torch.empty(plan.n_rows + 1, dtype=torch.int32, device=cuda)
        data = torch.empty(n + 16, dtype=torch.uint8, device=cuda)
        plan.decode_into(offs, data)
        assert np.array_equal(offs.cpu().numpy().astype(np.uint64), want_o)
        assert np.array_equal(data[:n].cpu().numpy(), want_b)
    plan.close()


DICT_KIND_IDS = [2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 15, 16] + list(range(17, 28))


@pytest.mark.parametrize("n_dict", [600, 20000, 70000])
def test_single_pass_dict_decode_every_size_class(cuda, n_dict):
    """The single-pass DICT decode (entries below 256 bytes: the packed row table exists): dictionary and row table
    in shared memory (600 entries) or read from global memory (20000, 70000), 16-bit code rows below 65535
    entries and 32-bit ones at 70000, empty and 1-3-byte entries, batches of long rows larger than the window."""
    from fastlanes_b200 import strings
    from fastlanes_b200 import workloads as W

    rng = np.random.default_rng(n_dict + 1)
    kind = rng.choice(4, n_dict, p=[0.1, 0.2, 0.5, 0.2])
    lens = rng.integers(np.array([0, 1, 4, 41])[kind], np.array([0, 3, 40, 255])[kind] + 1)
    doffs = np.zeros(n_dict + 1, np.uint64)
    doffs[1:] = np.cumsum(lens)
    dbytes = rng.integers(0, 256, int(doffs[-1]), dtype=np.uint8)
    codes = rng.integers(0, n_dict, 41 * 1024).astype(np.uint32)
    codes[7 * 1024:8 * 1024] = int(np.argmax(np.diff(doffs)))
    page, dic = strings.encode_string_dict(dbytes, doffs, codes)
    pb, pp = _dev(page, cuda, 3)
    db, dp = _dev(dic, cuda, 0)
    plan = strings.StringPlan(pp, page.size, dp, dic.size)
    offs, data = plan.decode(cuda)
    plan.close()
    assert W.dict_rows_match(offs, data, dbytes, doffs, codes)


def test_string_set_decodes_every_dict_page_in_one_launch(cuda, col_golden):
    """Every DICT-kind page of the reference's string pool (DICT with plain / FFOR / DELTA / patched codes,
    DICT_RLE, DICT_FRQ; each with its own dictionary) plus two columns of the DICT+FSST configuration's shape,
    decoded by one string set: one kernel launch, every column equal to the reference decoder's rows, twice in
    a row and as a CUDA graph replay."""
    import torch

    from fastlanes_b200 import _lib
    from fastlanes_b200 import primitives as P
    from fastlanes_b200 import strings
    from fastlanes_b200 import workloads as W

    keep, plans, wants = [], [], []
    for eid in DICT_KIND_IDS:
        page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
        pb, pp = _dev(page, cuda, eid % 4)
        db, dp = _dev(dic, cuda, 0)
        keep += [pb, db]
        plans.append(strings.StringPlan(pp, page.size, dp, dic.size))
        wants.append(("ref", _expected(col_golden, eid)))
    for seed in (11, 12):
        dbytes, doffs = W.string_dictionary(seed=seed)
        codes = W.zipf_codes(50 * 1024, seed=seed)
        page, dic = strings.encode_string_dict(dbytes, doffs, codes)
        pb, pp = _dev(page, cuda, 0)
        db, dp = _dev(dic, cuda, 0)
        keep += [pb, db]
        plans.append(strings.StringPlan(pp, page.size, dp, dic.size))
        wants.append(("gen", (dbytes, doffs, codes)))
    sizes = [p.measure() for p in plans]
    offs = [torch.full((p.n_rows + 1,), -1, dtype=torch.int32, device=cuda) for p in plans]
    data = [torch.full((n + 16,), 0xEE, dtype=torch.uint8, device=cuda) for n in sizes]
    sset = strings.StringSet(plans)
    sset.bind(offs, data)

    def check():
        torch.cuda.synchronize()
        for (kind, w), o, d, n in zip(wants, offs, data, sizes):
            if kind == "ref":
                assert np.array_equal(o.cpu().numpy().astype(np.uint64), w[0])
                assert np.array_equal(d[:n].cpu().numpy(), w[1])
            else:
                assert W.dict_rows_match(o, d[:n], *w)
            assert (d[n:] == 0xEE).all()

    _lib.lib.fls_gpu_launch_count(1)
    sset.decode()
    assert _lib.lib.fls_gpu_launch_count(1) == 1
    check()
    for o in offs:
        o.fill_(-1)
    sset.decode()
    check()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            sset.decode()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        for o in offs:
            o.fill_(-1)
        g.replay()
        check()
    del g
    sset.close()
    for p in plans:
        p.close()
    assert P.device_status() == 0


def test_fsst_column_with_and_without_escapes(cuda):
    """The single-pass FSST decode on a page of our own encoder where some vectors hold escape codes (rare bytes
    outside the symbol table: those vectors take the escape-aware total) and others none (their total is the sum
    of their symbol lengths), with empty, one-byte and long rows: every offset and byte as the input's."""
    from fastlanes_b200 import primitives as P
    from fastlanes_b200 import strings as S

    rng = np.random.default_rng(31)
    common = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz0123456789", np.uint8)
    n_vec = 48
    rows = []
    for v in range(n_vec):
        rare = v % 3 == 1  # every third vector: rows sprinkled with rare bytes
        for _ in range(1024):
            n = int(rng.choice([0, 1, 3, 9, 24, 200], p=[.1, .1, .2, .3, .25, .05]))
            r = common[rng.integers(0, common.size, n)]
            if rare and n:
                m = rng.random(n) < 0.2
                r = r.copy()
                r[m] = rng.integers(128, 256, int(m.sum()), dtype=np.uint8)
            rows.append(r)
    byts = np.concatenate(rows).astype(np.uint8)
    offs = np.zeros(len(rows) + 1, np.uint64)
    offs[1:] = np.cumsum([r.size for r in rows])
    table, comp, coffs = S.fsst_compress(byts, offs)
    assert (comp == 255).any()  # the page does hold escapes
    page, dic = S.fsst_page(table, comp, coffs)
    pb, pp = _dev(page, cuda, 1)
    db, dp = _dev(dic, cuda, 0)
    plan = S.StringPlan(pp, page.size, dp, dic.size)
    n = plan.measure()
    assert n == byts.size
    got_o, got_b = plan.decode(cuda)
    assert np.array_equal(got_o.cpu().numpy().astype(np.uint64), offs)
    assert np.array_equal(got_b.cpu().numpy(), byts)
    plan.close()
    assert P.device_status() == 0


def test_string_set_with_a_dictionary_too_large_for_shared_memory(cuda):
    """A string set whose largest dictionary (70,000 entries: 32-bit code rows) does not fit in shared memory
    decodes every column from global memory in one launch: a large-dictionary column, two small ones of 16-bit
    codes and a one-vector column, every offset and byte against the generator's rows, twice in a row."""
    import torch

    from fastlanes_b200 import primitives as P
    from fastlanes_b200 import strings
    from fastlanes_b200 import workloads as W

    rng = np.random.default_rng(77)
    cols = []
    for n_dict, n_vec in ((70000, 9), (300, 5), (4096, 12), (17, 1)):
        lens = rng.integers(0, 60, n_dict)
        doffs = np.zeros(n_dict + 1, np.uint64)
        doffs[1:] = np.cumsum(lens)
        dbytes = rng.integers(0, 256, int(doffs[-1]), dtype=np.uint8)
        codes = rng.integers(0, n_dict, n_vec * 1024).astype(np.uint32)
        cols.append((dbytes, doffs, codes))
    keep, plans = [], []
    for i, (dbytes, doffs, codes) in enumerate(cols):
        page, dic = strings.encode_string_dict(dbytes, doffs, codes)
        pb, pp = _dev(page, cuda, i % 4)
        db, dp = _dev(dic, cuda, 0)
        keep += [pb, db]
        plans.append(strings.StringPlan(pp, page.size, dp, dic.size))
    sizes = [p.measure() for p in plans]
    offs = [torch.full((p.n_rows + 1,), -1, dtype=torch.int32, device=cuda) for p in plans]
    data = [torch.full((n + 16,), 0xEE, dtype=torch.uint8, device=cuda) for n in sizes]
    sset = strings.StringSet(plans)
    sset.bind(offs, data)
    for _ in range(2):
        sset.decode()
        torch.cuda.synchronize()
        for (dbytes, doffs, codes), o, d, n in zip(cols, offs, data, sizes):
            assert W.dict_rows_match(o, d[:n], dbytes, doffs, codes)
            assert (d[n:] == 0xEE).all()
    sset.close()
    for p in plans:
        p.close()
    assert P.device_status() == 0
