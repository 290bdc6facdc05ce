"""The decode engine's device logic (make_plan / decode_vector of fastlanes_b200/csrc/fls_decode.cu), compiled
as host code and run on an emulated warp (32 threads + barrier), against the CPU oracle.  Catches layout and
indexing mistakes without a GPU; the same cases run on the B200 in test_primitives_gpu.py."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from tests.emu import build

TYPES = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}


@pytest.fixture(scope="module")
def emu():
    return ctypes.CDLL(build.build())


def P(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def batch(w, n_vec, rng):
    T = TYPES[w]
    bw = rng.integers(0, w + 1, n_vec).astype(np.uint8)
    base = rng.integers(0, np.iinfo(T).max, n_vec, dtype=np.uint64, endpoint=True).astype(T)
    chunks, offs, pos = [], [], 0
    for v in range(n_vec):
        b = int(bw[v])
        x = rng.integers(0, np.iinfo(np.uint64).max, 1024, dtype=np.uint64, endpoint=True)
        if b < 64:
            x &= np.uint64((1 << b) - 1)
        x = (x.astype(T) + base[v]).astype(T)
        p = oracle.ffor(x, b, base[v]).view(np.uint8)
        chunks.append(p)
        offs.append(pos)
        pos += p.size
    return np.concatenate(chunks + [np.zeros(256, np.uint8)]), np.array(offs, np.uint64), bw, base


def run(emu, w, enc, order, packed, off, bw, base, lane_base, n):
    out = np.zeros(n * 1024, TYPES[w])
    st = emu.emu_unffor(w, enc, order, P(packed), P(off), P(bw), P(None if base is None else base.view(np.uint8)),
                        P(None if lane_base is None else lane_base.view(np.uint8)), ctypes.c_uint64(n), P(out))
    return out, st


@pytest.mark.parametrize("w", [8, 16, 32, 64])
@pytest.mark.parametrize("order", [0, 1])
def test_emulated_unffor(emu, w, order):
    rng = np.random.default_rng(11 + w)
    n = 24
    _, _, bw, base = batch(w, n, rng)
    bw[:2] = [0, w]  # always cover the edge widths
    packed, off, _, _ = _rebuild(w, bw, base, rng)
    got, st = run(emu, w, 1, order, packed, off, bw, base, None, n)
    assert st == 0
    assert np.array_equal(got, oracle.unffor_batch(packed, off, bw, base, order == 1))


def _rebuild(w, bw, base, rng):
    T = TYPES[w]
    chunks, offs, pos = [], [], 0
    for v in range(bw.size):
        b = int(bw[v])
        x = rng.integers(0, np.iinfo(np.uint64).max, 1024, dtype=np.uint64, endpoint=True)
        if b < 64:
            x &= np.uint64((1 << b) - 1)
        x = (x.astype(T) + base[v]).astype(T)
        p = oracle.ffor(x, b, base[v]).view(np.uint8)
        chunks.append(p)
        offs.append(pos)
        pos += p.size
    return np.concatenate(chunks + [np.zeros(256, np.uint8)]), np.array(offs, np.uint64), bw, base


@pytest.mark.parametrize("w", [8, 16, 32, 64])
@pytest.mark.parametrize("order", [0, 1])
def test_emulated_rsum_and_delta(emu, w, order):
    T = TYPES[w]
    rng = np.random.default_rng(21 + w)
    n = 12
    L = 1024 // w
    lb = rng.integers(0, np.iinfo(np.uint64).max, n * L, dtype=np.uint64, endpoint=True).astype(T)
    packed, off, bw, base = batch(w, n, rng)
    got, st = run(emu, w, 2, order, packed, off, bw, base, lb, n)
    assert st == 0
    assert np.array_equal(got, oracle.delta_batch(packed, off, bw, base, lb, order == 1))


@pytest.mark.parametrize("order", [0, 1])
def test_emulated_delta_u64_small_widths(emu, order):
    """64-bit DELTA vectors of every bit width 0..27 with FOR bases below and at 2^26: the 32-bit running-sum
    path (widths up to 26, compile-time layouts up to 16) and the general one on either side of its bounds."""
    rng = np.random.default_rng(77)
    bw = np.array(list(range(28)) + [7, 16, 26], np.uint8)
    base = rng.integers(0, 1 << 26, bw.size, dtype=np.uint64)
    base[-3:] = [(1 << 26) - 1, 1 << 26, 0]
    lb = rng.integers(0, np.iinfo(np.uint64).max, bw.size * 16, dtype=np.uint64, endpoint=True)
    packed, off, _, _ = _rebuild(64, bw, base, rng)
    got, st = run(emu, 64, 2, order, packed, off, bw, base, lb, bw.size)
    assert st == 0
    assert np.array_equal(got, oracle.delta_batch(packed, off, bw, base, lb, order == 1))


@pytest.mark.parametrize("w", [8, 16, 32, 64])
def test_emulated_untranspose(emu, w):
    T = TYPES[w]
    rng = np.random.default_rng(31 + w)
    n = 6
    x = rng.integers(0, np.iinfo(np.uint64).max, n * 1024, dtype=np.uint64, endpoint=True).astype(T)
    got, st = run(emu, w, 0, 1, x.view(np.uint8), None, None, None, None, n)
    assert st == 0
    want = np.concatenate([oracle.untranspose_i(x[v * 1024:(v + 1) * 1024].copy()) for v in range(n)])
    assert np.array_equal(got, want)


def test_emulated_rejects_bit_width_above_type(emu):
    rng = np.random.default_rng(3)
    packed, off, bw, base = batch(32, 3, rng)
    bw[1] = 33
    _, st = run(emu, 32, 1, 0, packed, off, bw, base, None, 3)
    assert st & 2


@pytest.mark.parametrize("eid", [0, 1, 6, 7, 11, 16, 17, 22])
@pytest.mark.parametrize("order", [0, 1])
def test_emulated_reference_int64_pages(emu, col_golden, eid, order):
    """Reference-encoded int64 pages through the product's host page walker and the emulated warp decode."""
    page = np.ascontiguousarray(col_golden[f"i64_{eid}_page"])
    dic = np.ascontiguousarray(col_golden[f"i64_{eid}_dict"])
    want = col_golden[f"i64_{eid}_input"].view(np.uint64)
    n = want.size
    out = np.zeros(n, np.uint64)
    st = emu.emu_decode_page(P(page), ctypes.c_uint64(page.size), P(dic) if dic.size else None,
                             ctypes.c_uint64(dic.size), 64, order, P(out))
    assert st == 0
    if order == 1:
        assert np.array_equal(out, want)
    else:
        assert np.array_equal(out, np.concatenate([oracle.transpose_i(want[v * 1024:(v + 1) * 1024].copy())
                                                   for v in range(n // 1024)]))


def test_emulated_rejects_dictionary_code_out_of_range(emu, col_golden):
    page = np.ascontiguousarray(col_golden["i64_17_page"])
    dic = np.ascontiguousarray(col_golden["i64_17_dict"]).copy()
    # shrink the dictionary's entry count below the largest code in use
    dic[4:8] = np.frombuffer(np.uint32(3).tobytes(), np.uint8)
    dic[12:20] = np.frombuffer(np.uint64(3 * 8).tobytes(), np.uint8)
    out = np.zeros(3 * 1024, np.uint64)
    st = emu.emu_decode_page(P(page), ctypes.c_uint64(page.size), P(dic), ctypes.c_uint64(dic.size), 64, 1, P(out))
    assert st & 4


@pytest.mark.parametrize("eid", [2, 4, 5, 12, 13, 14])
@pytest.mark.parametrize("order", [0, 1])
def test_emulated_reference_patched_pages(emu, col_golden, eid, order):
    """Patched FFOR / DELTA pages of the reference (S / B / LL patches) through the device decode logic."""
    page = col_golden[f"i64patch_{eid}_page"]
    want = col_golden[f"i64patch_{eid}_input"]
    out = np.zeros(want.size, np.int64)
    st = emu.emu_decode_page(P(page), ctypes.c_uint64(page.size), None, ctypes.c_uint64(0), 64, order, P(out))
    assert st == 0, st
    if order == 1:
        assert np.array_equal(out, want)
    else:
        tw = np.concatenate([oracle.transpose_i(want.view(np.uint64)[v * 1024:(v + 1) * 1024]) for v in
                             range(want.size // 1024)]).view(np.int64)
        assert np.array_equal(out, tw)


def _emu_row(emu, twelve, sym, ln, data):
    data = np.ascontiguousarray(data, np.uint8)
    out = np.zeros(8 * data.size + 16, np.uint8)
    emu.emu_fsst_row.restype = ctypes.c_uint64
    n = emu.emu_fsst_row(int(twelve), P(sym), P(ln), P(data if data.size else np.zeros(1, np.uint8)),
                         ctypes.c_uint32(data.size), P(out))
    return out[:n].copy()


@pytest.mark.parametrize("eid", [13, 28])
def test_emulated_fsst_rows_match_oracle(emu, col_golden, eid):
    """The device FSST (pool id 13) and FSST12 (id 28) row decoders, compiled as host code: every row of the
    reference's page, and random byte strings of every length 0..40 (escapes, trailing lone FSST12 bytes,
    codes past the symbol count), decode as the oracle does; the length the lengths pass counts equals the
    bytes written."""
    from oracle import pages

    twelve = eid == 28
    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    table = oracle.fsst12_decode_table if twelve else oracle.fsst_decode_table
    dec = oracle.fsst12_decode if twelve else oracle.fsst_decode
    _, sym, ln = table(dic[8:])
    pg = pages.parse_page(page)
    for v in range(pg.vec_c):
        data = pg.vector_slice(v, 0)
        ends = oracle.untranspose_i(np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32).copy())
        start = 0
        for i in range(1024):
            row = data[start:ends[i]]
            assert np.array_equal(_emu_row(emu, twelve, sym, ln, row), dec(sym, ln, row)), (v, i)
            start = ends[i]
    rng = np.random.default_rng(eid)
    for n in list(range(41)) * 20:
        row = rng.integers(0, 256, n, dtype=np.uint8)
        assert np.array_equal(_emu_row(emu, twelve, sym, ln, row), dec(sym, ln, row)), n


@pytest.mark.parametrize("d0", [0, 1, 2, 3, 6])
def test_emulated_fsst_whole_word_rows(emu, col_golden, d0):
    """fsst_put_row (the FSST materialising pass's row writer) on a window full of garbage: a vector's rows
    written one after another from byte d0 reproduce the oracle's bytes exactly, nothing before d0 in the first
    word but zeros, and the last word zero past the end (the next rows OR into it)."""
    from oracle import pages

    page, dic = col_golden["str_13_page"], col_golden["str_13_dict"]
    _, sym, ln = oracle.fsst_decode_table(dic[8:])
    pg = pages.parse_page(page)
    rng = np.random.default_rng(d0)
    for v in range(pg.vec_c):
        data = np.ascontiguousarray(pg.vector_slice(v, 0))
        ends = oracle.untranspose_i(np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32).copy())
        starts = np.concatenate([[0], ends[:-1]])
        rows = [oracle.fsst_decode(sym, ln, data[s:e]) for s, e in zip(starts, ends)]
        # plus rows with escapes, an escape at the very end, and empty rows
        extra = [np.array([255, 65, 1, 255], np.uint8), np.zeros(0, np.uint8), np.array([255], np.uint8)]
        comp = np.concatenate([data[s:e] for s, e in zip(starts, ends)] + extra)
        lens = np.concatenate([np.asarray(ends) - np.asarray(starts), [e.size for e in extra]]).astype(np.uint64)
        coffs = np.zeros(lens.size + 1, np.uint64)
        coffs[1:] = np.cumsum(lens)
        rows += [oracle.fsst_decode(sym, ln, e) for e in extra]
        want = np.concatenate(rows)
        win = rng.integers(0, 1 << 32, (d0 + want.size) // 4 + 64, dtype=np.uint64).astype(np.uint32)
        emu.emu_fsst_put_rows.restype = ctypes.c_uint64
        n = emu.emu_fsst_put_rows(P(sym), P(ln), P(comp), P(coffs), ctypes.c_uint32(lens.size), ctypes.c_uint32(d0),
                                  P(win))
        got = win.view(np.uint8)
        assert n == want.size
        assert np.array_equal(got[d0:d0 + n], want), v
        assert not got[(d0 // 4) * 4:d0].any()
        end = d0 + n
        assert not got[end:(end + 3) // 4 * 4].any()


@pytest.mark.parametrize("d0", [0, 1, 2, 3, 5])
def test_emulated_put_row_window_protocol(emu, d0):
    """put_row (the DICT / BYTE_ARR materialising pass's row writer) on a window full of garbage: rows of 0..9
    bytes (many empty or shorter than a word) and some long ones, from any source offset, written one after
    another from byte d0 reproduce the source bytes, zeros before d0 in the first word and past the end."""
    rng = np.random.default_rng(100 + d0)
    src = rng.integers(0, 256, 1 << 14, dtype=np.uint8)
    n = 2000
    lens = rng.choice([0, 1, 2, 3, 4, 5, 7, 9, 40, 300], n, p=[.2, .15, .15, .1, .1, .1, .05, .05, .05, .05])
    lens = lens.astype(np.uint32)
    starts = rng.integers(0, src.size - 301, n).astype(np.uint32)
    want = np.concatenate([src[s:s + l] for s, l in zip(starts, lens)])
    win = rng.integers(0, 1 << 32, (d0 + want.size) // 4 + 64, dtype=np.uint64).astype(np.uint32)
    emu.emu_put_rows.restype = ctypes.c_uint64
    got_n = emu.emu_put_rows(P(src.view(np.uint32)), P(starts), P(lens), ctypes.c_uint32(n), ctypes.c_uint32(d0),
                             P(win))
    got = win.view(np.uint8)
    assert got_n == want.size
    assert np.array_equal(got[d0:d0 + want.size], want)
    assert not got[(d0 // 4) * 4:d0].any()
    end = d0 + want.size
    assert not got[end:(end + 3) // 4 * 4].any()


def _aligned(n, fill, align=16):
    raw = np.full(n + align, fill, np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n]


def _emu_stream(emu, fsst, sym, ln, ends, comp, shift, vbase):
    """stream_vector (both passes) on an emulated warp: comp placed at byte `shift` of a 16-byte aligned buffer,
    output at byte vbase of a sentinel-filled buffer.  Returns (lengths total, offsets, output buffer, bad)."""
    buf = _aligned(comp.size + shift + 16, 0x5A)
    buf[shift:shift + comp.size] = comp
    ends = np.ascontiguousarray(ends, np.uint32)
    cap = vbase + 8 * max(comp.size, 1) + 64
    out = _aligned(cap, 0xEE)
    offs = np.zeros(1025, np.uint32)
    tot_len = ctypes.c_uint64()
    bad = ctypes.c_int()
    emu.emu_stream_vector.restype = ctypes.c_uint64
    tot = emu.emu_stream_vector(int(fsst), P(sym), P(ln), P(ends), ctypes.c_void_p(buf.ctypes.data + shift),
                                ctypes.c_uint32(comp.size), ctypes.c_uint64(vbase), P(offs), P(out),
                                ctypes.byref(tot_len), ctypes.byref(bad))
    return tot, tot_len.value, offs, out, bad.value


def _check_stream(emu, fsst, sym, ln, rows, shift, vbase):
    comp = np.concatenate(rows) if rows else np.zeros(0, np.uint8)
    ends = np.cumsum([r.size for r in rows]).astype(np.uint32)
    dec = [oracle.fsst_decode(sym, ln, r) if fsst else r for r in rows]
    want = np.concatenate(dec)
    want_off = vbase + np.concatenate([[0], np.cumsum([d.size for d in dec])])
    tot, tot_len, offs, out, bad = _emu_stream(emu, fsst, sym, ln, ends, comp.astype(np.uint8), shift, vbase)
    assert bad == 0
    assert tot == tot_len == want.size
    assert np.array_equal(offs, want_off.astype(np.uint32))
    assert np.array_equal(out[vbase:vbase + want.size], want)
    assert (out[:vbase] == 0xEE).all() and (out[vbase + want.size:] == 0xEE).all()


@pytest.mark.parametrize("shift,vbase", [(0, 0), (1, 5), (2, 16), (3, 13)])
def test_emulated_stream_decode_reference_vectors(emu, col_golden, shift, vbase):
    """The code-parallel FSST column decoder (stream_vector, both passes) on every vector of the reference's FSST
    page and on the same rows as a BYTE_ARR vector: offsets and bytes equal the oracle's row-by-row decode, at
    any source alignment and output position, and nothing outside the vector's output range is written."""
    from oracle import pages

    page, dic = col_golden["str_13_page"], col_golden["str_13_dict"]
    _, sym, ln = oracle.fsst_decode_table(dic[8:])
    pg = pages.parse_page(page)
    for v in range(pg.vec_c):
        data = np.ascontiguousarray(pg.vector_slice(v, 0))
        ends = oracle.untranspose_i(np.frombuffer(pg.vector_slice(v, 1, 4096).tobytes(), np.uint32).copy())
        starts = np.concatenate([[0], ends[:-1]])
        rows = [data[s:e] for s, e in zip(starts, ends)]
        _check_stream(emu, True, sym, ln, rows, shift, vbase)
        _check_stream(emu, False, sym, ln, rows, shift, vbase)


@pytest.mark.parametrize("seed", range(6))
def test_emulated_stream_decode_escapes_and_ragged_rows(emu, col_golden, seed):
    """Rows full of escapes (runs of 255, an escape as a row's last byte, a literal 255), empty rows, rows of
    one byte and rows of hundreds, so that chunk boundaries fall inside escapes and rows: the stream decoder
    equals the oracle's row decoder."""
    dic = col_golden["str_13_dict"]
    _, sym, ln = oracle.fsst_decode_table(dic[8:])
    rng = np.random.default_rng(1000 + seed)
    lens = rng.choice([0, 1, 2, 3, 4, 7, 12, 40, 300], 1024, p=[.2, .1, .1, .1, .1, .1, .1, .15, .05])
    p255 = [0.0, 0.05, 0.3, 0.7][seed % 4]
    rows = []
    for n in lens:
        r = rng.integers(0, 256, n, dtype=np.uint8)
        r[rng.random(n) < p255] = 255
        rows.append(r)
    _check_stream(emu, True, sym, ln, rows, seed % 4, (7 * seed) % 17)
    _check_stream(emu, False, sym, ln, rows, seed % 4, (7 * seed) % 17)


def test_emulated_stream_decode_refuses_bad_rows(emu, col_golden):
    """Row ends that decrease, or end past the vector's bytes: the vector is refused (every row empty, total 0)
    by both passes."""
    dic = col_golden["str_13_dict"]
    _, sym, ln = oracle.fsst_decode_table(dic[8:])
    comp = np.arange(200, dtype=np.uint8)
    for ends in (np.r_[np.arange(1, 101), np.full(924, 50)], np.r_[np.arange(1, 1024), [201]]):
        tot, tot_len, offs, out, bad = _emu_stream(emu, True, sym, ln, ends.astype(np.uint32), comp, 1, 3)
        assert bad == 3 and tot == tot_len == 0
        assert (offs == 3).all()


@pytest.mark.parametrize("seed", range(8))
def test_emulated_fsst_plain_total(emu, col_golden, seed):
    """The single-pass FSST kernel's total of a vector without escapes (fsst_plain_total): the sum of its codes'
    symbol lengths, at every source alignment and length (empty, shorter than a word, ragged ends); any escape
    inside [0, L) is reported, and so is nothing outside it except the documented false alarm (a 254 right above
    an out-of-range 255 in the same word), which is always on the safe side."""
    dic = col_golden["str_13_dict"]
    _, sym, ln = oracle.fsst_decode_table(dic[8:])
    lens = np.asarray(ln, np.int64).copy()
    lens[255] = 0
    rng = np.random.default_rng(77 + seed)
    for L in [0, 1, 2, 3, 4, 5, 7, 127, 128, 129, 1000, 4099, int(rng.integers(1, 20000))]:
        for shift in range(4):
            buf = _aligned(L + 16, 0)
            # the bytes around the range: 255 everywhere outside (the worst case for the zero-byte test)
            buf[:] = 255
            body = rng.integers(0, 255, L, dtype=np.uint8)  # no escape
            buf[shift:shift + L] = body
            tot = ctypes.c_uint32()
            plain = emu.emu_fsst_plain_total(P(np.ascontiguousarray(ln, np.uint8)), ctypes.c_void_p(buf.ctypes.data + shift),
                                             ctypes.c_uint32(L), ctypes.byref(tot))
            # a false alarm needs a 254 as the range's first byte (right above the 255 before it)
            false_alarm_possible = L > 0 and shift > 0 and body[0] == 254
            if not false_alarm_possible:
                assert plain == 1, (L, shift)
            if plain:
                assert tot.value == int(lens[body].sum()), (L, shift)
            if L:
                # one escape anywhere inside the range is always seen
                pos = int(rng.integers(0, L))
                buf[shift + pos] = 255
                plain = emu.emu_fsst_plain_total(P(np.ascontiguousarray(ln, np.uint8)),
                                                 ctypes.c_void_p(buf.ctypes.data + shift), ctypes.c_uint32(L),
                                                 ctypes.byref(tot))
                assert plain == 0, (L, shift, pos)
