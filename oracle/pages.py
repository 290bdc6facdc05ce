"""TEST INFRASTRUCTURE — restatement of the reference's page framing, used as the checker for the GPU
column decoders.

Page bytes (src/cor/eng/compressor.cpp:68-86, src/cor/lyt/page/page.cpp:63-139,
src/cor/lyt/page/entry_point.cpp:21-41, include/fls/cor/lyt/page/page_hdr.hpp:8-15):
    [PageHdr: exp_t u8, var u8, reserved u16, vec_c u16, pad u16]
    [arr_c x u32: absolute offset of each buffer]
    [(vec_c - 1) x arr_c x u32: per-vector entry points; vector 0 starts at 0 in every buffer]
    [buffer 0] ... [buffer arr_c - 1]
"""
import struct

import numpy as np

from . import oracle

# (exp_t, var) -> number of buffers, from the compress RPN tables (des_buf_c) of include/fls/cor/exp/*/*_exp.hpp
ARR_C = {
    (2, 1): 1,  # UNCOMPRESSED
    (3, 1): 2,  # BYTE_ARR: bytes, end offsets
    (4, 1): 3,  # FFOR NO_PATCH: bw, base, packed
    (5, 1): 4,  # DELTA NO_PATCH: lane bases, bw, base, packed
    (4, 2): 5,  # FFOR LL_PATCH: exceptions, (exc_c, first position), bw, base, packed
    (4, 3): 5,  # FFOR S_PATCH: exceptions, (exc_c, positions), bw, base, packed
    (4, 4): 5,  # FFOR B_PATCH: exceptions, 1024-bit position bitmap, bw, base, packed
    (4, 5): 5,  # FFOR S_PATCH_REC: as S_PATCH, exceptions rec-compressed
    (5, 2): 6,  # DELTA LL_PATCH: lane bases, then as FFOR LL_PATCH
    (5, 3): 6,  # DELTA S_PATCH
    (5, 4): 6,  # DELTA B_PATCH
    (5, 5): 6,  # DELTA B_PATCH_REC: as B_PATCH, exceptions rec-compressed
    (6, 1): 2,  # RLE UNCOMPRESSED: run values, u16 index
    (6, 2): 5,  # RLE DELTA_NO_PATCH: run values, lane bases, bw, base, packed (u16 index)
    (6, 3): 2,  # RLE UNCOMPRESSED_REC: run values rec-compressed, raw u16 index
    (6, 4): 5,  # RLE DELTA_NO_PATCH_REC: as above, run values rec-compressed
    (6, 5): 5,  # RLE DELTA_NO_PATCH_REC2: run values and the u16 rsum bases rec-compressed (rle_exp.hpp:99-110)
    (7, 1): 2,  # FSST: bytes, end offsets
    (7, 2): 5,  # FSST DELTA_NO_PATCH: bytes, lane bases, bw, base, packed (u32 end offsets)
    (20, 1): 2,  # FSST12: bytes, end offsets (src/cor/lyt/vec.cpp:208-248)
    (20, 2): 5,  # FSST12 DELTA_NO_PATCH: as FSST DELTA_NO_PATCH
    (8, 1): 1,  # DICT UNCOMPRESSED: u32 codes
    (8, 2): 3,  # DICT FFOR_NO_PATCH
    (8, 7): 4,  # DICT DELTA_NO_PATCH
    (8, 3): 5,  # DICT FFOR_LL_PATCH: u32 codes as FFOR LL_PATCH (dict_exp.hpp:62-75)
    (8, 4): 5,  # DICT FFOR_S_PATCH
    (8, 5): 5,  # DICT FFOR_B_PATCH
    (8, 6): 5,  # DICT FFOR_S_PATCH_REC
    (8, 8): 6,  # DICT DELTA_LL_PATCH: u32 codes as DELTA LL_PATCH
    (8, 9): 6,  # DICT DELTA_S_PATCH
    (8, 10): 6,  # DICT DELTA_B_PATCH
    (8, 11): 6,  # DICT DELTA_B_PATCH_REC
    (11, 1): 2,  # DICT_RLE UNCOMPRESSED: u32 code runs, u16 index
    (11, 2): 5,  # DICT_RLE DELTA_NO_PATCH
    (11, 3): 2,  # DICT_RLE UNCOMPRESSED_REC
    (11, 4): 5,  # DICT_RLE DELTA_NO_PATCH_REC
}
# DICT_FRQ (exp_t 9) pages are DICT pages (dict_frq_exp derives dict_exp, dict_exp.hpp:208): same variants and
# buffers, the dictionary built in frequency order
ARR_C.update({(9, var): n for (et, var), n in list(ARR_C.items()) if et == 8})


class Page:
    def __init__(self, b):
        self.b = np.ascontiguousarray(b, np.uint8)
        self.exp_t, self.var, _, self.vec_c, _ = struct.unpack("<BBHHH", self.b[:8].tobytes())
        self.arr_c = ARR_C[(self.exp_t, self.var)]
        self.off = np.frombuffer(self.b[8:8 + 4 * self.arr_c].tobytes(), np.uint32).astype(np.int64)
        n_ep = (self.vec_c - 1) * self.arr_c
        s = 8 + 4 * self.arr_c
        self.ep = np.frombuffer(self.b[s:s + 4 * n_ep].tobytes(), np.uint32).astype(np.int64).reshape(-1, self.arr_c)
        ends = list(self.off[1:]) + [self.b.size]
        self.buf_size = [int(ends[i] - self.off[i]) for i in range(self.arr_c)]

    def ep_of(self, v, i):
        return 0 if v == 0 else int(self.ep[v - 1, i])

    def vector_slice(self, v, i, size=None):
        start = self.ep_of(v, i)
        end = start + size if size is not None else (self.ep_of(v + 1, i) if v + 1 < self.vec_c else self.buf_size[i])
        return self.b[self.off[i] + start:self.off[i] + end]


def parse_page(b):
    return Page(b)


def _le(b, dtype):
    return np.frombuffer(np.ascontiguousarray(b).tobytes(), dtype)


def rec_buffer(b, elem=np.uint64):
    """HzlDeCmp::decompress_buf (src/cor/eng/hzl_de_cmp.cpp:28-77): a chain of blocks, each a rec_hdr
    {bw u8, pad u8, exc_c u16, base[8]}; bw = 255 ends the chain with base = byte count of raw bytes, any other
    bw is an FFOR block of 1024 values of the buffer's element type followed by its exceptions
    (hzl_cmp.cpp:43-127 writes them): uint64 for 64-bit values and dictionary entries, idx_t = uint32
    (include/fls/common/alias.hpp:17) for DICT_RLE run codes.  Returns (decoded bytes, consumed bytes)."""
    out = []
    pos = 0
    while True:
        bw = int(b[pos])
        exc_c = int(struct.unpack("<H", b[pos + 2:pos + 4].tobytes())[0])
        base_raw = b[pos + 4:pos + 12]
        pos += 12
        if bw == 255:
            sz = int(struct.unpack("<Q", base_raw.tobytes())[0])
            out.append(b[pos:pos + sz])
            pos += sz
            return np.concatenate(out) if out else np.zeros(0, np.uint8), pos
        # an FFOR block of 1024 values (generated unffor keeps positions), then exc_c u16 positions and exc_c
        # values patched over the unpacked ones
        et = np.dtype(elem)
        base = np.frombuffer(base_raw.tobytes()[:et.itemsize], et)[0]
        packed = np.frombuffer(b[pos:pos + bw * 128].tobytes(), et)
        vals = oracle.unffor(packed, bw, base, et.type)
        pos += bw * 128
        exc_pos = np.frombuffer(b[pos:pos + 2 * exc_c].tobytes(), np.uint16)
        pos += 2 * exc_c
        exc_val = np.frombuffer(b[pos:pos + et.itemsize * exc_c].tobytes(), et)
        pos += et.itemsize * exc_c
        vals[exc_pos.astype(np.int64)] = exc_val
        out.append(np.frombuffer(vals.tobytes(), np.uint8))


STREAM_W = {2: None, 4: None, 5: None}


def _stream(pg, v, first, ws, enc, T, lane_bases=None):
    """Decode one 1024-value stream of width ws stored from buffer index `first` on; returns transposed.
    lane_bases: a DELTA stream's decoded rsum bases (rec-compressed buffer), indexed by the entry points."""
    if enc == "raw":
        return _le(pg.vector_slice(v, first, 128 * ws), T).copy()
    if enc == "ffor":
        bw = int(pg.vector_slice(v, first, 1)[0])
        base = _le(pg.vector_slice(v, first + 1, ws // 8), T)[0]
        packed = _le(pg.vector_slice(v, first + 2, bw * 128), T)
        return oracle.unffor(packed, bw, base, T)
    if lane_bases is not None:
        lb = _le(lane_bases[pg.ep_of(v, first):pg.ep_of(v, first) + 128], T).copy()
    else:
        lb = _le(pg.vector_slice(v, first, 128), T).copy()
    bw = int(pg.vector_slice(v, first + 1, 1)[0])
    base = _le(pg.vector_slice(v, first + 2, ws // 8), T)[0]
    packed = _le(pg.vector_slice(v, first + 3, bw * 128), T)
    return oracle.rsum(oracle.unffor(packed, bw, base, T), lb)


# (exp_t, var) of the patched FFOR / DELTA variants -> patch kind, exceptions rec-compressed
PATCHED = {(4, 2): ("ll", False), (4, 3): ("s", False), (4, 4): ("b", False), (4, 5): ("s", True),
           (5, 2): ("ll", False), (5, 3): ("s", False), (5, 4): ("b", False), (5, 5): ("b", True)}
# DICT with patched u32 codes (dict_exp.hpp:31-41, FFOR_* and DELTA_* variants) -> patch kind, rec exceptions,
# delta-coded
DICT_PATCHED = {(8, 3): ("ll", False, False), (8, 4): ("s", False, False), (8, 5): ("b", False, False),
                (8, 6): ("s", True, False), (8, 8): ("ll", False, True), (8, 9): ("s", False, True),
                (8, 10): ("b", False, True), (8, 11): ("b", True, True)}


def _patch(vals, kind, exc_bytes, side, base, T):
    """One vector's patch over its unpacked values (transposed positions), after unffor:
    s  (src/cor/prm/patch/s_patch/s_patch_decompress.cpp): side = exc_c u16, then exc_c u16 positions;
    b  (b_patch_decompress.cpp, patch.cpp:71-83): side = 16 uint64 bitmap words, exceptions in bit order;
    ll (ll_patch_decompress.cpp): side = exc_c u16, first position u16; the packed value at an exception is
       the distance to the next one minus one (offset = out[cur] - base + 1 in the type)."""
    T = np.dtype(T)
    exc = np.frombuffer(exc_bytes.tobytes(), T)
    if kind == "s":
        sel = np.frombuffer(side.tobytes()[: 2 * (1 + int(np.frombuffer(side.tobytes()[:2], np.uint16)[0]))], np.uint16)
        c = int(sel[0])
        vals[sel[1:1 + c].astype(np.int64)] = exc[:c]
    elif kind == "b":
        pos = np.flatnonzero(np.unpackbits(np.asarray(side[:128], np.uint8), bitorder="little"))
        vals[pos] = exc[:pos.size]
    else:
        c, first = struct.unpack("<HH", side[:4].tobytes())
        mask = (1 << (T.itemsize * 8)) - 1
        cur = int(first)
        for i in range(c):
            off = (int(vals[cur]) - int(base) + 1) & mask
            vals[cur] = exc[i]
            cur = (cur + off) & mask
    return vals


def _patched_stream(pg, v, T, rec_exc, kind=None, delta=None):
    """Unpacked, patched and (DELTA) rsum-ed values of vector v of a patched FFOR / DELTA page (transposed);
    kind / delta given for the DICT pages' patched code streams."""
    if kind is None:
        kind, _ = PATCHED[(pg.exp_t, pg.var)]
        delta = pg.exp_t == 5
    first = 1 if delta else 0
    ws = np.dtype(T).itemsize * 8
    bw = int(pg.vector_slice(v, first + 2, 1)[0])
    base = _le(pg.vector_slice(v, first + 3, ws // 8), T)[0]
    vals = oracle.unffor(_le(pg.vector_slice(v, first + 4, bw * 128), T), bw, base, T)
    if rec_exc is not None:
        end = pg.ep_of(v + 1, first) if v + 1 < pg.vec_c else rec_exc.size
        exc = rec_exc[pg.ep_of(v, first):end]
    else:
        exc = pg.vector_slice(v, first)
    vals = _patch(vals, kind, exc, pg.vector_slice(v, first + 1), base, T)
    if delta:
        vals = oracle.rsum(vals, _le(pg.vector_slice(v, 0, 128), T).copy())
    return vals


def decode_int(page, dict_bytes=None, value_dtype=np.uint64, raw_dict=False):
    """Materialised (original-order) values of an integer page, as assert_eq.hpp:50-400 reconstructs them.
    raw_dict: the dictionary page holds its entry_c values raw after dict_hdr_t, as a double column's does
    (TDic<dbl_pt>::Decompress, src/cor/lyt/dic/dic.cpp:150-153); decode a double page with value_dtype uint64
    (the values' bit patterns)."""
    pg = parse_page(page)
    VT = np.dtype(value_dtype)
    W = VT.itemsize * 8
    dic = None
    if dict_bytes is not None and len(dict_bytes) > 8:
        db = np.asarray(dict_bytes, np.uint8)
        if raw_dict:
            entry_c = int(np.frombuffer(db[4:8].tobytes(), np.uint32)[0])
            dic = _le(db[8:8 + entry_c * VT.itemsize], VT)
        else:
            dic = _le(rec_buffer(db[8:], np.uint64 if W == 64 else np.uint32)[0], VT)
    out = np.empty(pg.vec_c * 1024, VT)
    et, var = (8 if pg.exp_t == 9 else pg.exp_t), pg.var
    rec_vals = None
    rec_lb = None
    if (et, var) == (6, 5):
        rec_lb = rec_buffer(pg.b[pg.off[1]:pg.off[1] + pg.buf_size[1]], np.uint16)[0]
    if et in (6, 11) and var in (3, 4) or (et, var) == (6, 5):
        # UNCOMPRESSED_REC / DELTA_NO_PATCH_REC: buffer 0 (run values / run codes) is one rec buffer; entry
        # points index its decoded bytes
        ve = np.uint32 if et == 11 or W == 32 else np.uint64
        rec_vals = rec_buffer(pg.b[pg.off[0]:pg.off[0] + pg.buf_size[0]], ve)[0]
    rec_exc = None
    if (et, var) in PATCHED and PATCHED[(et, var)][1]:
        b = 1 if et == 5 else 0
        rec_exc = rec_buffer(pg.b[pg.off[b]:pg.off[b] + pg.buf_size[b]], np.uint64 if W == 64 else np.uint32)[0]
    if (et, var) in DICT_PATCHED and DICT_PATCHED[(et, var)][1]:
        b = 1 if DICT_PATCHED[(et, var)][2] else 0
        rec_exc = rec_buffer(pg.b[pg.off[b]:pg.off[b] + pg.buf_size[b]], np.uint32)[0]  # the codes' type
    for v in range(pg.vec_c):
        if (et, var) in PATCHED:
            tr = _patched_stream(pg, v, VT, rec_exc)
        elif et == 2:
            tr = _stream(pg, v, 0, W, "raw", VT)
        elif et == 4:
            tr = _stream(pg, v, 0, W, "ffor", VT)
        elif et == 5:
            tr = _stream(pg, v, 0, W, "delta", VT)
        elif et in (6, 11):
            if rec_vals is not None:
                end = pg.ep_of(v + 1, 0) if v + 1 < pg.vec_c else rec_vals.size
                vals_buf = rec_vals[pg.ep_of(v, 0):end]
            else:
                vals_buf = pg.vector_slice(v, 0)
            vt = VT if et == 6 else np.dtype(np.uint32)
            vals = _le(vals_buf, vt)
            idx = _stream(pg, v, 1, 16, "raw" if var in (1, 3) else "delta", np.uint16, rec_lb)
            tr = vals[idx.astype(np.int64)]
            if et == 11:
                tr = dic[tr.astype(np.int64)]
        elif (et, var) in DICT_PATCHED:
            kind, _, delta = DICT_PATCHED[(et, var)]
            codes = _patched_stream(pg, v, np.uint32, rec_exc, kind, delta)
            tr = dic[codes.astype(np.int64)]
        elif et == 8:
            enc = {1: "raw", 2: "ffor", 7: "delta"}[var]
            codes = _stream(pg, v, 0, 32, enc, np.uint32)
            tr = dic[codes.astype(np.int64)]
        else:
            raise NotImplementedError((et, var))
        out[v * 1024:(v + 1) * 1024] = oracle.untranspose_i(np.ascontiguousarray(tr.astype(VT)))
    return out
