"""Generates the golden fixtures in this folder from the reference (cwida/FastLanes).

Run in a container that has the reference checked out and the reference oracle built
(``make -C oracle ref``)::

    python tests/golden/make_golden.py [REFERENCE_ROOT]

primitives.npz
    * every ``rand_arr_*`` golden vector of the reference's generated primitive tests
      (primitives/fls_generated/fallback/scalar_aav_uf1/fallback_scalar_aav_1024_uf1_{unpack,unffor}_helper.hpp),
      with the packed words the reference's own ``pack`` (base 0, as in ..._unpack_test.cpp) and ``ffor``
      (base 10, as in ..._unffor_test.cpp:44-52) produce for them (the words themselves for 8/16-bit types,
      a SHA-256 of the words for 32/64-bit types);
    * the ``range_ow*`` vectors of ..._{rsum,transpose,untranspose}_helper.hpp with the reference's
      transpose_i / untranspose_i / unrsum / rsum outputs.
columns.npz
    * small seeded columns encoded by the reference's column encoder (ExpColEncoder, verify on) for the
      expressions on the decode path, with the reference decoder's materialised output.

The reference's FSST table export leaves its last byte uninitialised for some tables (str_13_dict differs
in that byte from run to run); a regenerated file keeps the committed bytes of every existing array.
"""
import ctypes
import hashlib
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FLS_REFERENCE", "/root/reference")
PRIM = os.path.join(REF, "primitives/fls_generated/fallback/scalar_aav_uf1")
TYPES = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}

# Expressions of src/cor/exp_pool.cpp on the integer / string decode path.
I64_IDS = [0, 1, 6, 7, 11, 16, 17, 22, 27]
# The same expressions on columns large enough that the reference's rec compression (hzl_cmp.cpp:43-127)
# writes FFOR blocks with exceptions, not only a raw tail: dictionaries of ~3000 entries, ~2000 runs.
REC_IDS = [8, 9, 10, 16, 17, 22, 27]
# Patched FFOR / DELTA (src/cor/prm/patch/*) on columns with ~3% outliers / outlying gaps.
PATCH_IDS = [2, 3, 4, 5, 12, 13, 14, 15]
# DICT with patched FFOR / DELTA codes (dict_exp.hpp FFOR_*_PATCH, DELTA_*_PATCH): ~97 % of the rows take one of
# 16 values, the rest ~2000 rare ones, so the rare values' codes (assigned in first-occurrence order) are the
# patches' exceptions.
DPATCH_IDS = [18, 19, 20, 21, 22, 23, 24, 25, 26]
# DICT_FRQ (exp_t 9): the DICT expressions (dict_frq_exp derives dict_exp, dict_exp.hpp:208) over a dictionary
# built in frequency order; the same columns as the patched DICT ones.
FRQ_IDS = [28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38]
# The double pool (src/cor/exp_pool.cpp:104-137) through every expression the reference encodes and decodes for
# doubles: UNCOMPRESSED, RLE without rec buffers, DICT (a raw double dictionary, src/cor/lyt/dic/dic.cpp:150-153)
# with every code variant, DICT_RLE and DICT_FRQ.  Its RLE _REC variants (8-10) have no double form in the
# reference (THzlDeCmp<double>::decompress_buf aborts) and ALP (1) needs the ALP library, absent here.
F64_IDS = [0, 6, 7] + list(range(16, 39))
STR_IDS = [0, 2, 3, 8, 13, 14, 15, 16]
# the rest of the string pool (src/cor/exp_pool.cpp:70-99): BYTE_ARR DELTA_NO_PATCH (1), DICT with patched codes
# (4-7, 9-12), DICT_FRQ (17-27) and FSST12 (28, 29); the dictionary ones on columns whose rare strings' codes
# become the patches' exceptions
STR_MORE_IDS = [1, 4, 5, 6, 7, 9, 10, 11, 12] + list(range(17, 28)) + [28, 29]  # 28, 29: FSST12


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def parse_arrays(path):
    txt = open(path).read()
    out = {}
    for name, body in re.findall(r"(\w+)\[1024\] = \{([^}]*)\}", txt):
        out[name] = [int(x.strip().rstrip("UL")) for x in body.split(",") if x.strip()]
    return out


def primitives(ref):
    res = {}
    for kind, helper, base in (("unpack", "unpack", 0), ("unffor", "unffor", 10)):
        arrs = parse_arrays(os.path.join(PRIM, f"fallback_scalar_aav_1024_uf1_{helper}_helper.hpp"))
        for name, vals in arrs.items():
            m = re.match(r"rand_arr_\d+_b(\d+)_w(\d+)_arr", name)
            bw, w = int(m.group(1)), int(m.group(2))
            T = TYPES[w]
            x = np.array(vals, dtype=np.uint64).astype(T)
            packed = np.zeros(1024, T)
            if kind == "unpack":
                getattr(ref, f"ref_pack_u{w}")(ptr(x), ptr(packed), ctypes.c_uint8(bw))
            else:
                b = np.array([base], T)
                getattr(ref, f"ref_ffor_u{w}")(ptr(x), ptr(packed), ctypes.c_uint8(bw), ptr(b))
            key = f"{kind}_w{w}_b{bw}"
            words = packed[: bw * (1024 // w)].copy()
            res[key + "_in"] = x
            # the packed words pin the bit layout; wide ones are kept as a digest to keep the fixture small
            if w <= 16:
                res[key + "_packed"] = words
            res[key + "_packed_sha256"] = np.frombuffer(hashlib.sha256(words.tobytes()).digest(), np.uint8)
    for w, T in TYPES.items():
        arrs = parse_arrays(os.path.join(PRIM, "fallback_scalar_aav_1024_uf1_rsum_helper.hpp"))
        rng = np.array(arrs[f"range_ow{w}"], dtype=np.uint64).astype(T)
        tr = np.zeros(1024, T)
        un = np.zeros(1024, T)
        getattr(ref, f"ref_transpose_i_u{w}")(ptr(rng), ptr(tr))
        getattr(ref, f"ref_untranspose_i_u{w}")(ptr(rng), ptr(un))
        padded = np.concatenate([tr, np.zeros(1024, T)])  # the generated unrsum reads one row past the vector
        delta = np.zeros(1024, T)
        getattr(ref, f"ref_unrsum_u{w}")(ptr(padded), ptr(delta))
        lanes = 1024 // w
        bases = tr[:lanes].copy()
        back = np.zeros(1024, T)
        getattr(ref, f"ref_rsum_u{w}")(ptr(delta), ptr(back), ptr(bases))
        res[f"range_w{w}"] = rng
        res[f"range_w{w}_transposed"] = tr
        res[f"range_w{w}_untransposed"] = un
        res[f"range_w{w}_delta"] = delta
        res[f"range_w{w}_bases"] = bases
        res[f"range_w{w}_rsum"] = back
    return res


def i64_column(eid, rng, n):
    if eid in (6, 7):
        runs = rng.geometric(1 / 8, n)
        vals = rng.integers(0, 10**6, runs.size)
        return np.repeat(vals, runs)[:n].astype(np.int64)
    if eid == 11:
        return (1_600_000_000_000_000_000 + np.cumsum(rng.geometric(0.1, n))).astype(np.int64)
    if eid in (16, 17, 22):
        return (rng.integers(0, 300, n) * 7919 - 5000).astype(np.int64)
    if eid == 27:
        runs = rng.geometric(1 / 6, n)
        return np.repeat(rng.integers(0, 40, runs.size) * 1000 + 3, runs)[:n].astype(np.int64)
    if eid == 1:
        return (rng.integers(0, 1 << 13, n) - 4000).astype(np.int64)
    return rng.integers(-(1 << 62), 1 << 62, n).astype(np.int64)


def rec_column(eid, rng, n):
    if eid in (16, 17, 22):
        return (rng.integers(0, 3000, n) * 7919 - 5000).astype(np.int64)
    runs = rng.geometric(1 / 2, n)
    if eid == 27:
        return np.repeat(rng.integers(0, 40, runs.size) * 1000 + 3, runs)[:n].astype(np.int64)
    # a few far-off run values become the FFOR blocks' exceptions
    vals = rng.integers(0, 10**6, runs.size)
    vals[rng.integers(0, runs.size, 8)] = rng.integers(-(1 << 60), 1 << 60, 8)
    return np.repeat(vals, runs)[:n].astype(np.int64)


def patch_column(eid, rng, n):
    if eid <= 5:
        x = (rng.integers(0, 1 << 10, n) + 5000).astype(np.int64)
        out = rng.random(n) < 0.03
        x[out] = rng.integers(-(1 << 40), 1 << 40, out.sum())
        return x
    gaps = rng.geometric(0.1, n)
    big = rng.random(n) < 0.03
    gaps[big] = rng.integers(1 << 20, 1 << 30, big.sum())
    return (1_600_000_000_000_000_000 + np.cumsum(gaps)).astype(np.int64)


def dpatch_column(eid, rng, n):
    common = rng.integers(-(1 << 40), 1 << 40, 16)
    rare = rng.integers(-(1 << 40), 1 << 40, 4000)
    x = common[rng.integers(0, 16, n)]
    out = rng.random(n) < 0.03
    x[out] = rare[rng.integers(0, rare.size, out.sum())]
    return x.astype(np.int64)


def f64_column(eid, rng, n):
    """Doubles with the equality structure of the int64 columns of the same expression (x / 4 is exact and
    one-to-one below 2^53); UNCOMPRESSED also carries infinities, NaNs, signed zeros and subnormals."""
    if eid == 0:
        x = rng.normal(0, 1e6, n)
        x[rng.integers(0, n, 64)] = [np.inf, -np.inf, np.nan, -0.0, 5e-324, -2.2250738585072014e-308, 1e308,
                                     0.1] * 8
        return x
    src = i64_column(eid, rng, n) if eid in (6, 7, 16, 17, 22, 27) else dpatch_column(eid, rng, n)
    return src.astype(np.float64) / 4


def str_column(eid, rng, n):
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789-_", np.uint8)
    tokens = [bytes(alphabet[rng.integers(0, 64, rng.integers(2, 7))]) for _ in range(64)]
    distinct = [b"".join(tokens[t] for t in rng.integers(0, 64, rng.integers(1, 6))) for _ in range(300)]
    if eid in (15, 16):
        runs = rng.geometric(1 / 5, n)
        col = [distinct[k] for k in np.repeat(rng.integers(0, 300, runs.size), runs)[:n]]
    elif eid in STR_MORE_IDS and eid not in (1, 28, 29):
        k = rng.integers(0, 16, n)
        rare = rng.random(n) < 0.03
        k[rare] = rng.integers(16, 300, rare.sum())
        col = [distinct[x] for x in k]
    else:
        col = [distinct[k] for k in rng.integers(0, 300, n)]
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in col])
    return np.frombuffer(b"".join(col), np.uint8).copy(), offs


def columns(ref):
    res = {}
    n = 3 * 1024
    cap = 1 << 22
    for eid in I64_IDS:
        rng = np.random.default_rng(1000 + eid)
        col = i64_column(eid, rng, n)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_i64(ptr(col), ctypes.c_uint64(n), ctypes.c_uint8(eid), 1, ptr(page), ctypes.c_uint64(cap),
                                ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        out = np.zeros(n, np.int64)
        nv = ctypes.c_uint64()
        rc = ref.ref_decode_i64(ptr(page), ptr(dic), ds, ptr(out), ctypes.c_uint64(n // 1024), ctypes.byref(nv))
        assert rc == 0 and nv.value == n // 1024, (eid, rc)
        assert np.array_equal(out, col), eid
        res[f"i64_{eid}_input"] = col
        res[f"i64_{eid}_page"] = page[: ps.value].copy()
        res[f"i64_{eid}_dict"] = dic[: ds.value].copy()
        # the reference decoder reproduces the input for every int64 expression (asserted above)
    for eid in REC_IDS:
        rng = np.random.default_rng(3000 + eid)
        # REC2 (id 10) also rec-compresses the u16 rsum bases (64 per vector): 20 vectors give one FFOR block
        m = (20 if eid == 10 else 4) * 1024
        col = rec_column(eid, rng, m)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_i64(ptr(col), ctypes.c_uint64(m), ctypes.c_uint8(eid), 1, ptr(page), ctypes.c_uint64(cap),
                                ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        out = np.zeros(m, np.int64)
        nv = ctypes.c_uint64()
        rc = ref.ref_decode_i64(ptr(page), ptr(dic), ds, ptr(out), ctypes.c_uint64(m // 1024), ctypes.byref(nv))
        assert rc == 0 and np.array_equal(out, col), (eid, rc)
        res[f"i64rec_{eid}_input"] = col
        res[f"i64rec_{eid}_page"] = page[: ps.value].copy()
        res[f"i64rec_{eid}_dict"] = dic[: ds.value].copy()
    for eid in PATCH_IDS:
        rng = np.random.default_rng(4000 + eid)
        col = patch_column(eid, rng, n)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_i64(ptr(col), ctypes.c_uint64(n), ctypes.c_uint8(eid), 1, ptr(page), ctypes.c_uint64(cap),
                                ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        res[f"i64patch_{eid}_input"] = col
        res[f"i64patch_{eid}_page"] = page[: ps.value].copy()
    for eid in DPATCH_IDS:
        rng = np.random.default_rng(5000 + eid)
        m = 4 * 1024
        col = dpatch_column(eid, rng, m)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_i64(ptr(col), ctypes.c_uint64(m), ctypes.c_uint8(eid), 1, ptr(page), ctypes.c_uint64(cap),
                                ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        res[f"i64dpatch_{eid}_input"] = col
        res[f"i64dpatch_{eid}_page"] = page[: ps.value].copy()
        res[f"i64dpatch_{eid}_dict"] = dic[: ds.value].copy()
    for eid in FRQ_IDS:
        rng = np.random.default_rng(6000 + eid)
        m = 4 * 1024
        col = dpatch_column(eid, rng, m)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_i64(ptr(col), ctypes.c_uint64(m), ctypes.c_uint8(eid), 1, ptr(page), ctypes.c_uint64(cap),
                                ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        res[f"i64frq_{eid}_input"] = col
        res[f"i64frq_{eid}_page"] = page[: ps.value].copy()
        res[f"i64frq_{eid}_dict"] = dic[: ds.value].copy()
    for eid in F64_IDS:
        rng = np.random.default_rng(8000 + eid)
        m = 4 * 1024
        col = f64_column(eid, rng, m)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_f64(ptr(col), ctypes.c_uint64(m), ctypes.c_uint8(eid), 1, ptr(page), ctypes.c_uint64(cap),
                                ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        out = np.zeros(m, np.float64)
        nv = ctypes.c_uint64()
        rc = ref.ref_decode_f64(ptr(page), ptr(dic), ds, ptr(out), ctypes.c_uint64(m // 1024), ctypes.byref(nv))
        assert rc == 0 and nv.value == m // 1024, (eid, rc)
        assert np.array_equal(out.view(np.uint64), col.view(np.uint64)), eid
        res[f"f64_{eid}_input"] = col
        res[f"f64_{eid}_page"] = page[: ps.value].copy()
        res[f"f64_{eid}_dict"] = dic[: ds.value].copy()
    for eid in STR_IDS + STR_MORE_IDS:
        rng = np.random.default_rng(2000 + eid if eid in STR_IDS else 7000 + eid)
        byts, offs = str_column(eid, rng, n)
        page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
        rc = ref.ref_encode_str(ptr(byts), ptr(offs), ctypes.c_uint64(n), ctypes.c_uint8(eid), 1, ptr(page),
                                ctypes.c_uint64(cap), ctypes.byref(ps), ptr(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
        assert rc == 0, (eid, rc)
        ob, oo, nr = np.zeros(cap, np.uint8), np.zeros(n + 1, np.uint64), ctypes.c_uint64()
        rc = ref.ref_decode_str(ptr(page), ptr(dic), ds, ptr(ob), ctypes.c_uint64(cap), ptr(oo), ctypes.c_uint64(n),
                                ctypes.byref(nr))
        assert rc == 0, (eid, rc)
        res[f"str_{eid}_input_bytes"] = byts
        res[f"str_{eid}_input_offsets"] = offs
        res[f"str_{eid}_page"] = page[: ps.value].copy()
        res[f"str_{eid}_dict"] = dic[: ds.value].copy()
        if not (np.array_equal(oo, offs) and np.array_equal(ob[: oo[-1]], byts)):
            # string DICT pages: the reference encoder stores each dictionary entry with its predecessor's
            # length (TDic::serialize writes start offsets, HzlCmp::FSST reads them as end offsets), so the
            # reference decoder's output differs from the input; it is what a drop-in decoder must return.
            res[f"str_{eid}_decoded_bytes"] = ob[: oo[-1]].copy()
            res[f"str_{eid}_decoded_offsets"] = oo
    return res


def main():
    ref = ctypes.CDLL(os.path.join(REPO, "oracle/_ref/libfls_ref.so"))
    np.savez_compressed(os.path.join(HERE, "primitives.npz"), **primitives(ref))
    cols = columns(ref)
    old = os.path.join(HERE, "columns.npz")
    if os.path.exists(old):
        prev = np.load(old)
        cols.update({k: prev[k] for k in prev.files if k in cols})
    np.savez_compressed(old, **cols)
    for f in ("primitives.npz", "columns.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
