"""Generates str_dict_1m.npz: a 1 Mi-row string DICT page (string pool id 3: DICT FFOR_NO_PATCH codes over an
FSST-compressed dictionary, src/cor/exp_pool.cpp:69) written by the reference's own column encoder, for the
full-size parity test of the string decoder (tests/test_strings_gpu.py).

Run where the reference is checked out and its oracle built (``make -C oracle ref``)::

    python tests/golden/make_str_dict_1m.py [REFERENCE_ROOT]

The column has the DICT+FSST configuration's shape: a 4096-entry dictionary of 5-40-byte strings made of
Zipf(1.2)-chosen tokens, rows Zipf(1.1) over it.  The fixture keeps the page, the dictionary page and the
reference decoder's dictionary (entry c as the reference decodes it; its encoder stores every entry with its
predecessor's length, so these differ from the input strings) and the code the reference gave every dictionary
value.  The rows are regenerated by row_codes(): row_values() mapped through those codes; the script asserts
that row r of the reference decoder's whole output is entry row_codes()[r] of that dictionary.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
N_ROWS = 1 << 20
N_DICT = 4096


def dictionary(seed=41):
    """N_DICT strings of uniform length 5..40 over a 64-symbol alphabet, each built from Zipf(1.2)-chosen tokens
    out of 256 seeded 2..6-byte tokens (inverse-CDF sampling on uniform draws)."""
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789-_", np.uint8)
    tokens = [bytes(alphabet[rng.integers(0, 64, rng.integers(2, 7))]) for _ in range(256)]
    cdf = np.cumsum(np.arange(1, 257, dtype=np.float64) ** -1.2)
    picks = np.searchsorted(cdf / cdf[-1], rng.random(N_DICT * 64))
    out, j = [], 0
    for _ in range(N_DICT):
        target = int(rng.integers(5, 41))
        s = b""
        while len(s) < target:
            s += tokens[min(int(picks[j]), 255)]
            j += 1
        out.append(s[:target])
    return out


def row_values(seed=42):
    """N_ROWS indices into dictionary(), Zipf(1.1) over its N_DICT entries (inverse CDF on uniform draws)."""
    rng = np.random.default_rng(seed)
    cdf = np.cumsum(np.arange(1, N_DICT + 1, dtype=np.float64) ** -1.1)
    return np.minimum(np.searchsorted(cdf / cdf[-1], rng.random(N_ROWS)), N_DICT - 1)


def row_codes(code_of_value):
    """The reference's code of every row: code_of_value[value] (the fixture's mapping, read from the page)."""
    return np.asarray(code_of_value)[row_values()].astype(np.uint32)


def page_codes(page):
    """The page's code stream in row order, decoded by the oracle (DICT FFOR_NO_PATCH: unffor + untranspose)."""
    sys.path.insert(0, REPO)
    from oracle import oracle
    from oracle import pages

    pg = pages.parse_page(page)
    return np.concatenate([oracle.untranspose_i(np.ascontiguousarray(pages._stream(pg, v, 0, 32, "ffor", np.uint32)))
                           for v in range(pg.vec_c)])


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FLS_REFERENCE", "/root/reference")
    assert os.path.isdir(ref_root), ref_root
    ref = ctypes.CDLL(os.path.join(REPO, "oracle/_ref/libfls_ref.so"))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    strs = dictionary()
    vals = row_values()
    col = [strs[v] for v in vals]
    byts = np.frombuffer(b"".join(col), np.uint8).copy()
    offs = np.zeros(N_ROWS + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in col])
    cap = 1 << 26
    page, dic = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
    ps, ds = ctypes.c_uint64(), ctypes.c_uint64()
    rc = ref.ref_encode_str(P(byts), P(offs), ctypes.c_uint64(N_ROWS), ctypes.c_uint8(3), 1, P(page),
                            ctypes.c_uint64(cap), ctypes.byref(ps), P(dic), ctypes.c_uint64(cap), ctypes.byref(ds))
    assert rc == 0, rc
    ob, oo, nr = np.zeros(1 << 27, np.uint8), np.zeros(N_ROWS + 1, np.uint64), ctypes.c_uint64()
    rc = ref.ref_decode_str(P(page), P(dic), ds, P(ob), ctypes.c_uint64(ob.size), P(oo), ctypes.c_uint64(N_ROWS),
                            ctypes.byref(nr))
    assert rc == 0 and nr.value == N_ROWS, (rc, nr.value)
    # the reference's code of every dictionary value (it numbers the entries itself), read from its page
    codes = page_codes(page[: ps.value])
    code_of_value = np.full(N_DICT, -1, np.int64)
    code_of_value[vals] = codes
    assert np.array_equal(code_of_value[vals], codes)  # one code per value
    # the reference decoder's dictionary: entry c = the decoded row where code c first occurs
    first = np.full(int(codes.max()) + 1, -1, np.int64)
    for r in range(N_ROWS - 1, -1, -1):
        first[codes[r]] = r
    assert (first >= 0).all()
    ent = [ob[int(oo[r]):int(oo[r + 1])] for r in first]
    dict_offsets = np.zeros(len(ent) + 1, np.uint64)
    dict_offsets[1:] = np.cumsum([e.size for e in ent])
    dict_bytes = np.concatenate(ent)
    # every row of the reference's output is its code's entry
    lens = np.diff(dict_offsets).astype(np.int64)[codes]
    assert np.array_equal(np.diff(oo).astype(np.int64), lens)
    starts = dict_offsets[:-1].astype(np.int64)[codes]
    idx = np.repeat(starts - oo[:-1].astype(np.int64), lens) + np.arange(int(oo[-1]))
    assert np.array_equal(ob[: int(oo[-1])], dict_bytes[idx])
    np.savez_compressed(os.path.join(HERE, "str_dict_1m.npz"), page=page[: ps.value].copy(),
                        dict=dic[: ds.value].copy(), ref_dict_bytes=dict_bytes, ref_dict_offsets=dict_offsets,
                        code_of_value=code_of_value.astype(np.int32),
                        n_decoded_bytes=np.uint64(oo[-1]))
    print("str_dict_1m.npz", os.path.getsize(os.path.join(HERE, "str_dict_1m.npz")), "decoded bytes", int(oo[-1]))


if __name__ == "__main__":
    main()
