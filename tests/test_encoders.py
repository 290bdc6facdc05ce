"""Host-side encoders of the engine (no GPU): FSST symbol tables and compression, checked against the
reference's own fsst_import + fsst_decompress and against the oracle's restatement."""
import ctypes

import numpy as np
import pytest

from oracle import oracle


def _strings(rng, n, alphabet=b"abcdefghijklmnopqrstuvwxyz0123456789-_ABCDEFGHIJKLMNOPQRSTUVWXYZ"):
    al = np.frombuffer(alphabet, np.uint8)
    toks = [bytes(al[rng.integers(0, al.size, rng.integers(2, 7))]) for _ in range(256)]
    p = rng.zipf(1.2, 100000) % 256
    out, j = [], 0
    for _ in range(n):
        s = b""
        while len(s) < rng.integers(5, 41):
            s += toks[p[j % p.size]]
            j += 1
        out.append(s[: max(5, min(len(s), 40))])
    out += [b"", b"\xff\x00\x01", bytes(range(256))]  # empty, escape-heavy and every byte value
    offs = np.zeros(len(out) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in out])
    return np.frombuffer(b"".join(out), np.uint8).copy(), offs


def test_fsst_round_trip_with_oracle_decoder():
    from fastlanes_b200 import strings

    rng = np.random.default_rng(0)
    byts, offs = _strings(rng, 3000)
    table, comp, coffs = strings.fsst_compress(byts, offs)
    used, sym, ln = oracle.fsst_decode_table(np.concatenate([table, np.zeros(64, np.uint8)]))
    assert used == table.size
    for i in range(offs.size - 1):
        got = oracle.fsst_decode(sym, ln, comp[int(coffs[i]):int(coffs[i + 1])])
        assert np.array_equal(got, byts[int(offs[i]):int(offs[i + 1])]), i
    assert comp.size < 0.8 * byts.size  # it compresses


@pytest.mark.skipif(oracle.reference is None, reason="reference library not built in this container")
def test_fsst_tables_decode_with_the_reference_fsst():
    from fastlanes_b200 import strings

    rng = np.random.default_rng(1)
    byts, offs = _strings(rng, 500)
    table, comp, coffs = strings.fsst_compress(byts, offs)
    tab = np.concatenate([table, np.zeros(2100, np.uint8)])
    out = np.zeros(4096, np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    oracle.reference.ref_fsst_decompress.restype = ctypes.c_int64
    for i in range(offs.size - 1):
        c = np.ascontiguousarray(comp[int(coffs[i]):int(coffs[i + 1])])
        n = oracle.reference.ref_fsst_decompress(P(tab), ctypes.c_uint64(c.size), P(c) if c.size else None,
                                                 ctypes.c_uint64(out.size), P(out))
        assert n == offs[i + 1] - offs[i]
        assert np.array_equal(out[:n], byts[int(offs[i]):int(offs[i + 1])]), i
