"""TEST INFRASTRUCTURE — Python face of the CPU oracle.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may import this module, and only as
the checker.  ``restated`` is the plain-C restatement (fls_oracle.c, always built); ``reference`` is the
reference project's own code compiled from its sources (oracle/_ref/libfls_ref.so, present only where it
was built).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED_PATH = os.path.join(HERE, "libfls_oracle.so")
REFERENCE_PATH = os.path.join(HERE, "_ref", "libfls_ref.so")
# the same sources built with -march=x86-64-v4 (AVX-512), for hosts that have those extensions
REFERENCE_V4_PATH = os.path.join(HERE, "_ref", "libfls_ref_v4.so")
TYPES = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _load(path):
    return ctypes.CDLL(path) if os.path.exists(path) else None


def _has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "").split()
    except OSError:
        return False
    return all(x in flags for x in ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"))


restated = _load(RESTATED_PATH)
REFERENCE_MARCH = "x86-64-v4" if os.path.exists(REFERENCE_V4_PATH) and _has_avx512() else "x86-64-v3"
reference = _load(REFERENCE_V4_PATH if REFERENCE_MARCH == "x86-64-v4" else REFERENCE_PATH)


def lib():
    if restated is None:
        raise RuntimeError(f"{RESTATED_PATH} missing: run `make -C oracle`")
    return restated


def _w(a):
    return {np.dtype(np.uint8): 8, np.dtype(np.uint16): 16, np.dtype(np.uint32): 32, np.dtype(np.uint64): 64}[a.dtype]


# ---- one vector -------------------------------------------------------------------------------------------
def transpose_i(x):
    out = np.empty_like(x)
    getattr(lib(), f"fls_o_transpose_i_u{_w(x)}")(_ptr(x), _ptr(out))
    return out


def untranspose_i(x):
    out = np.empty_like(x)
    getattr(lib(), f"fls_o_untranspose_i_u{_w(x)}")(_ptr(x), _ptr(out))
    return out


def ffor(x, bw, base):
    w = _w(x)
    out = np.zeros(1024, x.dtype)
    b = np.array([base], x.dtype)
    getattr(lib(), f"fls_o_ffor_u{w}")(_ptr(x), _ptr(out), ctypes.c_uint8(bw), _ptr(b))
    return out[: bw * (1024 // w)].copy()


def pack(x, bw):
    return ffor(x, bw, 0)


def unffor(packed, bw, base, dtype):
    w = _w(np.zeros(1, dtype))
    buf = np.zeros(1024, dtype)
    buf[: packed.size] = packed
    out = np.empty(1024, dtype)
    b = np.array([base], dtype)
    getattr(lib(), f"fls_o_unffor_u{w}")(_ptr(buf), _ptr(out), ctypes.c_uint8(bw), _ptr(b))
    return out


def unpack(packed, bw, dtype):
    return unffor(packed, bw, 0, dtype)


def rsum(deltas, lane_bases):
    out = np.empty_like(deltas)
    getattr(lib(), f"fls_o_rsum_u{_w(deltas)}")(_ptr(deltas), _ptr(out), _ptr(lane_bases))
    return out


def unrsum(x):
    out = np.empty_like(x)
    getattr(lib(), f"fls_o_unrsum_u{_w(x)}")(_ptr(x), _ptr(out))
    return out


def analyze(x):
    base = np.zeros(1, x.dtype)
    bw = getattr(lib(), f"fls_o_analyze_u{_w(x)}")(_ptr(x), _ptr(base))
    return int(bw) & 0xFF, base[0]


# ---- batches ----------------------------------------------------------------------------------------------
def unffor_batch(packed_bytes, byte_off, bw, base, original):
    """Decode a batch: vector v's packed words start at packed_bytes[byte_off[v]]."""
    dtype = base.dtype
    w = _w(base)
    words = np.frombuffer(packed_bytes.tobytes() + b"\0" * 16, dtype=dtype)
    word_off = (np.asarray(byte_off, np.uint64) // (w // 8)).astype(np.uint64)
    out = np.empty(bw.size * 1024, dtype)
    getattr(lib(), f"fls_o_unffor_batch_u{w}")(_ptr(words), _ptr(word_off), _ptr(bw.astype(np.uint8)), _ptr(base),
                                               ctypes.c_uint64(bw.size), ctypes.c_int(1 if original else 0), _ptr(out))
    return out


def delta_batch(packed_bytes, byte_off, bw, base, lane_bases, original):
    """DELTA decode of a batch: unffor, then rsum with 128-byte lane bases per vector."""
    dtype = base.dtype
    w = _w(base)
    L = 1024 // w
    tr = unffor_batch(packed_bytes, byte_off, bw, base, False).reshape(-1, 1024)
    lb = lane_bases.reshape(-1, L)
    out = np.empty_like(tr)
    for v in range(tr.shape[0]):
        r = rsum(tr[v].copy(), lb[v].copy())
        out[v] = untranspose_i(r) if original else r
    return out.reshape(-1)


def fsst_decode_table(table_bytes):
    sym = np.zeros(256, np.uint64)
    ln = np.zeros(256, np.uint8)
    used = lib().fls_o_fsst_import(_ptr(np.ascontiguousarray(table_bytes, np.uint8)), _ptr(sym), _ptr(ln))
    return int(used), sym, ln


def fsst_decode(sym, ln, data):
    data = np.ascontiguousarray(data, np.uint8)
    cap = max(8 * data.size, 1)
    out = np.zeros(cap, np.uint8)
    lib().fls_o_fsst_decode.restype = ctypes.c_uint64
    n = lib().fls_o_fsst_decode(_ptr(sym), _ptr(ln), _ptr(data), ctypes.c_uint64(data.size), _ptr(out),
                                ctypes.c_uint64(cap))
    return out[:n].copy()


def fsst12_decode_table(table_bytes):
    """FSST12 symbol table (4096 codes) from fsst12_export's bytes: (bytes used, symbols, lengths)."""
    t = np.ascontiguousarray(table_bytes, np.uint8)
    sym = np.zeros(4096, np.uint64)
    ln = np.zeros(4096, np.uint8)
    used = lib().fls_o_fsst12_import(_ptr(t), ctypes.c_uint64(t.size), _ptr(sym), _ptr(ln))
    return int(used), sym, ln


def fsst12_decode(sym, ln, data):
    data = np.ascontiguousarray(data, np.uint8)
    cap = max(8 * data.size, 1)
    out = np.zeros(cap, np.uint8)
    lib().fls_o_fsst12_decode.restype = ctypes.c_uint64
    n = lib().fls_o_fsst12_decode(_ptr(sym), _ptr(ln), _ptr(data), ctypes.c_uint64(data.size), _ptr(out),
                                  ctypes.c_uint64(cap))
    return out[:n].copy()
