"""String columns (DICT / DICT_RLE / DICT_FRQ with FSST dictionaries, FSST, FSST12, BYTE_ARR pages) decoded on the GPU into
Arrow-style offsets + bytes (fls_string_plan_* of include/fls_b200.h)."""
import ctypes

import torch

from ._lib import check, declare

_p = ctypes.c_void_p
_u64 = ctypes.c_uint64

_create = declare("fls_string_plan_create", ctypes.c_int, [_p, _u64, _p, _u64, ctypes.POINTER(_p)])
_rows = declare("fls_string_plan_rows", ctypes.c_int, [_p, ctypes.POINTER(_u64)])
_measure = declare("fls_string_plan_measure", ctypes.c_int, [_p, ctypes.POINTER(_u64), _p])
_decode = declare("fls_string_plan_decode", ctypes.c_int, [_p, _p, _p, _u64, _p])
_destroy = declare("fls_string_plan_destroy", ctypes.c_int, [_p])
_noalloc = declare("fls_gpu_decode_fsst_page_noalloc", ctypes.c_int, [_p, _u64, _p, _u64, _p, _p, _u64, _p, _p])
_set_create = declare("fls_string_set_create", ctypes.c_int, [_p, ctypes.c_uint32, ctypes.POINTER(_p)])
_set_bind = declare("fls_string_set_bind", ctypes.c_int, [_p, _p, _p, _p])
_set_decode = declare("fls_string_set_decode", ctypes.c_int, [_p, _p])
_set_destroy = declare("fls_string_set_destroy", ctypes.c_int, [_p])


def decode_fsst_page_noalloc(d_page, page_size, d_dict, dict_size, offsets, data, status, stream=None):
    """Allocation-free decode of an FSST / BYTE_ARR page into caller-owned offsets (int32, n_rows + 1) and data
    (uint8) tensors.  status: a zeroed int32 device tensor that receives the device-detected errors (FLS_DEV_*);
    returns the call's status code (0 = ok, -6 = page beyond the fixed scratch)."""
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    return _noalloc(d_page, page_size, d_dict, dict_size, offsets.data_ptr(), data.data_ptr(), data.numel(),
                    status.data_ptr() if status is not None else None, s)


class StringPlan:
    """Decoder of one string page; the page / dictionary device buffers must outlive it."""

    def __init__(self, d_page, page_size, d_dict=None, dict_size=0):
        h = _p()
        check(_create(d_page, page_size, d_dict, dict_size, ctypes.byref(h)), "fls_string_plan_create")
        self.handle = h
        n = _u64()
        check(_rows(h, ctypes.byref(n)), "rows")
        self.n_rows = n.value

    def measure(self, stream=None):
        n = _u64()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_measure(self.handle, ctypes.byref(n), s), "measure")
        return n.value

    def decode_into(self, offsets, data, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_decode(self.handle, offsets.data_ptr(), data.data_ptr(), data.numel(), s), "decode")

    def decode(self, device="cuda"):
        n_bytes = self.measure()
        offsets = torch.empty(self.n_rows + 1, dtype=torch.int32, device=device)
        data = torch.empty(max(n_bytes, 16), dtype=torch.uint8, device=device)
        self.decode_into(offsets, data)
        return offsets, data[:n_bytes]

    def close(self):
        if self.handle:
            _destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StringSet:
    """Many DICT string plans decoded by one kernel launch (fls_string_set_*).  The plans and the bound output
    tensors must outlive the set; decode() only launches (capturable in a CUDA graph)."""

    def __init__(self, plans):
        arr = (_p * len(plans))(*[p.handle.value for p in plans])
        h = _p()
        check(_set_create(ctypes.cast(arr, _p), len(plans), ctypes.byref(h)), "fls_string_set_create")
        self.handle = h
        self.n = len(plans)

    def bind(self, offsets, data):
        """offsets / data: one int32 (n_rows + 1) and one uint8 tensor per plan."""
        import numpy as np

        offs = (_p * self.n)(*[o.data_ptr() for o in offsets])
        byts = (_p * self.n)(*[d.data_ptr() for d in data])
        caps = np.array([d.numel() for d in data], np.uint64)
        check(_set_bind(self.handle, ctypes.cast(offs, _p), ctypes.cast(byts, _p), caps.ctypes.data_as(_p)),
              "fls_string_set_bind")
        self._bound = (offsets, data)

    def decode(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_set_decode(self.handle, s), "fls_string_set_decode")

    def close(self):
        if self.handle:
            _set_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_fsst_compress = declare("fls_fsst_compress", ctypes.c_int, [_p, _p, _u64, _p, _u64, ctypes.POINTER(_u64), _p, _u64,
                                                             _p])
_enc_dict = declare("fls_encode_string_dict", ctypes.c_int, [_p, _p, ctypes.c_uint32, _p, _u64, _p, _u64,
                                                             ctypes.POINTER(_u64), _p, _u64, ctypes.POINTER(_u64)])


def _np_ptr(a):
    return a.ctypes.data_as(_p)


def fsst_compress(byts, offsets):
    """FSST-compress n strings given as (bytes, offsets[n + 1]) numpy arrays (host only).
    Returns (table bytes in fsst_export format, compressed bytes, compressed offsets[n + 1])."""
    import numpy as np

    byts = np.ascontiguousarray(byts, np.uint8)
    offsets = np.ascontiguousarray(offsets, np.uint64)
    n = offsets.size - 1
    table = np.zeros(2100, np.uint8)
    tl = _u64()
    comp = np.zeros(2 * byts.size + 16, np.uint8)
    coffs = np.zeros(n + 1, np.uint64)
    check(_fsst_compress(_np_ptr(byts), _np_ptr(offsets), n, _np_ptr(table), table.size, ctypes.byref(tl),
                         _np_ptr(comp), comp.size, _np_ptr(coffs)), "fls_fsst_compress")
    return table[: tl.value].copy(), comp[: int(coffs[-1])].copy(), coffs


def encode_string_dict(dict_bytes, dict_offsets, codes):
    """String DICT FFOR page of codes into a dictionary; returns (page bytes, dictionary page bytes)."""
    import numpy as np

    dict_bytes = np.ascontiguousarray(dict_bytes, np.uint8)
    dict_offsets = np.ascontiguousarray(dict_offsets, np.uint64)
    codes = np.ascontiguousarray(codes, np.uint32)
    page = np.zeros(codes.size * 4 + 65536, np.uint8)
    dic = np.zeros(8 + 2066 + 4 * (dict_offsets.size - 1) + 2 * dict_bytes.size + 64, np.uint8)
    ps, ds = _u64(), _u64()
    check(_enc_dict(_np_ptr(dict_bytes), _np_ptr(dict_offsets), dict_offsets.size - 1, _np_ptr(codes), codes.size,
                    _np_ptr(page), page.size, ctypes.byref(ps), _np_ptr(dic), dic.size, ctypes.byref(ds)),
          "fls_encode_string_dict")
    return page[: ps.value].copy(), dic[: ds.value].copy()


def _transposed_order():
    """Index array of the unified transposed layout: transposed[k] = original[idx[k]]."""
    import numpy as np

    k = np.arange(1024)
    order = np.array([0, 4, 2, 6, 1, 5, 3, 7])
    return (k % 16) * 64 + order[(k // 16) % 8] * 8 + k // 128


def encode_fsst_page(byts, offsets):
    """FSST column page (string pool expression 13, FSST UNCOMPRESSED) of n strings, n a multiple of 1024, and its
    dictionary page (dict_hdr_t + the exported symbol table).  Layout as the reference writes it
    (src/cor/lyt/vec.cpp:162-207): per vector its compressed bytes (buffer 0) and its 1024 cumulative END offsets
    within them, u32, transposed (buffer 1); entry points per vector after the first."""
    import numpy as np

    table, comp, coffs = fsst_compress(byts, offsets)
    return fsst_page(table, comp, coffs)


def fsst_page(table, comp, coffs):
    """The FSST column page and dictionary page of strings already compressed with `table` (fsst_compress's
    outputs: compressed bytes and their offsets[n + 1], n a multiple of 1024)."""
    import numpy as np

    coffs = np.ascontiguousarray(coffs, np.uint64)
    n = coffs.size - 1
    if n % 1024:
        raise ValueError("fsst_page: whole vectors only")
    vec_c = n // 1024
    if vec_c >= 1 << 16:
        raise ValueError("fsst_page: at most 65535 vectors")
    starts = coffs[0:n:1024]
    ends = (coffs[1:].reshape(vec_c, 1024) - starts[:, None]).astype(np.uint32)
    ends_t = ends[:, _transposed_order()]
    meta = 8 + 2 * 4 + 2 * 4 * max(vec_c - 1, 0)
    b0 = comp.size
    hdr = np.zeros(meta, np.uint8)
    hdr[0], hdr[1] = 7, 1
    hdr[4:6] = np.frombuffer(np.uint16(vec_c).tobytes(), np.uint8)
    hdr[8:16] = np.frombuffer(np.array([meta, meta + b0], np.uint32).tobytes(), np.uint8)
    if vec_c > 1:
        ep = np.stack([starts[1:].astype(np.uint32), (np.arange(1, vec_c) * 4096).astype(np.uint32)], axis=1)
        hdr[16:] = np.frombuffer(ep.astype("<u4").tobytes(), np.uint8)
    page = np.concatenate([hdr, comp, np.frombuffer(ends_t.astype("<u4").tobytes(), np.uint8)])
    dic = np.concatenate([np.array([7, 0, 0, 0, 0, 0, 0, 0], np.uint8), table])
    return page, dic
