"""Files: the reference's file pair data.fls + footer.json (Connection::to_fls / read_fls of the reference,
src/connection.cpp:102-128, src/reader/reader.cpp:19-61) on the GPU.

read_fls() loads columns into device tensors through fls_file_read (the C ABI).  write_fls() writes the same
container with page columns — the columns' row-group chunks encoded as reference pages, listed under "pages"
in each column's metadata — next to the reference's ZERO_COPY raw columns, so that a file readable by the
reference's footer parser carries compressed columns this library decodes on the GPU.
"""
import ctypes
import json
import os

import numpy as np

from . import pages as PG
from ._lib import check, declare

_p = ctypes.c_void_p
ZERO_COPY, PAGES, NO_DATA = 1, 2, 3
_NAMES = {PG.INT64: "INT64", PG.UINT64: "UINT64", PG.INT32: "INT32", PG.UINT32: "UINT32", PG.INT16: "INT16",
          PG.UINT16: "UINT16"}
_CODE = {np.dtype(v): k for k, v in PG.DTYPE_OF.items()}

_open = declare("fls_file_open", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_p)])
_shape = declare("fls_file_shape", ctypes.c_int, [_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)])
_column = declare("fls_file_column", ctypes.c_int, [_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint8),
                                                     ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)])
_read = declare("fls_file_read", ctypes.c_int, [_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
                                                 ctypes.POINTER(_p), _p])
_close = declare("fls_file_close", ctypes.c_int, [_p])


class FlsFile:
    """An opened file pair: shape and column kinds from footer.json (host only)."""

    def __init__(self, directory):
        h = _p()
        check(_open(os.fsencode(directory), ctypes.byref(h)), "fls_file_open")
        self.handle = h
        n, v = ctypes.c_uint32(), ctypes.c_uint64()
        check(_shape(h, ctypes.byref(n), ctypes.byref(v)), "fls_file_shape")
        self.n_cols, self.n_vec = n.value, v.value
        self.columns = []
        for i in range(self.n_cols):
            t, k, m = ctypes.c_uint8(), ctypes.c_uint8(), ctypes.c_uint64()
            check(_column(h, i, ctypes.byref(t), ctypes.byref(k), ctypes.byref(m)), "fls_file_column")
            self.columns.append({"data_type": t.value, "kind": k.value, "n_values": m.value})

    def read(self, cols=None, device="cuda", stream=None):
        """Device tensors of the given columns (all readable ones by default), in one fls_file_read."""
        import torch

        cols = [i for i, c in enumerate(self.columns) if c["kind"] != NO_DATA] if cols is None else list(cols)
        outs = []
        for i in cols:
            c = self.columns[i]
            dt = torch.from_numpy(np.zeros(1, PG.DTYPE_OF[c["data_type"]])).dtype
            outs.append(torch.empty(max(c["n_values"], 1), dtype=dt, device=device)[:c["n_values"]])
        idx = (ctypes.c_uint32 * len(cols))(*cols)
        ptrs = (_p * len(cols))(*[o.data_ptr() for o in outs])
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_read(self.handle, idx, len(cols), ptrs, s), "fls_file_read")
        return outs

    def close(self):
        if self.handle:
            _close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_fls(directory, cols=None, device="cuda"):
    f = FlsFile(directory)
    try:
        return f.read(cols, device)
    finally:
        f.close()


def write_fls(directory, columns, rowgroup_vectors=64):
    """columns: list of (values, expr): values a 1-D integer array of whole vectors; expr None for a raw
    ZERO_COPY column (the reference's own kind), else a page expression id (0, 1, 6, 11 through
    encode_from_memory; "dict" / "dict_rle" through encode_int_dict) applied per chunk of rowgroup_vectors."""
    os.makedirs(directory, exist_ok=True)
    blob, mtds = bytearray(), []
    n_vec = None
    for col_idx, (values, expr) in enumerate(columns):
        values = np.ascontiguousarray(values)
        if values.size % 1024:
            raise ValueError("columns hold whole vectors")
        code = _CODE[values.dtype]
        n_vec = values.size // 1024 if n_vec is None else n_vec
        m = {"col_ofs": len(blob), "is_determined": True, "logical_type": int(code),
             "logical_type_str": _NAMES[code]}
        if expr is None:
            m["Encoding RPN"] = {"operands": [{"col idx": col_idx}], "operators": ["ZERO_COPY", _NAMES[code]]}
            blob += values.tobytes()
        else:
            chunks = []
            for v0 in range(0, values.size // 1024, rowgroup_vectors):
                x = values[v0 * 1024:(v0 + rowgroup_vectors) * 1024]
                if expr in ("dict", "dict_rle"):
                    page, dic = PG.encode_int_dict(x, rle=expr == "dict_rle")
                else:
                    page, dic = PG.encode_from_memory(x, code, expr)[0], None
                ref = {"ofs": len(blob), "size": int(page.size), "dict_ofs": 0, "dict_size": 0,
                       "n_vec": x.size // 1024}
                blob += page.tobytes()
                if dic is not None:
                    ref["dict_ofs"], ref["dict_size"] = len(blob), int(dic.size)
                    blob += dic.tobytes()
                chunks.append(ref)
            m["Encoding RPN"] = {"operands": [{"col idx": col_idx}], "operators": ["FLS_PAGES", _NAMES[code]]}
            m["pages"] = chunks
        mtds.append(m)
    with open(os.path.join(directory, "data.fls"), "wb") as f:
        f.write(bytes(blob))
    footer = {"1: N VEC": int(n_vec or 0), "2: Rowgroup size": len(blob), "3: Column Metadatas": mtds}
    with open(os.path.join(directory, "footer.json"), "w") as f:
        json.dump(footer, f)
