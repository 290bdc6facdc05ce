"""Reference page columns and the reference's C API (include/fastlanes.h), on the GPU engine."""
import ctypes

import numpy as np

from ._lib import FlsError, check, declare

_p = ctypes.c_void_p
_u64 = ctypes.c_uint64

# data_t values of include/fastlanes.h
INT64, UINT64, INT32, UINT32, INT16, UINT16, DOUBLE = 5, 9, 4, 8, 3, 7, 1
DTYPE_OF = {INT64: np.int64, UINT64: np.uint64, INT32: np.int32, UINT32: np.uint32, INT16: np.int16,
            UINT16: np.uint16, DOUBLE: np.float64}


class PageColumn(ctypes.Structure):
    _fields_ = [("d_page", _p), ("page_size", _u64), ("d_dict", _p), ("dict_size", _u64), ("data_type", ctypes.c_uint8),
                ("order", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 6), ("d_out", _p)]


_decode_pages = declare("fls_gpu_decode_pages", ctypes.c_int, [ctypes.POINTER(PageColumn), ctypes.c_uint32, _p])
_decode_vectors = declare("fls_gpu_decode_page_vectors", ctypes.c_int, [ctypes.POINTER(PageColumn), ctypes.c_uint32,
                                                                        ctypes.c_uint32, _p])
_page_info = declare("fls_page_info", ctypes.c_int, [_p, _u64, ctypes.POINTER(ctypes.c_uint32),
                                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(_u64)])
_placement = declare("fls_page_placement", ctypes.c_int, [_p, _u64, ctypes.POINTER(ctypes.c_uint32)])
_enc_status = declare("fls_encode_from_memory_status", ctypes.c_int, [_p, _u64, _u64, _p, ctypes.POINTER(_u64),
                                                                        ctypes.POINTER(_u64), ctypes.c_uint8,
                                                                        ctypes.c_uint8])
_dec_checked = declare("fls_decode_to_memory_checked", ctypes.c_int, [_p, _u64, _p, _u64, ctypes.c_uint8,
                                                                       ctypes.POINTER(_u64)])
declare("encode_from_memory", ctypes.c_bool, [_p, _u64, _u64, _p, ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                                              ctypes.c_uint8, ctypes.c_uint8])
declare("decode_to_memory", None, [_p, _p, ctypes.c_uint8])
_ra_ranges = declare("fls_random_access_ranges", ctypes.c_int, [_p, _u64, ctypes.POINTER(_u64), _p])
_ra_decode = declare("fls_random_access_decode", ctypes.c_int, [_p, _u64, _u64, _p, _p, _p])
declare("init_random_access", None, [_p, _u64, ctypes.POINTER(_u64), _p])
declare("random_access", None, [_p, _u64, ctypes.POINTER(_u64), _p, _p, _p])
declare("fls_cpi_connection_open", _p, [])
declare("fls_cpi_connection_close", None, [_p])


def _ptr(a):
    return a.ctypes.data_as(_p)


def page_info(page):
    page = np.ascontiguousarray(page, np.uint8)
    e, v, n, a = (ctypes.c_uint32() for _ in range(4))
    m = _u64()
    check(_page_info(_ptr(page), page.size, ctypes.byref(e), ctypes.byref(v), ctypes.byref(n), ctypes.byref(a),
                     ctypes.byref(m)), "page_info")
    return {"exp_t": e.value, "var": v.value, "vec_c": n.value, "arr_c": a.value, "meta_size": m.value}


def placement(page):
    page = np.ascontiguousarray(page, np.uint8)
    s = ctypes.c_uint32()
    check(_placement(_ptr(page), page.size, ctypes.byref(s)), "placement")
    return s.value


_plan_pages = declare("fls_plan_create_pages", ctypes.c_int, [ctypes.POINTER(PageColumn), ctypes.c_uint32,
                                                                ctypes.POINTER(_p)])
_plan_decode = declare("fls_plan_decode", ctypes.c_int, [_p, _p])
_plan_destroy = declare("fls_plan_destroy", ctypes.c_int, [_p])
_plan_autotune = declare("fls_plan_autotune", ctypes.c_int, [_p, ctypes.c_int, _p])
_plan_variant = declare("fls_plan_variant_name", ctypes.c_char_p, [_p, ctypes.c_int])
_plan_graph = declare("fls_plan_decode_graph", ctypes.c_int, [_p, _p])


def _columns(columns):
    arr = (PageColumn * len(columns))()
    for i, c in enumerate(columns):
        a = arr[i]
        a.d_page, a.page_size = c["d_page"], c["page_size"]
        a.d_dict, a.dict_size = c.get("d_dict"), c.get("dict_size", 0)
        a.data_type, a.order, a.d_out = c["data_type"], c.get("order", 1), c["d_out"]
    return arr


class PagePlan:
    """fls_plan_create_pages: page metadata read once; decode() is one kernel launch."""

    def __init__(self, columns):
        h = _p()
        check(_plan_pages(_columns(columns), len(columns), ctypes.byref(h)), "fls_plan_create_pages")
        self.handle = h

    def decode(self, stream=None):
        import torch

        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_plan_decode(self.handle, s), "fls_plan_decode")

    def decode_graph(self, stream=None):
        """The plan's launches captured once in a CUDA graph, replayed on the stream."""
        import torch

        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_plan_graph(self.handle, s), "fls_plan_decode_graph")

    def autotune(self, reps=3, stream=None):
        """Pick the fastest geometry variant per launch segment (runs decodes); returns the variants' names."""
        import torch

        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(_plan_autotune(self.handle, reps, s), "fls_plan_autotune")
        return [n for n in (_plan_variant(self.handle, i).decode() for i in (0, 1)) if n]

    def close(self):
        if self.handle:
            _plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- predicate pushdown (src/primitive/predicate/equal.cpp of the reference) ------------------------------
PRED_EQ, PRED_NE, PRED_LT, PRED_LE, PRED_GT, PRED_GE = range(6)
BITMAP_AND, BITMAP_OR, BITMAP_ANDNOT = range(3)


class Predicate(ctypes.Structure):
    _fields_ = [("op", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 7), ("value", ctypes.c_int64)]


_plan_filter = declare("fls_plan_create_filter", ctypes.c_int, [ctypes.POINTER(PageColumn), ctypes.c_uint32,
                                                                  ctypes.POINTER(Predicate), ctypes.POINTER(_p)])
_to_selection = declare("fls_gpu_bitmap_to_selection", ctypes.c_int, [_p, _u64, _p, _p, _p])
_combine = declare("fls_gpu_bitmap_combine", ctypes.c_int, [_p, _p, _p, _u64, ctypes.c_int, _p])
_sel_and = declare("fls_gpu_selection_and", ctypes.c_int, [_p, _p, _p, _p, _p, _p, _u64, _p])


def _stream(stream):
    import torch

    return stream if stream is not None else torch.cuda.current_stream().cuda_stream


class FilterPlan(PagePlan):
    """fls_plan_create_filter: `column OP value` over page columns; each column's d_out receives vec_c * 128
    bytes (one 1024-bit bitmap per vector, bit i = value i in the column's order).  decode() evaluates.  The
    value is compared with every value widened to 64 bits (sign-extended for signed types); an unsigned
    column's constant is given as its uint64 bits or any Python int that wraps to them."""

    def __init__(self, columns, op, value):
        pr = Predicate()
        pr.op = op
        v = int(value) & (2**64 - 1)
        pr.value = v - 2**64 if v >= 2**63 else v
        h = _p()
        check(_plan_filter(_columns(columns), len(columns), ctypes.byref(pr), ctypes.byref(h)),
              "fls_plan_create_filter")
        self.handle = h


def bitmap_to_selection(d_bitmaps, n_vec, d_idx, d_count, stream=None):
    """SelectionDS idx_arr / n_selected_values per vector (u16) from bitmaps (device pointers)."""
    check(_to_selection(d_bitmaps, n_vec, d_idx, d_count, _stream(stream)), "fls_gpu_bitmap_to_selection")


def bitmap_combine(d_a, d_b, d_out, n_vec, op, stream=None):
    check(_combine(d_a, d_b, d_out, n_vec, op, _stream(stream)), "fls_gpu_bitmap_combine")


def selection_and(d_idx0, d_count0, d_idx1, d_count1, d_idx_out, d_count_out, n_vec, stream=None):
    """and_selection_ds_func per vector on index lists (device pointers)."""
    check(_sel_and(d_idx0, d_count0, d_idx1, d_count1, d_idx_out, d_count_out, n_vec, _stream(stream)),
          "fls_gpu_selection_and")


def decode_pages(columns, stream=None):
    """columns: list of dicts with d_page, page_size, d_dict, dict_size, data_type, order, d_out (device ptrs)."""
    import torch

    arr = (PageColumn * len(columns))()
    for i, c in enumerate(columns):
        a = arr[i]
        a.d_page, a.page_size = c["d_page"], c["page_size"]
        a.d_dict, a.dict_size = c.get("d_dict"), c.get("dict_size", 0)
        a.data_type, a.order, a.d_out = c["data_type"], c.get("order", 1), c["d_out"]
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(_decode_pages(arr, len(columns), s), "fls_gpu_decode_pages")


def decode_page_vectors(column, first_vec, n_vec, stream=None):
    """Vectors [first_vec, first_vec + n_vec) of one page into column["d_out"] (fls_gpu_decode_page_vectors)."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(_decode_vectors(_columns([column]), first_vec, n_vec, s), "fls_gpu_decode_page_vectors")


def encode_from_memory(values, data_type, expr_id, capacity=None):
    """fastlanes.h encode_from_memory on a host array; returns (page bytes, metadata size)."""
    values = np.ascontiguousarray(values, DTYPE_OF[data_type])
    cap = capacity if capacity is not None else values.nbytes * 2 + 65536
    out = np.zeros(cap, np.uint8)
    size, mtd = _u64(), _u64()
    rc = _enc_status(_ptr(values), values.size, cap, _ptr(out), ctypes.byref(size), ctypes.byref(mtd), data_type,
                     expr_id)
    if rc != 0:
        raise FlsError(f"encode_from_memory: {rc}")
    return out[: size.value].copy(), mtd.value


_enc_int_dict = declare("fls_encode_int_dict", ctypes.c_int, [_p, _u64, ctypes.c_int, ctypes.c_int, _p, _u64,
                                                            ctypes.POINTER(_u64), _p, _u64, ctypes.POINTER(_u64)])


def encode_int_dict(values, rle=False):
    """DICT (exp 8 var 2) or DICT_RLE (exp 11 var 2) pages of an integer host array (32 / 64-bit, whole
    vectors); returns (codes page, dictionary page)."""
    values = np.ascontiguousarray(values)
    w = values.dtype.itemsize * 8
    cap = values.size * 4 * 2 + 65536
    dcap = values.nbytes + 64
    page, dic = np.zeros(cap, np.uint8), np.zeros(dcap, np.uint8)
    ps, ds = _u64(), _u64()
    rc = _enc_int_dict(_ptr(values), values.size, w, 1 if rle else 0, _ptr(page), cap, ctypes.byref(ps), _ptr(dic),
                       dcap, ctypes.byref(ds))
    if rc != 0:
        raise FlsError(f"encode_int_dict: {rc}")
    return page[: ps.value].copy(), dic[: ds.value].copy()


def decode_to_memory(page, data_type, size=None):
    """fastlanes.h decode_to_memory on host bytes; returns the decoded values (original order)."""
    page = np.ascontiguousarray(page, np.uint8)
    info = page_info(page)
    out = np.zeros(info["vec_c"] * 1024, DTYPE_OF[data_type])
    n = _u64()
    check(_dec_checked(_ptr(page), page.size if size is None else size, _ptr(out), out.nbytes, data_type,
                       ctypes.byref(n)), "decode_to_memory")
    return out


def random_access_ranges(page, vector):
    """fastlanes.h init_random_access: the [offset, size] byte ranges of the buffers one vector of an INT64 page
    needs (host only; reads the page's metadata)."""
    page = np.ascontiguousarray(page, np.uint8)
    n = _u64()
    pairs = np.zeros(12, np.uint64)
    check(_ra_ranges(_ptr(page), vector, ctypes.byref(n), _ptr(pairs)), "init_random_access")
    return pairs[: 2 * n.value].reshape(-1, 2)


def random_access(page, vector, buffers, ranges):
    """fastlanes.h random_access: vector `vector` of an INT64 page from its loaded buffers (host arrays, one per
    range of random_access_ranges); returns its 1024 values in original order."""
    bufs = [np.ascontiguousarray(b, np.uint8) for b in buffers]
    ptrs = (_p * len(bufs))(*[b.ctypes.data for b in bufs])
    pairs = np.ascontiguousarray(ranges, np.uint64).reshape(-1)
    out = np.zeros(1024, np.int64)
    page = np.ascontiguousarray(page, np.uint8)
    check(_ra_decode(_ptr(page), vector, len(bufs), _ptr(pairs), ctypes.cast(ptrs, _p), _ptr(out)), "random_access")
    return out
