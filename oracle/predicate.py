"""TEST INFRASTRUCTURE — CPU restatement of the reference's predicate primitives (checker only).

The reference evaluates predicates per decoded vector of 1024 i64 values into a SelectionDS
(include/fls/expression/selection_ds.hpp:16-31): an index array of the selected positions in ascending order
plus their count (equal.cpp:12-28 eq_vector_constant_func via euqality_pt_func, :43-56 ge_tvec_cvec (>),
:73-86 lessthan_func (<)), and intersects two selections with a sorted merge (equal.cpp:100-119,
and_selection_ds_func).  Its bitmap form (SelectionDS::bitmap, 16 u64) is declared but not implemented
(equal.cpp:9-11); here bit i of word i / 64 is position i.  Operators EQ NE LT LE GT GE; values compared
widened to 64 bits (sign-extended for signed dtypes) against the constant read the same way.
"""
import numpy as np

EQ, NE, LT, LE, GT, GE = range(6)


def holds(values, op, value):
    """Boolean array of `values OP value` (values: any integer dtype; value: a Python int)."""
    x = np.asarray(values)
    wide = x.astype(np.int64) if np.issubdtype(x.dtype, np.signedinteger) else x.astype(np.uint64)
    c = np.array(value).astype(wide.dtype)
    return {EQ: wide == c, NE: wide != c, LT: wide < c, LE: wide <= c, GT: wide > c, GE: wide >= c}[op]


def bitmaps(values, op, value):
    """(n_vec, 16) uint64 bitmaps of consecutive 1024-value vectors."""
    h = holds(values, op, value).reshape(-1, 1024)
    bits = np.packbits(h.astype(np.uint8), axis=1, bitorder="little")  # (n_vec, 128) bytes, bit i = position i
    return np.ascontiguousarray(bits).view(np.uint64)


def selection(bitmap_row):
    """idx_arr / n_selected_values of one vector's bitmap (16 uint64): positions in ascending order."""
    bits = np.unpackbits(np.ascontiguousarray(bitmap_row).view(np.uint8), bitorder="little")
    idx = np.flatnonzero(bits).astype(np.uint16)
    return idx, idx.size


def select_vector(vec, op, value):
    """The reference's per-vector loop (equal.cpp:16-27 and alike): positions where the predicate holds."""
    sel = []
    for i, x in enumerate(np.asarray(vec).tolist()):
        if bool(holds(np.array([x], np.asarray(vec).dtype), op, value)[0]):
            sel.append(i)
    return np.array(sel, np.uint16)


def selection_and(idx0, n0, idx1, n1):
    """and_selection_ds_func (equal.cpp:100-119): sorted merge of two index lists."""
    i = j = 0
    out = []
    while i < n0 and j < n1:
        if idx0[i] < idx1[j]:
            i += 1
        elif idx0[i] > idx1[j]:
            j += 1
        else:
            out.append(int(idx0[i]))
            i += 1
            j += 1
    return np.array(out, np.uint16)
