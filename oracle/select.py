"""TEST INFRASTRUCTURE — CPU oracle for expression selection (the wizard and the learned selector).

Only tests/ and bench.py's cpu legs may import this module, and only as the checker.

The reference chooses a column's expression by encoding the column with every expression of its pool and keeping
the smallest result (src/encoder/exp_col_encoder.cpp:18-28 encode_all, :117-129 GetBest; pool in
src/cor/exp_pool.cpp:22-101).  This module restates that choice for the no-patch integer candidates as an exact
size model of the pages the engine's encoders emit, per (column, row-group) chunk of vectors:

    candidate 0  UNCOMPRESSED       (pool id 0)   page (2,1): [values]
    candidate 1  FFOR               (pool id 1)   page (4,1): [bw][base][packed]
    candidate 2  RLE DELTA_NO_PATCH (pool id 6)   page (6,2): [run values][u16 lane bases][bw][u16 base][packed]
    candidate 3  DELTA              (pool id 11)  page (5,1): [lane bases][bw][base][packed]
    candidate 4  DICT FFOR          (pool id 17)  dictionary page + page (8,2): [bw][u32 base][packed codes]
    candidate 5  DICT_RLE           (pool id 27*) dictionary page + page (11,2): [u32 run codes][...u16 index]

  * id 27 is DICT_RLE DELTA_NO_PATCH_REC in the reference; the engine's candidate keeps the run codes raw (the
    layout of the string pool's DICT_RLE DELTA_NO_PATCH, exp_pool.cpp:61).

A page of n vectors and arr_c buffers costs 8 + 4 * arr_c * n bytes of framing (page_hdr.hpp:8-15, one offset per
buffer, one entry point per buffer for vectors 1..n-1) plus its buffers.  The dictionary page is the 8-byte
dict_hdr_t (dic.hpp:32-41) and a rec buffer holding the entries raw (12-byte rec header with bw 255,
hzl_de_cmp.cpp:28-77).  Codes are assigned in first-occurrence order (dic_fac.cpp:19-40).

The learned selector (no reference counterpart) reads 32 statistics per vector (``features``) and runs an MLP
32 -> 128 -> 128 (ReLU) -> K softmax; ``mlp_forward``/``mlp_grad``/``adam`` restate it in float64.
"""
import numpy as np

from . import oracle as O

K = 6
N_FEAT = 32
HIDDEN = 128
POOL_IDS = (0, 1, 6, 11, 17, 27)
_UT = {32: np.uint32, 64: np.uint64}
_ST = {32: np.int32, 64: np.int64}


def _bits(d):
    d = int(d)
    return d.bit_length()


def _range_bits(x, w, signed):
    """bits of (max - min) in W-bit arithmetic, min/max taken signed or unsigned (ffor_analyze.cpp:77-102)."""
    x = np.asarray(x)
    v = x.view(_ST[w]) if signed else x.view(_UT[w])
    mx, mn = int(v.max()), int(v.min())
    return _bits((mx - mn) & ((1 << w) - 1))


def vector_parts(x, signed):
    """Exact per-vector quantities of the size model: (bwF, bwD, runs, bwI)."""
    x = np.ascontiguousarray(x)
    w = x.dtype.itemsize * 8
    bw_f = _range_bits(x, w, signed)
    deltas = O.unrsum(O.transpose_i(x))
    bw_d = _range_bits(deltas, w, signed)
    start = np.ones(1024, bool)
    start[1:] = x[1:] != x[:-1]
    runs = int(start.sum())
    idx = (np.cumsum(start) - 1).astype(np.uint16)
    bw_i = O.analyze(O.unrsum(O.transpose_i(idx)))[0]
    return bw_f, bw_d, runs, int(bw_i)


def chunk_dictionary(values):
    """Distinct count and first-occurrence codes of one chunk's values."""
    _, first, inv = np.unique(values, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    return order.size, rank[inv].astype(np.uint32)


def chunk_sizes(values, signed):
    """Exact encoded bytes of every candidate for one chunk (values: n_vec * 1024 of uint32 / uint64)."""
    values = np.ascontiguousarray(values)
    sz = values.dtype.itemsize
    nv = values.size // 1024
    parts = np.array([vector_parts(values[v * 1024:(v + 1) * 1024], signed) for v in range(nv)], np.int64)
    s_f, s_d, s_r, s_i = (int(parts[:, i].sum()) for i in range(4))
    d, codes = chunk_dictionary(values)
    s_c = sum(_bits(int(c.max()) - int(c.min())) for c in codes.reshape(nv, 1024))
    dict_page = 8 + 12 + d * sz
    return np.array([
        8 + 4 * nv + 1024 * sz * nv,
        8 + 12 * nv + nv + sz * nv + 128 * s_f,
        8 + 20 * nv + sz * s_r + 128 * nv + nv + 2 * nv + 128 * s_i,
        8 + 16 * nv + 128 * nv + nv + sz * nv + 128 * s_d,
        dict_page + 8 + 12 * nv + nv + 4 * nv + 128 * s_c,
        dict_page + 8 + 20 * nv + 4 * s_r + 128 * nv + nv + 2 * nv + 128 * s_i,
    ], np.uint64)


def column_chunks(n_vec, chunk_vectors=64):
    """(first vector, vector count) of every chunk of a column."""
    return [(c, min(chunk_vectors, n_vec - c)) for c in range(0, n_vec, chunk_vectors)]


# ---------------------------------------------------------------------------------------------------------
# Per-vector statistics of the learned selector
# ---------------------------------------------------------------------------------------------------------
def vector_stats(x, signed):
    """The integer statistics every feature is made of (exact)."""
    x = np.ascontiguousarray(x)
    w = x.dtype.itemsize * 8
    mask = (1 << w) - 1
    v = x.view(_ST[w]) if signed else x.view(_UT[w])
    vi = [int(t) for t in v]
    bw_f, bw_d, runs, bw_i = vector_parts(x, signed)
    vals, counts = np.unique(x, return_counts=True)
    mn, mx = min(vi), max(vi)
    inc = sum(1 for i in range(1, 1024) if vi[i] > vi[i - 1])
    dec = sum(1 for i in range(1, 1024) if vi[i] < vi[i - 1])
    bw_a = 0
    for i in range(1, 1024):
        d = (vi[i] - vi[i - 1]) & mask
        if d >> (w - 1):
            d = (-d) & mask
        bw_a = max(bw_a, _bits(d))
    maxrun, cur = 1, 1
    for i in range(1, 1024):
        cur = cur + 1 if vi[i] == vi[i - 1] else 1
        maxrun = max(maxrun, cur)
    cnt_top = 0
    if bw_f > 0:
        cnt_top = sum(1 for t in vi if (((t - mn) & mask) >> (bw_f - 1)) & 1)
    blk = sum(_range_bits(x[32 * b:32 * b + 32], w, signed) for b in range(32))
    mag = max(_bits(abs(t)) for t in vi) if signed else _bits(mx)
    return dict(w=w, signed=int(bool(signed)), bw_f=bw_f, bw_d=bw_d, runs=runs, bw_i=bw_i, dv=int(vals.size),
                top1=int(counts.max()), inc=inc, dec=dec, bw_a=bw_a, maxrun=maxrun, cnt_top=cnt_top, blk=blk,
                nzero=sum(1 for t in vi if t == 0), nmin=sum(1 for t in vi if t == mn),
                nmax=sum(1 for t in vi if t == mx), mag=mag)


def features(s):
    """32 float features of one vector from its statistics (float64 restatement of the device's float32)."""
    w, sz = s["w"], s["w"] // 8
    raw = 1024.0 * sz
    dv, r = s["dv"], s["runs"]
    cb = _bits(dv - 1)
    f = [
        s["bw_f"] / w, s["bw_d"] / w, r / 1024, s["bw_i"] / 16, dv / 1024, np.log2(dv) / 10, cb / 16,
        s["inc"] / 1023, s["dec"] / 1023, s["bw_a"] / w, s["maxrun"] / 1024, np.log2(1024 / r) / 10,
        s["top1"] / 1024, s["cnt_top"] / 1024, s["blk"] / (32 * w), w / 64, s["signed"],
        (1 + sz + 128 * s["bw_f"]) / raw, (129 + sz + 128 * s["bw_d"]) / raw,
        (r * sz + 131 + 128 * s["bw_i"]) / raw, (dv * sz + 5 + 128 * cb) / raw,
        (dv * sz + 4 * r + 131 + 128 * s["bw_i"]) / raw, s["mag"] / w, s["nzero"] / 1024, dv / r,
        np.log2(s["maxrun"]) / 10, _bits(s["top1"]) / 11, s["nmin"] / 1024, s["nmax"] / 1024,
        (s["bw_f"] - s["blk"] / 32) / w, 1.0 if s["bw_f"] == 0 else 0.0, 1.0 if s["dec"] == 0 else 0.0,
    ]
    return np.array(f, np.float64)


# ---------------------------------------------------------------------------------------------------------
# MLP 32 -> 128 -> 128 -> K, parameters flat: W1[32][128] b1[128] W2[128][128] b2[128] W3[128][K] b3[K]
# ---------------------------------------------------------------------------------------------------------
def param_count(k=K):
    return N_FEAT * HIDDEN + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN * k + k


def unpack_params(p, k=K):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((N_FEAT, HIDDEN), (HIDDEN,), (HIDDEN, HIDDEN), (HIDDEN,), (HIDDEN, k), (k,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def mlp_forward(p, x, k=K):
    w1, b1, w2, b2, w3, b3 = unpack_params(p, k)
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ w1 + b1, 0)
    h2 = np.maximum(h1 @ w2 + b2, 0)
    z = h2 @ w3 + b3
    e = np.exp(z - z.max(axis=1, keepdims=True))
    return e / e.sum(axis=1, keepdims=True), (x, h1, h2, z)


def mlp_grad(p, x, y, k=K):
    """Mean cross-entropy loss over the batch and its gradient (flat, the parameter layout)."""
    w1, b1, w2, b2, w3, b3 = unpack_params(p, k)
    prob, (x, h1, h2, z) = mlp_forward(p, x, k)
    n = x.shape[0]
    y = np.asarray(y, np.int64)
    loss = -np.mean(np.log(prob[np.arange(n), y]))
    dz = prob.copy()
    dz[np.arange(n), y] -= 1
    dz /= n
    gw3 = h2.T @ dz
    gb3 = dz.sum(0)
    dh2 = (dz @ w3.T) * (h2 > 0)
    gw2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    gw1 = x.T @ dh1
    gb1 = dh1.sum(0)
    return loss, np.concatenate([g.reshape(-1) for g in (gw1, gb1, gw2, gb2, gw3, gb3)])


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015, Algorithm 1); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
