"""Seeded synthetic workloads with the shapes of the FastLanes decode benchmarks, encoded on the GPU with this
library's own encoders (transpose_i -> ffor), so the packed bytes are exactly what the reference's
generated ffor would produce for the same values.

The reference measures on public datasets (public_bi, NextiaJD, ClickBench) that are not available here;
these generators stand in for them with the value distributions the benchmark configurations name.
"""
import ctypes

import numpy as np
import torch

from . import primitives as P
from ._lib import check, declare, lib

_p = ctypes.c_void_p


class _Batch(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint8), ("encoding", ctypes.c_uint8), ("order", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8), ("n_vec", ctypes.c_uint32), ("d_packed", _p), ("d_byte_off", _p),
                ("d_bw", _p), ("d_base", _p), ("d_lane_base", _p), ("d_out", _p)]


declare("fls_plan_create", ctypes.c_int, [ctypes.POINTER(_Batch), ctypes.c_uint32, _p, ctypes.c_uint64,
                                          ctypes.POINTER(_p)])
declare("fls_plan_create_ex", ctypes.c_int, [ctypes.POINTER(_Batch), ctypes.c_uint32, _p, ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.POINTER(_p)])
declare("fls_plan_decode", ctypes.c_int, [_p, _p])
declare("fls_plan_decode_grid", ctypes.c_int, [_p, ctypes.c_int, _p])
declare("fls_plan_destroy", ctypes.c_int, [_p])
declare("fls_plan_autotune", ctypes.c_int, [_p, ctypes.c_int, _p])
declare("fls_plan_variant_name", ctypes.c_char_p, [_p, ctypes.c_int])
declare("fls_plan_decode_graph", ctypes.c_int, [_p, _p])
declare("fls_plan_geometry", ctypes.c_int, [_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)])

_DT = {32: torch.uint32, 64: torch.uint64, 16: torch.uint16, 8: torch.uint8}
_SIGNED = {32: torch.int32, 64: torch.int64, 16: torch.int16, 8: torch.int8}


class FforColumn:
    """Packed FFOR vectors of one width, device resident: packed bytes, byte offsets, bw, base."""

    def __init__(self, width, packed, byte_off, bw, base, values=None):
        self.width, self.packed, self.byte_off, self.bw, self.base, self.values = (width, packed, byte_off, bw, base,
                                                                                   values)
        self.n_vec = bw.numel()

    @property
    def packed_bytes(self):
        return int((self.bw.to(torch.int64) * 128).sum().item())

    def algorithmic_read_bytes(self):
        """Packed words + per-vector bw byte + FOR base + 8-byte offset."""
        return self.packed_bytes + self.n_vec * (1 + self.width // 8 + 8)

    def decoded_bytes(self):
        return self.n_vec * 1024 * self.width // 8


def random_ffor_column(width, n_vec, rng, device, keep_values=False):
    """Vectors whose bit width is uniform in 0..width and whose base is uniform in [0, 2^width - 2^bw];
    values = base + uniform[0, 2^bw)."""
    bw = rng.integers(0, width + 1, n_vec)
    hi = (np.uint64(0) - (np.uint64(1) << bw.astype(np.uint64))) if width == 64 else \
        ((1 << width) - (1 << bw)).astype(np.uint64)
    if width == 64:
        hi = np.where(bw == 64, np.uint64(0), hi)  # 2^64 - 2^64 = 0
        hi = np.where(bw == 0, np.uint64(np.iinfo(np.uint64).max), hi)
    base = rng.integers(0, hi, dtype=np.uint64, endpoint=True)
    g = torch.Generator(device=device)
    g.manual_seed(int(rng.integers(0, 1 << 62)))
    bits = torch.randint(-(1 << 63), (1 << 63) - 1, (n_vec, 1024), dtype=torch.int64, device=device, generator=g)
    bw_t = torch.from_numpy(bw.astype(np.int64)).to(device)
    mask = torch.where(bw_t >= 64, torch.full_like(bw_t, -1), (torch.ones_like(bw_t) << bw_t.clamp(max=63)) - 1)
    base_i64 = torch.from_numpy(base.view(np.int64)).to(device)
    vals = (bits & mask[:, None]) + base_i64[:, None]
    if width < 64:
        vals = (vals & ((1 << width) - 1)).to(_SIGNED[width]).view(_DT[width])
    else:
        vals = vals.view(torch.uint64)
    vals = vals.reshape(-1).contiguous()
    tr = P.transpose_i(vals)
    bw_d = torch.from_numpy(bw.astype(np.uint8)).to(device)
    base_d = torch.from_numpy(base.astype(np.uint64)).to(device)
    if width < 64:
        base_d = base_d.view(torch.int64).to(_SIGNED[width]).view(_DT[width])
    else:
        base_d = base_d.view(torch.uint64)
    packed, off = P.ffor(tr, bw_d, base_d)
    return FforColumn(width, packed, off, bw_d, base_d, vals if keep_values else None)


class Plan:
    """A decode plan over several FFOR columns (fls_plan_create / fls_plan_decode)."""

    def __init__(self, columns, outs, order, queue=None, keep_order=False):
        batches = (_Batch * len(columns))()
        for i, (c, o) in enumerate(zip(columns, outs)):
            b = batches[i]
            b.width, b.encoding, b.order, b.n_vec = c.width, 1, order, c.n_vec
            b.d_packed, b.d_byte_off, b.d_bw, b.d_base = (c.packed.data_ptr(), c.byte_off.data_ptr(),
                                                          c.bw.data_ptr(), c.base.data_ptr())
            b.d_lane_base, b.d_out = None, o.data_ptr()
        self._keep = (columns, outs, queue)
        h = _p()
        n_items = queue.numel() if queue is not None else 0
        check(lib.fls_plan_create_ex(batches, len(columns), queue.data_ptr() if queue is not None else None, n_items,
                                     1 if keep_order else 0, ctypes.byref(h)), "fls_plan_create")
        self.handle = h

    def decode(self, stream=None, grid=0):
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib.fls_plan_decode_grid(self.handle, grid, s), "fls_plan_decode")

    def decode_graph(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib.fls_plan_decode_graph(self.handle, s), "fls_plan_decode_graph")

    def autotune(self, reps=3, stream=None):
        """Pick the fastest geometry variant per launch segment (runs decodes); returns the variants' names."""
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib.fls_plan_autotune(self.handle, reps, s), "fls_plan_autotune")
        return [n for n in (lib.fls_plan_variant_name(self.handle, i).decode() for i in (0, 1)) if n]

    def geometry(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib.fls_plan_geometry(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "geometry")
        return a.value, b.value, c.value

    def close(self):
        if self.handle:
            lib.fls_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bw_sweep(n32=65536, n64=32768, seed=0, device="cuda", keep_values=False):
    """Batched bit-width sweep: 64 Mi u32 + 32 Mi u64 values in 1024-value vectors, per-vector bit width uniform
    in 0..32 / 0..64, vectors of both widths interleaved in a shuffled work queue."""
    rng = np.random.default_rng(seed)
    c32 = random_ffor_column(32, n32, rng, device, keep_values)
    c64 = random_ffor_column(64, n64, rng, device, keep_values)
    items = np.concatenate([np.arange(n32, dtype=np.uint32), (1 << 24) | np.arange(n64, dtype=np.uint32)])
    items = items[rng.permutation(items.size)]
    queue = torch.from_numpy(items.view(np.int32)).to(device)
    return [c32, c64], queue


# ---------------------------------------------------------------------------------------------------------------
# Page workloads (host arrays -> reference-format pages through the engine's own encoders)
# ---------------------------------------------------------------------------------------------------------------
def ffor_u32_bw7(n_vec=1024, seed=0):
    """1024 vectors; per vector base ~ U[0, 2^20), values = base + U[0, 2^7); FOR with the drawn base at bw 7.
    Returns (packed bytes, byte offsets, bw, base, transposed values) as numpy arrays."""
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 1 << 20, n_vec).astype(np.uint32)
    vals = (rng.integers(0, 1 << 7, (n_vec, 1024)) + base[:, None]).astype(np.uint32)
    return base, vals


def delta_timestamps(n=32 << 20, seed=0):
    """Sorted int64 timestamps from 1.6e18 with geometric(p = 0.1, support >= 1, mean 10) gaps."""
    rng = np.random.default_rng(seed)
    gaps = rng.geometric(0.1, n).astype(np.int64)
    return (1_600_000_000_000_000_000 + np.cumsum(gaps)).astype(np.int64)


def rle_int32(n=32 << 20, seed=0):
    """int32 run values ~ U[0, 1e6) with geometric(mean 8) run lengths."""
    rng = np.random.default_rng(seed)
    runs = rng.geometric(1 / 8, n // 4 + 1024)
    vals = rng.integers(0, 10**6, runs.size).astype(np.int32)
    out = np.repeat(vals, runs)
    return out[:n].copy()


def string_dictionary(seed=0, n_dict=4096, n_tokens=256):
    """n_dict strings of uniform length 5..40 over a 64-symbol alphabet, each made of Zipf(1.2)-chosen tokens
    out of n_tokens seeded 2..6-byte tokens.  Returns (bytes, offsets[n_dict + 1])."""
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789-_", np.uint8)
    tokens = [bytes(alphabet[rng.integers(0, 64, rng.integers(2, 7))]) for _ in range(n_tokens)]
    picks = (rng.zipf(1.2, n_dict * 64) - 1) % n_tokens
    out, j = [], 0
    for _ in range(n_dict):
        target = int(rng.integers(5, 41))
        s = b""
        while len(s) < target:
            s += tokens[picks[j]]
            j += 1
        out.append(s[:target])
    offs = np.zeros(n_dict + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in out])
    return np.frombuffer(b"".join(out), np.uint8).copy(), offs


def zipf_codes(n_rows=16 << 20, n_dict=4096, a=1.1, seed=0):
    rng = np.random.default_rng(seed)
    return ((rng.zipf(a, n_rows) - 1) % n_dict).astype(np.uint32)


STRING_SELECTION_FAMILIES = ("dict_tokens", "dict_runs", "unique_tokens", "random_bytes", "few_long")


def _gather_rows(dbytes, doffs, codes):
    """Arrow (bytes, offsets) of rows = dictionary entries codes[r]."""
    lens = np.diff(doffs).astype(np.int64)[codes]
    offs = np.zeros(codes.size + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    idx = np.repeat(doffs[:-1][codes].astype(np.int64) - offs[:-1].astype(np.int64), lens)
    idx += np.arange(idx.size, dtype=np.int64)
    return dbytes[idx], offs


def dict_rows_device(dict_bytes, dict_offsets, codes, device="cuda", chunk_rows=1 << 22):
    """Arrow rows = dictionary entries codes[r], built on the device chunk by chunk: (bytes uint8, offsets
    int64[n + 1]) tensors."""
    db = torch.from_numpy(np.ascontiguousarray(dict_bytes, np.uint8)).to(device)
    do = torch.from_numpy(np.asarray(dict_offsets).astype(np.int64)).to(device)
    cd = torch.from_numpy(np.asarray(codes).astype(np.int64)).to(device)
    lens = (do[1:] - do[:-1])[cd]
    offs = torch.zeros(cd.numel() + 1, dtype=torch.int64, device=device)
    offs[1:] = torch.cumsum(lens, 0)
    out = torch.empty(int(offs[-1]) + 16, dtype=torch.uint8, device=device)
    for a in range(0, cd.numel(), chunk_rows):
        b = min(cd.numel(), a + chunk_rows)
        o0, o1 = int(offs[a]), int(offs[b])
        rows = torch.repeat_interleave(torch.arange(a, b, device=device), lens[a:b])
        out[o0:o1] = db[do[cd[rows]] + (torch.arange(o0, o1, device=device) - offs[rows])]
    return out, offs


def string_selection_column(rng, n_vec, family=None):
    """A seeded string column of n_vec vectors for expression selection: (bytes, offsets[n + 1] uint64, FSST
    table bytes trained on a sample of its rows).  Families: token dictionaries with Zipf codes (DICT), the same
    in runs (DICT_RLE), every row a fresh token string (FSST), random bytes (BYTE_ARR), a few long strings."""
    from .strings import fsst_compress

    n = n_vec * 1024
    family = family or STRING_SELECTION_FAMILIES[rng.integers(0, len(STRING_SELECTION_FAMILIES))]
    seed = int(rng.integers(0, 2 ** 31))
    if family in ("dict_tokens", "dict_runs"):
        dbytes, doffs = string_dictionary(seed=seed, n_dict=int(rng.integers(16, 4097)))
        d = doffs.size - 1
        if family == "dict_tokens":
            codes = _zipf_codes(n, d, float(rng.uniform(0.8, 1.5)), torch.Generator().manual_seed(seed), "cpu").numpy()
        else:
            runs = rng.geometric(1.0 / float(rng.uniform(2, 64)), n)
            codes = np.repeat(rng.integers(0, d, runs.size), runs)[:n]
        byts, offs = _gather_rows(dbytes, doffs, codes)
    elif family == "unique_tokens":
        dbytes, doffs = string_dictionary(seed=seed, n_dict=n)
        byts, offs = dbytes, doffs
    elif family == "random_bytes":
        lens = rng.integers(1, 41, n)
        offs = np.zeros(n + 1, np.uint64)
        offs[1:] = np.cumsum(lens)
        byts = rng.integers(0, 256, int(offs[-1]), dtype=np.uint8)
    else:  # few_long
        d = int(rng.integers(4, 17))
        lens = rng.integers(100, 256, d)
        doffs = np.zeros(d + 1, np.uint64)
        doffs[1:] = np.cumsum(lens)
        dbytes = rng.integers(97, 123, int(doffs[-1]), dtype=np.uint8)
        codes = _zipf_codes(n, d, 1.2, torch.Generator().manual_seed(seed), "cpu").numpy()
        byts, offs = _gather_rows(dbytes, doffs, codes)
    m = min(n, 4096)  # the table is trained on the column's first rows
    table, _, _ = fsst_compress(byts[:int(offs[m])], offs[:m + 1])
    return np.ascontiguousarray(byts, np.uint8), offs, table


def dict_rows_match(offsets, data, dict_bytes, dict_offsets, codes, chunk_rows=1 << 22):
    """Whole-buffer parity of decoded DICT string rows: `offsets` (int32, n + 1) and `data` (uint8) on the device
    against the rows the generator meant -- row r is dictionary entry codes[r] -- built on the device by a
    gather over the dictionary, chunk by chunk, every byte compared.  dict_bytes / dict_offsets / codes: host
    arrays."""
    dev = data.device
    db = torch.from_numpy(np.ascontiguousarray(dict_bytes, np.uint8)).to(dev)
    do = torch.from_numpy(np.asarray(dict_offsets).astype(np.int64)).to(dev)
    cd = torch.from_numpy(np.asarray(codes).astype(np.int64)).to(dev)
    n = cd.numel()
    lens = (do[1:] - do[:-1])[cd]
    want = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    want[1:] = torch.cumsum(lens, 0)
    if offsets.numel() != n + 1 or not torch.equal(offsets.to(torch.int64) & 0xFFFFFFFF, want):
        return False
    if data.numel() < int(want[-1]):
        return False
    for a in range(0, n, chunk_rows):
        b = min(n, a + chunk_rows)
        o0, o1 = int(want[a]), int(want[b])
        rows = torch.repeat_interleave(torch.arange(a, b, device=dev), lens[a:b])
        src = do[cd[rows]] + (torch.arange(o0, o1, device=dev) - want[rows])
        if not torch.equal(data[o0:o1], db[src]):
            return False
    return True


# ---- integer columns for expression selection ------------------------------------------------------------
SELECTION_FAMILIES = ("for_u32", "for_i64", "delta_i64", "rle", "dict_i32", "dict_rle", "noise")


def _zipf_codes(n, d, a, g, device):
    """n codes over d entries with P(k) proportional to 1 / (k + 1)^a (inverse CDF)."""
    k = torch.arange(1, d + 1, dtype=torch.float64, device=device)
    cdf = torch.cumsum(k.pow(-a), 0)
    cdf /= cdf[-1].clone()
    u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
    return torch.searchsorted(cdf, u).clamp_(max=d - 1)


def _runs(n, mean, g, device):
    """Run id of each of n positions, run lengths geometric with the given mean."""
    m = int(n / mean * 2) + 16
    lens = torch.empty(m, device=device, dtype=torch.float64).geometric_(1.0 / mean, generator=g).long()
    ends = torch.cumsum(lens, 0)
    pos = torch.arange(n, device=device, dtype=torch.int64)
    return torch.searchsorted(ends, pos, right=True)


def selection_column(rng, n_vec, device="cuda", family=None):
    """One seeded integer column of n_vec vectors from a family of the mixed row-group workload, with random
    parameters: FOR u32 / i64 (random bit width), sorted i64 timestamps (geometric gaps), runs (geometric
    lengths, mean 2..64), low-cardinality int32 dictionaries (16..65,536 entries, Zipf 0.8..1.5), the same with
    runs, and incompressible noise.  Returns (tensor, is_signed): int32 / int64 on `device`."""
    fam = family or SELECTION_FAMILIES[rng.choice(len(SELECTION_FAMILIES), p=(.2, .2, .15, .15, .15, .1, .05))]
    g = torch.Generator(device=device)
    g.manual_seed(int(rng.integers(0, 2 ** 62)))
    n = n_vec * 1024
    if fam == "for_u32":
        bw = int(rng.integers(0, 33))
        base = int(rng.integers(0, 2 ** 32 - 2 ** bw + 1))
        v = torch.randint(0, 2 ** bw, (n,), generator=g, device=device, dtype=torch.int64) + base
        return v.to(torch.int32), False
    if fam == "for_i64":
        bw = int(rng.integers(0, 63))
        base = int(rng.integers(-2 ** 62, 2 ** 62 - 2 ** bw + 1))
        return torch.randint(0, 2 ** bw, (n,), generator=g, device=device, dtype=torch.int64) + base, True
    if fam == "delta_i64":
        mean = float(np.exp(rng.uniform(0, np.log(4096))))
        gaps = torch.empty(n, device=device, dtype=torch.float64).geometric_(1.0 / max(mean, 1.0), generator=g)
        t0 = 1_600_000_000_000_000_000 + int(rng.integers(0, 2 ** 40))
        return torch.cumsum(gaps.long() - 1, 0) + t0, True
    if fam == "rle":
        wide = bool(rng.integers(0, 2))
        run = _runs(n, float(rng.uniform(2, 64)), g, device)
        bw = int(rng.integers(1, 41 if wide else 32))
        vals = torch.randint(0, 2 ** bw, (int(run[-1]) + 1,), generator=g, device=device, dtype=torch.int64)
        v = vals[run]
        return (v, True) if wide else (v.to(torch.int32), False)
    if fam in ("dict_i32", "dict_rle"):
        d = int(np.exp(rng.uniform(np.log(16), np.log(65536))))
        bw = int(rng.integers(8, 32))
        dic = torch.randint(-2 ** bw, 2 ** bw, (d,), generator=g, device=device, dtype=torch.int64)
        a = float(rng.uniform(0.8, 1.5))
        if fam == "dict_i32":
            codes = _zipf_codes(n, d, a, g, device)
        else:
            run = _runs(n, float(rng.uniform(2, 64)), g, device)
            codes = _zipf_codes(int(run[-1]) + 1, d, a, g, device)[run]
        return dic[codes].to(torch.int32), True
    wide = bool(rng.integers(0, 2))
    v = torch.randint(-2 ** 62, 2 ** 62, (n,), generator=g, device=device, dtype=torch.int64) * 2 + 1
    return (v, True) if wide else (v.to(torch.int32), False)


# ---- the mixed row-group workload ------------------------------------------------------------------------
MIXED_KINDS = ("for", "delta", "rle", "dict", "strings")


def mixed_rowgroup_columns(rng, n_cols=256, device="cuda", min_vec=64, max_vec=4096):
    """Columns of uneven lengths (U[min_vec, max_vec] vectors, i.e. 64 Ki..4 Mi values) whose types are drawn
    uniformly from: u32 / i64 FOR with a random bit width; sorted i64 timestamps; runs (geometric mean 2..64);
    low-cardinality int32 Zipf dictionaries (16..65,536 entries, Zipf 0.8..1.5); FSST-able strings (a
    4096-entry dictionary of 5..40-byte token strings, Zipf(1.1) codes).  Returns (integer columns as
    (tensor, is_signed), string columns as (dictionary bytes, offsets, codes))."""
    ints, strs = [], []
    for _ in range(n_cols):
        kind = MIXED_KINDS[rng.integers(0, len(MIXED_KINDS))]
        n_vec = int(rng.integers(min_vec, max_vec + 1))
        if kind == "strings":
            seed = int(rng.integers(0, 2 ** 31))
            dbytes, doffs = string_dictionary(seed=seed)
            strs.append((dbytes, doffs, zipf_codes(n_vec * 1024, seed=seed + 1)))
            continue
        fam = {"for": ("for_u32", "for_i64")[rng.integers(0, 2)], "delta": "delta_i64", "rle": "rle",
               "dict": "dict_i32"}[kind]
        ints.append(selection_column(rng, n_vec, device, fam))
    return ints, strs


def fsst_rows(n_rows=8 << 20, seed=0):
    """The string column of the DICT+FSST configuration (dictionary strings picked by Zipf(1.1) codes) as an FSST
    column: every row FSST-compressed with one symbol table, built as the dictionary entries compressed once and
    gathered by code (the same bytes as compressing each row with that table).  Returns (table, compressed
    bytes, compressed offsets[n + 1], plain bytes, plain offsets[n + 1])."""
    from .strings import fsst_compress

    dbytes, doffs = string_dictionary(seed)
    codes = zipf_codes(n_rows, seed=seed)
    table, comp, coffs = fsst_compress(dbytes, doffs)

    def gather(src, offs):
        lens = np.diff(offs).astype(np.int64)[codes]
        out_offs = np.zeros(codes.size + 1, np.uint64)
        out_offs[1:] = np.cumsum(lens)
        idx = np.repeat(offs[:-1][codes].astype(np.int64) - out_offs[:-1].astype(np.int64), lens)
        idx += np.arange(idx.size, dtype=np.int64)
        return src[idx], out_offs

    cb, co = gather(comp, coffs.astype(np.uint64))
    pb, po = gather(dbytes, doffs.astype(np.uint64))
    return table, cb, co, pb, po
