"""Row groups of integer columns: every (column, row-group) chunk encoded with its own expression (chosen by
``select``), the pages placed in one device buffer, and all chunks decoded by one persistent launch.

Reference shape: a row group's columns each hold one expression per row group (include/fls/footer/
rowgroup_footer.hpp:23-75, src/reader/reader.cpp:19-61 reads them back chunk by chunk through the
Engine); here the reader is one page plan whose work queue spans every vector of every chunk.
"""
import numpy as np
import torch

from . import pages as PG
from .select import POOL_IDS


def shard_chunks(chunk_bytes, world_size):
    """Contiguous chunk ranges [begin, end) for each of world_size ranks with about equal bytes each (chunks are
    independent, so ranks decode their ranges with no exchange).  Every rank computes the same split."""
    w = np.asarray(chunk_bytes, np.float64)
    if world_size < 1:
        raise ValueError("world_size must be positive")
    prefix = np.concatenate([[0.0], np.cumsum(w)])
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world_size):
        # first boundary at or after r / world_size of the bytes, never before the previous cut
        cuts.append(max(cuts[-1], int(np.searchsorted(prefix, total * r / world_size, side="left"))))
    cuts.append(len(w))
    return [(cuts[r], cuts[r + 1]) for r in range(world_size)]


_DT = {(4, True): PG.INT32, (4, False): PG.UINT32, (8, True): PG.INT64, (8, False): PG.UINT64}
_UNSIGNED = {4: np.uint32, 8: np.uint64}


def encode_chunk(values, signed, candidate):
    """Pages of one chunk (host array of whole vectors) under selection candidate 0..5; returns
    (page, dictionary page or None)."""
    x = values if signed else values.view(_UNSIGNED[values.dtype.itemsize])
    if candidate <= 3:
        page, _ = PG.encode_from_memory(x, _DT[(values.dtype.itemsize, signed)], POOL_IDS[candidate])
        return page, None
    return PG.encode_int_dict(x, rle=candidate == 5)


class RowGroupSet:
    """Encoded chunks of a set of columns and their decoder.

    columns: list of (int32 / int64 tensor, is_signed); chunks: (col, first vector, vector count) arrays;
    choice: candidate per chunk.  The pages live in one device buffer, each at a 16-byte aligned offset
    (fls_page_placement), the dictionaries in another; outputs are one tensor per column (original order)."""

    def __init__(self, columns, chunks, choice, device="cuda", chunk_range=None):
        col, first, count = chunks
        choice = np.asarray(choice)
        if chunk_range is not None:  # one rank's share (shard_chunks): only these chunks are encoded and decoded
            b, e = chunk_range
            col, first, count, choice = col[b:e], first[b:e], count[b:e], choice[b:e]
        host = [t.cpu().numpy() for t, _ in columns]
        self.signed = [s for _, s in columns]
        pages, dicts, self.page_bytes, self.dict_bytes = [], [], 0, 0
        for c in range(len(col)):
            x = host[col[c]][int(first[c]) * 1024:(int(first[c]) + int(count[c])) * 1024]
            p, d = encode_chunk(x, self.signed[col[c]], int(choice[c]))
            pages.append(p)
            dicts.append(d)
            self.page_bytes += p.size
            self.dict_bytes += 0 if d is None else d.size
        # one buffer for the pages (each placed so its packed words start 16-byte aligned), one for dictionaries
        pos, blob, off = 64, [], []
        for p in pages:
            shift = PG.placement(p)
            start = (pos + 15) // 16 * 16 + shift
            blob.append((start, p))
            off.append(start)
            pos = start + p.size + 16
        buf = np.zeros(pos + 64, np.uint8)
        for start, p in blob:
            buf[start:start + p.size] = p
        dpos, dblob, doff = 0, [], []
        for d in dicts:
            if d is None:
                doff.append(None)
                continue
            start = (dpos + 15) // 16 * 16
            dblob.append((start, d))
            doff.append(start)
            dpos = start + d.size
        dbuf = np.zeros(max(dpos, 16) + 16, np.uint8)
        for start, d in dblob:
            dbuf[start:start + d.size] = d
        self.d_pages = torch.from_numpy(buf).to(device)
        self.d_dicts = torch.from_numpy(dbuf).to(device)
        self.outputs = [torch.empty_like(t, device=device) for t, _ in columns]
        base, dbase = self.d_pages.data_ptr(), self.d_dicts.data_ptr()
        self.columns = []
        for c in range(len(col)):
            t = self.outputs[col[c]]
            self.columns.append(dict(
                d_page=base + off[c], page_size=pages[c].size,
                d_dict=(dbase + doff[c]) if doff[c] is not None else None,
                dict_size=0 if dicts[c] is None else dicts[c].size,
                data_type=_DT[(t.element_size(), self.signed[col[c]])], order=1,
                d_out=t.data_ptr() + int(first[c]) * 1024 * t.element_size()))
        self.plan = PG.PagePlan(self.columns) if len(col) else None
        self.values = int(sum(int(n) * 1024 for n in count))
        self.value_bytes = int(sum(int(count[c]) * 1024 * self.outputs[col[c]].element_size() for c in range(len(col))))

    def decode(self, stream=None, graph=True):
        """Every chunk of the set: one plan, one persistent launch per kernel family present, replayed from a
        CUDA graph (graph=False launches directly)."""
        if self.plan is None:
            return
        if graph:
            self.plan.decode_graph(stream)
        else:
            self.plan.decode(stream)

    def autotune(self, reps=3):
        """Geometry variants chosen on this set's own data (see PagePlan.autotune)."""
        return self.plan.autotune(reps) if self.plan is not None else []

    def close(self):
        if self.plan is not None:
            self.plan.close()


class StringColumnSet:
    """String columns of a row-group set, each a DICT page (the string pool's DICT FFOR_NO_PATCH, id 3) over an
    FSST-compressed dictionary, all decoded by one string set (one kernel launch) into Arrow offsets + bytes.

    columns: list of (dictionary bytes, dictionary offsets, codes) host arrays.  decode() only launches
    (capturable in a CUDA graph together with the integer plan)."""

    def __init__(self, columns, device="cuda"):
        from . import strings as S

        self.plans, self.outputs, self._keep = [], [], []
        self.page_bytes = self.dict_bytes = self.rows = self.value_bytes = 0
        for dbytes, doffs, codes in columns:
            page, dic = S.encode_string_dict(dbytes, doffs, codes)
            shift = PG.placement(page)
            pb = torch.zeros(page.size + 64, dtype=torch.uint8, device=device)
            pb[shift:shift + page.size] = torch.from_numpy(page).to(device)
            db = torch.from_numpy(dic).to(device)
            plan = S.StringPlan(pb.data_ptr() + shift, page.size, db.data_ptr(), dic.size)
            n = plan.measure()
            offs = torch.empty(plan.n_rows + 1, dtype=torch.int32, device=device)
            data = torch.empty(n + 16, dtype=torch.uint8, device=device)
            self._keep.append((pb, db))
            self.plans.append(plan)
            self.outputs.append((offs, data, n))
            self.page_bytes += page.size
            self.dict_bytes += dic.size
            self.rows += plan.n_rows
            self.value_bytes += 4 * (plan.n_rows + 1) + n
        self.set = S.StringSet(self.plans)
        self.set.bind([o for o, _, _ in self.outputs], [d for _, d, _ in self.outputs])

    def decode(self, streams=None, join=True):
        """Every column's decode (one launch); with `streams`, on streams[0], ordered after the current stream
        and (with `join`) the current stream after it, so it overlaps other work on the current stream, also
        inside a CUDA graph capture.  join(streams) closes the fork."""
        if not streams:
            self.set.decode()
            return
        cur = torch.cuda.current_stream()
        streams[0].wait_stream(cur)
        with torch.cuda.stream(streams[0]):
            self.set.decode(stream=streams[0].cuda_stream)
        if join:
            self.join(streams)

    @staticmethod
    def join(streams):
        torch.cuda.current_stream().wait_stream(streams[0])

    def check(self, columns):
        """Every column's offsets and every byte against the generator's rows (row r is dictionary entry
        codes[r]), compared whole on the device."""
        from .workloads import dict_rows_match

        return all(dict_rows_match(offs, data[:n], dbytes, doffs, codes)
                   for (dbytes, doffs, codes), (offs, data, n) in zip(columns, self.outputs))

    def close(self):
        self.set.close()
        for p in self.plans:
            p.close()
