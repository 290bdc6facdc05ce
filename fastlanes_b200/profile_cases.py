"""Small, self-checking workloads of each kernel family, for profilers (``ncu -k <kernel> ...``).

    python -m fastlanes_b200.profile_cases strings --rows 8388608 --reps 3
    python -m fastlanes_b200.profile_cases rle --values 16777216 --reps 3
    python -m fastlanes_b200.profile_cases delta --values 16777216 --reps 3
    python -m fastlanes_b200.profile_cases mixed --columns 32 --reps 3
    python -m fastlanes_b200.profile_cases select --columns 32 --reps 3
    python -m fastlanes_b200.profile_cases filter --values 16777216 --reps 3
    python -m fastlanes_b200.profile_cases select_strings --columns 12 --reps 3

Each case builds its input, decodes (or selects) once and checks the result, then repeats the call `reps`
times, and prints one line with the mean time of the repeats (CUDA events; not a benchmark number).
"""
import argparse
import sys

import numpy as np
import torch


def _timed(fn, reps):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / max(reps, 1)


def case_strings(a):
    from . import pages as PG
    from . import strings as S
    from . import workloads as W

    dbytes, doffs = W.string_dictionary()
    codes = W.zipf_codes(a.rows)
    page, dic = S.encode_string_dict(dbytes, doffs, codes)
    shift = PG.placement(page)
    pb = torch.zeros(page.size + 64, dtype=torch.uint8, device="cuda")
    pb[shift:shift + page.size] = torch.from_numpy(page).cuda()
    db = torch.from_numpy(dic).cuda()
    plan = S.StringPlan(pb.data_ptr() + shift, page.size, db.data_ptr(), dic.size)
    n = plan.measure()
    offs = torch.empty(plan.n_rows + 1, dtype=torch.int32, device="cuda")
    data = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
    plan.decode_into(offs, data)
    lens = np.diff(doffs).astype(np.int64)
    want = np.zeros(codes.size + 1, np.int64)
    want[1:] = np.cumsum(lens[codes])
    if not np.array_equal(offs.cpu().numpy().astype(np.int64), want):
        raise SystemExit("strings: offsets mismatch")
    ms = _timed(lambda: plan.decode_into(offs, data), a.reps)
    plan.close()
    return f"strings rows={a.rows} bytes={n} ms={ms:.4f}"


def _page_case(values, dtype, expr, reps, name, autotune=False):
    from . import pages as PG

    page, _ = PG.encode_from_memory(values, dtype, expr)
    shift = PG.placement(page)
    buf = torch.zeros(page.size + 64, dtype=torch.uint8, device="cuda")
    buf[shift:shift + page.size] = torch.from_numpy(page).cuda()
    out = torch.empty(values.size, dtype=torch.from_numpy(values[:1]).dtype, device="cuda")
    plan = PG.PagePlan([dict(d_page=buf.data_ptr() + shift, page_size=page.size, data_type=dtype, order=1,
                             d_out=out.data_ptr())])
    plan.decode()
    if not np.array_equal(out.cpu().numpy(), values):
        raise SystemExit(f"{name}: mismatch")
    tuned = plan.autotune() if autotune else []
    ms = _timed(plan.decode, reps)
    plan.close()
    return f"{name} values={values.size} page={page.size} variants={tuned} ms={ms:.4f}"


def case_rle(a):
    from . import pages as PG
    from . import workloads as W

    return _page_case(W.rle_int32(a.values), PG.INT32, 6, a.reps, "rle", a.autotune)


def case_delta(a):
    from . import pages as PG
    from . import workloads as W

    return _page_case(W.delta_timestamps(a.values), PG.INT64, 11, a.reps, "delta", a.autotune)


def case_filter(a):
    """Filter plan (predicate pushdown) on the DELTA page of `values` sorted int64 timestamps: x > median."""
    from . import pages as PG
    from . import workloads as W

    values = W.delta_timestamps(a.values)
    page, _ = PG.encode_from_memory(values, PG.INT64, 11)
    shift = PG.placement(page)
    buf = torch.zeros(page.size + 64, dtype=torch.uint8, device="cuda")
    buf[shift:shift + page.size] = torch.from_numpy(page).cuda()
    c = int(np.median(values))
    bm = torch.empty(values.size // 8, dtype=torch.uint8, device="cuda")
    plan = PG.FilterPlan([dict(d_page=buf.data_ptr() + shift, page_size=page.size, data_type=PG.INT64, order=1,
                               d_out=bm.data_ptr())], PG.PRED_GT, c)
    plan.decode()
    want = np.packbits((values > c).astype(np.uint8).reshape(-1, 1024), axis=1, bitorder="little")
    if not np.array_equal(bm.cpu().numpy().reshape(-1, 128), want):
        raise SystemExit("filter: mismatch")
    ms = _timed(plan.decode, a.reps)
    plan.close()
    return f"filter values={values.size} page={page.size} ms={ms:.4f}"


def _columns(a):
    from . import workloads as W

    rng = np.random.default_rng(1)
    return [W.selection_column(rng, int(rng.integers(64, a.max_vectors + 1))) for _ in range(a.columns)]


def case_mixed(a):
    from . import rowgroups as RG
    from . import select as SL

    cols = _columns(a)
    plan = SL.SelectionPlan(cols)
    _, best, _ = plan.wizard()
    rg = RG.RowGroupSet(cols, plan.chunks(), best.cpu().numpy())
    rg.decode()
    torch.cuda.synchronize()
    if not all(torch.equal(o, t) for o, (t, _) in zip(rg.outputs, cols)):
        raise SystemExit("mixed: mismatch")
    if a.autotune:
        rg.autotune()
    rg.decode()  # (re)captures the plan's graph outside the timed repeats
    ms = _timed(rg.decode, a.reps)
    res = f"mixed chunks={plan.n_chunks} values={rg.values} read={rg.page_bytes + rg.dict_bytes} ms={ms:.4f}"
    rg.close()
    plan.close()
    return res


def case_select(a):
    from . import select as SL

    cols = _columns(a)
    plan = SL.SelectionPlan(cols)
    params = SL.mlp_init(0)
    plan.wizard()
    plan.learned(params, 8)
    ms = _timed(lambda: plan.learned(params, 8), a.reps)
    wms = _timed(plan.wizard, a.reps)
    res = f"select chunks={plan.n_chunks} ms={ms:.4f} wizard_ms={wms:.4f}"
    plan.close()
    return res


def case_select_strings(a):
    """Expression selection over string columns shaped as the mixed configuration's (4096-entry token
    dictionaries, Zipf(1.1) codes; --columns columns of 64 vectors ... --max-vectors vectors): the wizard and the
    learned path (an untrained network, no wizard fallback), each timed with CUDA events."""
    from . import select as SL
    from . import strings as S
    from . import workloads as W

    rng = np.random.default_rng(1)
    cols = []
    for _ in range(a.columns):
        seed = int(rng.integers(0, 2 ** 31))
        dbytes, doffs = W.string_dictionary(seed=seed)
        codes = W.zipf_codes(int(rng.integers(64, a.max_vectors + 1)) * 1024, seed=seed + 1)
        sb, so = W.dict_rows_device(dbytes, doffs, codes, "cuda")
        table, _, _ = S.fsst_compress(dbytes, doffs)
        cols.append((sb, so, table))
    plan = SL.StrSelectionPlan(cols)
    params = SL.mlp_init(0)
    plan.wizard()
    plan.learned(params, 8)
    wms = _timed(plan.wizard, a.reps)
    ms = _timed(lambda: plan.learned(params, 8), a.reps)
    res = f"select_strings chunks={plan.n_chunks} ms={ms:.4f} wizard_ms={wms:.4f}"
    plan.close()
    return res


def case_fsst(a):
    """The DICT+FSST configuration's rows as an FSST column (string pool id 13)."""
    from . import strings as S
    from . import workloads as W

    table, cb, co, pbytes, poffs = W.fsst_rows(a.rows)
    page, dic = S.fsst_page(table, cb, co)
    pg = torch.from_numpy(page).cuda()
    dc = torch.from_numpy(dic).cuda()
    plan = S.StringPlan(pg.data_ptr(), page.size, dc.data_ptr(), dic.size)
    n = plan.measure()
    offs = torch.empty(plan.n_rows + 1, dtype=torch.int32, device="cuda")
    data = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
    plan.decode_into(offs, data)
    if n != pbytes.size or not np.array_equal(offs.cpu().numpy().astype(np.int64), poffs.astype(np.int64)):
        raise SystemExit("fsst: offsets mismatch")
    if not torch.equal(data[:n], torch.from_numpy(pbytes).cuda()):
        raise SystemExit("fsst: bytes mismatch")
    ms = _timed(lambda: plan.decode_into(offs, data), a.reps)
    plan.close()
    return f"fsst rows={a.rows} bytes={n} compressed={cb.size} ms={ms:.4f}"


CASES = {"strings": case_strings, "rle": case_rle, "delta": case_delta, "mixed": case_mixed, "select": case_select,
         "filter": case_filter, "fsst": case_fsst, "select_strings": case_select_strings}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--rows", type=int, default=8 << 20)
    ap.add_argument("--values", type=int, default=16 << 20)
    ap.add_argument("--columns", type=int, default=32)
    ap.add_argument("--max-vectors", type=int, default=1024)
    ap.add_argument("--autotune", action="store_true", help="pick the plan's geometry variants first (as bench.py)")
    a = ap.parse_args(argv)
    print(CASES[a.case](a))
    return 0


if __name__ == "__main__":
    sys.exit(main())
