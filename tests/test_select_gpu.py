"""Expression selection on the GPU against the CPU oracle (oracle/select.py): exact per-vector quantities and
chunk sizes, the features, the MLP's forward / gradient / Adam kernels, training and the learned selector."""
import numpy as np
import pytest

from oracle import select as SEL

pytestmark = pytest.mark.gpu

FAMS = ("for_u32", "for_i64", "delta_i64", "rle", "dict_i32", "dict_rle", "noise")


def _cols(seed=0, n_vec=3, fams=FAMS, reps=2):
    import torch

    from fastlanes_b200 import workloads as W

    rng = np.random.default_rng(seed)
    cols = [W.selection_column(rng, n_vec, "cpu", f) for f in fams for _ in range(reps)]
    return [(t.cuda(), s) for t, s in cols], [(t.numpy(), s) for t, s in cols]


def _edge_cols():
    """Constant, ramp, alternating signs, the all-ones 64-bit value (the hash's empty key), full-range."""
    import torch

    rng = np.random.default_rng(5)
    h = [
        (np.full(2048, 7, np.int32), False),
        (np.arange(2048, dtype=np.int64), True),
        (np.tile(np.array([-1, 1], np.int64), 1024), True),
        (np.tile(np.array([-1, 1], np.int64), 1024), False),
        (np.where(rng.random(2048) < 0.5, -1, 3).astype(np.int64), False),
        (rng.integers(-2 ** 31, 2 ** 31, 2048).astype(np.int32), True),
        (np.repeat(np.arange(128, dtype=np.int32), 16), False),
    ]
    return [(torch.from_numpy(x).cuda(), s) for x, s in h], h


def _unsigned(x):
    return x.view(np.uint32 if x.dtype.itemsize == 4 else np.uint64)


def test_vector_parts_exact(cuda):
    from fastlanes_b200 import select as S

    dcols, hcols = _cols()
    e_d, e_h = _edge_cols()
    dcols += e_d
    hcols += e_h
    plan = S.SelectionPlan(dcols)
    got = plan.vector_parts().cpu().numpy().astype(np.uint32)
    i = 0
    for x, sgn in hcols:
        u = _unsigned(x)
        for v in range(u.size // 1024):
            bw_f, bw_d, runs, bw_i = SEL.vector_parts(u[v * 1024:(v + 1) * 1024], sgn)
            p = int(got[i])
            assert (p & 127, (p >> 7) & 127, (p >> 14) & 31, p >> 19) == (bw_f, bw_d, bw_i, runs), (i, x.dtype, sgn)
            i += 1
    assert i == got.size
    plan.close()


@pytest.mark.parametrize("chunk_vectors", [2, 3])
def test_wizard_sizes_exact(cuda, chunk_vectors):
    from fastlanes_b200 import select as S

    dcols, hcols = _cols(1, n_vec=5, reps=1)
    e_d, e_h = _edge_cols()
    dcols += e_d
    hcols += e_h
    plan = S.SelectionPlan(dcols, chunk_vectors)
    sizes, best, dn = plan.wizard()
    sizes, best, dn = sizes.cpu().numpy(), best.cpu().numpy(), dn.cpu().numpy()
    col, first, count = plan.chunks()
    for c in range(plan.n_chunks):
        x, sgn = hcols[col[c]]
        u = _unsigned(x)[int(first[c]) * 1024:(int(first[c]) + int(count[c])) * 1024]
        want = SEL.chunk_sizes(u, sgn)
        assert sizes[c].tolist() == want.astype(np.int64).tolist(), (c, x.dtype, sgn)
        assert best[c] == int(np.argmin(want))
        assert dn[c] == SEL.chunk_dictionary(u)[0]
    plan.close()


def _many_distinct_cols():
    """Full 64-vector chunks around the chunk dictionary's shared-memory capacity (12,288 distinct values):
    exactly at it and one past it, 13,000 and 40,000 values spread over the chunk, 65,536 distinct full-range
    values with the all-ones key among them, and a chunk whose second half brings 20,000 new values after a
    first half of 6,000.  Each column is 84 vectors: a full chunk and a partial one."""
    import torch

    rng = np.random.default_rng(17)
    n = 84 * 1024

    def spread(d, dtype):
        pool = rng.permutation(np.arange(d, dtype=np.int64) * 7919 + 11).astype(dtype)
        return pool[np.concatenate([np.arange(d), rng.integers(0, d, n - d)])[rng.permutation(n)]]

    full = rng.integers(-2 ** 63, 2 ** 63 - 1, n, dtype=np.int64)
    full[[5, 4097, 70000]] = -1
    half = np.concatenate([rng.integers(0, 6000, 32 * 1024), rng.integers(6000, 26000, n - 32 * 1024)])
    h = [
        (spread(12288, np.int64), True),
        (spread(12289, np.int64), False),
        (spread(13000, np.int32), True),
        (spread(40000, np.int32), False),
        (full, True),
        (half.astype(np.int64), True),
    ]
    return [(torch.from_numpy(x).cuda(), s) for x, s in h], h


def test_wizard_sizes_exact_for_chunks_of_many_distinct_values(cuda):
    """64-vector chunks past the shared-memory dictionary's capacity go through the hash buckets: the same exact
    dictionary sizes, code widths and candidate sizes as the oracle's."""
    from fastlanes_b200 import select as S

    dcols, hcols = _many_distinct_cols()
    plan = S.SelectionPlan(dcols, 64)
    sizes, best, dn = plan.wizard()
    sizes, best, dn = sizes.cpu().numpy(), best.cpu().numpy(), dn.cpu().numpy()
    col, first, count = plan.chunks()
    assert plan.n_chunks == 2 * len(hcols)
    for c in range(plan.n_chunks):
        x, sgn = hcols[col[c]]
        u = _unsigned(x)[int(first[c]) * 1024:(int(first[c]) + int(count[c])) * 1024]
        want = SEL.chunk_sizes(u, sgn)
        assert dn[c] == SEL.chunk_dictionary(u)[0], (c, x.dtype, sgn)
        assert sizes[c].tolist() == want.astype(np.int64).tolist(), (c, x.dtype, sgn)
        assert best[c] == int(np.argmin(want))
    from fastlanes_b200 import primitives as P

    assert P.device_status() == 0
    plan.close()


def test_wizard_sizes_equal_encoded_page_sizes(cuda):
    """Candidates 0 / 1 / 2 / 3 are exactly the pages fastlanes.h's encoder writes (ids 0, 1, 6, 11)."""
    from fastlanes_b200 import pages as PG
    from fastlanes_b200 import select as S

    dcols, hcols = _cols(2, n_vec=4, fams=("for_i64", "delta_i64", "rle", "for_u32"), reps=1)
    plan = S.SelectionPlan(dcols, 4)
    sizes = plan.wizard()[0].cpu().numpy()
    dt = {(8, True): PG.INT64, (8, False): PG.UINT64, (4, True): PG.INT32, (4, False): PG.UINT32}
    for c, (x, sgn) in enumerate(hcols):
        for cand, expr in ((0, 0), (1, 1), (2, 6), (3, 11)):
            page, _ = PG.encode_from_memory(x if sgn else _unsigned(x), dt[(x.dtype.itemsize, sgn)], expr)
            assert page.size == sizes[c, cand], (c, cand)
    plan.close()


def test_dictionary_candidates_equal_encoded_sizes_and_round_trip(cuda):
    """Candidates 4 / 5 are exactly the int DICT / DICT_RLE pages fls_encode_int_dict writes (codes page +
    dictionary page), and those pages decode back to the column."""
    import torch

    from fastlanes_b200 import pages as PG
    from fastlanes_b200 import select as S

    dcols, hcols = _cols(4, n_vec=3, fams=("dict_i32", "dict_rle", "rle", "for_i64"), reps=1)
    plan = S.SelectionPlan(dcols, 3)
    sizes = plan.wizard()[0].cpu().numpy()
    dt = {(8, True): PG.INT64, (8, False): PG.UINT64, (4, True): PG.INT32, (4, False): PG.UINT32}
    for c, (x, sgn) in enumerate(hcols):
        for cand, rle in ((4, False), (5, True)):
            page, dic = PG.encode_int_dict(x, rle=rle)
            assert page.size + dic.size == sizes[c, cand], (c, cand)
            dp = torch.from_numpy(np.concatenate([page, np.zeros(64, np.uint8)])).cuda()
            dd = torch.from_numpy(dic).cuda()
            out = torch.empty(x.size, dtype=torch.from_numpy(x[:1]).dtype, device="cuda")
            PG.decode_pages([dict(d_page=dp.data_ptr(), page_size=page.size, d_dict=dd.data_ptr(),
                                  dict_size=dic.size, data_type=dt[(x.dtype.itemsize, sgn)], order=1,
                                  d_out=out.data_ptr())])
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy(), x), (c, cand)
    plan.close()


def test_features_match_oracle(cuda):
    from fastlanes_b200 import select as S

    dcols, hcols = _cols(3, n_vec=2, reps=1)
    e_d, e_h = _edge_cols()
    dcols += e_d
    hcols += e_h
    plan = S.SelectionPlan(dcols)
    feat, rc = plan.features(1)
    feat = feat.cpu().numpy()
    i = 0
    for x, sgn in hcols:
        u = _unsigned(x)
        for v in range(u.size // 1024):
            want = SEL.features(SEL.vector_stats(u[v * 1024:(v + 1) * 1024], sgn))
            assert np.allclose(feat[i], want, rtol=1e-5, atol=1e-6), (i, np.flatnonzero(~np.isclose(feat[i], want)))
            i += 1
    # sampling: vectors 0, 2, ... of every chunk
    f2, rc2 = plan.features(2)
    assert f2.shape[0] == sum((u.size // 1024 + 1) // 2 for u, _ in hcols)
    plan.close()


def test_mlp_forward_and_gradient_match_oracle(cuda):
    import torch

    from fastlanes_b200 import select as S

    rng = np.random.default_rng(4)
    p = rng.normal(0, 0.2, SEL.param_count()).astype(np.float32)
    x = rng.uniform(0, 1, (200, SEL.N_FEAT)).astype(np.float32)
    y = rng.integers(0, SEL.K, 200)
    pd, xd = torch.from_numpy(p).cuda(), torch.from_numpy(x).cuda()
    prob = S.mlp_forward(pd, xd).cpu().numpy()
    want, _ = SEL.mlp_forward(p, x)
    assert np.allclose(prob, want, rtol=1e-4, atol=1e-6)
    loss, g = S.mlp_grad(pd, xd, torch.from_numpy(y).cuda())
    wl, wg = SEL.mlp_grad(p, x, y)
    assert abs(loss - wl) <= 1e-4 * abs(wl)
    g = g.cpu().numpy()
    assert np.allclose(g, wg, rtol=1e-3, atol=1e-6 * np.abs(wg).max())


def test_adam_step_matches_oracle(cuda):
    import torch

    from fastlanes_b200 import select as S

    rng = np.random.default_rng(6)
    n = SEL.param_count()
    p, g, m, v = (rng.normal(0, 1, n).astype(np.float32) for _ in range(4))
    v = np.abs(v)
    pd, gd, md, vd = (torch.from_numpy(a.copy()).cuda() for a in (p, g, m, v))
    S.adam_step(pd, gd, md, vd, 3, lr=1e-2)
    wp, wm, wv = SEL.adam(p.astype(np.float64), g, m, v, 3, lr=1e-2)
    assert np.allclose(pd.cpu().numpy(), wp, rtol=1e-5, atol=1e-6)
    assert np.allclose(md.cpu().numpy(), wm, rtol=1e-5, atol=1e-7)
    assert np.allclose(vd.cpu().numpy(), wv, rtol=1e-5, atol=1e-7)


def test_training_replays_match_stepwise_adam(cuda):
    """fls_sel_train (graph replays) equals the same minibatches through mlp_grad + adam_step."""
    import torch

    from fastlanes_b200 import select as S

    rng = np.random.default_rng(8)
    x = torch.from_numpy(rng.uniform(0, 1, (512, SEL.N_FEAT)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.integers(0, SEL.K, 512).astype(np.int32)).cuda()
    p0 = S.mlp_init(3)
    p1 = p0.clone()
    hist = S.train(p1, x, y, epochs=2, batch=128, lr=1e-2, seed=5)
    prng = np.random.default_rng(5)
    perm = np.concatenate([prng.permutation(512) for _ in range(2)])
    p2 = p0.clone()
    m, v = torch.zeros_like(p2), torch.zeros_like(p2)
    for s in range(8):
        idx = torch.from_numpy(perm[s * 128:(s + 1) * 128].astype(np.int64)).cuda()
        loss, g = S.mlp_grad(p2, x[idx], y[idx])
        assert abs(loss - hist[s]) <= 1e-4 * abs(loss) + 1e-6
        S.adam_step(p2, g, m, v, s + 1, lr=1e-2)
    assert torch.allclose(p1, p2, rtol=1e-4, atol=1e-6)


def test_learned_selection_after_training(cuda):
    """Trained on wizard labels, the selector's choices lose little against the wizard on held-out chunks, and
    a threshold above every confidence sends every chunk to the wizard (choices then equal the wizard's)."""
    import torch

    from fastlanes_b200 import select as S
    from fastlanes_b200 import workloads as W

    params, hist = S.train_selector(n_chunks=600, seed=11, epochs=12, batch=512, lr=2e-3)
    assert hist[-20:].mean() < hist[:20].mean() * 0.6
    rng = np.random.default_rng(99)
    cols = [W.selection_column(rng, 64) for _ in range(150)]
    plan = S.SelectionPlan(cols)
    sizes, best, _ = plan.wizard()
    choice, conf, nfb = plan.learned(params, stride=8)
    assert nfb == 0
    loss = S.ratio_loss(sizes, choice)
    untrained, _, _ = plan.learned(S.mlp_init(1), stride=8)
    assert loss < 0.05 and loss < S.ratio_loss(sizes, untrained)
    choice_fb, _, nfb = plan.learned(params, stride=8, threshold=1.01)
    assert nfb == plan.n_chunks
    assert torch.equal(choice_fb, best)
    plan.close()


def test_rowgroups_every_candidate_in_one_launch(cuda):
    """Chunks encoded with every candidate (chosen at random per chunk) decode bit-exactly through one page
    plan spanning all chunks of all columns."""
    import torch

    from fastlanes_b200 import rowgroups as RG
    from fastlanes_b200 import select as S

    dcols, _ = _cols(7, n_vec=6, reps=1)
    plan = S.SelectionPlan(dcols, 2)
    rng = np.random.default_rng(0)
    choice = rng.integers(0, S.K, plan.n_chunks)
    choice[:S.K] = np.arange(S.K)
    rg = RG.RowGroupSet(dcols, plan.chunks(), choice)
    rg.decode()
    torch.cuda.synchronize()
    for o, (t, _) in zip(rg.outputs, dcols):
        assert torch.equal(o, t)
    rg.close()
    plan.close()
