"""The selection oracle pinned on the CPU: its size model against the reference's own encoded pages, and its
MLP gradient against finite differences."""
import numpy as np
import pytest

from oracle import select as SEL


@pytest.mark.parametrize("expr,cand", [(0, 0), (1, 1), (6, 2), (11, 3)])
def test_size_model_matches_reference_pages(col_golden, expr, cand):
    """The reference's encoder (pool ids 0 / 1 / 6 / 11 on int64) wrote pages of exactly the modelled size."""
    x = col_golden[f"i64_{expr}_input"].view(np.uint64)
    assert int(SEL.chunk_sizes(x, True)[cand]) == col_golden[f"i64_{expr}_page"].size


def test_dict_codes_page_matches_reference(col_golden):
    """DICT (id 17): the codes page the reference wrote has the modelled size with first-occurrence codes; only
    the dictionary page differs (the reference FFOR-packs the entries, the engine stores them raw)."""
    x = col_golden["i64_17_input"].view(np.uint64)
    d, _ = SEL.chunk_dictionary(x)
    codes_page = int(SEL.chunk_sizes(x, True)[4]) - (8 + 12 + 8 * d)
    assert codes_page == col_golden["i64_17_page"].size


def test_chunk_dictionary_first_occurrence_order():
    x = np.array([5, 3, 5, 9, 3, 1] * 171 + [5] * (1024 - 6 * 171), np.uint32)
    d, codes = SEL.chunk_dictionary(x)
    assert d == 4
    assert codes[:6].tolist() == [0, 1, 0, 2, 1, 3]


def test_vector_parts_edge_vectors():
    const = np.full(1024, 7, np.uint32)
    assert SEL.vector_parts(const, False) == (0, 0, 1, 0)
    ramp = np.arange(1024, dtype=np.uint64)
    # chains run over contiguous original positions: deltas 1 (0 at chain starts), index deltas 1
    assert SEL.vector_parts(ramp, False) == (10, 1, 1024, 1)
    blocks = np.repeat(np.arange(64, dtype=np.uint32), 16)  # runs start only at chain starts
    assert SEL.vector_parts(blocks, False)[2:] == (64, 0)
    neg = np.array([-1, 1] * 512, np.int64).view(np.uint64)
    assert SEL.vector_parts(neg, True)[0] == 2       # signed range 2
    assert SEL.vector_parts(neg, False)[0] == 64     # unsigned range 2^64 - 2


def test_features_of_a_constant_vector():
    f = SEL.features(SEL.vector_stats(np.full(1024, 3, np.uint32), False))
    assert f.shape == (32,)
    assert f[0] == 0 and f[2] == 1 / 1024 and f[4] == 1 / 1024 and f[10] == 1.0 and f[30] == 1.0


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, SEL.param_count())
    x = rng.uniform(0, 1, (16, SEL.N_FEAT))
    y = rng.integers(0, SEL.K, 16)
    _, g = SEL.mlp_grad(p, x, y)
    idx = rng.choice(p.size, 60, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = SEL.mlp_grad(q, x, y)
        q[i] -= 2 * eps
        lm, _ = SEL.mlp_grad(q, x, y)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_adam_first_step_moves_by_lr():
    p = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    q, m, v = SEL.adam(p, g, np.zeros(4), np.zeros(4), 1, lr=0.01)
    assert np.allclose(q[:3], -0.01 * np.sign(g[:3]), atol=1e-9) and q[3] == 0
