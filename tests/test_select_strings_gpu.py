"""Expression selection for string columns (fls_sel_plan_create_strings): the wizard's page sizes against the
pages the reference's own encoder wrote for the same rows (BYTE_ARR, DICT over an FSST dictionary, FSST,
DICT_RLE), and the learned selector against the wizard on seeded string chunks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# wizard candidate index of the string pool ids whose pages the fixtures hold
CAND = {0: 0, 3: 1, 13: 2, 15: 3}


def _plan(cuda, byts, offs, table):
    import torch

    from fastlanes_b200 import select as SL

    b = torch.from_numpy(np.ascontiguousarray(byts, np.uint8)).to(cuda)
    o = torch.from_numpy(np.asarray(offs, np.uint64).astype(np.int64)).to(cuda)
    return SL.StrSelectionPlan([(b, o, np.asarray(table, np.uint8))], 64), (b, o)


def _distinct_first_occurrence(byts, offs):
    rows = [bytes(byts[int(offs[i]):int(offs[i + 1])]) for i in range(offs.size - 1)]
    seen, dist = {}, []
    for r in rows:
        if r not in seen:
            seen[r] = len(dist)
            dist.append(r)
    d_offs = np.zeros(len(dist) + 1, np.uint64)
    d_offs[1:] = np.cumsum([len(x) for x in dist])
    return np.frombuffer(b"".join(dist), np.uint8).copy(), d_offs, np.array([seen[r] for r in rows], np.uint32)


@pytest.mark.parametrize("eid", [0, 13])
def test_string_wizard_size_is_the_reference_page_size(cuda, col_golden, eid):
    """BYTE_ARR and FSST: the size of the reference's page (and, for FSST, its exported table) for the same
    rows, with the reference's own symbol table."""
    byts, offs = col_golden[f"str_{eid}_input_bytes"], col_golden[f"str_{eid}_input_offsets"]
    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    table = dic[8:] if dic.size else col_golden["str_13_dict"][8:]  # BYTE_ARR's size needs no table
    plan, keep = _plan(cuda, byts, offs, table)
    sizes, best, dn = plan.wizard()
    plan.close()
    assert int(sizes[0, CAND[eid]].item()) == page.size + dic.size
    assert int(sizes[0, 4].item()) == -1 and int(sizes[0, 5].item()) == -1  # UINT64_MAX: no such candidate


@pytest.mark.parametrize("eid", [3, 15])
def test_string_wizard_dictionary_sizes(cuda, col_golden, eid):
    """DICT and DICT_RLE: the codes page as the reference writes it for the same rows, plus the dictionary page
    with every entry's true compressed length, as this engine's encoder writes it (the reference's encoder
    compresses entry i with the length of entry i - 1, so its dictionary pages hold other bytes)."""
    from fastlanes_b200 import strings as S

    byts, offs = col_golden[f"str_{eid}_input_bytes"], col_golden[f"str_{eid}_input_offsets"]
    page = col_golden[f"str_{eid}_page"]
    dbytes, doffs, codes = _distinct_first_occurrence(byts, offs)
    table, _, _ = S.fsst_compress(dbytes, doffs)
    _, own_dict = S.encode_string_dict(dbytes, doffs, codes)
    plan, keep = _plan(cuda, byts, offs, table)
    sizes, best, dn = plan.wizard()
    plan.close()
    assert int(dn[0].item()) == doffs.size - 1
    assert int(sizes[0, CAND[eid]].item()) == page.size + own_dict.size


def test_string_wizard_picks_the_family_winner_and_the_learned_selector_agrees(cuda):
    """Seeded chunks of every string family: labels from the wizard, an MLP trained on them (the integer
    selector's architecture and kernels), then held-out chunks chosen by both; the learned choice costs at most
    1 % more bytes."""
    import torch

    from fastlanes_b200 import select as SL
    from fastlanes_b200 import workloads as W

    feat, y, sizes, best = SL.labelled_string_vectors(120, seed=3, chunk_vectors=8)
    counts = np.bincount(best.cpu().numpy(), minlength=6)
    assert counts[:4].sum() == best.numel() and (counts[:4] > 0).sum() >= 3, counts
    params = SL.mlp_init(1)
    hist = SL.train(params, feat, y, epochs=30, batch=256, lr=2e-3)
    assert hist[-20:].mean() < hist[:20].mean()
    rng = np.random.default_rng(99)
    cols = []
    for _ in range(60):
        byts, offs, table = W.string_selection_column(rng, 8)
        cols.append((torch.from_numpy(byts).cuda(), torch.from_numpy(offs.astype(np.int64)).cuda(), table))
    plan = SL.StrSelectionPlan(cols, 8)
    sz, wbest, _ = plan.wizard()
    choice, conf, n_fb = plan.learned(params, stride=2, threshold=0.0)
    plan.close()
    assert int(choice.max().item()) < 4
    loss = SL.ratio_loss(sz[:, :4], choice)
    assert loss <= 0.01, (loss, (choice == wbest).float().mean().item())
