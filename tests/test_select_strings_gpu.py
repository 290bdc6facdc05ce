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


@pytest.mark.parametrize("eid", [0, 3, 13, 15])
def test_string_wizard_size_is_the_reference_page_size(cuda, col_golden, eid):
    byts, offs = col_golden[f"str_{eid}_input_bytes"], col_golden[f"str_{eid}_input_offsets"]
    page, dic = col_golden[f"str_{eid}_page"], col_golden[f"str_{eid}_dict"]
    # the symbol table the reference's pages use (BYTE_ARR has none: its size does not depend on one)
    table = dic[8:] if dic.size else col_golden["str_13_dict"][8:]
    plan, keep = _plan(cuda, byts, offs, table)
    sizes, best, dn = plan.wizard()
    plan.close()
    assert int(sizes[0, CAND[eid]].item()) == page.size + dic.size
    assert int(sizes[0, 4].item()) == -1 and int(sizes[0, 5].item()) == -1  # UINT64_MAX: no such candidate


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
