"""The reference's file pair (data.fls + footer.json, written by the reference's own Connection::to_fls from a
seeded CSV: tests/golden/fls_ref, made by tests/golden/make_fls_fixture.py) opened by fls_file_open, and the
GPU read of it and of this library's page container (fls_file_read)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "golden", "fls_ref")
NAMES = ["RANGE_0_1000", "CONSTANT_INT", "EQUAL_TO_RANGE", "BIG_SIGNED", "SORTED"]


def _stored(x):
    """What the reference's to_fls stores for a ZERO_COPY column: its first vector n_vec times
    (PhysicalExpr::PointTo, src/expression/physical_expression.cpp:5, is empty, so the vectorized store
    writes the vector the column's TypedVector points at for every vector index)."""
    return np.tile(x[:1024], x.size // 1024)


def test_reference_file_footer_and_layout():
    """Host only: shape and column kinds from the reference's footer; its ZERO_COPY columns are raw vectors
    at col_ofs, CONSTANT / EQUAL columns store nothing."""
    from fastlanes_b200 import files as F

    f = F.FlsFile(REF_DIR)
    want = np.load(os.path.join(REF_DIR, "values.npz"))
    assert (f.n_cols, f.n_vec) == (5, 3)
    kinds = [c["kind"] for c in f.columns]
    assert kinds == [F.ZERO_COPY, F.NO_DATA, F.NO_DATA, F.ZERO_COPY, F.ZERO_COPY]
    raw = np.fromfile(os.path.join(REF_DIR, "data.fls"), np.uint8)
    footer = json.load(open(os.path.join(REF_DIR, "footer.json")))
    for i, m in enumerate(footer["3: Column Metadatas"]):
        if kinds[i] == F.ZERO_COPY:
            o = m["col_ofs"]
            assert np.array_equal(raw[o:o + 3 * 8192].view(np.int64), _stored(want[NAMES[i]]))
    f.close()


def test_malformed_footers_are_refused(tmp_path):
    from fastlanes_b200 import _lib
    from fastlanes_b200 import files as F

    (tmp_path / "data.fls").write_bytes(bytes(8192))
    bad = ['{"1: N VEC": 1}', '{"1: N VEC": 1, "3: Column Metadatas": [{"col_ofs": 0}]}',
           '{"1: N VEC": 2, "3: Column Metadatas": [{"col_ofs": 0, "logical_type": 5, '
           '"Encoding RPN": {"operators": ["ZERO_COPY", "INT64"]}}]}',  # 2 vectors > the 8 KB file
           '{"1: N VEC": 1, "3: Column Metadatas": [', 'not json']
    for text in bad:
        (tmp_path / "footer.json").write_text(text)
        with pytest.raises(_lib.FlsError):
            F.FlsFile(str(tmp_path))


@pytest.mark.gpu
def test_reference_file_read_on_the_gpu(cuda):
    from fastlanes_b200 import _lib
    from fastlanes_b200 import files as F

    want = np.load(os.path.join(REF_DIR, "values.npz"))
    f = F.FlsFile(REF_DIR)
    got = f.read([0, 3, 4])
    for t, name in zip(got, (NAMES[0], NAMES[3], NAMES[4])):
        assert np.array_equal(t.cpu().numpy(), _stored(want[name]))
    with pytest.raises(_lib.FlsError):
        f.read([1])  # a CONSTANT column: the reference's file holds no value for it
    f.close()


@pytest.mark.gpu
def test_page_container_round_trip(cuda, tmp_path):
    """write_fls with raw and page columns (FFOR, DELTA, RLE, DICT, DICT_RLE; 32 / 64-bit; several row-group
    chunks per column) and read_fls back on the GPU: every column bit-exact; the footer stays readable by the
    reference's keys."""
    from fastlanes_b200 import files as F
    from fastlanes_b200 import workloads as W

    rng = np.random.default_rng(3)
    n = 150 * 1024
    cols = [
        (rng.integers(0, 1 << 20, n).astype(np.uint32), 1),
        (W.delta_timestamps(n), 11),
        (W.rle_int32(n), 6),
        (rng.integers(-5, 5, n).astype(np.int64) * 1000003, "dict"),
        (np.repeat(rng.integers(0, 300, n // 16), 16).astype(np.int32), "dict_rle"),
        (rng.integers(-10**18, 10**18, n, dtype=np.int64), None),
        (rng.integers(0, 1 << 40, n).astype(np.uint64), 1),
    ]
    F.write_fls(str(tmp_path), cols, rowgroup_vectors=64)
    f = F.FlsFile(str(tmp_path))
    assert [c["kind"] for c in f.columns] == [F.PAGES] * 5 + [F.ZERO_COPY, F.PAGES]
    got = f.read()
    for t, (x, _) in zip(got, cols):
        assert np.array_equal(t.cpu().numpy(), x)
    # a subset, in another order
    got = f.read([6, 2])
    assert np.array_equal(got[0].cpu().numpy(), cols[6][0]) and np.array_equal(got[1].cpu().numpy(), cols[2][0])
    f.close()
    footer = json.load(open(tmp_path / "footer.json"))
    assert footer["1: N VEC"] == 150 and len(footer["3: Column Metadatas"]) == 7
