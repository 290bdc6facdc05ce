"""Writes tests/golden/fls_ref/: a file pair (data.fls + footer.json) written by the reference's own
Connection::read(dir).to_fls(out) (compiled from its sources into oracle/_ref/libfls_ref.so), from a seeded
CSV + schema.json made here, plus values.npz with the CSV's columns.

    make -C oracle ref && python tests/golden/make_fls_fixture.py
"""
import ctypes
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle  # noqa: E402


def main():
    if oracle.reference is None:
        raise SystemExit("oracle/_ref/libfls_ref.so missing: run `make -C oracle ref`")
    rng = np.random.default_rng(2024)
    n = 3 * 1024
    cols = {
        "RANGE_0_1000": rng.integers(0, 1000, n),
        "CONSTANT_INT": np.full(n, 42),
        "EQUAL_TO_RANGE": None,
        "BIG_SIGNED": rng.integers(-10**15, 10**15, n),
        "SORTED": np.cumsum(rng.integers(0, 20, n)),
    }
    cols["EQUAL_TO_RANGE"] = cols["RANGE_0_1000"].copy()
    out = os.path.join(HERE, "fls_ref")
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "in")
        os.makedirs(src)
        with open(os.path.join(src, "schema.json"), "w") as f:
            json.dump({"columns": [{"name": k, "type": "integer"} for k in cols]}, f, indent=2)
        with open(os.path.join(src, "data.csv"), "w") as f:
            for i in range(n):
                f.write("|".join(str(int(cols[k][i])) for k in cols) + "\n")
        dst = os.path.join(tmp, "out")
        os.makedirs(dst)
        if oracle.reference.ref_csv_to_fls(src.encode(), dst.encode()) != 0:
            raise SystemExit("the reference's to_fls failed")
        os.makedirs(out, exist_ok=True)
        for name in ("data.fls", "footer.json"):
            shutil.copy(os.path.join(dst, name), os.path.join(out, name))
    np.savez_compressed(os.path.join(out, "values.npz"), **{k: np.asarray(v, np.int64) for k, v in cols.items()})
    print("wrote", out)


if __name__ == "__main__":
    main()
