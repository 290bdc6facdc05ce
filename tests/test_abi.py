"""The C-ABI library loads and exports every entry point declared in include/*.h (no device calls)."""
import glob
import os
import re

from tests.conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:int|void|bool|uint64_t|int64_t|uint32_t|connection_cpi\s*\*)\s*\*?\s*(\w+)\s*\(",
                             txt, re.M):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_all_declared():
    from fastlanes_b200 import _lib

    declared = _declared()
    assert len(declared) > 30
    missing = [n for n in sorted(declared) if not hasattr(_lib.lib, n)]
    assert not missing, missing


def test_python_signatures_cover_declarations():
    from fastlanes_b200 import _lib
    import fastlanes_b200  # noqa: F401  (declares the later entry points)

    declared = _declared()
    unbound = sorted(declared - set(_lib.exported_symbols()))
    assert not unbound, unbound
