"""B200-native decode engine for FastLanes' cascading lightweight encodings.

The compute path is libfls_b200.so (hand-written sm_100a CUDA behind a C ABI, include/fls_b200.h); this
package is the Python face of that ABI.
"""
from . import _lib  # noqa: F401  (raises if the CUDA library is missing)
from . import primitives  # noqa: F401
from . import pages  # noqa: F401
from . import strings  # noqa: F401
from . import select  # noqa: F401
from . import workloads  # noqa: F401
from . import files  # noqa: F401

__all__ = ["files", "pages", "primitives", "select", "strings", "workloads"]
