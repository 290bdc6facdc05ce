"""Loads libfls_b200.so (the CUDA decode engine) and declares its C ABI (include/fls_b200.h).

There is no fallback: if the library is missing or does not load, importing this module raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfls_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing; build it with `make -C fastlanes_b200/csrc` (sm_100a)")

lib = ctypes.CDLL(LIB_PATH)

_p = ctypes.c_void_p
_u8 = ctypes.c_uint8
_u64 = ctypes.c_uint64
_i = ctypes.c_int

# name -> (restype, argtypes)
_SIGS = {
    "fls_gpu_status": (_i, [_i]),
    "fls_gpu_launch_count": (_u64, [_i]),
    "fls_gpu_test_stalled_copy": (_i, [_p, _p, _p, _p, _p, _u64, _u64, ctypes.c_uint32, _p]),
}
for w in (8, 16, 32, 64):
    _SIGS[f"fls_gpu_unpack_u{w}"] = (_i, [_p, _p, _p, _p, _u64, _i, _p])
    _SIGS[f"fls_gpu_unffor_u{w}"] = (_i, [_p, _p, _p, _p, _p, _u64, _i, _p])
    _SIGS[f"fls_gpu_rsum_u{w}"] = (_i, [_p, _p, _p, _u64, _i, _p])
    _SIGS[f"fls_gpu_untranspose_i_u{w}"] = (_i, [_p, _p, _u64, _p])
    _SIGS[f"fls_gpu_transpose_i_u{w}"] = (_i, [_p, _p, _u64, _p])
    _SIGS[f"fls_gpu_ffor_u{w}"] = (_i, [_p, _p, _p, _p, _p, _u64, _p])
for w in (16, 32, 64):
    _SIGS[f"fls_gpu_unffor_rsum_u{w}"] = (_i, [_p, _p, _p, _p, _p, _p, _u64, _i, _p])
    _SIGS[f"fls_gpu_unrsum_u{w}"] = (_i, [_p, _p, _u64, _p])
    _SIGS[f"fls_gpu_analyze_u{w}"] = (_i, [_p, _p, _p, _u64, _i, _p])

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def declare(name, restype, argtypes):
    """Declare a further symbol of the library (used by the modules that wrap later entry points)."""
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    _SIGS[name] = (restype, argtypes)
    return f


def exported_symbols():
    return sorted(_SIGS)


class FlsError(RuntimeError):
    pass


_CODES = {-1: "FLS_ERR_ARG", -2: "FLS_ERR_CUDA", -3: "FLS_ERR_FORMAT", -4: "FLS_ERR_UNSUPPORTED", -5: "FLS_ERR_BW"}


def check(rc, what=""):
    if rc != 0:
        raise FlsError(f"{what}: {_CODES.get(rc, rc)}")
    return rc
