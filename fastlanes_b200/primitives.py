"""Batched device versions of the reference's generated primitives (include/fls_gen/*), on torch CUDA tensors.

Names and argument meaning follow ``generated::<op>::fallback::scalar::<op>``; every call decodes a batch of
1024-value vectors instead of one, and returns the output tensor.  Tensors hold unsigned integers of the
primitive's width (torch.uint8/uint16/uint32/uint64).  ``order`` is TRANSPOSED (the primitive's own output)
or ORIGINAL (untransposed, as Materializer::Materialize returns it).
"""
import torch

from ._lib import check, lib

TRANSPOSED = 0
ORIGINAL = 1

_WIDTH = {torch.uint8: 8, torch.uint16: 16, torch.uint32: 32, torch.uint64: 64}
_DTYPE = {8: torch.uint8, 16: torch.uint16, 32: torch.uint32, 64: torch.uint64}


def _stream():
    return ctypes_stream(torch.cuda.current_stream())


def ctypes_stream(s):
    return s.cuda_stream


def _ptr(t):
    return None if t is None else t.data_ptr()


def width_of(t):
    return _WIDTH[t.dtype]


def packed_offsets(bw, width):
    """Byte offset of every vector in a dense concatenation of packed vectors (bw*128 bytes each)."""
    sizes = bw.to(torch.int64) * 128
    off = torch.zeros_like(sizes)
    off[1:] = torch.cumsum(sizes, 0)[:-1]
    return off.to(torch.uint64)


def unpack(packed, bw, byte_off=None, order=TRANSPOSED, width=None):
    """generated::unpack: bit-unpack every vector (packed words of vector v at byte byte_off[v])."""
    w = width or width_of(packed)
    n = bw.numel()
    out = torch.empty(n * 1024, dtype=_DTYPE[w], device=packed.device)
    check(getattr(lib, f"fls_gpu_unpack_u{w}")(_ptr(packed), _ptr(out), _ptr(bw), _ptr(byte_off), n, order,
                                               _stream()), "unpack")
    return out


def unffor(packed, bw, base, byte_off=None, order=TRANSPOSED):
    """generated::unffor: unpack + frame-of-reference add (wrapping in the type)."""
    w = width_of(base)
    n = bw.numel()
    out = torch.empty(n * 1024, dtype=_DTYPE[w], device=base.device)
    check(getattr(lib, f"fls_gpu_unffor_u{w}")(_ptr(packed), _ptr(out), _ptr(bw), _ptr(base), _ptr(byte_off), n,
                                               order, _stream()), "unffor")
    return out


def rsum(deltas, lane_base, order=TRANSPOSED):
    """generated::rsum: per-lane running sum of 1024 transposed deltas, seeded by 1024/W lane bases."""
    w = width_of(deltas)
    n = deltas.numel() // 1024
    out = torch.empty_like(deltas)
    check(getattr(lib, f"fls_gpu_rsum_u{w}")(_ptr(deltas), _ptr(out), _ptr(lane_base), n, order, _stream()), "rsum")
    return out


def unffor_rsum(packed, bw, base, lane_base, byte_off=None, order=TRANSPOSED):
    """Fused DELTA decode: unffor then rsum (ffor_decompress + rsum_decompress of the reference)."""
    w = width_of(base)
    n = bw.numel()
    out = torch.empty(n * 1024, dtype=_DTYPE[w], device=base.device)
    check(getattr(lib, f"fls_gpu_unffor_rsum_u{w}")(_ptr(packed), _ptr(out), _ptr(bw), _ptr(base), _ptr(lane_base),
                                                    _ptr(byte_off), n, order, _stream()), "unffor_rsum")
    return out


def untranspose_i(x):
    """generated::untranspose::untranspose_i (untranspose_o is the same permutation)."""
    w = width_of(x)
    out = torch.empty_like(x)
    check(getattr(lib, f"fls_gpu_untranspose_i_u{w}")(_ptr(x), _ptr(out), x.numel() // 1024, _stream()),
          "untranspose_i")
    return out


untranspose_o = untranspose_i


def transpose_i(x):
    """generated::transpose::transpose_i (transpose_o is the same permutation)."""
    w = width_of(x)
    out = torch.empty_like(x)
    check(getattr(lib, f"fls_gpu_transpose_i_u{w}")(_ptr(x), _ptr(out), x.numel() // 1024, _stream()), "transpose_i")
    return out


transpose_o = transpose_i


def ffor(x, bw, base=None):
    """generated::ffor (base None = generated::pack): returns (packed bytes, byte offsets)."""
    w = width_of(x)
    n = x.numel() // 1024
    off = packed_offsets(bw, w)
    total = int((bw.to(torch.int64) * 128).sum().item())
    out = torch.zeros(max(total, 16), dtype=torch.uint8, device=x.device)
    check(getattr(lib, f"fls_gpu_ffor_u{w}")(_ptr(x), _ptr(out), _ptr(bw), _ptr(base), _ptr(off), n, _stream()),
          "ffor")
    return out, off


def pack(x, bw):
    return ffor(x, bw, None)


def unrsum(x):
    """generated::unrsum: deltas along each lane (first element of a lane becomes 0)."""
    w = width_of(x)
    out = torch.empty_like(x)
    check(getattr(lib, f"fls_gpu_unrsum_u{w}")(_ptr(x), _ptr(out), x.numel() // 1024, _stream()), "unrsum")
    return out


def analyze(x, signed=False):
    """Per-vector FOR base and bit width (ffor_analyze): returns (bw uint8, base)."""
    w = width_of(x)
    n = x.numel() // 1024
    bw = torch.empty(n, dtype=torch.uint8, device=x.device)
    base = torch.empty(n, dtype=x.dtype, device=x.device)
    check(getattr(lib, f"fls_gpu_analyze_u{w}")(_ptr(x), _ptr(bw), _ptr(base), n, int(signed), _stream()), "analyze")
    return bw, base


def device_status(reset=True):
    """OR of device-side error bits since the last reset (synchronises)."""
    return lib.fls_gpu_status(int(reset))


def stalled_unffor(packed, bw, base, byte_off, stall_vector, spin_limit):
    """fls_gpu_test_stalled_copy (failure injection): unffor u32 where vector `stall_vector`'s staging copy is
    armed but never issued, so its bounded wait runs out.  Returns (output, call status); the device status
    word then carries FLS_DEV_TIMEOUT."""
    n = bw.numel()
    out = torch.zeros(n * 1024, dtype=torch.uint32, device=base.device)
    rc = lib.fls_gpu_test_stalled_copy(_ptr(packed), _ptr(out), _ptr(bw), _ptr(base), _ptr(byte_off), n, stall_vector,
                                       spin_limit, _stream())
    return out, rc
