"""WAH (word-aligned hybrid) compressed bitmaps: the reference's
compressed-bitmap baseline (merle/wahGpu.cuh, merle/host/wahCpu.h,
ssb/wah-demo.cu) on this library's kernels.

Names follow the reference's:

- ``wah_compress`` / ``wah_decompress``: ``wahCompress`` and ``wahDecomp``
  (merle/wahGpuCmprs.cu:172-198, 34-47), between this library's bitmaps and
  WAH streams (``order``: ``abi.WAH_LSB`` puts row 31g + j of group g at bit j,
  ``abi.WAH_MSB`` at bit 30 - j);
- ``wah_and`` / ``wah_or`` / ``wah_xor``: ``wahAnd`` / ``wahOr`` / ``wahXor``
  (merle/wahGpu.cuh:11-30): canonical streams in, a canonical stream out;
- ``load_wah_file`` / ``save_wah_file``: ``loadWahFile``
  (merle/host/wahConv.c:93-109) and the matching writer.

A decompressed stream is an ordinary bitmap, so it can be a bin of an
``ops.Col`` operand of a virtual bitmap program (the compressed-operand hook
``vprg::_cmprs_adapt_run`` that the reference declares at primitive.cuh:334-337
but never defines).  Device arrays are torch uint32-typed int32 tensors on
CUDA; the library fails loudly if its CUDA build is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import abi, check, lib


def _torch():
    import torch
    return torch


def _ptr(t) -> int | None:
    return int(t.data_ptr()) if t is not None and t.numel() else None


def _stream(stream) -> int | None:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def wah_groups(nrows: int) -> int:
    return int(lib().mb_wah_groups(nrows))


def wah_compress(bitmap, nrows: int, order: int = abi.WAH_LSB, stream=None):
    """Device bitmap (int32 tensor, >= ceil(nrows/32) words) -> device WAH
    stream (int32 tensor of exactly the stream's words)."""
    torch = _torch()
    cap = max(1, wah_groups(nrows))
    out = torch.empty(cap, dtype=torch.int32, device=bitmap.device if nrows else "cuda")
    n = C.c_uint64()
    check(lib().mb_wah_encode(_ptr(bitmap) if nrows else None, nrows, order, _ptr(out), cap, C.byref(n),
                              _stream(stream)))
    return out[:n.value].clone()


def wah_decompress(wah, nrows: int, order: int = abi.WAH_LSB, stream=None):
    """Device WAH stream -> device bitmap of mb_bitmap_stride(nrows) words."""
    torch = _torch()
    stride = int(lib().mb_bitmap_stride(nrows))
    out = torch.empty(max(1, stride), dtype=torch.int32, device=wah.device if wah.numel() else "cuda")
    check(lib().mb_wah_decode(_ptr(wah), wah.numel(), order, nrows, _ptr(out), _stream(stream)))
    return out[:stride]


def wah_ngroups(wah, stream=None) -> int:
    n = C.c_uint64()
    check(lib().mb_wah_ngroups(_ptr(wah), wah.numel(), C.byref(n), _stream(stream)))
    return n.value


def _op(op: int, a, b, ngroups: int | None, stream=None):
    torch = _torch()
    if ngroups is None:
        ngroups = max(wah_ngroups(a, stream), wah_ngroups(b, stream))
    cap = max(1, ngroups)
    out = torch.empty(cap, dtype=torch.int32, device=a.device)
    n = C.c_uint64()
    check(lib().mb_wah_op(op, _ptr(a), a.numel(), _ptr(b), b.numel(), ngroups, _ptr(out), cap, C.byref(n),
                          _stream(stream)))
    return out[:n.value].clone()


def wah_and(a, b, ngroups: int | None = None, stream=None):
    return _op(abi.WAH_AND, a, b, ngroups, stream)


def wah_or(a, b, ngroups: int | None = None, stream=None):
    return _op(abi.WAH_OR, a, b, ngroups, stream)


def wah_xor(a, b, ngroups: int | None = None, stream=None):
    return _op(abi.WAH_XOR, a, b, ngroups, stream)


def save_wah_file(path: str | Path, words: np.ndarray, ngroups: int) -> None:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    check(lib().mb_wah_save(str(path).encode(), w.ctypes.data if len(w) else None, len(w), ngroups))


def load_wah_file(path: str | Path) -> tuple[np.ndarray, int]:
    """(stream words, groups) of a file in the reference's layout."""
    n, g = C.c_uint64(), C.c_uint64()
    check(lib().mb_wah_load(str(path).encode(), None, 0, C.byref(n), C.byref(g)))
    w = np.zeros(max(1, n.value), np.uint32)
    check(lib().mb_wah_load(str(path).encode(), w.ctypes.data, len(w), C.byref(n), C.byref(g)))
    return w[:n.value], g.value
