"""merle_b200 - B200-native (sm_100a) fused bitmap-index query engine.

The engine itself is the CUDA/C++ shared library libmerleb200.so with the C ABI
of include/merle_b200.h.  This package loads it (ctypes) and mirrors the
reference's host-side operator interface for tests and benchmarks.  There is no
CPU fallback: if the library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import abi

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB_PATH = PKG / "libmerleb200.so"
HEADER = ROOT / "include" / "merle_b200.h"

_lib: C.CDLL | None = None


class MbError(RuntimeError):
    """A C ABI call returned a non-OK mb_status."""

    def __init__(self, status: int, msg: str):
        name = abi.STATUS_NAMES[status] if 0 <= status < len(abi.STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """The loaded CUDA library.  Raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m merle_b200.build` "
                "(there is no CPU fallback)")
        _lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        abi.bind(_lib, abi.SIGNATURES)
    return _lib


def check(status: int) -> None:
    if status != abi.MB_OK:
        raise MbError(status, lib().mb_last_error().decode(errors="replace"))


__all__ = ["abi", "lib", "check", "MbError", "LIB_PATH", "HEADER"]
