"""Device-buffer plumbing for tests and benchmarks (torch allocates, the CUDA
library computes).  Nothing here computes a query result."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, check, lib

_TORCH_DT = {1: "uint8", 2: "int16", 4: "int32", 8: "int64"}


def torch():
    import torch as T
    return T


def empty(n: int, width: int, zero: bool = False):
    """Device buffer of n elements of `width` bytes (16-byte aligned)."""
    T = torch()
    dt = getattr(T, _TORCH_DT[width])
    f = T.zeros if zero else T.empty
    return f(max(int(n), 1), dtype=dt, device="cuda")


def to_host(t, np_dtype) -> np.ndarray:
    """Copy a device buffer to a numpy array reinterpreted as np_dtype."""
    a = t.detach().cpu().numpy()
    return a.view(np_dtype)


def from_host(a: np.ndarray):
    T = torch()
    w = a.dtype.itemsize
    b = np.ascontiguousarray(a).view({1: np.uint8, 2: np.int16, 4: np.int32, 8: np.int64}[w])
    return T.from_numpy(b.copy()).cuda()


def stream_ptr() -> int:
    return int(torch().cuda.current_stream().cuda_stream)


class DevStar:
    """Star-schema fact and dimension columns generated on the device by
    mb_gen_star / mb_gen_star_dims."""

    NARROW = {"orderdate": 2, "quantity": 1, "discount": 1, "suppcity": 1}
    FACT = ["custkey", "partkey", "suppkey", "orderdate", "quantity", "discount", "extendedprice",
            "revenue", "supplycost", "suppcity"]

    def __init__(self, seed: int, k: int, n: int, width4: bool = False, row0: int = 0):
        self.seed, self.k, self.n, self.width4 = seed, k, n, width4
        self.cols = {f: empty(n, 4 if width4 else self.NARROW.get(f, 4)) for f in self.FACT}
        sc = abi.mb_star_cols(**{f: int(t.data_ptr()) for f, t in self.cols.items()})
        check(lib().mb_gen_star(seed, k, row0, n, 1 if width4 else 0, C.byref(sc), stream_ptr()))
        lg = 0
        while (2 << lg) <= k:
            lg += 1
        self.ncust, self.nsupp, self.npart = 30000 * k, 2000 * k, 200000 * (1 + lg)
        self.custcity = empty(self.ncust + 1, 1)
        self.suppcity = empty(self.nsupp + 1, 1)
        self.partmfgr = empty(self.npart + 1, 2)
        check(lib().mb_gen_star_dims(seed, k, self.custcity.data_ptr(), self.suppcity.data_ptr(),
                                     self.partmfgr.data_ptr(), stream_ptr()))

    def __getitem__(self, k):
        return self.cols[k]

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.cols.values())


class DevFlat:
    """The flat 5-column int32 table generated by mb_gen_flat."""

    def __init__(self, seed: int, n: int):
        self.seed, self.n = seed, n
        self.cols = {c: empty(n, 4) for c in "abcde"}
        check(lib().mb_gen_flat(seed, 0, n, *[self.cols[c].data_ptr() for c in "abcde"], stream_ptr()))

    def __getitem__(self, k):
        return self.cols[k]


def src_of(col, fk=None, checked: bool = True) -> abi.mb_src:
    s = abi.mb_src()
    s.col = int(col.data_ptr())
    s.width = int(col.element_size())
    if fk is not None:
        s.fk = int(fk.data_ptr())
        s.dimsz = int(col.numel()) if checked else 0
    return s


def bitmap_create(src: abi.mb_src, n: int, lo, hi, pop: bool = True):
    """Bin bitmaps of one column on the device: (slab [nbins x stride] words, popcounts)."""
    L = lib()
    lo = np.ascontiguousarray(lo, np.uint64)
    hi = np.ascontiguousarray(hi, np.uint64)
    nb = len(lo)
    stride = int(L.mb_bitmap_stride(n))
    slab = empty(nb * stride, 4, zero=True)
    pc = empty(nb, 8, zero=True) if pop else None
    check(L.mb_bitmap_create(C.byref(src), n, lo.ctypes.data_as(C.POINTER(C.c_uint64)),
                             hi.ctypes.data_as(C.POINTER(C.c_uint64)), nb, slab.data_ptr(), stride,
                             pc.data_ptr() if pc is not None else None, stream_ptr()))
    return slab.view(nb, stride), pc


def bitmap_create_levels(src: abi.mb_src, n: int, levels, pop: bool = True):
    """Several bin levels of one column in one pass (mb_bitmap_create_levels):
    levels = [(lo, hi), ...]; returns [(slab [nbins x stride] words, popcounts)]
    per level."""
    L = lib()
    stride = int(L.mb_bitmap_stride(n))
    arr = (abi.mb_level * max(1, len(levels)))()
    keep, outs = [], []
    for i, (lo, hi) in enumerate(levels):
        lo = np.ascontiguousarray(lo, np.uint64)
        hi = np.ascontiguousarray(hi, np.uint64)
        nb = len(lo)
        slab = empty(nb * stride, 4, zero=True)
        pc = empty(nb, 8, zero=True) if pop else None
        keep += [lo, hi]
        arr[i].lo = lo.ctypes.data_as(C.POINTER(C.c_uint64))
        arr[i].hi = hi.ctypes.data_as(C.POINTER(C.c_uint64))
        arr[i].nbins = nb
        arr[i].out = slab.data_ptr()
        arr[i].popcounts = pc.data_ptr() if pc is not None else None
        outs.append((slab.view(nb, stride), pc))
    check(L.mb_bitmap_create_levels(C.byref(src), n, arr, len(levels), stride, stream_ptr()))
    return outs


def vprg_grpby(prg: abi.mb_vprg, op: abi.mb_op, nr_grp: int, launch: abi.mb_launch | None = None,
               out=None, nq=None):
    L = lib()
    out = out if out is not None else empty(nr_grp, 8)
    nq = nq if nq is not None else empty(1, 8)
    check(L.mb_vprg_grpby(C.byref(prg), C.byref(op), nr_grp, out.data_ptr(), nq.data_ptr(),
                          C.byref(launch) if launch is not None else None, stream_ptr()))
    return out, nq


def join_grpby(n: int, op: abi.mb_op, nr_grp: int):
    L = lib()
    out = empty(nr_grp, 8)
    nq = empty(1, 8)
    check(L.mb_join_grpby(n, C.byref(op), nr_grp, out.data_ptr(), nq.data_ptr(), stream_ptr()))
    return out, nq
