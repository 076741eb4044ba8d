"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the reference's
own CPU oracle compiled from its sources (oracle/_ref/libcpuref.so).

TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the checker, never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from merle_b200 import abi

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libcpuref.so"

P = C.c_void_p
U32, U64, I64, I32 = C.c_uint32, C.c_uint64, C.c_int64, C.c_int32

SIGS = {
    "orc_is_nochk": (I32, [C.POINTER(abi.mb_vprg)]),
    "orc_bitmap_create": (None, [C.POINTER(abi.mb_src), U64, P, P, U32, P, U64, P]),
    "orc_vprg_eval": (None, [C.POINTER(abi.mb_vprg), I32, P, P]),
    "orc_op_row": (I32, [C.POINTER(abi.mb_op), U64, I32, U32, P, P]),
    "orc_vprg_grpby": (None, [C.POINTER(abi.mb_vprg), C.POINTER(abi.mb_op), U32, P, P]),
    "orc_join_grpby": (None, [U64, C.POINTER(abi.mb_op), U32, P, P]),
    "orc_bitmap_to_rows": (U64, [P, P, U64, P]),
    "orc_sector_count": (U64, [P, U64, U32]),
    "orc_gen_flat": (None, [U64, U64, U64, P, P, P, P, P]),
    "orc_gen_star": (None, [U64, U32, U64, U64, I32, C.POINTER(abi.mb_star_cols)]),
    "orc_gen_star_dims": (None, [U64, U32, P, P, P]),
    "orc_date_to_year": (U32, [U32]),
    "orc_s1": (I64, [P, U64, U32, U32, U32, U32, U32, U32, P]),
    "orc_s2": (None, [P, U64, U32, U32, U32, U32, P, U32, P]),
    "orc_s3": (None, [P, U64, U32, U32, U32, U32, U32, U32, P, U32, P]),
    "orc_s4": (None, [P, U64, U32, U32, U32, U32, U32, U32, U32, U32, P, U32, P]),
    "orc_synth": (None, [P, P, U32, P, P, P, U64, U64, U64, U64, U64, U64, U64, P, P]),
    "orc_flat_query": (I64, [P, P, P, P, P, U64, I32, I32, P, U32, I32, I32, P]),
}

_lib = None
_ref = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        for n, (r, a) in SIGS.items():
            f = getattr(_lib, n)
            f.restype, f.argtypes = r, a
    return _lib


def ref() -> C.CDLL | None:
    """The reference's own cpuref.c / synth cpuref.c, or None if not built."""
    global _ref
    if _ref is None and REF_LIB.exists():
        _ref = C.CDLL(str(REF_LIB), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        _ref.s1ref.restype = U64
        _ref.s1ref.argtypes = [P, C.c_size_t, C.c_uint16, C.c_uint16, C.c_uint8, C.c_uint8, C.c_uint8, C.c_uint8]
        _ref.s2ref.restype = None
        _ref.s2ref.argtypes = [P, C.c_size_t, U32, U32, C.c_uint8, C.c_uint8, P]
        _ref.s3ref.restype = None
        _ref.s3ref.argtypes = [P, C.c_size_t, C.c_uint8, C.c_uint8, C.c_uint8, C.c_uint8, C.c_uint16, C.c_uint16, P]
        _ref.s4ref.restype = None
        _ref.s4ref.argtypes = [P, C.c_size_t, C.c_uint8, C.c_uint8, C.c_uint8, C.c_uint8, C.c_uint16,
                               C.c_uint16, C.c_uint16, C.c_uint16, P]
        _ref.ssb_cpujoin.restype = C.POINTER(U32)
        _ref.ssb_cpujoin.argtypes = [P, C.c_size_t]
        _ref.synth_ref.restype = None
        _ref.synth_ref.argtypes = [P, C.c_size_t, U64, U64, U64, U64, U64, U64, P]
        _ref.window_zipf.restype = C.POINTER(C.c_double)
        _ref.window_zipf.argtypes = [C.c_double, C.c_size_t, C.c_size_t]
    return _ref


def ptr(a: np.ndarray) -> int:
    return int(a.ctypes.data)


# ------------------------------------------------------------- data holders
class SsbSchema(C.Structure):
    """struct ssb_schema (ssb/ssbdemo.h:41-49): host pointers for cpuref."""
    _fields_ = [(n, C.c_void_p) for n in (
        "loCustKey", "loPartKey", "loOrderDate", "loExtendedPrice", "loRevenue", "loSupplyCost",
        "loQuantity", "loDiscount", "loSuppCity", "custMktSegment", "custCity", "partName",
        "partMfgr", "partColor", "partType", "partSize", "partContainer")]


class OrcSsb(C.Structure):
    """struct orc_ssb of oracle.h."""
    _fields_ = [(n, C.c_void_p) for n in (
        "loCustKey", "loPartKey", "loOrderDate", "loExtendedPrice", "loRevenue", "loSupplyCost",
        "loQuantity", "loDiscount", "loSuppCity", "custCity", "partMfgr")]


class SynthSchema(C.Structure):
    """struct synth_schema (synth/synthdemo.h:16-23)."""
    _fields_ = [("bitwidth", C.c_uint32), ("factattr1", C.c_void_p), ("factattr2", C.c_void_p),
                ("fkey", C.c_void_p), ("dimattr1", C.c_void_p), ("dimattr2", C.c_void_p)]


class StarHost:
    """Star-schema columns on the host in the reference's ssb_schema widths."""

    FACT = ["custkey", "partkey", "suppkey", "orderdate", "quantity", "discount", "extendedprice",
            "revenue", "supplycost", "suppcity"]

    def __init__(self, seed: int, k: int, n: int, row0: int = 0, width4: bool = False):
        L = lib()
        nw = {"orderdate": np.uint16, "quantity": np.uint8, "discount": np.uint8, "suppcity": np.uint8}
        self.n, self.k, self.seed = n, k, seed
        self.cols = {}
        for f in self.FACT:
            dt = np.uint32 if width4 else nw.get(f, np.uint32)
            self.cols[f] = np.zeros(n, dtype=dt)
        sc = abi.mb_star_cols(**{f: ptr(a) for f, a in self.cols.items()})
        L.orc_gen_star(seed, k, row0, n, 1 if width4 else 0, C.byref(sc))
        nc, ns, np_ = 30000 * k, 2000 * k, star_npart(k)
        self.custcity = np.zeros(nc + 1, np.uint8)
        self.suppcity = np.zeros(ns + 1, np.uint8)
        self.partmfgr = np.zeros(np_ + 1, np.uint16)
        L.orc_gen_star_dims(seed, k, ptr(self.custcity), ptr(self.suppcity), ptr(self.partmfgr))

    def __getitem__(self, k):
        return self.cols[k]

    def narrow(self) -> "StarHost":
        """A view in the reference's ssb_schema widths (for cpuref)."""
        o = object.__new__(StarHost)
        o.n, o.k, o.seed = self.n, self.k, self.seed
        nw = {"orderdate": np.uint16, "quantity": np.uint8, "discount": np.uint8, "suppcity": np.uint8}
        o.cols = {f: a.astype(nw.get(f, np.uint32)) for f, a in self.cols.items()}
        o.custcity, o.suppcity, o.partmfgr = self.custcity, self.suppcity, self.partmfgr
        return o

    def ssb_schema(self) -> SsbSchema:
        s = self.narrow()
        self._narrow = s
        return SsbSchema(loCustKey=ptr(s["custkey"]), loPartKey=ptr(s["partkey"]),
                         loOrderDate=ptr(s["orderdate"]), loExtendedPrice=ptr(s["extendedprice"]),
                         loRevenue=ptr(s["revenue"]), loSupplyCost=ptr(s["supplycost"]),
                         loQuantity=ptr(s["quantity"]), loDiscount=ptr(s["discount"]),
                         loSuppCity=ptr(s["suppcity"]), custCity=ptr(s.custcity), partMfgr=ptr(s.partmfgr))

    def orc_ssb(self) -> OrcSsb:
        s = self.narrow()
        self._narrow2 = s
        return OrcSsb(loCustKey=ptr(s["custkey"]), loPartKey=ptr(s["partkey"]),
                      loOrderDate=ptr(s["orderdate"]), loExtendedPrice=ptr(s["extendedprice"]),
                      loRevenue=ptr(s["revenue"]), loSupplyCost=ptr(s["supplycost"]),
                      loQuantity=ptr(s["quantity"]), loDiscount=ptr(s["discount"]),
                      loSuppCity=ptr(s["suppcity"]), custCity=ptr(s.custcity), partMfgr=ptr(s.partmfgr))


def star_npart(k: int) -> int:
    lg = 0
    while (2 << lg) <= k:
        lg += 1
    return 200000 * (1 + lg)


def gen_flat(seed: int, n: int, row0: int = 0) -> dict:
    cols = {c: np.zeros(n, np.int32) for c in "abcde"}
    lib().orc_gen_flat(seed, row0, n, *[ptr(cols[c]) for c in "abcde"])
    return cols


# ------------------------------------------------------------- oracle calls
def bitmap_create(src: abi.mb_src, n: int, lo, hi, stride: int | None = None):
    lo = np.ascontiguousarray(lo, np.uint64)
    hi = np.ascontiguousarray(hi, np.uint64)
    nb = len(lo)
    W = (n + 31) // 32
    stride = stride or W
    out = np.zeros(nb * stride, np.uint32)
    pop = np.zeros(nb, np.uint64)
    lib().orc_bitmap_create(C.byref(src), n, ptr(lo), ptr(hi), nb, ptr(out), stride, ptr(pop))
    return out.reshape(nb, stride), pop


def vprg_eval(p: abi.mb_vprg, chk: bool):
    W = (p.factsz + 31) // 32
    po = np.zeros(W, np.uint32)
    un = np.zeros(W, np.uint32)
    lib().orc_vprg_eval(C.byref(p), 1 if chk else 0, ptr(po), ptr(un))
    return po, un


def vprg_grpby(p: abi.mb_vprg, op: abi.mb_op, nr_grp: int):
    out = np.zeros(nr_grp, np.int64)
    nq = np.zeros(1, np.uint64)
    lib().orc_vprg_grpby(C.byref(p), C.byref(op), nr_grp, ptr(out), ptr(nq))
    return out, int(nq[0])


def join_grpby(n: int, op: abi.mb_op, nr_grp: int):
    out = np.zeros(nr_grp, np.int64)
    nq = np.zeros(1, np.uint64)
    lib().orc_join_grpby(n, C.byref(op), nr_grp, ptr(out), ptr(nq))
    return out, int(nq[0])


def bitmap_to_rows(poss: np.ndarray, unc: np.ndarray | None, n: int) -> np.ndarray:
    rows = np.zeros(max(1, int(np.unpackbits(poss.view(np.uint8)).sum())), np.uint32)
    cnt = lib().orc_bitmap_to_rows(ptr(poss), ptr(unc) if unc is not None else None, n, ptr(rows))
    return rows[:cnt]


def sector_count(rowbits: np.ndarray, n: int, width: int) -> int:
    return int(lib().orc_sector_count(ptr(rowbits), n, width))
