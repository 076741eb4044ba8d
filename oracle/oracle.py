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
WAH_REF_LIB = HERE / "_ref" / "libwahref.so"

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
    "orc_wah_encode": (U64, [P, U64, U32, P]),
    "orc_wah_decode": (None, [P, U64, U32, U64, P, U64]),
    "orc_wah_op": (U64, [U32, P, U64, P, U64, U64, P]),
}

_lib = None
_ref = None
_wahref = None


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


def wah_ref() -> C.CDLL | None:
    """The reference's CPU WAH code (merle/host/wahCpu.c, wahConv.c), or None
    if not built."""
    global _wahref
    if _wahref is None and WAH_REF_LIB.exists():
        _wahref = C.CDLL(str(WAH_REF_LIB), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        _wahref.wahCmprsCPU.restype = C.c_size_t
        _wahref.wahCmprsCPU.argtypes = [P, C.c_size_t, P]
        _wahref.wahAndCPU.restype = C.c_void_p
        _wahref.wahAndCPU.argtypes = [P, P, P, P, P, P]
        _wahref.loadWahFile.restype = C.c_void_p
        _wahref.loadWahFile.argtypes = [C.c_char_p]
    return _wahref


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
        o.cols = {f: a.astype(nw.get(f, np.uint32), copy=False) for f, a in self.cols.items()}
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


def ngroups(tmpl: int, p) -> int:
    """Group count of a template query: the size of the reference's output
    array for it (s1ref one sum; s2ref 7 x mfgr width; s3ref a x b x years;
    s4ref a x b x years with its /10 and /40 scalings; ssb/cpuref.c:141-242)."""
    def years(dmin, dmax):
        return 1 if dmax <= dmin else _year(dmax - 1) - _year(dmin) + 1
    if tmpl == 1:
        return 1
    if tmpl == 2:
        return 7 * (p[1] - p[0]) if p[1] > p[0] else 1
    if tmpl == 3:
        a, b = p[1] - p[0], p[3] - p[2]
        if p[1] - p[0] >= 50:
            a, b = p[1] // 10 - p[0] // 10, p[3] // 10 - p[2] // 10
        return max(1, a * b * years(p[4], p[5]))
    a, b = p[3] - p[2], p[5] - p[4]
    if p[3] - p[2] >= 50:
        a = p[3] // 10 - p[2] // 10
    if p[5] - p[4] >= 200:
        b = p[5] // 40 - p[4] // 40
    return max(1, a * b * years(p[6], p[7]))


def _year(d: int) -> int:
    """ssbDateToYear (ssb/ssbdemo.h:28-39): day 0 = 1992-01-01 -> year index."""
    return int(np.searchsorted(np.array(_YEARS[1:]), d, side="right"))


def ref_answers(schema: "SsbSchema", n: int, qs, threads: int):
    """Each template query through the reference's own s1ref..s4ref
    (ssb/cpuref.c:141-242) over the first n rows of schema, one query per
    thread on `threads` threads (ssb_cpujoin's shape, ssb/cpuref.c:244-302):
    (answers, seconds).  An answer is the uint64 sum of s1ref, or the uint32
    group array s2ref..s4ref fill (ngroups values)."""
    import time
    from concurrent.futures import ThreadPoolExecutor
    r = ref()
    if r is None:
        raise RuntimeError("oracle/_ref/libcpuref.so is not built")

    def one(q):
        t = int(q.tmpl)
        k = {1: 6, 2: 4, 3: 6, 4: 8}[t]
        p = tuple(int(q.p[i]) for i in range(k))
        if t == 1:
            return np.array([r.s1ref(C.byref(schema), n, *p)], np.uint64)
        out = np.zeros(ngroups(t, p) + 1, np.uint32)  # one spare word: nothing may land there
        f = {2: r.s2ref, 3: r.s3ref, 4: r.s4ref}[t]
        f(C.byref(schema), n, *p, out.ctypes.data)
        if out[-1] != 0:
            raise RuntimeError(f"reference wrote past its group array for {t} {p}")
        return out[:-1]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max(1, threads)) as ex:
        res = list(ex.map(one, qs))
    return res, time.perf_counter() - t0


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


# ------------------------------------------------- algorithmic bytes (roofline)
# The canonical index of the star schema (levels coarse to fine) and, per
# template, the columns a plan must gather for every qualifying row (the key
# and value sources of s1op..s4op, ssb/lambdas.cuh:19-152) and the dimension
# arrays it probes.
_YEARS = [0, 366, 731, 1096, 1461, 1827, 2192, 2557]
_DM = [31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31]
_MONTHS = []
_d = 0
for _y in range(1992, 1999):
    for _m in range(12):
        _MONTHS.append(_d)
        _d += _DM[_m] + (1 if (_m == 1 and _y % 4 == 0) else 0)
_MONTHS.append(_d)
INDEX_LEVELS = {
    "date": (0, 2557, [_YEARS, _MONTHS]),
    "discount": (0, 11, [list(range(0, 12))]),
    "quantity": (1, 51, [list(range(1, 52))]),
    "custcity": (0, 250, [list(range(0, 251, 50)), list(range(0, 251, 10))]),
    "suppcity": (0, 250, [list(range(0, 251, 50)), list(range(0, 251, 10))]),
    "partmfgr": (0, 1000, [list(range(0, 1001, 200)), list(range(0, 1001, 40))]),
}
PREDS = {1: [("date", 0, 1), ("discount", 2, 3), ("quantity", 4, 5)],
         2: [("partmfgr", 0, 1), ("suppcity", 2, 3)],
         3: [("custcity", 0, 1), ("suppcity", 2, 3), ("date", 4, 5)],
         4: [("custcity", 0, 1), ("suppcity", 2, 3), ("partmfgr", 4, 5), ("date", 6, 7)]}
GATHER = {1: ["extendedprice", "discount"], 2: ["partkey", "orderdate", "revenue"],
          3: ["custkey", "suppcity", "orderdate", "revenue"],
          4: ["suppcity", "orderdate", "partkey", "revenue", "supplycost"]}
DIMS = {1: [], 2: ["partmfgr"], 3: ["custcity"], 4: ["partmfgr"]}


def _exact_bins(levels, lo, hi):
    """Bins of the coarsest-first exact cover of [lo, hi), or None."""
    x, n = lo, 0
    while x < hi:
        for b in levels:
            if x in b:
                j = b.index(x)
                if j + 1 < len(b) and b[j + 1] <= hi:
                    x, n = b[j + 1], n + 1
                    break
        else:
            return None
    return n


def canonical_bitmaps(tmpl: int, p) -> int:
    """Per predicate the fewer of (bins covering the range) and (bins covering
    its complement); a range no exact cover reaches counts its finest-level
    bins, edge bins included.  Full ranges read nothing."""
    total = 0
    for col, a, b in PREDS[tmpl]:
        dlo, dhi, levels = INDEX_LEVELS[col]
        lo, hi = max(p[a], dlo), min(p[b], dhi)
        if lo >= hi or (lo == dlo and hi == dhi):
            continue
        cands = []
        d = _exact_bins(levels, lo, hi)
        if d is not None:
            cands.append(d)
        c1 = _exact_bins(levels, dlo, lo) if dlo < lo else 0
        c2 = _exact_bins(levels, hi, dhi) if hi < dhi else 0
        if c1 is not None and c2 is not None:
            cands.append(c1 + c2)
        if not cands:
            f = levels[-1]
            cands.append(sum(1 for j in range(len(f) - 1) if f[j + 1] > lo and f[j] < hi))
        total += min(cands)
    return total


def canonical_bins(tmpl: int, p) -> set:
    """The bitmaps (column, level, bin) of canonical_bitmaps' choice per
    predicate: the exact cover or the exact cover of the complement, whichever
    has fewer bins (the finest level's bins when no exact cover exists)."""
    out = set()
    for col, a, b in PREDS[tmpl]:
        dlo, dhi, levels = INDEX_LEVELS[col]
        lo, hi = max(p[a], dlo), min(p[b], dhi)
        if lo >= hi or (lo == dlo and hi == dhi):
            continue

        def cover(x, y):
            bins = []
            while x < y:
                for li, bnd in enumerate(levels):
                    if x in bnd:
                        j = bnd.index(x)
                        if j + 1 < len(bnd) and bnd[j + 1] <= y:
                            bins.append((col, li, j))
                            x = bnd[j + 1]
                            break
                else:
                    return None
            return bins
        cands = []
        d = cover(lo, hi)
        if d is not None:
            cands.append(d)
        c1 = cover(dlo, lo) if dlo < lo else []
        c2 = cover(hi, dhi) if hi < dhi else []
        if c1 is not None and c2 is not None:
            cands.append(c1 + c2)
        if not cands:
            f = levels[-1]
            li = len(levels) - 1
            cands.append([(col, li, j) for j in range(len(f) - 1) if f[j + 1] > lo and f[j] < hi])
        out.update(min(cands, key=len))
    return out


def qualifying_mask(star: "StarHost", tmpl: int, p, nrows: int | None = None) -> np.ndarray:
    """Rows among the first nrows (default: all) that satisfy every predicate
    of the query (numpy, vectorised)."""
    n = star.n if nrows is None else min(nrows, star.n)
    cache = getattr(star, "_joined", None)
    if cache is None or cache[0] != n:
        c = {k: v[:n] for k, v in star.cols.items()}
        vals = {"date": c["orderdate"], "discount": c["discount"], "quantity": c["quantity"],
                "suppcity": c["suppcity"], "custcity": star.custcity[c["custkey"]],
                "partmfgr": star.partmfgr[c["partkey"]]}
        star._joined = cache = (n, vals)
    vals = cache[1]
    m = np.ones(n, bool)
    for col, a, b in PREDS[tmpl]:
        v = vals[col]
        m &= (v >= p[a]) & (v < p[b])
    return m


def algo_bytes(star: "StarHost", scale: float, nrows: int, tmpl: int, p, ngroups: int, widths: dict,
               sample_n: int | None = None) -> dict:
    """Plan-independent algorithmic bytes of one query over `nrows` rows:
    canonical bitmaps + the 32-byte sectors of every gathered column that hold
    a qualifying row (counted exactly on the first sample_n rows of the host
    table `star`, scaled by `scale`) + probed dimension arrays + the int64
    group outputs."""
    W = (nrows + 31) // 32
    bm = canonical_bitmaps(tmpl, p) * W * 4
    m = qualifying_mask(star, tmpl, p, sample_n)
    rows = np.flatnonzero(m)
    sec = 0
    for col in GATHER[tmpl]:
        w = widths[col]
        sec += len(np.unique(rows // (32 // w))) * 32
    dims = sum(len(getattr(star, d)) * getattr(star, d).dtype.itemsize for d in DIMS[tmpl])
    return {"bitmap": bm, "gather": int(sec * scale), "dims": dims, "out": 8 * ngroups,
            "total": int(bm + sec * scale + dims + 8 * ngroups), "rows": int(len(rows) * scale)}


# ---------------------------------------------------------------- WAH streams
def wah_encode(bitmap: np.ndarray, nrows: int, order: int = 0) -> np.ndarray:
    bm = np.ascontiguousarray(bitmap, dtype=np.uint32)
    G = (nrows + 30) // 31
    out = np.zeros(max(1, G), np.uint32)
    n = lib().orc_wah_encode(ptr(bm), nrows, order, ptr(out))
    return out[:n].copy()


def wah_decode(wah: np.ndarray, nrows: int, order: int = 0) -> np.ndarray:
    w = np.ascontiguousarray(wah, dtype=np.uint32)
    stride = ((nrows + 31) // 32 + 31) // 32 * 32
    bm = np.zeros(max(1, stride), np.uint32)
    lib().orc_wah_decode(ptr(w) if len(w) else None, len(w), order, nrows, ptr(bm), stride)
    return bm[:stride]


def wah_op(op: int, a: np.ndarray, b: np.ndarray, ngroups: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    out = np.zeros(max(1, ngroups), np.uint32)
    n = lib().orc_wah_op(op, ptr(a) if len(a) else None, len(a), ptr(b) if len(b) else None, len(b), ngroups,
                         ptr(out))
    return out[:n].copy()
