"""Host-side mirror of the reference's operator interface.

Reference names are kept so that code and tests read like the reference's:

- ``Instr`` / ``Vprg`` / ``Col``: ``vprg::instr``, ``vprg`` and ``col``
  (primitive.cuh:135-198);
- ``s1op`` .. ``s4op``: the SSB op functors (ssb/lambdas.cuh:19-152);
- ``synth_op``: the synthetic star query's ``_op`` (synth/synthdemo.cu:7-53);
- ``flat_op``: the flat-table query (a range AND b in a set AND c range,
  SUM(e*d)).

Each builder turns the functor's fields into the declarative ``mb_op`` of the
C ABI.  Columns are passed as numpy arrays (host pointers: for the CPU oracle)
or torch tensors (device pointers: for the CUDA library); the builder keeps a
reference to every buffer so pointers stay valid while the descriptor lives.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Sequence

from . import abi

# ssbDateToYear thresholds (ssb/ssbdemo.h:10-26): day numbers from 1992-01-01.
SSBDATE_920101 = 0
SSBDATE_930101 = 366
SSBDATE_940101 = 731
SSBDATE_940201 = 762
SSBDATE_940204 = 765
SSBDATE_940211 = 772
SSBDATE_940301 = 790
SSBDATE_940501 = 851
SSBDATE_940901 = 974
SSBDATE_950101 = 1096
SSBDATE_960101 = 1461
SSBDATE_970101 = 1827
SSBDATE_971201 = 2161
SSBDATE_980101 = 2192
SSBDATE_990101 = 2557
YEAR_START = [0, 366, 731, 1096, 1461, 1827, 2192, 2557]


def date_to_year(d: int) -> int:
    """ssbDateToYear (ssb/ssbdemo.h:28-39)."""
    y = 0
    for k in range(1, 7):
        if d >= YEAR_START[k]:
            y = k
    return y


def ptr_width(x: Any) -> tuple[int, int]:
    """(address, element bytes) of a numpy array or torch tensor."""
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr()), int(x.element_size())
    return int(x.ctypes.data), int(x.dtype.itemsize)


def nelem(x: Any) -> int:
    return int(x.numel()) if hasattr(x, "numel") else int(x.size)


@dataclass
class Src:
    """A value source: col[row], or col[fk[row]] when fk is given."""
    col: Any
    fk: Any = None
    checked: bool = True  # keys >= len(col) eliminate the row


@dataclass
class Op:
    """Builder of an mb_op: sources, AND of OR-clauses, key fields, value."""
    srcs: list = field(default_factory=list)
    clauses: list = field(default_factory=list)   # [[(src, lo, hi), ...], ...]
    keys: list = field(default_factory=list)      # [(src, xform, div, base, mul)]
    vkind: int = abi.V_ONE
    va: int = 0
    vb: int = 0

    def to_c(self) -> abi.mb_op:
        o = abi.mb_op()
        if len(self.srcs) > abi.MB_MAXSRC:
            raise ValueError("too many sources")
        o.nsrc = len(self.srcs)
        keep = []
        for i, s in enumerate(self.srcs):
            p, w = ptr_width(s.col)
            o.src[i].col = p
            o.src[i].width = w
            keep.append(s.col)
            if s.fk is not None:
                o.src[i].fk = ptr_width(s.fk)[0]
                o.src[i].dimsz = nelem(s.col) if s.checked else 0
                keep.append(s.fk)
        o.nclause = len(self.clauses)
        t = 0
        for c, cl in enumerate(self.clauses):
            o.clause_len[c] = len(cl)
            for (src, lo, hi) in cl:
                o.terms[t].src, o.terms[t].lo, o.terms[t].hi = src, lo, hi
                t += 1
        o.nkey = len(self.keys)
        for k, (src, xf, div, base, mul) in enumerate(self.keys):
            kk = o.keys[k]
            kk.src, kk.xform, kk.div, kk.base, kk.mul = src, xf, div, base & 0xFFFFFFFF, mul & 0xFFFFFFFF
        o.vkind, o.va, o.vb = self.vkind, self.va, self.vb
        o._keep = keep  # type: ignore[attr-defined]
        return o


def s1op(dateMin, dateMax, loOrderDate, discntMin, discntMax, loDiscount, qtyMin, qtyMax, loQuantity,
         extendedPrice) -> Op:
    """s1op (ssb/lambdas.cuh:19-38): SUM(extendedprice * discount), 1 group."""
    return Op(srcs=[Src(loOrderDate), Src(loDiscount), Src(loQuantity), Src(extendedPrice)],
              clauses=[[(0, dateMin, dateMax)], [(1, discntMin, discntMax)], [(2, qtyMin, qtyMax)]],
              keys=[], vkind=abi.V_MUL, va=3, vb=1)


def s2op(loPartKey, pMfgrMin, pMfgrMax, partMfgr, sCityMin, sCityMax, loSuppCity, loOrderDate,
         loRevenue) -> Op:
    """s2op (ssb/lambdas.cuh:40-62): group (mfgr - min) + year * (max - min)."""
    return Op(srcs=[Src(loSuppCity), Src(partMfgr, loPartKey), Src(loOrderDate), Src(loRevenue)],
              clauses=[[(0, sCityMin, sCityMax)], [(1, pMfgrMin, pMfgrMax)]],
              keys=[(1, abi.X_ID, 1, pMfgrMin, 1), (2, abi.X_YEAR, 1, 0, pMfgrMax - pMfgrMin)],
              vkind=abi.V_COL, va=3)


def s3op(loCustKey, cCityMin, cCityMax, custCity, sCityMin, sCityMax, loSuppCity, dateMin, dateMax,
         loOrderDate, loRevenue) -> Op:
    """s3op (ssb/lambdas.cuh:64-102): group a*b*(year-ymin) + a*(cCity-cmin) + (sCity-smin),
    cities scaled to nations (/10) when the customer range spans >= 50 cities."""
    cmn, cmx, smn, smx = cCityMin, cCityMax, sCityMin, sCityMax
    xf, div = abi.X_ID, 1
    if cCityMax - cCityMin >= 50:
        cmn, cmx, smn, smx = cmn // 10, cmx // 10, smn // 10, smx // 10
        xf, div = abi.X_DIV, 10
    a, b = cmx - cmn, smx - smn
    ymin = date_to_year(dateMin)
    return Op(srcs=[Src(loSuppCity), Src(loOrderDate), Src(custCity, loCustKey), Src(loRevenue)],
              clauses=[[(0, sCityMin, sCityMax)], [(1, dateMin, dateMax)], [(2, cCityMin, cCityMax)]],
              keys=[(1, abi.X_YEAR, 1, ymin, a * b), (2, xf, div, cmn, a), (0, xf, div, smn, 1)],
              vkind=abi.V_COL, va=3)


def s4op(loCustKey, loPartKey, cCityMin, cCityMax, custCity, sCityMin, sCityMax, loSuppCity, pMfgrMin,
         pMfgrMax, partMfgr, dateMin, dateMax, loOrderDate, loRevenue, loSupplyCost) -> Op:
    """s4op (ssb/lambdas.cuh:104-152): value revenue - supplycost, group
    a*b*(year-ymin) + a*(sCity-smin) + (mfgr-pmin) with /10 and /40 scaling."""
    smn, smx, sxf, sdiv = sCityMin, sCityMax, abi.X_ID, 1
    if sCityMax - sCityMin >= 50:
        smn, smx, sxf, sdiv = smn // 10, smx // 10, abi.X_DIV, 10
    pmn, pmx, pxf, pdiv = pMfgrMin, pMfgrMax, abi.X_ID, 1
    if pMfgrMax - pMfgrMin >= 200:
        pmn, pmx, pxf, pdiv = pmn // 40, pmx // 40, abi.X_DIV, 40
    a, b = smx - smn, pmx - pmn
    ymin = date_to_year(dateMin)
    return Op(srcs=[Src(loSuppCity), Src(loOrderDate), Src(custCity, loCustKey), Src(partMfgr, loPartKey),
                    Src(loRevenue), Src(loSupplyCost)],
              clauses=[[(0, sCityMin, sCityMax)], [(1, dateMin, dateMax)], [(2, cCityMin, cCityMax)],
                       [(3, pMfgrMin, pMfgrMax)]],
              keys=[(1, abi.X_YEAR, 1, ymin, a * b), (0, sxf, sdiv, smn, a), (3, pxf, pdiv, pmn, 1)],
              vkind=abi.V_SUB, va=4, vb=5)


def synth_op(factattr1, factattr2, fkey, dimattr1, dimattr2, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi) -> Op:
    """_op (synth/synthdemo.cu:7-53): (a1 in R1 OR a2 in R2) AND dim.a1 in R3,
    GROUP BY dim.a2 (256 groups), COUNT.  The reference does not bound-check
    the key (checked=False keeps that)."""
    return Op(srcs=[Src(factattr1), Src(factattr2), Src(dimattr1, fkey, checked=False),
                    Src(dimattr2, fkey, checked=False)],
              clauses=[[(0, fa1lo, fa1hi), (1, fa2lo, fa2hi)], [(2, da1lo, da1hi)]],
              keys=[(3, abi.X_ID, 1, 0, 1)], vkind=abi.V_ONE)


def flat_op(a, b, c, d, e, alo, ahi, bset: Sequence[int], clo, chi) -> Op:
    """a in [alo,ahi) AND b in bset AND c in [clo,chi): SUM(int64 e*d), 1 group."""
    return Op(srcs=[Src(a), Src(b), Src(c), Src(d), Src(e)],
              clauses=[[(0, alo, ahi)], [(1, v, v + 1) for v in bset], [(2, clo, chi)]],
              keys=[], vkind=abi.V_MUL, va=4, vb=3)


@dataclass
class Col:
    """mybmpidx::col: middle bins inside the range, optional edge bins."""
    middle: list = field(default_factory=list)
    leftmost: Any = None
    rightmost: Any = None

    def is_nochk(self) -> bool:
        return self.leftmost is None and self.rightmost is None


def Instr(opcode: int, dstreg: int = 0, src1: int = 0, src2: int = 0) -> tuple:
    return (opcode, dstreg, src1, src2)


@dataclass
class Vprg:
    """mybmpidx::vprg: memory operands + instructions; result in r0."""
    factsz: int
    cols: list
    instrs: list

    def is_nochk(self) -> bool:
        return all(c.is_nochk() for c in self.cols)

    def to_c(self) -> abi.mb_vprg:
        p = abi.mb_vprg()
        p.factsz = self.factsz
        if len(self.cols) > abi.MB_MAXCOLS or len(self.instrs) > abi.MB_MAXNINSTR:
            raise ValueError("program exceeds MB_MAXCOLS / MB_MAXNINSTR")
        p.ncols = len(self.cols)
        keep = []
        for i, c in enumerate(self.cols):
            arr = (C.c_void_p * max(1, len(c.middle)))(*[ptr_width(m)[0] for m in c.middle])
            keep.append(arr)
            keep.extend(c.middle)
            p.cols[i].nmiddle = len(c.middle)
            p.cols[i].middle = C.cast(arr, C.POINTER(C.c_void_p))
            if c.leftmost is not None:
                p.cols[i].leftmost = ptr_width(c.leftmost)[0]
                keep.append(c.leftmost)
            if c.rightmost is not None:
                p.cols[i].rightmost = ptr_width(c.rightmost)[0]
                keep.append(c.rightmost)
        for i, ins in enumerate(self.instrs):
            p.instrs[i].opcode, p.instrs[i].dstreg, p.instrs[i].src1, p.instrs[i].src2 = ins
        p._keep = keep  # type: ignore[attr-defined]
        return p
