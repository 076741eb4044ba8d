"""Shared test helpers: the reference's SSB query set and recipe layouts.

The 13 SSB parameterisations are those of ssb_cpujoin (ssb/cpuref.c:252-298);
the recipe inputs follow s1bmp..s4bmp (ssb/controlled-demo.cu:206-283).  Every
builder works on host numpy arrays (for the CPU oracle) or device torch tensors
(for the CUDA library) alike, through merle_b200.ops.
"""
from __future__ import annotations

import numpy as np

from merle_b200 import abi, ops

# (template, args, nr_grp) in result-slot order (ssb/cpuref.c:252-298).
SSB13 = [
    ("s1", (366, 731, 1, 4, 0, 25), 1),
    ("s1", (731, 762, 4, 7, 26, 36), 1),
    ("s1", (765, 772, 5, 8, 26, 36), 1),
    ("s2", (40, 80, 150, 200), 280),
    ("s2", (260, 268, 200, 250), 56),
    ("s2", (260, 261, 50, 100), 7),
    ("s3", (200, 250, 200, 250, 0, 2192), 150),
    ("s3", (190, 200, 190, 200, 0, 2192), 600),
    ("s3", (51, 55, 51, 55, 0, 2192), 96),
    ("s3", (51, 55, 51, 55, 2161, 2192), 16),
    ("s4", (150, 200, 150, 200, 0, 400, 0, 2557), 350),
    ("s4", (150, 200, 150, 200, 0, 400, 1827, 2557), 100),
    ("s4", (150, 200, 190, 200, 120, 160, 1827, 2557), 800),
]
SLOTS = np.cumsum([0] + [g for _, _, g in SSB13])
NODIM = 0xFFFFFFFF


def nbit_of(x) -> int:
    return ops.ptr_width(x)[1] * 8


def ssb_op(star, q: str, a: tuple) -> ops.Op:
    """The reference op functor for one query, over columns of `star`
    (a mapping with custkey, partkey, orderdate, ... and dims custcity/partmfgr)."""
    c = star
    if q == "s1":
        dmin, dmax, dimin, dimax, qmin, qmax = a
        return ops.s1op(dmin, dmax, c["orderdate"], dimin, dimax, c["discount"], qmin, qmax, c["quantity"],
                        c["extendedprice"])
    if q == "s2":
        pmin, pmax, smin, smax = a
        return ops.s2op(c["partkey"], pmin, pmax, c.partmfgr, smin, smax, c["suppcity"], c["orderdate"],
                        c["revenue"])
    if q == "s3":
        cmin, cmax, smin, smax, dmin, dmax = a
        return ops.s3op(c["custkey"], cmin, cmax, c.custcity, smin, smax, c["suppcity"], dmin, dmax,
                        c["orderdate"], c["revenue"])
    cmin, cmax, smin, smax, pmin, pmax, dmin, dmax = a
    return ops.s4op(c["custkey"], c["partkey"], cmin, cmax, c.custcity, smin, smax, c["suppcity"], pmin, pmax,
                    c.partmfgr, dmin, dmax, c["orderdate"], c["revenue"], c["supplycost"])


def ssb_recipe(star, q: str, a: tuple):
    """(preds, instrs) of s1bmp..s4bmp: preds = [(fk|None, attr, min, max)]."""
    c = star
    L, A = abi.ORM, abi.ANDM
    if q == "s1":
        dmin, dmax, dimin, dimax, qmin, qmax = a
        return ([(None, c["orderdate"], dmin, dmax), (None, c["discount"], dimin, dimax),
                 (None, c["quantity"], qmin, qmax)], [(L, 0, 0, 0), (A, 0, 1, 0), (A, 0, 2, 0)])
    if q == "s2":
        pmin, pmax, smin, smax = a
        return ([(c["partkey"], c.partmfgr, pmin, pmax), (None, c["suppcity"], smin, smax)],
                [(L, 0, 0, 0), (A, 0, 1, 0)])
    if q == "s3":
        cmin, cmax, smin, smax, dmin, dmax = a
        return ([(c["custkey"], c.custcity, cmin, cmax), (None, c["suppcity"], smin, smax),
                 (None, c["orderdate"], dmin, dmax)], [(L, 0, 0, 0), (A, 0, 1, 0), (A, 0, 2, 0)])
    cmin, cmax, smin, smax, pmin, pmax, dmin, dmax = a
    preds = [(c["custkey"], c.custcity, cmin, cmax), (None, c["suppcity"], smin, smax),
             (c["partkey"], c.partmfgr, pmin, pmax), (None, c["orderdate"], dmin, dmax)]
    ins = [(L, 0, 0, 0), (A, 0, 1, 0), (A, 0, 2, 0), (A, 0, 3, 0)]
    if dmin <= 0 and dmax >= 2557:  # s4bmp drops a full date range (controlled-demo.cu:280-281)
        preds, ins = preds[:3], ins[:3]
    return preds, ins


def recipe_ranges(kind: str, preds):
    """Per predicate: (middle ranges, leftmost range|None, rightmost range|None)
    of recipe::perfect / many_or / candchk (bmpidx_create.cu:228-316), with the
    reference's uint32 arithmetic."""
    M = 0xFFFFFFFF
    out = []
    for i, (_, _, mn, mx) in enumerate(preds):
        step = ((mx - mn) & M) // 3
        if kind == "perfect":
            out.append(([(mn, mx)], None, None))
        elif kind == "many_or" or (kind == "candchk" and i >= 2):
            out.append(([(mn, mx)], None, None) if step == 0 else
                       ([(mn, mn + step), (mn + step, mn + 2 * step), (mn + 2 * step, mx)], None, None))
        elif i == 0:
            if step == 0:
                out.append(([], (mn, mx + 1), None))
            else:
                lo = max(mn, step // 2) - step // 2
                out.append(([(mn + step, mn + 2 * step), (mn + 2 * step, mx)], (lo, mn + step), None))
        else:
            if step == 0:
                out.append(([], None, ((mn - 1) & M, mx)))
            else:
                out.append(([(mn, mn + step), (mn + step, mn + 2 * step)], None,
                            (mn + 2 * step, mx + step // 2)))
    return out


def host_bitmap(orc, fk, attr, n, lo, hi):
    """One bitmap built by the oracle (create_select / create_join)."""
    s = abi.mb_src()
    s.col = orc.ptr(attr)
    s.width = attr.dtype.itemsize
    if fk is not None:
        s.fk = orc.ptr(fk)
        s.dimsz = 0
    bm, _ = orc.bitmap_create(s, n, [lo], [hi])
    return bm[0].copy()


def host_recipe(orc, kind: str, preds, instrs, n):
    """The recipe's program over oracle-built host bitmaps."""
    cols = []
    for (fk, attr, _, _), (mids, left, right) in zip(preds, recipe_ranges(kind, preds)):
        c = ops.Col(middle=[host_bitmap(orc, fk, attr, n, lo, hi) for lo, hi in mids])
        if left is not None:
            c.leftmost = host_bitmap(orc, fk, attr, n, *left)
        if right is not None:
            c.rightmost = host_bitmap(orc, fk, attr, n, *right)
        cols.append(c)
    return ops.Vprg(n, cols, instrs)
