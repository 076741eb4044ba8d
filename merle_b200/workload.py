"""Seeded query workloads over the star schema (the four templates of
mb_query): the reference's 13 SSB parameterisations (ssb/cpuref.c:252-298)
and seeded random mixes.

Every generated query keeps the reference's group-index formula well inside
its group count, so the reference's own CPU code (which indexes its output
array without a bound check, ssb/cpuref.c:203,240) can run it: template 3 uses
equally wide customer and supplier ranges, template 4 a part range whose
(scaled) width is at least the supplier range's.
"""
from __future__ import annotations

import numpy as np

from . import abi

YEAR_START = [0, 366, 731, 1096, 1461, 1827, 2192, 2557]
_DM = [31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31]
MONTH_START = []
_d = 0
for _y in range(1992, 1999):
    for _m in range(12):
        MONTH_START.append(_d)
        _d += _DM[_m] + (1 if (_m == 1 and _y % 4 == 0) else 0)
MONTH_START.append(_d)

SSB13 = [
    (1, (366, 731, 1, 4, 0, 25)), (1, (731, 762, 4, 7, 26, 36)), (1, (765, 772, 5, 8, 26, 36)),
    (2, (40, 80, 150, 200)), (2, (260, 268, 200, 250)), (2, (260, 261, 50, 100)),
    (3, (200, 250, 200, 250, 0, 2192)), (3, (190, 200, 190, 200, 0, 2192)), (3, (51, 55, 51, 55, 0, 2192)),
    (3, (51, 55, 51, 55, 2161, 2192)),
    (4, (150, 200, 150, 200, 0, 400, 0, 2557)), (4, (150, 200, 150, 200, 0, 400, 1827, 2557)),
    (4, (150, 200, 190, 200, 120, 160, 1827, 2557)),
]
TEMPLATE_NAME = {1: "s1", 2: "s2", 3: "s3", 4: "s4"}


def ssb13() -> list[abi.mb_query]:
    return [abi.query(t, *p) for t, p in SSB13]


def as_tuple(q: abi.mb_query) -> tuple[int, tuple]:
    n = {1: 6, 2: 4, 3: 6, 4: 8}[q.tmpl]
    return q.tmpl, tuple(int(q.p[i]) for i in range(n))


def _date_range(r: np.random.Generator, level: str):
    if level == "year":
        y0 = int(r.integers(0, 7))
        y1 = int(r.integers(y0 + 1, min(7, y0 + 3) + 1))
        return YEAR_START[y0], YEAR_START[y1]
    if level == "month":
        m0 = int(r.integers(0, 84))
        m1 = int(r.integers(m0 + 1, min(84, m0 + 13) + 1))
        return MONTH_START[m0], MONTH_START[m1]
    if level == "week":
        d0 = int(r.integers(0, 2550))
        return d0, d0 + 7
    d0 = int(r.integers(0, 2500))
    return d0, d0 + int(r.integers(1, 400))


def _city_range(r: np.random.Generator, level: str, width: int | None = None):
    if level == "region":
        x = int(r.integers(0, 5)) * 50
        return x, x + 50
    if level == "nation":
        x = int(r.integers(0, 25)) * 10
        return x, x + 10
    w = width or int(r.integers(1, 10))
    x = int(r.integers(0, 250 - w + 1))
    return x, x + w


def random_query(r: np.random.Generator, tmpl: int | None = None, narrow: float = 0.3) -> abi.mb_query:
    """One seeded query; `narrow` is the chance of city / brand / week level
    constants (very selective) instead of region / category / year level."""
    t = int(tmpl or r.integers(1, 5))
    fine = r.random() < narrow
    if t == 1:
        d = _date_range(r, "week" if fine else str(r.choice(["year", "month", "any"])))
        di0 = int(r.integers(0, 9))
        q0 = int(r.integers(1, 45))
        qw = int(r.integers(1, 11)) if fine else int(r.integers(5, 26))
        return abi.query(1, d[0], d[1], di0, di0 + int(r.integers(1, 4)), q0, min(51, q0 + qw))
    if t == 2:
        if fine:
            b = int(r.integers(0, 1000 - 8))
            m = (b, b + int(r.integers(1, 9)))
        else:
            c = int(r.integers(0, 25)) * 40
            m = (c, c + 40) if r.random() < 0.7 else (c // 200 * 200, c // 200 * 200 + 200)
        s = _city_range(r, "city" if fine else str(r.choice(["region", "nation"])))
        return abi.query(2, m[0], m[1], s[0], s[1])
    if t == 3:
        lvl = "city" if fine else str(r.choice(["region", "nation"]))
        w = int(r.integers(1, 10)) if lvl == "city" else None
        c = _city_range(r, lvl, w)
        s = _city_range(r, lvl, w if w else None)
        if lvl != "city" and (s[1] - s[0]) != (c[1] - c[0]):
            s = (s[0], s[0] + c[1] - c[0])
        d = _date_range(r, "week" if fine else "year")
        return abi.query(3, c[0], c[1], s[0], s[1], d[0], d[1])
    c = _city_range(r, "nation" if fine else "region")
    s = _city_range(r, str(r.choice(["city", "nation"])) if fine else "region")
    sw = (s[1] - s[0]) // 10 if s[1] - s[0] >= 50 else s[1] - s[0]
    if r.random() < 0.5:
        p0 = int(r.integers(0, 4)) * 200
        p = (p0, p0 + 400)                       # two mfgrs: /40 scaling, 10 categories
    else:
        w = max(sw, int(r.integers(10, 41)))
        p0 = int(r.integers(0, 1000 - w))
        p = (p0, p0 + w)
    if (p[1] - p[0]) >= 200 and (p[1] - p[0]) // 40 < sw:
        p = (0, 400)
    d = _date_range(r, "year") if r.random() < 0.6 else (0, 2557)
    return abi.query(4, c[0], c[1], s[0], s[1], p[0], p[1], d[0], d[1])


def random_mix(seed: int, n: int, narrow: float = 0.3) -> list[abi.mb_query]:
    r = np.random.default_rng(seed)
    return [random_query(r, None, narrow) for _ in range(n)]


# ------------------------------------------------ selectivity-spanning mix
NDAYS, NCITY, NMFGR = 2556, 250, 1000


def est_selectivity(q: abi.mb_query) -> float:
    """Expected fraction of fact rows a query selects on the star schema's
    distributions (order date uniform over 2,556 days, quantity U[1,50],
    discount U[0,10], customer / supplier city U[0,249] and part mfgr code
    U[0,999] per dimension row, foreign keys uniform): the product of the
    predicates' fractions."""
    t, p = as_tuple(q)

    def frac(lo, hi, dom_lo, dom_hi):
        return max(0, min(hi, dom_hi) - max(lo, dom_lo)) / (dom_hi - dom_lo)
    if t == 1:
        return frac(p[0], p[1], 0, NDAYS) * frac(p[2], p[3], 0, 11) * frac(p[4], p[5], 1, 51)
    if t == 2:
        return frac(p[0], p[1], 0, NMFGR) * frac(p[2], p[3], 0, NCITY)
    if t == 3:
        return frac(p[0], p[1], 0, NCITY) * frac(p[2], p[3], 0, NCITY) * frac(p[4], p[5], 0, NDAYS)
    return (frac(p[0], p[1], 0, NCITY) * frac(p[2], p[3], 0, NCITY) * frac(p[4], p[5], 0, NMFGR)
            * frac(p[6], p[7], 0, NDAYS))


def _loguni_int(r: np.random.Generator, lo: int, hi: int) -> int:
    """An integer in [lo, hi], log-uniformly distributed."""
    return int(min(hi, max(lo, round(float(np.exp(r.uniform(np.log(lo), np.log(hi + 0.999))) - 0.499)))))


def _span(r: np.random.Generator, width: int, dom: int, align: int = 1) -> tuple[int, int]:
    """[x, x + width) inside [0, dom), x a multiple of align."""
    x = int(r.integers(0, (dom - width) // align + 1)) * align
    return x, x + width


def broad_query(r: np.random.Generator, tmpl: int) -> abi.mb_query:
    """A query of template tmpl whose range widths are drawn log-uniformly,
    so that its selectivity can lie anywhere from the template's least to
    the whole table.  The reference's group-index formulas stay inside their
    group counts (its CPU code writes its output without a bound check,
    ssb/cpuref.c:157-242): template 3 takes equally wide customer and supplier
    ranges, aligned to nations (10 cities) when 50 or more wide (the /10
    scaling); template 4 aligns a supplier range of 50 or more to nations and a
    part range of 200 or more to categories (the /40 scaling), the part
    range's scaled width at least the supplier range's."""
    if tmpl == 1:
        d = _span(r, _loguni_int(r, 1, NDAYS), NDAYS)
        di = _span(r, _loguni_int(r, 1, 11), 11)
        qw = _loguni_int(r, 1, 50)
        q0 = int(r.integers(1, 51 - qw + 1))
        return abi.query(1, d[0], d[1], di[0], di[1], q0, q0 + qw)
    if tmpl == 2:
        m = _span(r, _loguni_int(r, 1, NMFGR), NMFGR)
        s = _span(r, _loguni_int(r, 1, NCITY), NCITY)
        return abi.query(2, m[0], m[1], s[0], s[1])
    if tmpl == 3:
        w = _loguni_int(r, 1, NCITY)
        if w >= 50:
            w = w // 10 * 10
            c, s = _span(r, w, NCITY, 10), _span(r, w, NCITY, 10)
        else:
            c, s = _span(r, w, NCITY), _span(r, w, NCITY)
        d = _span(r, _loguni_int(r, 1, NDAYS), NDAYS)
        return abi.query(3, c[0], c[1], s[0], s[1], d[0], d[1])
    c = _span(r, _loguni_int(r, 1, NCITY), NCITY)
    sw = _loguni_int(r, 1, NCITY)
    if sw >= 50:
        sw = sw // 10 * 10
        s = _span(r, sw, NCITY, 10)
        ssc = sw // 10
    else:
        s = _span(r, sw, NCITY)
        ssc = sw
    pw = max(_loguni_int(r, 1, NMFGR), ssc)
    if pw >= 200 and max(pw // 40, ssc) * 40 > NMFGR:
        pw = 199  # the scaled part range cannot reach the supplier range's width: stay unscaled
    if pw >= 200:
        pw = max(pw // 40, ssc) * 40
        p = _span(r, pw, NMFGR, 40)
    else:
        p = _span(r, pw, NMFGR)
    d = _span(r, _loguni_int(r, 1, NDAYS), NDAYS)
    return abi.query(4, c[0], c[1], s[0], s[1], p[0], p[1], d[0], d[1])


def span_mix(seed: int, n: int, lo: float = 1e-6, hi: float = 0.5, tries: int = 4000) -> list[abi.mb_query]:
    """n queries of the four templates (in turn) whose expected
    selectivities (est_selectivity) follow a log-uniform spread over
    [lo, hi]: for each query a target drawn log-uniformly, then the closest of
    up to `tries` broad_query draws (within 10 % ends the search).  The
    first and last targets are lo and hi themselves, so the mix reaches both
    ends."""
    r = np.random.default_rng(seed)
    targets = np.exp(r.uniform(np.log(lo), np.log(hi), n))
    if n >= 2:
        targets[0], targets[-1] = lo, hi
    out = []
    for i, tgt in enumerate(targets):
        t = 2 if (i == n - 1 and n >= 2) else 1 + i % 4  # template 2 reaches the widest end most easily
        best, best_err = None, np.inf
        for _ in range(tries):
            q = broad_query(r, t)
            s = est_selectivity(q)
            if s <= 0:
                continue
            err = abs(np.log(s / tgt))
            if err < best_err:
                best, best_err = q, err
                if err < 0.1:
                    break
        out.append(best)
    return out
