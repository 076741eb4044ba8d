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
