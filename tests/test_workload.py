"""The benchmark's selectivity-spanning query mix (workload.span_mix): it
reaches both ends of [1e-6, 0.5], covers the four templates, and every
query keeps the reference's group index inside its group array, so the
reference's own CPU code (which writes that array without a bound check,
ssb/cpuref.c:157-242) can answer it.  Then the mix through the reference's
s1ref..s4ref equals the oracle's int64 restatement mod 2^32 on a small
table."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from merle_b200 import workload as WL


def _year(d):
    from oracle import oracle as O
    return O._year(d)


def _max_group(t, p):
    """Largest group index the reference's formulas (ssb/cpuref.c:157-242)
    produce for any row passing the query's filters, by enumeration of the
    dimension values and years in range."""
    years = range(_year(p[-2]), _year(max(p[-2], p[-1] - 1)) + 1)
    ymin = _year(p[-2])
    if t == 2:
        return max((m - p[0]) + y * (p[1] - p[0]) for m in range(p[0], p[1]) for y in years)
    if t == 3:
        c0, c1, s0, s1 = p[:4]
        sc = c1 - c0 >= 50
        best = 0
        for c in range(c0, c1):
            for s in range(s0, s1):
                cc, ss, cm, cx, sm, sx = c, s, c0, c1, s0, s1
                if sc:
                    cc, ss, cm, cx, sm, sx = c // 10, s // 10, c0 // 10, c1 // 10, s0 // 10, s1 // 10
                a, b = cx - cm, sx - sm
                for y in years:
                    best = max(best, a * b * (y - ymin) + a * (cc - cm) + (ss - sm))
        return best
    s0, s1, m0, m1 = p[2:6]
    best = 0
    ssc, msc = s1 - s0 >= 50, m1 - m0 >= 200
    for s in range(s0, s1):
        ss, sm, sx = (s // 10, s0 // 10, s1 // 10) if ssc else (s, s0, s1)
        for m in range(m0, m1):
            mm, mn, mx = (m // 40, m0 // 40, m1 // 40) if msc else (m, m0, m1)
            a, b = sx - sm, mx - mn
            best = max(best, max(a * b * (y - ymin) + a * (ss - sm) + (mm - mn) for y in years))
    return best


@pytest.mark.parametrize("seed,n", [(3, 64), (5, 256)])
def test_span_mix_group_index_in_bounds(seed, n):
    from oracle import oracle as O
    for q in WL.span_mix(seed, n):
        t, p = WL.as_tuple(q)
        if t == 1:
            continue
        assert _max_group(t, p) < O.ngroups(t, p), (t, p)


def test_span_mix_reaches_both_ends():
    qs = WL.span_mix(3, 64)
    s = np.array([WL.est_selectivity(q) for q in qs])
    assert s.min() <= 1.5e-6 and s.max() >= 0.4
    assert {q.tmpl for q in qs} == {1, 2, 3, 4}
    # log-uniform: about a sixth of the decades' span in each sixth
    dec = np.log10(s)
    assert np.histogram(dec, bins=4, range=(-6, np.log10(0.5)))[0].min() >= 8


def test_span_mix_seeded():
    a = [WL.as_tuple(q) for q in WL.span_mix(3, 16)]
    b = [WL.as_tuple(q) for q in WL.span_mix(3, 16)]
    assert a == b


def test_span_mix_reference_equals_oracle(orc):
    """s1ref..s4ref over a 300,000-row star table equal the oracle's int64
    restatement, mod 2^32 for the group arrays."""
    if orc.ref() is None:
        pytest.skip("oracle/_ref not built")
    n = 300_000
    star = orc.StarHost(2, 1, n)
    schema = star.ssb_schema()
    od = star.orc_ssb()
    qs = WL.span_mix(3, 64)
    got, _ = orc.ref_answers(schema, n, qs, 4)
    L = orc.lib()
    for q, g in zip(qs, got):
        t, p = WL.as_tuple(q)
        ng = orc.ngroups(t, p)
        if t == 1:
            want = L.orc_s1(C.byref(od), n, *p, None)
            assert int(g[0]) == want % (1 << 64), p
            continue
        out = np.zeros(ng, np.int64)
        f = {2: L.orc_s2, 3: L.orc_s3, 4: L.orc_s4}[t]
        f(C.byref(od), n, *p, out.ctypes.data, ng, None)
        np.testing.assert_array_equal(g, out.astype(np.uint64).astype(np.uint32), err_msg=str((t, p)))
