"""CPU tests that pin the oracle to the reference.

- the generator's Zipf table is exact, and generated values match the
  committed golden heads;
- the oracle's direct restatements and its declarative-op path reproduce the
  reference's own ssb_cpujoin / synth_ref outputs (tests/golden/, produced by
  the reference's functions) mod 2^32, and agree with each other in int64;
- the fused plan over every recipe layout (perfect / many_or / candchk, i.e.
  nochk and chk algebra) equals the no-index plan, the reference's own
  differential check (ssb/cpuref.c:326-349, synth/cpuref.c:236-241);
- when the reference's CPU oracle is built (oracle/_ref), it is called live.
"""
from __future__ import annotations

import ctypes as C
import json
import re
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi, ops
from tests import helpers as H

GOLDEN = Path(__file__).resolve().parent / "golden"
G = json.loads((GOLDEN / "golden.json").read_text())
ROOT = Path(__file__).resolve().parent.parent


def test_zipf_table_is_exact():
    text = (ROOT / "include" / "merle_b200_gen.h").read_text()
    body = text[text.index("#define MBG_ZIPF64_TABLE"):]
    body = body[:body.index("}")]
    vals = [int(v) for v in re.findall(r"(\d+)ULL", body)]
    Hs = [Fraction(0)]
    for j in range(1, 65):
        Hs.append(Hs[-1] + Fraction(1, j))
    want = [int((Hs[k + 1] / Hs[64]) * (1 << 32)) for k in range(64)]
    assert vals == want


def test_generator_heads(orc):
    f = orc.gen_flat(1, 16)
    assert {k: v.tolist() for k, v in f.items()} == G["flat_head"]
    s = orc.StarHost(2, 1, 16)
    assert {k: v.tolist() for k, v in s.cols.items()} == G["star_head"]
    assert s.custcity[:16].tolist() == G["star_dims_head"]["custcity"]
    assert s.partmfgr[:16].tolist() == G["star_dims_head"]["partmfgr"]


def test_generator_row_ranges_compose(orc):
    # any row range regenerates the same values (counter-based)
    full = orc.gen_flat(7, 1000)
    part = orc.gen_flat(7, 300, row0=500)
    for c in "abcde":
        assert np.array_equal(full[c][500:800], part[c])
    a = orc.StarHost(3, 2, 1000)
    b = orc.StarHost(3, 2, 100, row0=900)
    for c in a.cols:
        assert np.array_equal(a[c][900:], b[c])


def test_generator_distributions(orc):
    n = 200_000
    f = orc.gen_flat(1, n)
    assert f["a"].min() == 0 and f["a"].max() == 999
    assert f["c"].min() == 1 and f["c"].max() == 50
    assert f["d"].min() == 0 and f["d"].max() == 10
    assert f["e"].min() >= 90000 and f["e"].max() < 10500000
    # Zipf(1) over 64 values: P(v) = 1/((v+1) H64)
    h = sum(1.0 / k for k in range(1, 65))
    freq = np.bincount(f["b"], minlength=64) / n
    for v in (0, 1, 3, 7, 11, 63):
        assert abs(freq[v] - 1.0 / ((v + 1) * h)) < 0.01
    s = orc.StarHost(2, 20, n)
    assert s["orderdate"].max() <= 2555 and s["quantity"].min() == 1 and s["discount"].max() == 10
    assert np.all(s["extendedprice"] % s["quantity"] == 0)  # quantity * partprice
    price = s["extendedprice"] // s["quantity"]
    assert price.min() >= 90000 and price.max() <= 110000
    assert np.all(s["revenue"] == (s["extendedprice"].astype(np.uint64) * (100 - s["discount"]) // 100))


@pytest.fixture(scope="module")
def star(orc):
    g = G["ssb13"]
    return orc.StarHost(g["seed"], g["k"], g["n"])


def _golden_ssb():
    return np.load(GOLDEN / "ssb13_ref_u32.npy")


def _direct(orc, star, q, a, ng):
    d = star.orc_ssb()
    n = star.n
    out = np.zeros(ng, np.int64)
    nq = np.zeros(1, np.uint64)
    L = orc.lib()
    if q == "s1":
        v = L.orc_s1(C.byref(d), n, *a, orc.ptr(nq))
        out[0] = v
    elif q == "s2":
        L.orc_s2(C.byref(d), n, *a, orc.ptr(out), ng, orc.ptr(nq))
    elif q == "s3":
        L.orc_s3(C.byref(d), n, *a, orc.ptr(out), ng, orc.ptr(nq))
    else:
        L.orc_s4(C.byref(d), n, *a, orc.ptr(out), ng, orc.ptr(nq))
    return out, int(nq[0])


def test_ssb13_direct_matches_reference_golden(orc, star):
    gold = _golden_ssb()
    for i, (q, a, ng) in enumerate(H.SSB13):
        out, _ = _direct(orc, star, q, a, ng)
        np.testing.assert_array_equal(out.astype(np.uint32), gold[H.SLOTS[i]:H.SLOTS[i + 1]], err_msg=f"{q}{a}")


def test_ssb13_declarative_join_matches_direct(orc, star):
    for q, a, ng in H.SSB13:
        want, nqw = _direct(orc, star, q, a, ng)
        op = H.ssb_op(star, q, a).to_c()
        got, nq = orc.join_grpby(star.n, op, ng)
        np.testing.assert_array_equal(got, want, err_msg=f"{q}{a}")
        assert nq == nqw


@pytest.mark.parametrize("kind", ["perfect", "many_or", "candchk"])
def test_ssb13_fused_recipes_match_join(orc, star, kind):
    for q, a, ng in H.SSB13:
        preds, ins = H.ssb_recipe(star, q, a)
        prg = H.host_recipe(orc, kind, preds, ins, star.n)
        op = H.ssb_op(star, q, a).to_c()
        got, nq = orc.vprg_grpby(prg.to_c(), op, ng)
        want, nqw = orc.join_grpby(star.n, op, ng)
        np.testing.assert_array_equal(got, want, err_msg=f"{kind} {q}{a}")
        assert nq == nqw
        if kind == "candchk":
            assert not prg.is_nochk()


def test_ssb13_live_reference(orc, star):
    ref = orc.ref()
    if ref is None:
        pytest.skip("oracle/_ref not built (no reference tree)")
    schema = star.ssb_schema()
    res = ref.ssb_cpujoin(C.byref(schema), star.n)
    live = np.ctypeslib.as_array(res, shape=(int(H.SLOTS[-1]),)).copy()
    np.testing.assert_array_equal(live, _golden_ssb())


def _synth(orc, bw):
    from tests.golden.make_golden import synth_tables
    return synth_tables(bw)


def test_synth_matches_reference_golden(orc):
    gold = np.load(GOLDEN / "synth_ref_u32.npy")
    g = G["synth"]
    n = g["n"]
    i = 0
    for bw in g["bitwidths"]:
        a1, a2, fk, d1, d2 = _synth(orc, bw)
        for case in g["cases"]:
            out = np.zeros(256, np.int64)
            nq = np.zeros(1, np.uint64)
            orc.lib().orc_synth(orc.ptr(a1), orc.ptr(a2), bw, orc.ptr(fk), orc.ptr(d1), orc.ptr(d2), n, *case,
                                orc.ptr(out), orc.ptr(nq))
            np.testing.assert_array_equal(out.astype(np.uint32), gold[i])
            op = ops.synth_op(a1, a2, fk, d1, d2, *case).to_c()
            got, _ = orc.join_grpby(n, op, 256)
            np.testing.assert_array_equal(got, out)
            # the OR program of synth_bmp (synth/synthdemo.cu:389-391) over each recipe layout
            preds = [(None, a1, case[0], case[1]), (None, a2, case[2], case[3]), (fk, d1, case[4], case[5])]
            ins = [(abi.ORM, 0, 0, 0), (abi.ORM, 0, 1, 0), (abi.ANDM, 0, 2, 0)]
            for kind in ("perfect", "many_or", "candchk"):
                prg = H.host_recipe(orc, kind, preds, ins, n)
                got, _ = orc.vprg_grpby(prg.to_c(), op, 256)
                np.testing.assert_array_equal(got, out, err_msg=f"bw{bw} {case} {kind}")
            i += 1


def test_flat_query(orc):
    n = 100_003  # ragged: not a multiple of 32
    f = orc.gen_flat(1, n)
    bset = np.array([3, 7, 11], np.int32)
    cnt = np.zeros(1, np.uint64)
    want = orc.lib().orc_flat_query(*[orc.ptr(f[c]) for c in "abcde"], n, 200, 450, orc.ptr(bset), 3, 0, 25,
                                    orc.ptr(cnt))
    op = ops.flat_op(f["a"], f["b"], f["c"], f["d"], f["e"], 200, 450, [3, 7, 11], 0, 25).to_c()
    got, nq = orc.join_grpby(n, op, 1)
    assert got[0] == want and nq == int(cnt[0])
    # the index of the flat table: a in 100 width-10 bins, b and c equality bins
    def src(x):
        s = abi.mb_src()
        s.col, s.width = orc.ptr(x), 4
        return s
    abins, _ = orc.bitmap_create(src(f["a"]), n, np.arange(0, 1000, 10), np.arange(10, 1010, 10))
    bbins, _ = orc.bitmap_create(src(f["b"]), n, np.arange(64), np.arange(1, 65))
    cbins, _ = orc.bitmap_create(src(f["c"]), n, np.arange(1, 51), np.arange(2, 52))
    prg = ops.Vprg(n, [ops.Col(middle=[abins[j] for j in range(20, 45)]),
                       ops.Col(middle=[bbins[3], bbins[7], bbins[11]]),
                       ops.Col(middle=[cbins[j] for j in range(0, 24)])],
                   [(abi.ORM, 0, 0, 0), (abi.ANDM, 0, 1, 0), (abi.ANDM, 0, 2, 0)])
    got, nq = orc.vprg_grpby(prg.to_c(), op, 1)
    assert got[0] == want and nq == int(cnt[0])
    po, _ = orc.vprg_eval(prg.to_c(), False)
    assert int(np.unpackbits(po.view(np.uint8)).sum()) == int(cnt[0])


def test_bitmap_create_matches_numpy(orc):
    n = 70_001
    f = orc.gen_flat(3, n)
    s = abi.mb_src()
    s.col, s.width = orc.ptr(f["a"]), 4
    lo, hi = [0, 100, 250, 999, 5], [100, 250, 999, 1000, 6]
    bms, pop = orc.bitmap_create(s, n, lo, hi)
    for j in range(len(lo)):
        bits = ((f["a"] >= lo[j]) & (f["a"] < hi[j])).astype(np.uint8)
        want = np.packbits(np.pad(bits, (0, (-n) % 32)), bitorder="little").view(np.uint32)
        np.testing.assert_array_equal(bms[j], want)
        assert pop[j] == bits.sum()


def test_vbp_chk_algebra_small_exhaustive(orc):
    # The chk algebra on single words against a direct per-row statement of the
    # (possible, uncertain) semantics of primitive.cuh:255-332 for programs whose
    # NOT never sees an uncertain row.
    rng = np.random.default_rng(0)
    n = 32 * 64
    W = n // 32
    for trial in range(20):
        mids = [rng.integers(0, 2**32, W, dtype=np.uint64).astype(np.uint32) for _ in range(3)]
        edge = rng.integers(0, 2**32, W, dtype=np.uint64).astype(np.uint32)
        c0 = ops.Col(middle=[mids[0]], leftmost=edge)
        c1 = ops.Col(middle=[mids[1], mids[2]])
        prg = ops.Vprg(n, [c0, c1], [(abi.ORM, 0, 0, 0), (abi.ANDM, 0, 1, 0)])
        p, u = orc.vprg_eval(prg.to_c(), True)
        cert0 = mids[0]
        poss0 = mids[0] | edge
        unc0 = edge  # ORM from empty registers: u = u_src & ~p_prev (primitive.cuh:321)
        m1 = mids[1] | mids[2]
        want_p = np.where(poss0 != 0, poss0 & m1, 0).astype(np.uint32)
        want_u = np.where(poss0 != 0, unc0 & want_p, unc0).astype(np.uint32)
        np.testing.assert_array_equal(p, want_p)
        np.testing.assert_array_equal(u, want_u)
        assert np.all((p & ~cert0 & ~edge) == 0)


def test_bitmap_to_rows_ascending(orc):
    rng = np.random.default_rng(1)
    n = 10_000
    W = (n + 31) // 32
    po = rng.integers(0, 2**32, W, dtype=np.uint64).astype(np.uint32)
    un = rng.integers(0, 2**32, W, dtype=np.uint64).astype(np.uint32) & po
    rows = orc.bitmap_to_rows(po, un, n)
    ids = rows & 0x7FFFFFFF
    assert np.all(np.diff(ids.astype(np.int64)) > 0) and ids.max() < n


def test_window_zipf_golden():
    # restated window_zipf (synth/window_zipf.c:13-67) against the reference's values
    def wz(skew, n, win):
        eta = 0.0
        sign = 1.0
        for k in range(1, 50001):
            eta += sign / (k ** skew)
            sign = -sign
        zeta = eta / (1.0 - 2.0 ** (1.0 - skew))
        kp = [0.0] + [1.0 / (k ** skew) for k in range(1, n + win + 1)]
        return [sum(kp[x + 1:x + win + 1]) / zeta for x in range(n)]
    for skew, vals in G["window_zipf"].items():
        got = wz(float(skew), 64, 60)
        np.testing.assert_allclose(got, vals, rtol=1e-12)
