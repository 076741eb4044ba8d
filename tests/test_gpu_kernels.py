"""GPU parity tests of the L2 kernels through the C ABI.

Every result is compared with the CPU oracle (oracle/) on the same seeded
inputs, and query results also with the reference's own outputs
(tests/golden/, mod 2^32).  Integer work: everything is bit-exact.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi, check, device as D, ops
from tests import helpers as H

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
G = json.loads((GOLDEN / "golden.json").read_text())


def host(t, dt):
    return D.to_host(t, dt)


@pytest.fixture(scope="module")
def stars(cuda, orc, mb):
    g = G["ssb13"]
    dev = D.DevStar(g["seed"], g["k"], g["n"])
    ref = orc.StarHost(g["seed"], g["k"], g["n"])
    return dev, ref


def test_device_generator_matches_oracle(stars, cuda, orc):
    dev, ref = stars
    cuda.cuda.synchronize()
    for f in dev.FACT:
        np.testing.assert_array_equal(host(dev[f], ref[f].dtype), ref[f], err_msg=f)
    np.testing.assert_array_equal(host(dev.custcity, np.uint8), ref.custcity)
    np.testing.assert_array_equal(host(dev.suppcity, np.uint8), ref.suppcity)
    np.testing.assert_array_equal(host(dev.partmfgr, np.uint16), ref.partmfgr)
    # width4 layout holds the same values
    d4 = D.DevStar(ref.seed, ref.k, 5000, width4=True)
    for f in dev.FACT:
        np.testing.assert_array_equal(host(d4[f], np.uint32), ref[f][:5000].astype(np.uint32), err_msg=f)
    fl = D.DevFlat(1, 70_001)
    hf = orc.gen_flat(1, 70_001)
    for c in "abcde":
        np.testing.assert_array_equal(host(fl[c], np.int32), hf[c])


BIN_CASES = {
    "equal_w1": (np.arange(0, 50), np.arange(1, 51)),           # equality bins (match_any path)
    "equal_w10": (np.arange(0, 250, 10), np.arange(10, 260, 10)),
    "sorted_gaps": ([0, 3, 50, 51, 200, 240, 241], [2, 40, 51, 52, 230, 241, 250]),
    "overlap": ([0, 10, 5, 100, 0], [20, 30, 250, 101, 1]),     # ballot path
    "few": ([0, 100], [100, 250]),
    "empty_bin": ([0, 7, 9], [5, 7, 250]),
}


@pytest.mark.parametrize("case", list(BIN_CASES))
@pytest.mark.parametrize("n", [1, 31, 33, 4096, 70_001, 300_000])
def test_bitmap_create_fact_column(stars, orc, case, n):
    dev, ref = stars
    lo, hi = BIN_CASES[case]
    col = ref["suppcity"][:n]
    s = abi.mb_src()
    s.col, s.width = orc.ptr(col), 1
    want, wpop = orc.bitmap_create(s, n, lo, hi)
    got, gpop = D.bitmap_create(D.src_of(dev["suppcity"]), n, lo, hi)
    W = (n + 31) // 32
    gh = host(got, np.uint32).reshape(len(lo), -1)
    np.testing.assert_array_equal(gh[:, :W], want[:, :W])
    assert np.all(gh[:, W:] == 0)
    np.testing.assert_array_equal(host(gpop, np.uint64), wpop)


@pytest.mark.parametrize("width", [1, 2, 4])
def test_bitmap_create_widths_and_many_bins(stars, orc, cuda, width):
    dev, ref = stars
    n = ref.n
    src = {1: "quantity", 2: "orderdate", 4: "revenue"}[width]
    col = ref[src]
    hi_v = int(col.max()) + 1
    nb = 300 if width != 1 else 60  # >256 bins: split into several passes
    edges = np.linspace(0, hi_v, nb + 1).astype(np.uint64)
    lo, hi = edges[:-1], edges[1:]
    s = abi.mb_src()
    s.col, s.width = orc.ptr(col), width
    want, wpop = orc.bitmap_create(s, n, lo, hi)
    got, gpop = D.bitmap_create(D.src_of(dev[src]), n, lo, hi)
    W = (n + 31) // 32
    np.testing.assert_array_equal(host(got, np.uint32).reshape(nb, -1)[:, :W], want)
    np.testing.assert_array_equal(host(gpop, np.uint64), wpop)


def test_bitmap_create_join(stars, orc):
    dev, ref = stars
    n = ref.n
    # customer region bins through custkey -> custCity, part category bins through partkey -> partMfgr
    for fkname, dim_dev, dim_h, lo, hi in [
            ("custkey", dev.custcity, ref.custcity, np.arange(0, 250, 50), np.arange(50, 300, 50)),
            ("partkey", dev.partmfgr, ref.partmfgr, np.arange(0, 1000, 40), np.arange(40, 1040, 40))]:
        s = abi.mb_src()
        s.col, s.fk, s.width, s.dimsz = orc.ptr(dim_h), orc.ptr(ref[fkname]), dim_h.dtype.itemsize, 0
        want, wpop = orc.bitmap_create(s, n, lo, hi)
        got, gpop = D.bitmap_create(D.src_of(dim_dev, dev[fkname], checked=False), n, lo, hi)
        W = (n + 31) // 32
        np.testing.assert_array_equal(host(got, np.uint32).reshape(len(lo), -1)[:, :W], want)
        np.testing.assert_array_equal(host(gpop, np.uint64), wpop)
    # keys >= dimsz give no bit (create_join, bmpidx_create.cu:99)
    short = dev.custcity[:1000]
    s = abi.mb_src()
    s.col, s.fk, s.width, s.dimsz = orc.ptr(ref.custcity[:1000]), orc.ptr(ref["custkey"]), 1, 1000
    want, _ = orc.bitmap_create(s, n, [0], [250])
    got, _ = D.bitmap_create(D.src_of(short, dev["custkey"], checked=True), n, [0], [250])
    np.testing.assert_array_equal(host(got, np.uint32).reshape(1, -1)[:, :(n + 31) // 32], want)


LEVEL_CASES = {
    # the engine's hierarchies: years + months of a date, regions + nations of a city
    "date": ("orderdate", [(np.array([0, 366, 731, 1096, 1461, 1827, 2192]),
                            np.array([366, 731, 1096, 1461, 1827, 2192, 2557]))], True),
    "city": ("suppcity", [(np.arange(0, 250, 50), np.arange(50, 300, 50)),
                          (np.arange(0, 250, 10), np.arange(10, 260, 10))], False),
    "quantity": ("quantity", [(np.arange(1, 51), np.arange(2, 52))], False),
    # a level with gaps, values outside every bin, and three levels at once
    "gaps3": ("suppcity", [([0, 3, 50, 51, 200, 240], [2, 40, 51, 52, 230, 241]),
                           (np.arange(0, 240, 60), np.arange(60, 300, 60)),
                           (np.arange(5, 245, 5), np.arange(10, 250, 5))], False),
    # 4 x 200 bins: their word tiles exceed shared memory, one pass per level
    "wide4": ("suppcity", [(np.arange(0, 200), np.arange(1, 201)), (np.arange(10, 210), np.arange(11, 211)),
                           (np.arange(20, 220), np.arange(21, 221)), (np.arange(49, 249), np.arange(50, 250))],
              False),
    # overlapping bins in one level: that level falls back to its own pass
    "overlap": ("suppcity", [(np.arange(0, 250, 50), np.arange(50, 300, 50)),
                             ([0, 10, 5], [20, 30, 250])], False),
}


@pytest.mark.parametrize("case", list(LEVEL_CASES))
@pytest.mark.parametrize("n", [1, 31, 33, 4095, 4097, 100_003, 300_000])
def test_bitmap_create_levels(stars, orc, case, n):
    """One pass over a column builds several levels of bins: each level
    equals its own single-level oracle pass word for word, tails zero,
    popcounts exact."""
    dev, ref = stars
    colname, levels, months = LEVEL_CASES[case]
    if months:
        from merle_b200 import workload as WL
        ms = np.array(WL.MONTH_START)
        levels = levels + [(ms[:-1], ms[1:])]
    col = ref[colname][:n]
    s = abi.mb_src()
    s.col, s.width = orc.ptr(col), col.dtype.itemsize
    got = D.bitmap_create_levels(D.src_of(dev[colname]), n, levels)
    W = (n + 31) // 32
    for (lo, hi), (slab, pc) in zip(levels, got):
        want, wpop = orc.bitmap_create(s, n, lo, hi)
        gh = host(slab, np.uint32).reshape(len(lo), -1)
        np.testing.assert_array_equal(gh[:, :W], want[:, :W], err_msg=case)
        assert np.all(gh[:, W:] == 0)
        np.testing.assert_array_equal(host(pc, np.uint64), wpop)


def test_bitmap_create_levels_join(stars, orc):
    """Regions and nations of the customer city through custkey -> custCity in
    one pass, and keys >= dimsz give no bit."""
    dev, ref = stars
    n = ref.n
    levels = [(np.arange(0, 250, 50), np.arange(50, 300, 50)), (np.arange(0, 250, 10), np.arange(10, 260, 10))]
    for dimsz, dim_dev, dim_h in [(0, dev.custcity, ref.custcity), (1000, dev.custcity[:1000], ref.custcity[:1000])]:
        s = abi.mb_src()
        s.col, s.fk, s.width, s.dimsz = orc.ptr(dim_h), orc.ptr(ref["custkey"]), 1, dimsz
        got = D.bitmap_create_levels(D.src_of(dim_dev, dev["custkey"], checked=dimsz != 0), n, levels)
        W = (n + 31) // 32
        for (lo, hi), (slab, pc) in zip(levels, got):
            want, wpop = orc.bitmap_create(s, n, lo, hi)
            np.testing.assert_array_equal(host(slab, np.uint32).reshape(len(lo), -1)[:, :W], want)
            np.testing.assert_array_equal(host(pc, np.uint64), wpop)


def _device_recipe(mb, dev, kind, preds, instrs, n):
    r = abi.mb_recipe()
    r.factsz = n
    for i, (fk, attr, mn, mx) in enumerate(preds):
        r.nbit[i] = attr.element_size() * 8
        r.min[i], r.max[i] = mn & 0xFFFFFFFF, mx & 0xFFFFFFFF
        r.dimsz[i] = 0xFFFFFFFF
        r.fk[i] = fk.data_ptr() if fk is not None else None
        r.attr[i] = attr.data_ptr()
    ins = (abi.mb_instr * abi.MB_MAXNINSTR)()
    for i, t in enumerate(instrs):
        ins[i].opcode, ins[i].dstreg, ins[i].src1, ins[i].src2 = t
    o = abi.mb_owned_vprg()
    k = {"perfect": abi.RECIPE_PERFECT, "many_or": abi.RECIPE_MANY_OR, "candchk": abi.RECIPE_CANDCHK}[kind]
    check(mb.lib().mb_recipe_build(C.byref(r), k, ins, C.byref(o), D.stream_ptr()))
    return o


# (group strategy, warps per CTA, CTAs per SM, words per lane, staging): staging 0 runs the
# TMA-staged kernel, 1 the direct-load kernel
LAUNCHES = [None, (abi.GRP_SHARED, 4, 0, 4, 1), (abi.GRP_GLOBAL, 8, 1, 2, 1), (abi.GRP_HASH, 16, 0, 1, 1),
            (abi.GRP_GLOBAL, 8, 0, 4, 0), (abi.GRP_SHARED, 8, 0, 1, 0), (abi.GRP_HASH, 8, 2, 2, 0),
            (abi.GRP_AUTO, 8, 0, 4, 0)]


@pytest.mark.parametrize("kind", ["perfect", "many_or", "candchk"])
def test_fused_ssb13_recipes(stars, orc, mb, cuda, kind):
    dev, ref = stars
    gold = np.load(GOLDEN / "ssb13_ref_u32.npy")
    n = ref.n
    for i, (q, a, ng) in enumerate(H.SSB13):
        preds_d, ins = H.ssb_recipe(dev, q, a)
        owned = _device_recipe(mb, dev, kind, preds_d, ins, n)
        # the device recipe's bitmaps equal the oracle-built ones
        preds_h, _ = H.ssb_recipe(ref, q, a)
        prg_h = H.host_recipe(orc, kind, preds_h, ins, n)
        op_h = H.ssb_op(ref, q, a).to_c()
        want, nqw = orc.vprg_grpby(prg_h.to_c(), op_h, ng)
        np.testing.assert_array_equal(want.astype(np.uint32), gold[H.SLOTS[i]:H.SLOTS[i + 1]])
        op_d = H.ssb_op(dev, q, a).to_c()
        for L in LAUNCHES:
            la = abi.mb_launch(*L) if L else None
            out, nq = D.vprg_grpby(owned.prg, op_d, ng, la)
            cuda.cuda.synchronize()
            np.testing.assert_array_equal(host(out, np.int64), want, err_msg=f"{kind} {q}{a} {L}")
            assert int(host(nq, np.uint64)[0]) == nqw
        check(mb.lib().mb_owned_vprg_release(C.byref(owned)))


def test_join_ssb13(stars, orc, cuda):
    dev, ref = stars
    for q, a, ng in H.SSB13:
        want, nqw = orc.join_grpby(ref.n, H.ssb_op(ref, q, a).to_c(), ng)
        out, nq = D.join_grpby(ref.n, H.ssb_op(dev, q, a).to_c(), ng)
        np.testing.assert_array_equal(host(out, np.int64), want, err_msg=f"{q}{a}")
        assert int(host(nq, np.uint64)[0]) == nqw


@pytest.mark.parametrize("width,n,offset", [(8, 100_003, 0), (4, 128 * 300 + 77, 0), (2, 4097, 0),
                                            (1, 131, 0), (4, 50_001, 1)])
def test_join_screen_widths_tails_alignment(orc, cuda, width, n, offset):
    """The no-index scan's screen: one range on a fact column of each width
    (four rows a lane from one vector load), row counts that end inside a
    128-row chunk, and a column that is not 16-byte aligned (the per-row
    screen); SUM(b * c) and the row count equal the oracle's."""
    rng = np.random.default_rng(width * 1000 + n)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width]
    a_full = rng.integers(0, 200, n + offset).astype(dt)
    b = rng.integers(0, 1000, n).astype(np.uint32)
    c = rng.integers(0, 50, n).astype(np.uint32)
    a = a_full[offset:]
    def op(cols):
        return ops.Op(srcs=[ops.Src(cols[0]), ops.Src(cols[1]), ops.Src(cols[2])],
                      clauses=[[(0, 40, 90)], [(2, 5, 45)]], keys=[], vkind=abi.V_MUL, va=1, vb=2).to_c()
    want, nqw = orc.join_grpby(n, op((np.ascontiguousarray(a), b, c)), 1)
    da_full = D.from_host(a_full)
    da = da_full[offset:] if offset else da_full
    out, nq = D.join_grpby(n, op((da, D.from_host(b), D.from_host(c))), 1)
    assert int(host(out, np.int64)[0]) == int(want[0]) and int(host(nq, np.uint64)[0]) == nqw


def test_materialised_stages(stars, orc, mb, cuda):
    dev, ref = stars
    n = ref.n
    L = mb.lib()
    for kind in ("perfect", "candchk"):
        for q, a, ng in H.SSB13[::3]:
            preds_d, ins = H.ssb_recipe(dev, q, a)
            owned = _device_recipe(mb, dev, kind, preds_d, ins, n)
            preds_h, _ = H.ssb_recipe(ref, q, a)
            prg_h = H.host_recipe(orc, kind, preds_h, ins, n)
            chk = not prg_h.is_nochk()
            po_w, un_w = orc.vprg_eval(prg_h.to_c(), chk)
            W = (n + 31) // 32
            po = D.empty(W, 4)
            un = D.empty(W, 4)
            pc = D.empty(1, 8, zero=True)
            check(L.mb_vprg_eval(C.byref(owned.prg), int(chk), po.data_ptr(), un.data_ptr(), pc.data_ptr(),
                                 D.stream_ptr()))
            np.testing.assert_array_equal(host(po, np.uint32), po_w)
            if chk:
                np.testing.assert_array_equal(host(un, np.uint32), un_w)
            assert int(host(pc, np.uint64)[0]) == int(np.unpackbits(po_w.view(np.uint8)).sum())
            rows_w = orc.bitmap_to_rows(po_w, un_w if chk else None, n)
            rows = D.empty(max(len(rows_w), 1), 4)
            cnt = D.empty(1, 8)
            check(L.mb_bitmap_to_rows(po.data_ptr(), un.data_ptr() if chk else None, n, rows.data_ptr(),
                                      cnt.data_ptr(), D.stream_ptr()))
            assert int(host(cnt, np.uint64)[0]) == len(rows_w)
            np.testing.assert_array_equal(host(rows, np.uint32)[:len(rows_w)], rows_w)
            op_d = H.ssb_op(dev, q, a).to_c()
            out = D.empty(ng, 8)
            nq = D.empty(1, 8)
            check(L.mb_rows_grpby(rows.data_ptr(), cnt.data_ptr(), rows.numel(), C.byref(op_d), ng,
                                  out.data_ptr(), nq.data_ptr(), D.stream_ptr()))
            want, nqw = orc.vprg_grpby(prg_h.to_c(), H.ssb_op(ref, q, a).to_c(), ng)
            np.testing.assert_array_equal(host(out, np.int64), want)
            assert int(host(nq, np.uint64)[0]) == nqw
            check(L.mb_owned_vprg_release(C.byref(owned)))


def test_synth_golden(orc, mb, cuda):
    from tests.golden.make_golden import synth_tables
    gold = np.load(GOLDEN / "synth_ref_u32.npy")
    g = G["synth"]
    n = g["n"]
    i = 0
    for bw in g["bitwidths"]:
        a1, a2, fk, d1, d2 = synth_tables(bw)
        t = [D.from_host(x) for x in (a1, a2, fk, d1, d2)]
        for case in g["cases"]:
            op = ops.synth_op(*t, *case).to_c()
            preds = [(None, t[0], case[0], case[1]), (None, t[1], case[2], case[3]), (t[2], t[3], case[4], case[5])]
            ins = [(abi.ORM, 0, 0, 0), (abi.ORM, 0, 1, 0), (abi.ANDM, 0, 2, 0)]
            for kind in ("perfect", "many_or", "candchk"):
                owned = _device_recipe(mb, None, kind, preds, ins, n)
                out, _ = D.vprg_grpby(owned.prg, op, 256)
                np.testing.assert_array_equal(host(out, np.int64).astype(np.uint32), gold[i], err_msg=f"{bw} {case} {kind}")
                check(mb.lib().mb_owned_vprg_release(C.byref(owned)))
            out, _ = D.join_grpby(n, op, 256)
            np.testing.assert_array_equal(host(out, np.int64).astype(np.uint32), gold[i])
            i += 1


@pytest.mark.parametrize("n", [1, 31, 32, 33, 4095, 4097, 100_003])
def test_edge_sizes_and_not_tail(orc, cuda, n):
    """Ragged sizes; a program ending in NOT sets no bit at rows >= n."""
    f = orc.gen_flat(9, n)
    fd = D.DevFlat(9, n)
    s = abi.mb_src()
    s.col, s.width = orc.ptr(f["a"]), 4
    bh, _ = orc.bitmap_create(s, n, [0], [300])
    bd, _ = D.bitmap_create(D.src_of(fd["a"]), n, [0], [300])
    # nochk program: the op's clauses are not re-evaluated, every selected row counts
    op_h = ops.flat_op(f["a"], f["b"], f["c"], f["d"], f["e"], 0, 1000, [1], 0, 100).to_c()
    op_d = ops.flat_op(fd["a"], fd["b"], fd["c"], fd["d"], fd["e"], 0, 1000, [1], 0, 100).to_c()
    ins = [(abi.ORM, 1, 0, 0), (abi.NOT, 0, 1, 0)]
    ph = ops.Vprg(n, [ops.Col(middle=[bh[0]])], ins).to_c()
    pd = ops.Vprg(n, [ops.Col(middle=[bd[0]])], ins).to_c()
    want, nqw = orc.vprg_grpby(ph, op_h, 1)
    assert nqw == int((f["a"] >= 300).sum())
    for L in LAUNCHES:
        out, nq = D.vprg_grpby(pd, op_d, 1, abi.mb_launch(*L) if L else None)
        assert int(host(out, np.int64)[0]) == int(want[0]) and int(host(nq, np.uint64)[0]) == nqw


def test_empty_inputs(cuda, mb):
    L = mb.lib()
    out = D.empty(4, 8)
    nq = D.empty(1, 8)
    p = ops.Vprg(0, [], []).to_c()
    op = ops.Op().to_c()
    check(L.mb_vprg_grpby(C.byref(p), C.byref(op), 4, out.data_ptr(), nq.data_ptr(), None, D.stream_ptr()))
    assert np.all(host(out, np.int64) == 0) and host(nq, np.uint64)[0] == 0
    check(L.mb_join_grpby(0, C.byref(op), 4, out.data_ptr(), nq.data_ptr(), D.stream_ptr()))
    # a program with no instructions selects nothing
    fd = D.DevFlat(1, 1000)
    p = ops.Vprg(1000, [], []).to_c()
    op = ops.flat_op(fd["a"], fd["b"], fd["c"], fd["d"], fd["e"], 0, 1000, [1], 0, 100).to_c()
    check(L.mb_vprg_grpby(C.byref(p), C.byref(op), 1, out.data_ptr(), nq.data_ptr(), None, D.stream_ptr()))
    assert host(nq, np.uint64)[0] == 0


def test_flat_query_full_size(orc, cuda):
    """The 24M-row flat table: 214-bitmap index, the 52-bitmap program."""
    n = 24_000_000
    f = orc.gen_flat(1, n)
    fd = D.DevFlat(1, n)
    bset = np.array([3, 7, 11], np.int32)
    cnt = np.zeros(1, np.uint64)
    want = orc.lib().orc_flat_query(*[orc.ptr(f[c]) for c in "abcde"], n, 200, 450, orc.ptr(bset), 3, 0, 25,
                                    orc.ptr(cnt))
    ab, _ = D.bitmap_create(D.src_of(fd["a"]), n, np.arange(0, 1000, 10), np.arange(10, 1010, 10))
    bb, _ = D.bitmap_create(D.src_of(fd["b"]), n, np.arange(64), np.arange(1, 65))
    cb, cpop = D.bitmap_create(D.src_of(fd["c"]), n, np.arange(1, 51), np.arange(2, 52))
    np.testing.assert_array_equal(host(cpop, np.uint64), np.bincount(f["c"], minlength=52)[1:51])
    prg = ops.Vprg(n, [ops.Col(middle=[ab[j] for j in range(20, 45)]), ops.Col(middle=[bb[3], bb[7], bb[11]]),
                       ops.Col(middle=[cb[j] for j in range(0, 24)])],
                   [(abi.ORM, 0, 0, 0), (abi.ANDM, 0, 1, 0), (abi.ANDM, 0, 2, 0)]).to_c()
    op = ops.flat_op(fd["a"], fd["b"], fd["c"], fd["d"], fd["e"], 200, 450, [3, 7, 11], 0, 25).to_c()
    out, nq = D.vprg_grpby(prg, op, 1)
    assert int(host(out, np.int64)[0]) == int(want)
    assert int(host(nq, np.uint64)[0]) == int(cnt[0])
