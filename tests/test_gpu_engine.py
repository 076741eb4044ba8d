"""GPU tests of the engine C ABI (mb_engine_*): resident star schema,
canonical index, rule planner, every plan kind, against the CPU oracle and the
reference's own outputs."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi, workload as WL
from merle_b200.engine import Engine
from tests import helpers as H

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
G = json.loads((GOLDEN / "golden.json").read_text())


def oracle_query(orc, star, q):
    t, a = WL.as_tuple(q)
    ng = Engine.ngroups(q)
    op = H.ssb_op(star, WL.TEMPLATE_NAME[t], a).to_c()
    return orc.join_grpby(star.n, op, ng)


@pytest.fixture(scope="module")
def eng(cuda, mb):
    g = G["ssb13"]
    e = Engine(0)
    e.gen_star(g["seed"], g["k"], g["n"])
    e.build_index()
    yield e
    e.close()


@pytest.fixture(scope="module")
def star(orc):
    g = G["ssb13"]
    return orc.StarHost(g["seed"], g["k"], g["n"])


def test_engine_info(eng):
    i = eng.info()
    assert i["nbitmaps"] == 242 and i["nrows"] == G["ssb13"]["n"]
    assert i["index_bytes"] >= 242 * (G["ssb13"]["n"] // 8)


def test_engine_ssb13_matches_reference(eng, star, orc):
    gold = np.load(GOLDEN / "ssb13_ref_u32.npy")
    for i, q in enumerate(WL.ssb13()):
        out, nq, st = eng.query(q)
        np.testing.assert_array_equal(out.astype(np.uint32), gold[H.SLOTS[i]:H.SLOTS[i + 1]], err_msg=str(WL.as_tuple(q)))
        want, nqw = oracle_query(orc, star, q)
        np.testing.assert_array_equal(out, want)
        assert nq == nqw and st.nbitmaps >= 1


PLANS = [
    dict(kind=abi.PLAN_FUSED),
    dict(kind=abi.PLAN_SCAN),
    dict(kind=abi.PLAN_MATERIALISED),
    dict(kind=abi.PLAN_FUSED, materialise=0b1011),
    dict(kind=abi.PLAN_MATERIALISED, materialise=0b0101),
    dict(kind=abi.PLAN_FUSED, order_mode=1, launch=(abi.GRP_GLOBAL, 4, 0, 2, 1)),
    dict(kind=abi.PLAN_FUSED, launch=(abi.GRP_HASH, 16, 1, 1, 1)),
    dict(kind=abi.PLAN_FUSED, launch=(abi.GRP_GLOBAL, 8, 0, 1, 0)),
]


def mkplan(d) -> abi.mb_plan:
    p = abi.mb_plan()
    p.kind = d.get("kind", 0)
    p.order_mode = d.get("order_mode", 0)
    p.materialise = d.get("materialise", 0)
    if "launch" in d:
        p.launch = abi.mb_launch(*d["launch"])
    return p


def test_engine_random_mix_all_plans(eng, star, orc):
    qs = WL.random_mix(11, 40, narrow=0.4)
    for q in qs:
        want, nqw = oracle_query(orc, star, q)
        for d in PLANS:
            out, nq, _ = eng.query(q, mkplan(d))
            np.testing.assert_array_equal(out, want, err_msg=f"{WL.as_tuple(q)} {d}")
            assert nq == nqw


def test_engine_edge_predicates(eng, star, orc):
    qs = [
        abi.query(1, 0, 2557, 0, 11, 1, 51),        # every predicate full: all rows
        abi.query(1, 100, 100, 0, 11, 1, 51),       # empty date range
        abi.query(1, 2556, 4000, 10, 11, 50, 51),   # ranges clipped at the domain end
        abi.query(2, 0, 1000, 0, 250),              # full mfgr and city ranges
        abi.query(2, 37, 41, 3, 4),                 # brands across a category edge, one city
        abi.query(3, 0, 250, 0, 250, 0, 2557),
        abi.query(3, 13, 17, 201, 205, 59, 1500),   # city level: edge bins both sides
        abi.query(4, 0, 50, 0, 50, 0, 1000, 366, 2557),
    ]
    for q in qs:
        want, nqw = oracle_query(orc, star, q)
        for d in PLANS:
            out, nq, _ = eng.query(q, mkplan(d))
            np.testing.assert_array_equal(out, want, err_msg=f"{WL.as_tuple(q)} {d}")
            assert nq == nqw


def test_engine_width4_and_host_load(cuda, star, orc, mb):
    g = G["ssb13"]
    e4 = Engine(0)
    e4.gen_star(g["seed"], g["k"], g["n"], width4=True)
    e4.build_index()
    # host load of the same table in ssb_schema widths (ssb_load's H2D step)
    n = star.n
    s = star.narrow()
    h = abi.mb_star_host(nrows=n, ncust=len(s.custcity), nsupp=len(s.suppcity), npart=len(s.partmfgr))
    for f, c in [("custkey", "custkey"), ("partkey", "partkey"), ("orderdate", "orderdate"),
                 ("extendedprice", "extendedprice"), ("revenue", "revenue"), ("supplycost", "supplycost"),
                 ("quantity", "quantity"), ("discount", "discount"), ("suppcity", "suppcity")]:
        setattr(h, f, s[c].ctypes.data)
    h.custcity = s.custcity.ctypes.data
    h.partmfgr = s.partmfgr.ctypes.data
    eh = Engine(0)
    eh.load_star(h)
    eh.build_index()
    for q in WL.ssb13() + WL.random_mix(5, 12):
        want, nqw = oracle_query(orc, star, q)
        for e in (e4, eh):
            out, nq, _ = e.query(q)
            np.testing.assert_array_equal(out, want, err_msg=str(WL.as_tuple(q)))
            assert nq == nqw
    e4.close()
    eh.close()


def test_engine_keys_outside_dimension(cuda, star, orc, mb):
    """A loaded table whose customer and part keys partly leave their
    dimensions: the index build's join passes count those keys, the engine
    keeps probing through the keys instead of denormalised columns, and the
    plans and the batched scan answer as the oracle (such rows are
    eliminated)."""
    import copy
    s = star.narrow()
    b = copy.copy(s)
    b.cols = {k: v.copy() for k, v in s.cols.items()}
    b.cols["custkey"][::97] = len(s.custcity) + 3
    b.cols["partkey"][5::113] = len(s.partmfgr) + 11
    n = star.n
    h = abi.mb_star_host(nrows=n, ncust=len(s.custcity), nsupp=len(s.suppcity), npart=len(s.partmfgr))
    for f in ("custkey", "partkey", "orderdate", "extendedprice", "revenue", "supplycost", "quantity", "discount",
              "suppcity"):
        setattr(h, f, b.cols[f].ctypes.data)
    h.custcity = s.custcity.ctypes.data
    h.partmfgr = s.partmfgr.ctypes.data
    e = Engine(0)
    try:
        e.load_star(h)
        e.build_index()
        assert e.info()["denorm_bytes"] == 0  # the keys are probed
        qs = WL.ssb13() + WL.random_mix(11, 12)
        wants = [oracle_query(orc, b, q) for q in qs]
        for q, (want, nqw) in zip(qs, wants):
            out, nq, _ = e.query(q)
            np.testing.assert_array_equal(out, want, err_msg=str(WL.as_tuple(q)))
            assert nq == nqw
        out, nq = e.query_batch(qs)
        np.testing.assert_array_equal(out, np.concatenate([w for w, _ in wants]))
        np.testing.assert_array_equal(nq, np.array([x for _, x in wants], np.uint64))
    finally:
        e.close()


def test_engine_errors(eng, mb):
    out = np.zeros(8, np.int64)
    q = abi.query(9, 1, 2)
    st = mb.lib().mb_engine_query(eng.handle, C.byref(q), None, out.ctypes.data, None, None)
    assert st == abi.MB_ERR_INVALID
    e = Engine(0)
    q = abi.query(1, 0, 10, 0, 1, 1, 2)
    assert mb.lib().mb_engine_query(e.handle, C.byref(q), None, out.ctypes.data, None, None) == abi.MB_ERR_INVALID
    e.close()


def _batch_oracle(orc, star, qs):
    outs, nqs = [], []
    for q in qs:
        o, n = oracle_query(orc, star, q)
        outs.append(o)
        nqs.append(n)
    return np.concatenate(outs) if outs else np.zeros(0, np.int64), np.array(nqs, np.uint64)


BATCH_OPTS = [
    (0, 0, 0, 0, abi.PREFETCH_AUTO),
    (1, 8, 2, 0, abi.PREFETCH_NONE),
    (2, 16, 3, 0, abi.PREFETCH_ALL),
    (4, 16, 0, 0, abi.PREFETCH_AUTO),
    (2, 4, 1, 2, abi.PREFETCH_AUTO),
    (2, 12, 0, 0, abi.PREFETCH_AUTO),
    (6, 16, 0, 0, abi.PREFETCH_AUTO),
    (6, 12, 1, 3, abi.PREFETCH_NONE),
    (2, 16, 0, 0, abi.PREFETCH_AUTO, 1),   # group tables of at most 1 KB
    (4, 8, 0, 0, abi.PREFETCH_AUTO, 16),
    (1, 2, 0, 0, abi.PREFETCH_AUTO),       # one worker warp per CTA
]


def _mix_with_edges():
    return WL.ssb13() + WL.random_mix(21, 40, narrow=0.4) + [
        abi.query(1, 100, 100, 0, 11, 1, 51), abi.query(1, 0, 2557, 0, 11, 1, 51), abi.query(2, 37, 41, 3, 4),
        abi.query(3, 13, 17, 201, 205, 59, 1500), abi.query(4, 0, 50, 0, 50, 0, 1000, 366, 2557)]


@pytest.mark.parametrize("opts", BATCH_OPTS)
def test_engine_batch_matches_oracle(eng, star, orc, mb, opts):
    """The batched scan through the device-memory entry point, on every
    launch shape, against the oracle (edge cases: empty, full, candidate
    checks on both sides)."""
    import torch
    L = mb.lib()
    qs = _mix_with_edges()
    want, wn = _batch_oracle(orc, star, qs)
    n = len(qs)
    qarr = (abi.mb_query * n)(*qs)
    total = int(L.mb_queries_layout(qarr, n, None))
    assert total == len(want)
    out = torch.zeros(total, dtype=torch.int64, device="cuda")
    nq = torch.zeros(n, dtype=torch.int64, device="cuda")
    o = abi.mb_batch_opts(*opts)
    mb.check(L.mb_engine_enqueue_batch(eng.handle, qarr, n, C.byref(o), out.data_ptr(), nq.data_ptr()))
    mb.check(L.mb_engine_sync(eng.handle, None, 0))
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    np.testing.assert_array_equal(nq.cpu().numpy().astype(np.uint64), wn)


@pytest.mark.parametrize("table_kb", [0, 1])
def test_engine_batch_span_mix_matches_oracle(eng, star, orc, table_kb):
    """The selectivity-spanning mix (1e-6 .. 0.5, wide multi-group queries
    summing into shared group tables) through the batched scan, against the
    oracle; and with the tables held to 1 KB (global atomics instead)."""
    qs = WL.span_mix(3, 64)
    want, wn = _batch_oracle(orc, star, qs)
    o = abi.mb_batch_opts()
    o.table_kb = table_kb
    out, nq = eng.query_batch(qs, o)
    np.testing.assert_array_equal(out, want)
    np.testing.assert_array_equal(nq, wn)


def test_engine_batch_host_api_and_split(eng, star, orc):
    qs = WL.random_mix(33, 300, narrow=0.3)  # > MB_BATCH_MAX: three launches
    want, wn = _batch_oracle(orc, star, qs)
    out, nq = eng.query_batch(qs)
    np.testing.assert_array_equal(out, want)
    np.testing.assert_array_equal(nq, wn)


def test_engine_batch_alone_equals_in_mix(eng):
    """Every query's results are the same alone (a batch of one, and the
    single-query path) as inside a mix of 64."""
    qs = WL.random_mix(3, 64, narrow=0.3)
    out, nq = eng.query_batch(qs)
    offs = np.concatenate([[0], np.cumsum([Engine.ngroups(q) for q in qs])])
    for i in range(0, 64, 7):
        a, an = eng.query_batch([qs[i]])
        np.testing.assert_array_equal(a, out[offs[i]:offs[i + 1]])
        assert an[0] == nq[i]
        b, bn, _ = eng.query(qs[i])
        np.testing.assert_array_equal(b, a)
        assert bn == an[0]


def test_engine_batch_invalid_options(eng, mb):
    L = mb.lib()
    qs = WL.random_mix(4, 2)
    qarr = (abi.mb_query * 2)(*qs)
    out = np.zeros(4096, np.int64)
    for bad in [(3, 0, 0, 0, 0), (0, 17, 0, 0, 0), (0, 1, 0, 0, 0), (0, 0, 5, 0, 0), (0, 0, 0, 0, 3),
                (0, 0, 0, 0, 0, 228)]:
        o = abi.mb_batch_opts(*bad)
        assert L.mb_engine_query_batch(eng.handle, qarr, 2, C.byref(o), out.ctypes.data, None) == abi.MB_ERR_INVALID


def _batch_info(eng, mb, qs, opts=None):
    L = mb.lib()
    n = len(qs)
    qarr = (abi.mb_query * n)(*qs)
    infos = (abi.mb_batch_launch_info * 8)()
    nl, na = C.c_uint32(0), C.c_uint32(0)
    mb.check(L.mb_engine_batch_info(eng.handle, qarr, n, C.byref(opts) if opts else None, infos, 8,
                                    C.byref(nl), C.byref(na)))
    return list(infos)[:nl.value], na.value


def test_engine_batch_stages_only_rows_it_reads(eng, mb):
    """A batch stages exactly the union of the rows its queries read, one
    tensor copy per run of consecutive rows."""
    q = abi.query(1, 366, 731, 1, 4, 0, 25)  # one year bin, three discount bins, quantity bins
    li, na = _batch_info(eng, mb, [q])
    assert na == 0 and len(li) == 1
    assert li[0].queries == 1 and li[0].staged_rows <= 30 and 1 <= li[0].copies <= 4
    qs = WL.random_mix(3, 64, narrow=0.3)
    li, na = _batch_info(eng, mb, qs)
    assert len(li) == 1 and li[0].queries + na == 64
    assert li[0].staged_rows <= 242 and li[0].copies <= 48
    assert li[0].words_per_lane in (1, 2, 4) and 1 <= li[0].warps <= 16


def test_engine_batch_graph_replays(eng, star, orc, mb):
    import torch
    L = mb.lib()
    qs = _mix_with_edges()
    want, wn = _batch_oracle(orc, star, qs)
    n = len(qs)
    qarr = (abi.mb_query * n)(*qs)
    out = torch.full((len(want),), -1, dtype=torch.int64, device="cuda")
    nq = torch.zeros(n, dtype=torch.int64, device="cuda")
    g = C.c_void_p()
    mb.check(L.mb_batch_graph_create(eng.handle, qarr, n, None, out.data_ptr(), nq.data_ptr(), C.byref(g)))
    try:
        for _ in range(3):
            out.fill_(-1)
            torch.cuda.synchronize()
            mb.check(L.mb_batch_graph_launch(g))
            mb.check(L.mb_engine_sync(eng.handle, None, 0))
            np.testing.assert_array_equal(out.cpu().numpy(), want)
            np.testing.assert_array_equal(nq.cpu().numpy().astype(np.uint64), wn)
    finally:
        mb.check(L.mb_batch_graph_destroy(g))


def test_engine_batch_autotune(eng, star, orc, mb):
    L = mb.lib()
    qs = WL.random_mix(5, 64, narrow=0.3)
    n = len(qs)
    qarr = (abi.mb_query * n)(*qs)
    best = abi.mb_batch_opts()
    ms, tried = C.c_float(0), C.c_uint32(0)
    mb.check(L.mb_engine_tune_batch(eng.handle, qarr, n, 2, C.byref(best), C.byref(ms), C.byref(tried)))
    assert tried.value >= 9 and 0 < ms.value < 1e3
    assert best.words_per_lane in (1, 2, 4, 6) and best.warps in (8, 12, 16)
    want, wn = _batch_oracle(orc, star, qs)
    out, nq = eng.query_batch(qs, best)
    np.testing.assert_array_equal(out, want)
    np.testing.assert_array_equal(nq, wn)


def test_engine_denormalised_equals_probe(cuda, star, orc):
    """The index over denormalised dimension columns and the one that probes
    the dimensions through the foreign keys give the same results, on the
    plan kinds and through the batch."""
    g = G["ssb13"]
    ep = Engine(0)
    ep.gen_star(g["seed"], g["k"], g["n"])
    ep.build_index(probe_dims=True)
    ed = Engine(0)
    ed.gen_star(g["seed"], g["k"], g["n"])
    ed.build_index()
    assert ep.info()["denorm"] == 0 and ed.info()["denorm"] == 1
    assert ed.info()["denorm_bytes"] == 3 * g["n"]
    qs = WL.ssb13() + WL.random_mix(8, 24, narrow=0.4)
    for q in qs:
        want, nqw = oracle_query(orc, star, q)
        for e in (ep, ed):
            for d in PLANS[:3]:
                out, nq, _ = e.query(q, mkplan(d))
                np.testing.assert_array_equal(out, want, err_msg=f"{WL.as_tuple(q)} {d}")
                assert nq == nqw
    want, wn = _batch_oracle(orc, star, qs)
    for e in (ep, ed):
        out, nq = e.query_batch(qs)
        np.testing.assert_array_equal(out, want)
        np.testing.assert_array_equal(nq, wn)
    ep.close()
    ed.close()


def test_engine_index_file_roundtrip(cuda, mb, tmp_path):
    """An index saved to a file and loaded into a fresh engine over the same
    table answers every query as the built one; a damaged file or a file for
    another table is refused."""
    g = G["ssb13"]
    a = Engine(0)
    a.gen_star(g["seed"], g["k"], g["n"])
    a.build_index()
    f = tmp_path / "star.mbix"
    a.save_index(f)
    b = Engine(0)
    b.gen_star(g["seed"], g["k"], g["n"])
    b.load_index(f)
    assert b.info()["nbitmaps"] == a.info()["nbitmaps"] and b.info()["index_bytes"] == a.info()["index_bytes"]
    qs = WL.ssb13() + WL.random_mix(51, 30, narrow=0.4)
    for q in qs:
        oa, na, _ = a.query(q)
        ob, nb, _ = b.query(q)
        np.testing.assert_array_equal(oa, ob)
        assert na == nb
    ba, bna = a.query_batch(qs)
    bb, bnb = b.query_batch(qs)
    np.testing.assert_array_equal(ba, bb)
    np.testing.assert_array_equal(bna, bnb)
    raw = bytearray(f.read_bytes())
    raw[len(raw) // 2] ^= 0x40
    bad = tmp_path / "bad.mbix"
    bad.write_bytes(bytes(raw))
    with pytest.raises(mb.MbError) as ei:
        b.load_index(bad)
    assert ei.value.status == abi.MB_ERR_IO
    c = Engine(0)
    c.gen_star(g["seed"], g["k"], g["n"] + 1000)
    with pytest.raises(mb.MbError) as ei:
        c.load_index(f)
    assert ei.value.status == abi.MB_ERR_INVALID
    for e in (a, b, c):
        e.close()


def test_engine_index_planner(cuda, mb, tmp_path):
    """The index-memory planner drops levels to fit a budget (the workload's
    estimated bytes rise), an index built with its choice answers every query
    as the full one, and an index file keeps the choice."""
    g = G["ssb13"]
    e = Engine(0)
    e.gen_star(g["seed"], g["k"], g["n"])
    e.build_index()
    full = e.info()["index_bytes"]
    qs = WL.random_mix(61, 200, narrow=0.3)
    m_all, b_all, w_all = e.plan_index(qs, full)
    assert m_all == abi.MB_LEVELS_ALL and b_all == full
    m, b, w = e.plan_index(qs, int(full * 0.6))
    assert b <= full * 0.6 and m != abi.MB_LEVELS_ALL and w >= w_all
    want = [e.query(q)[:2] for q in qs[:40]]
    wb = e.query_batch(qs[:40])
    e.build_index_levels(m)
    assert e.info()["index_bytes"] == b
    for q, (o, n) in zip(qs[:40], want):
        out, nq, _ = e.query(q)
        np.testing.assert_array_equal(out, o)
        assert nq == n
    ob, nb = e.query_batch(qs[:40])
    np.testing.assert_array_equal(ob, wb[0])
    np.testing.assert_array_equal(nb, wb[1])
    f = tmp_path / "small.mbix"
    e.save_index(f)
    e2 = Engine(0)
    e2.gen_star(g["seed"], g["k"], g["n"])
    e2.load_index(f)
    assert e2.info()["index_bytes"] == b
    out, nq, _ = e2.query(qs[0])
    np.testing.assert_array_equal(out, want[0][0])
    with pytest.raises(mb.MbError):
        e.plan_index(qs, full // 10)  # below the smallest index (one level per column)
    with pytest.raises(mb.MbError):
        e.build_index_levels(0x3fe & ~0x3)  # no date level
    e.close()
    e2.close()
