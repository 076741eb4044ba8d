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


def test_engine_errors(eng, mb):
    out = np.zeros(8, np.int64)
    q = abi.query(9, 1, 2)
    st = mb.lib().mb_engine_query(eng.handle, C.byref(q), None, out.ctypes.data, None, None)
    assert st == abi.MB_ERR_INVALID
    e = Engine(0)
    q = abi.query(1, 0, 10, 0, 1, 1, 2)
    assert mb.lib().mb_engine_query(e.handle, C.byref(q), None, out.ctypes.data, None, None) == abi.MB_ERR_INVALID
    e.close()
