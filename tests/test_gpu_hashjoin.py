"""GPU parity tests of the Crystal-style hash-join plan (mb_hash_join_grpby,
the engine's MB_PLAN_HASH): the 13 SSB queries against the oracle's no-index
plan and the reference's own answers (golden); the synthetic star query with
two attributes on one key and a mixed OR clause; tables small enough for
shared memory and too large for it; a dimension no row passes; the limits;
and the engine's hash plan against its other plans on the mix, with and
without denormalised dimension columns.  Integer work: bit-exact."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi, check, device as D, ops
from merle_b200 import workload as WL
from merle_b200.engine import Engine
from tests import helpers as H

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
G = json.loads((GOLDEN / "golden.json").read_text())


def host(t, dt):
    return D.to_host(t, dt)


def hash_join(n: int, op: abi.mb_op, nr_grp: int):
    out, nq = D.empty(nr_grp, 8), D.empty(1, 8)
    check(D.lib().mb_hash_join_grpby(n, C.byref(op), nr_grp, out.data_ptr(), nq.data_ptr(), D.stream_ptr()))
    return host(out, np.int64), int(host(nq, np.uint64)[0])


@pytest.fixture(scope="module")
def stars(cuda, orc, mb):
    g = G["ssb13"]
    return D.DevStar(g["seed"], g["k"], g["n"]), orc.StarHost(g["seed"], g["k"], g["n"])


def test_hash_join_ssb13(stars, orc):
    dev, ref = stars
    gold = np.load(GOLDEN / "ssb13_ref_u32.npy")
    for i, (q, a, ng) in enumerate(H.SSB13):
        want, nqw = orc.join_grpby(ref.n, H.ssb_op(ref, q, a).to_c(), ng)
        got, nq = hash_join(ref.n, H.ssb_op(dev, q, a).to_c(), ng)
        np.testing.assert_array_equal(got, want, err_msg=f"{q}{a}")
        assert nq == nqw
        np.testing.assert_array_equal(got.astype(np.uint32), gold[H.SLOTS[i]:H.SLOTS[i + 1]])


def test_hash_join_large_and_small_tables(stars, orc):
    """A part filter every part passes (a table far over the shared-memory
    limit, probed in global memory) and a narrow one (staged per CTA)."""
    dev, ref = stars
    for a in [(0, 1000, 0, 250), (0, 1000, 150, 200), (260, 261, 0, 250)]:
        want, nqw = orc.join_grpby(ref.n, H.ssb_op(ref, "s2", a).to_c(), 1000)
        got, nq = hash_join(ref.n, H.ssb_op(dev, "s2", a).to_c(), 1000)
        np.testing.assert_array_equal(got, want, err_msg=f"{a}")
        assert nq == nqw


def test_hash_join_no_dimension_row_passes(stars):
    dev, _ = stars
    got, nq = hash_join(dev.n, H.ssb_op(dev, "s3", (251, 255, 0, 250, 0, 2557)).to_c(), 150)
    assert nq == 0 and not got.any()


def test_hash_join_synth_two_attributes_on_one_key(orc, cuda):
    """The synthetic star query with bounds-checked keys: both dimension
    attributes ride in one table; the fact OR clause runs first."""
    from tests.golden.make_golden import synth_tables
    n = G["synth"]["n"]
    for bw in G["synth"]["bitwidths"]:
        a1, a2, fk, d1, d2 = synth_tables(bw)
        t = [D.from_host(x) for x in (a1, a2, fk, d1, d2)]
        for case in G["synth"]["cases"]:
            def op_of(c):
                return ops.Op(srcs=[ops.Src(c[0]), ops.Src(c[1]), ops.Src(c[3], c[2]), ops.Src(c[4], c[2])],
                              clauses=[[(0, case[0], case[1]), (1, case[2], case[3])], [(2, case[4], case[5])]],
                              keys=[(3, abi.X_ID, 1, 0, 1)], vkind=abi.V_ONE).to_c()
            want, nqw = orc.join_grpby(n, op_of((a1, a2, fk, d1, d2)), 256)
            got, nq = hash_join(n, op_of(t), 256)
            np.testing.assert_array_equal(got, want, err_msg=f"{bw} {case}")
            assert nq == nqw


def test_hash_join_limits(stars, mb):
    dev, _ = stars
    # four attributes on one key: more than a table entry carries
    op = ops.Op(srcs=[ops.Src(dev.custcity, dev["custkey"])] * 4,
                clauses=[[(0, 0, 100)]], keys=[], vkind=abi.V_ONE).to_c()
    out, nq = D.empty(1, 8), D.empty(1, 8)
    assert mb.lib().mb_hash_join_grpby(dev.n, C.byref(op), 1, out.data_ptr(), nq.data_ptr(),
                                       D.stream_ptr()) == abi.MB_ERR_UNSUPPORTED
    assert mb.lib().mb_hash_join_grpby(dev.n, C.byref(op), 0, out.data_ptr(), nq.data_ptr(),
                                       D.stream_ptr()) == abi.MB_ERR_INVALID


@pytest.mark.parametrize("probe_dims", [False, True])
def test_engine_hash_plan(cuda, mb, probe_dims):
    e = Engine(0)
    try:
        e.gen_star(2, 4, 6_000_000)
        e.build_index(probe_dims=probe_dims)
        plan = abi.mb_plan()
        plan.kind = abi.PLAN_HASH
        for q in WL.ssb13() + WL.random_mix(5, 40, narrow=0.4):
            want, nqw, _ = e.query(q)
            got, nq, _ = e.query(q, plan)
            np.testing.assert_array_equal(got, want, err_msg=f"{WL.as_tuple(q)}")
            assert nq == nqw
        bad = abi.mb_plan()
        bad.kind = 9
        with pytest.raises(mb.MbError):
            e.query(WL.ssb13()[0], bad)
    finally:
        e.close()


@pytest.mark.parametrize("width,n,offset", [(8, 100_003, 0), (4, 128 * 300 + 77, 0), (2, 4097, 0),
                                            (1, 131, 0), (4, 50_001, 1)])
def test_hash_probe_screen_widths_tails_alignment(orc, cuda, width, n, offset):
    """The hash probe's screen: one range on a fact column of each width (four
    rows a lane from one vector load), row counts that end inside a 128-row
    chunk, and a column that is not 16-byte aligned (the generic screen), next
    to a dimension clause through a foreign key (so a table is built and
    probed); SUM(b * c) and the row count equal the oracle's no-index plan."""
    rng = np.random.default_rng(width * 7000 + n)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width]
    a_full = rng.integers(0, 200, n + offset).astype(dt)
    b = rng.integers(0, 1000, n).astype(np.uint32)
    c = rng.integers(0, 50, n).astype(np.uint32)
    dim = rng.integers(0, 1000, 5000).astype(np.uint16)
    fk = rng.integers(0, 5000, n).astype(np.uint32)
    a = a_full[offset:]

    def op(cols):
        return ops.Op(srcs=[ops.Src(cols[0]), ops.Src(cols[1]), ops.Src(cols[2]), ops.Src(cols[3], cols[4])],
                      clauses=[[(0, 40, 90)], [(3, 100, 700)]], keys=[], vkind=abi.V_MUL, va=1, vb=2).to_c()
    want, nqw = orc.join_grpby(n, op((np.ascontiguousarray(a), b, c, dim, fk)), 1)
    da_full = D.from_host(a_full)
    da = da_full[offset:] if offset else da_full
    got, nq = hash_join(n, op((da, D.from_host(b), D.from_host(c), D.from_host(dim), D.from_host(fk))), 1)
    assert int(got[0]) == int(want[0]) and nq == nqw
