"""Parity at the benchmark configurations' full sizes.

Against the reference's own CPU code (ssb/cpuref.c s1ref..s4ref, compiled
from its sources into oracle/_ref, run over every row of a host copy of the
table generated by the oracle): at 120M rows the selectivity-spanning
64-query mix and the 13 SSB queries through the batched scan (rule and
learned batch plans) and the plain path, and the SSB queries through every
plan kind (fused, materialised, no-index scan, hash joins); at 600M rows the
mix through the batched scan.  The reference sums uint32 (its s1ref a
uint64), so (uint32) of every int64 group sum must equal its value.

Through properties that hold at any size: at 600M rows the batched scan
answers every query of the 64-query mix exactly as the plain path does; at
1.8B rows (row ids above 2^30, 132 GB resident) the answers of the whole table
equal the sums of the answers of its two halves, each half generated and
indexed on its own (group sums and row counts are additive over row ranges)."""
from __future__ import annotations

import numpy as np
import pytest

from merle_b200 import shard, workload as WL
from merle_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _reference(orc, k, n, qs):
    """The reference's answers over the whole table (host copy), or skip."""
    import os
    if orc.ref() is None:
        pytest.skip("oracle/_ref (the reference's cpuref) not built")
    try:
        import psutil
        if psutil.virtual_memory().available < n * 40:
            pytest.skip("host memory too small for the table")
    except ImportError:
        pass
    star = orc.StarHost(2, k, n)
    ans, _ = orc.ref_answers(star.ssb_schema(), n, qs, os.cpu_count() or 1)
    return ans


def _assert_reference(qs, answers, out, nqs=None):
    """(uint32) of our int64 group sums equal the reference's uint32 arrays;
    s1ref's uint64 sum equals ours as uint64."""
    off = 0
    for q, a in zip(qs, answers):
        ng = Engine.ngroups(q)
        mine = np.asarray(out[off:off + ng])
        if int(q.tmpl) == 1:
            assert int(mine[0]) % (1 << 64) == int(a[0]), WL.as_tuple(q)
        else:
            np.testing.assert_array_equal(mine.astype(np.uint64).astype(np.uint32), a, err_msg=str(WL.as_tuple(q)))
        off += ng


def _batch_learned(e, qs):
    """The batch under the committed learned batch planner (or the rule's
    plan if the weights are absent)."""
    from pathlib import Path
    from merle_b200 import lib
    from merle_b200.planner import MLP
    w = Path(__file__).resolve().parent.parent / "merle_b200" / "weights" / "batch_planner.f32"
    if not w.exists():
        return e.query_batch(qs)
    m = MLP.load(w)
    try:
        lib().mb_engine_set_batch_planner(e.handle, m.handle)
        return e.query_batch(qs)  # no options: the engine plans the batch with its network
    finally:
        lib().mb_engine_set_batch_planner(e.handle, None)
        m.close()


def test_120M_every_plan_matches_reference(cuda, mb, orc):
    from merle_b200 import abi
    n = 120_000_000
    qs = WL.span_mix(3, 64) + WL.ssb13()
    want = _reference(orc, 20, n, qs)
    e = Engine(0)
    try:
        e.gen_star(2, 20, n, width4=True)
        e.build_index()
        out, _ = e.query_batch(qs, abi.mb_batch_opts())
        _assert_reference(qs, want, out)
        out, _ = _batch_learned(e, qs)
        _assert_reference(qs, want, out)
        out, _ = _plain(e, qs)
        _assert_reference(qs, want, out)
        ssb = WL.ssb13()
        for kind in (abi.PLAN_MATERIALISED, abi.PLAN_SCAN, abi.PLAN_HASH):
            plan = abi.mb_plan()
            plan.kind = kind
            outs = [e.query(q, plan)[0] for q in ssb]
            _assert_reference(ssb, want[64:], np.concatenate(outs))
    finally:
        e.close()


def test_600M_batch_matches_reference(cuda, mb, orc):
    n = 600_000_000
    qs = WL.span_mix(3, 64)
    want = _reference(orc, 100, n, qs)
    e = Engine(0)
    try:
        e.gen_star(2, 100, n, width4=True)
        e.build_index()
        out, _ = _batch_learned(e, qs)
        _assert_reference(qs, want, out)
    finally:
        e.close()


def _plain(e, qs):
    outs, nqs = [], []
    for q in qs:
        o, n, _ = e.query(q)
        outs.append(o)
        nqs.append(n)
    return np.concatenate(outs), np.array(nqs, np.uint64)


def test_600M_batch_equals_plain(cuda, mb):
    """The batched scan, the plain path, the no-index scan and the hash-join
    plan agree on every query (the last two on the SSB queries)."""
    from merle_b200 import abi
    e = Engine(0)
    try:
        e.gen_star(2, 100, 600_000_000, width4=True)
        e.build_index()
        qs = WL.random_mix(3, 64, 0.3)
        out, nq = e.query_batch(qs)
        want, wn = _plain(e, qs)
        np.testing.assert_array_equal(out, want)
        np.testing.assert_array_equal(nq, wn)
        for kind in (abi.PLAN_SCAN, abi.PLAN_HASH):
            plan = abi.mb_plan()
            plan.kind = kind
            for q in WL.ssb13():
                o1, n1, _ = e.query(q)
                o2, n2, _ = e.query(q, plan)
                np.testing.assert_array_equal(o2, o1, err_msg=f"kind {kind} {WL.as_tuple(q)}")
                assert n2 == n1
    finally:
        e.close()


def test_1800M_halves_add_up(cuda, mb):
    total = 1_800_000_000
    half = total // 2
    qs = WL.ssb13() + WL.random_mix(17, 19, 0.3)
    parts = []
    for rank in (0, 1):
        row0, n = shard.row_range(rank, half)
        e = Engine(0)
        try:
            e.gen_star(2, 300, n, width4=True, row0=row0)
            e.build_index()
            parts.append(_plain(e, qs))
        finally:
            e.close()
    e = Engine(0)
    try:
        e.gen_star(2, 300, total, width4=True)
        e.build_index()
        out, nq = e.query_batch(qs)
        one, onq = _plain(e, qs[:6])
    finally:
        e.close()
    np.testing.assert_array_equal(out, parts[0][0] + parts[1][0])
    np.testing.assert_array_equal(nq, parts[0][1] + parts[1][1])
    k = sum(Engine.ngroups(q) for q in qs[:6])
    np.testing.assert_array_equal(one, out[:k])
    np.testing.assert_array_equal(onq, nq[:6])
