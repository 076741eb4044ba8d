"""Parity at the benchmark configurations' full sizes, through properties
that hold at any size (the CPU oracle is too slow there): at 600M rows the
batched scan answers every query of the 64-query mix exactly as the plain
path does, and the no-index scan and the hash-join plan answer the SSB
queries as the index plan does; at 1.8B rows (row ids above 2^30, 132 GB resident) the answers of
the whole table equal the sums of the answers of its two halves, each half
generated and indexed on its own (group sums and row counts are additive over
row ranges)."""
from __future__ import annotations

import numpy as np
import pytest

from merle_b200 import shard, workload as WL
from merle_b200.engine import Engine

pytestmark = pytest.mark.gpu


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
