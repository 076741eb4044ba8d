"""World-size-2 test of the row-sharded path on CPU (gloo): each rank takes
its row range of the star schema, answers the queries over it (the oracle
stands in for the GPU engine here), and merle_b200.shard.combine sums the
tables; the sums equal the answers over all the rows at once."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from merle_b200 import workload as WL

K, ROWS_PER_RANK, WORLD = 1, 150_000, 2


def _queries():
    return WL.ssb13() + WL.random_mix(9, 12, narrow=0.4)


def _answers(star, qs):
    from merle_b200.engine import Engine
    from tests import helpers as H
    from oracle import oracle as O
    outs, nqs = [], []
    for q in qs:
        t, a = WL.as_tuple(q)
        o, n = O.join_grpby(star.n, H.ssb_op(star, WL.TEMPLATE_NAME[t], a).to_c(), Engine.ngroups(q))
        outs.append(np.asarray(o, np.int64))
        nqs.append(n)
    return np.concatenate(outs), np.array(nqs, np.int64)


def _rank(rank, port, result):
    import torch.distributed as dist
    from merle_b200 import shard
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        row0, n = shard.row_range(rank, ROWS_PER_RANK)
        star = O.StarHost(2, K, n, row0=row0)
        out, nq = _answers(star, _queries())
        t_out, t_nq = torch.from_numpy(out.copy()), torch.from_numpy(nq.copy())
        shard.combine(t_out, t_nq)
        if rank == 0:
            result["out"] = t_out.numpy().copy()
            result["nq"] = t_nq.numpy().copy()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_row_shards_sum_to_whole_table(orc):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    result = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, result)) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    star = orc.StarHost(2, K, ROWS_PER_RANK * WORLD)
    want, wn = _answers(star, _queries())
    np.testing.assert_array_equal(result["out"], want)
    np.testing.assert_array_equal(result["nq"], wn)


def test_row_range():
    from merle_b200 import shard
    assert shard.row_range(3, 100) == (300, 100)
    with pytest.raises(ValueError):
        shard.row_range(0, 0)
