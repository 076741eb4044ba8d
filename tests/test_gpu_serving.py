"""GPU tests of the serving loop (mb_server_*): every answer under Poisson
load, in batched and plain mode, equals the engine's answer for the query
alone; admission holds reservations under the budget and rejects what can
never fit; cancellation and host-side fault injection (failed arena
allocation, failed launch, slow launch) end the affected requests with their
status while the rest are answered.  No GPU fault is made."""
from __future__ import annotations

import numpy as np
import pytest

from merle_b200 import abi, workload as WL
from merle_b200 import serving as SV
from merle_b200.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng(cuda, mb):
    e = Engine(0)
    e.gen_star(2, 4, 24_000_000)
    e.build_index()
    yield e
    e.close()


@pytest.fixture(scope="module")
def mix():
    return WL.ssb13() + WL.random_mix(41, 240, narrow=0.4)


@pytest.fixture(scope="module")
def alone(eng, mix):
    res = []
    for q in mix:
        out, nq, _ = eng.query(q)
        res.append((out, nq))
    return res


def _layout(qs):
    offs = np.cumsum([0] + [Engine.ngroups(q) for q in qs])
    return offs


@pytest.mark.parametrize("mode,rate,min_batch", [(abi.SERVE_BATCHED, 20000.0, 0), (abi.SERVE_BATCHED, 2000.0, 0),
                                                 (abi.SERVE_BATCHED, 20000.0, 1), (abi.SERVE_BATCHED, 2000.0, 1),
                                                 (abi.SERVE_PLAIN, 20000.0, 0)])
def test_serving_results_equal_alone(eng, mix, alone, mode, rate, min_batch):
    with SV.Server(eng, mode, min_batch=min_batch) as s:
        out, info = s.run_load(mix, rate, seed=3)
        st = s.stats()
    offs = _layout(mix)
    for i, q in enumerate(mix):
        assert info[i].status == abi.MB_OK
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], alone[i][0], err_msg=str(WL.as_tuple(q)))
        assert info[i].nqual == alone[i][1]
        assert info[i].t_submit_us <= info[i].t_launch_us <= info[i].t_done_us
    assert st["completed"] == len(mix) and st["failed"] == 0
    if mode == abi.SERVE_BATCHED and rate >= 20000 and min_batch == 1:
        assert st["launches"] < len(mix) and st["scan_launches"] == st["launches"]  # requests shared launches
    if mode == abi.SERVE_BATCHED:
        assert st["launched_queries"] == len(mix)
    if mode == abi.SERVE_PLAIN:
        assert st["launches"] == len(mix)
    r = SV.summarize(info, rate)
    assert r["ok"] == len(mix) and r["p99_ms"] >= r["p50_ms"] > 0


def test_admission_budget_bounds_reservations(eng, mix, alone):
    # room for about 3000 groups in flight: launches wait for each other
    budget = 24 * 1024
    with SV.Server(eng, abi.SERVE_BATCHED, mem_budget=budget, max_inflight=4) as s:
        out, info = s.run_load(mix, 50000.0, seed=4)
        st = s.stats()
    offs = _layout(mix)
    big = [i for i, q in enumerate(mix) if 8 * (Engine.ngroups(q) + 1) > budget]
    for i in range(len(mix)):
        if i in big:
            assert info[i].status == abi.MB_ERR_REJECTED
        else:
            assert info[i].status == abi.MB_OK
            np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], alone[i][0])
    assert st["peak_reserved"] <= budget
    assert st["rejected"] == len(big)


def test_request_larger_than_budget_is_rejected(eng):
    q = abi.query(2, 0, 1000, 0, 250)  # 7 * 1000 groups
    with SV.Server(eng, abi.SERVE_BATCHED, mem_budget=4096) as s:
        out = np.zeros(Engine.ngroups(q), np.int64)
        rid = s.submit(q, out)
        assert s.wait(rid, 10_000).status == abi.MB_ERR_REJECTED


def test_cancel_and_injected_faults(eng, mix, alone):
    offs = _layout(mix)
    with SV.Server(eng, abi.SERVE_BATCHED, max_batch=8, max_inflight=1) as s:
        # a slow first launch keeps the rest queued; then fail two launches
        s.inject(abi.FAULT_SLOW, 1, 200_000)
        outs = [np.zeros(offs[i + 1] - offs[i], np.int64) for i in range(len(mix))]
        ids = [s.submit(q, outs[i]) for i, q in enumerate(mix[:64])]
        cancelled = {i for i in range(40, 64, 3) if s.cancel(ids[i])}
        assert cancelled  # queued behind the held launch
        s.inject(abi.FAULT_ALLOC, 1)
        s.inject(abi.FAULT_LAUNCH, 1)
        infos = [s.wait(r, 60_000) for r in ids]
        st = s.stats()
    failed = [i for i, inf in enumerate(infos) if inf.status in (abi.MB_ERR_OOM, abi.MB_ERR_CUDA)]
    assert {infos[i].status for i in failed} <= {abi.MB_ERR_OOM, abi.MB_ERR_CUDA}
    assert st["failed"] == len(failed) and len(failed) > 0
    for i, inf in enumerate(infos):
        if i in cancelled:
            assert inf.status == abi.MB_ERR_CANCELLED
        elif i not in failed:
            assert inf.status == abi.MB_OK
            np.testing.assert_array_equal(outs[i], alone[i][0])
    # the held launch took at least the injected 200 ms
    assert infos[0].t_done_us - infos[0].t_submit_us >= 200_000
    assert st["cancelled"] == len(cancelled)


def test_wait_timeout_and_unknown_id(eng, mb):
    with SV.Server(eng, abi.SERVE_BATCHED, max_inflight=1) as s:
        s.inject(abi.FAULT_SLOW, 1, 300_000)
        q = WL.ssb13()[0]
        out = np.zeros(1, np.int64)
        rid = s.submit(q, out)
        with pytest.raises(mb.MbError):
            s.wait(rid, 1)  # not done within 1 ms: MB_ERR_TIMEOUT
        assert s.wait(rid, 60_000).status == abi.MB_OK
        with pytest.raises(mb.MbError):
            s.wait(rid, 1)  # already handed out


@pytest.mark.parametrize("mode,min_batch,rate", [(abi.SERVE_PLAIN, 0, 5000.0), (abi.SERVE_BATCHED, 65, 50000.0)])
def test_learned_planner_in_the_serving_loop(eng, mix, alone, mode, min_batch, rate):
    """Plain mode plans each request at the front of the queue; batched mode
    held to the plain path (min_batch above max_batch) plans a launch's query
    with the queued ones ahead of it in one planner call."""
    from merle_b200 import planner as P
    m = P.MLP(seed=5)  # untrained: any candidate may come out, answers must not change
    try:
        from merle_b200 import lib, check
        check(lib().mb_engine_set_planner(eng.handle, m.handle))
        with SV.Server(eng, mode, use_planner=True, mem_budget=1 << 30, min_batch=min_batch) as s:
            out, info = s.run_load(mix[:60], rate, seed=6)
            st = s.stats()
        check(lib().mb_engine_set_planner(eng.handle, None))
    finally:
        m.close()
    offs = _layout(mix[:60])
    plans = set()
    for i in range(60):
        assert info[i].status == abi.MB_OK
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], alone[i][0])
        assert info[i].nqual == alone[i][1] and info[i].batch_size == 1
        plans.add(info[i].plan)
    assert plans <= set(range(P.NC))
    assert st["launches"] == 60 and st["scan_launches"] == 0


def test_device_wait_runs_out(eng, mix, alone, mb):
    """A batched launch whose first staged tile is armed but never filled
    (mb_engine_test_stall): the bounded wait for it runs out after a few
    thousand tries, the kernel records the wait in the device error word and
    returns, and the call reports MB_ERR_TIMEOUT with zeroed results; the
    engine answers the next batch correctly.  In the server exactly the
    requests of the stalled launch end with MB_ERR_TIMEOUT and every other
    request is answered as alone."""
    from merle_b200 import lib
    qs = mix[:24]
    lib().mb_engine_test_stall(eng.handle, 1, 4096)
    with pytest.raises(mb.MbError) as ei:
        eng.query_batch(qs)
    assert ei.value.status == abi.MB_ERR_TIMEOUT and "code 1" in str(ei.value)
    out, nq = eng.query_batch(qs)  # the stall was one launch: this one is whole
    offs = _layout(qs)
    for i in range(len(qs)):
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], alone[i][0])
        assert nq[i] == alone[i][1]
    # the server: every launch on the batched scan, one at a time
    with SV.Server(eng, abi.SERVE_BATCHED, min_batch=1, max_inflight=1) as s:
        lib().mb_engine_test_stall(eng.handle, 1, 4096)
        out, info = s.run_load(mix, 20000.0, seed=5)
        st = s.stats()
    offs = _layout(mix)
    stalled = {i.launch for i in info if i.status == abi.MB_ERR_TIMEOUT}
    assert len(stalled) == 1, stalled
    for i, q in enumerate(mix):
        if info[i].launch in stalled:
            assert info[i].status == abi.MB_ERR_TIMEOUT
            continue
        assert info[i].status == abi.MB_OK
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], alone[i][0], err_msg=str(WL.as_tuple(q)))
        assert info[i].nqual == alone[i][1]
    assert st["failed"] == sum(1 for i in info if i.status == abi.MB_ERR_TIMEOUT) > 0
