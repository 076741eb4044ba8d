"""CPU tests of the serving loop's host parts: the Poisson arrival generator
and the latency summary."""
from __future__ import annotations

import numpy as np
import pytest

from merle_b200 import abi, serving as SV


def test_poisson_arrivals_are_exponential(mb):
    rate = 5000.0
    t = SV.poisson_arrivals(7, rate, 200_000)
    gaps = np.diff(np.concatenate([[0.0], t])) / 1e6
    assert (gaps > 0).all() and np.all(np.diff(t) > 0)
    assert gaps.mean() == pytest.approx(1 / rate, rel=0.01)
    assert gaps.std() == pytest.approx(1 / rate, rel=0.02)  # exponential: sd = mean
    # P(gap > x) = exp(-rate x) at a few quantiles
    for q in (0.5, 1.0, 2.0, 4.0):
        assert (gaps > q / rate).mean() == pytest.approx(np.exp(-q), abs=0.005)
    np.testing.assert_array_equal(t, SV.poisson_arrivals(7, rate, 200_000))
    assert not np.array_equal(t[:100], SV.poisson_arrivals(8, rate, 100))


def test_poisson_arrivals_rejects_bad_rate(mb):
    with pytest.raises(mb.MbError):
        SV.poisson_arrivals(1, 0.0, 10)


def test_summarize():
    infos = []
    for i in range(100):
        r = abi.mb_request_info()
        r.status = abi.MB_OK if i < 98 else abi.MB_ERR_REJECTED
        r.t_submit_us = i * 1000.0
        r.t_launch_us = r.t_submit_us + 100
        r.t_done_us = r.t_submit_us + 1000.0 * (1 + (i % 10))
        r.batch_size = 4
        r.launch = i // 4
        infos.append(r)
    s = SV.summarize(infos, 1000.0)
    assert s["ok"] == 98 and s["statuses"] == {"MB_OK": 98, "MB_ERR_REJECTED": 2}
    assert s["p50_ms"] == pytest.approx(np.percentile([1 + (i % 10) for i in range(98)], 50))
    assert s["mean_batch"] == 4 and s["queue_p50_ms"] == pytest.approx(0.1)
