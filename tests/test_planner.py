"""CPU tests of the learned planner's pieces that need no GPU: the network
oracle (its gradients against finite differences, its bfloat16 rounding
against torch's), and the host logic that turns timings into targets and
regret figures."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp as OM


def _params(rng, nin, nh, nout, scale=0.4):
    n = nh * nin + nh + nh * nh + nh + nout * nh + nout
    return rng.normal(0, scale, n)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    nin, nh, nout, n = 6, 8, 4, 20
    p = _params(rng, nin, nh, nout)
    x = rng.normal(0, 1, (n, nin))
    t = rng.normal(0, 1, (n, nout))
    mask = (rng.random((n, nout)) < 0.7).astype(float)
    loss, g = OM.loss_and_grad(p, x, t, mask, nin, nh, nout)
    eps = 1e-6
    num = np.zeros_like(p)
    for i in range(len(p)):
        d = np.zeros_like(p)
        d[i] = eps
        num[i] = (OM.loss_and_grad(p + d, x, t, mask, nin, nh, nout)[0]
                  - OM.loss_and_grad(p - d, x, t, mask, nin, nh, nout)[0]) / (2 * eps)
    # ReLU kinks are measure-zero for these inputs; central differences in
    # float64 agree to ~1e-8
    np.testing.assert_allclose(g, num, rtol=1e-5, atol=1e-7)
    assert loss > 0


def test_oracle_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.normal(0, 10, 5000), rng.normal(0, 1e-3, 5000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, -3.5, 65504.0])]).astype(np.float32)
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(OM.bf16(a), want)


def test_oracle_forward_bf16_close_to_fp32():
    rng = np.random.default_rng(2)
    p = _params(rng, 32, 64, 12, 0.2)
    x = rng.random((50, 32))
    y, _ = OM.forward(p, x, 32, 64, 12)
    yb, _ = OM.forward(p, x, 32, 64, 12, bf=True)
    assert np.max(np.abs(y - yb)) < 0.05 * (1 + np.max(np.abs(y)))


def test_targets_and_regret_report():
    from merle_b200 import planner as P
    times = np.array([[2.0, 1.0, 4.0] + [np.nan] * (P.NC - 3),
                      [1.0, 3.0, 1.5] + [np.nan] * (P.NC - 3)])
    t, m = P.targets(times)
    np.testing.assert_allclose(t[0, :3], np.log([2.0, 1.0, 4.0]), rtol=1e-6)
    np.testing.assert_allclose(t[1, :3], np.log([1.0, 3.0, 1.5]), rtol=1e-6)
    assert m[:, :3].all() and not m[:, 3:].any()
    full = np.nan_to_num(times, nan=1e9)
    r = P.regret_report(full, np.array([1, 0]))
    assert r["regret_mean"] == pytest.approx(1.0)
    assert r["rule_regret_mean"] == pytest.approx(1.5)
    assert r["speedup_vs_rule_total"] == pytest.approx(3.0 / 2.0)
    r2 = P.regret_report(full, np.array([2, 2]))
    assert r2["regret_max"] == pytest.approx(4.0)
    assert r2["regret_total"] == pytest.approx(5.5 / 2.0)
