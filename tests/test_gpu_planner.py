"""GPU tests of the learned planner: the network's forward and backward
kernels against the CPU oracle (oracle/mlp.py), training on the GPU, the
features and candidate plans of the engine (every candidate gives the oracle's
answer), and what the trained network gains over the rule planner on
held-out queries."""
from __future__ import annotations

import numpy as np
import pytest

from merle_b200 import workload as WL
from merle_b200 import planner as P
from merle_b200.engine import Engine
from oracle import mlp as OM

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net(cuda, mb):
    m = P.MLP(32, 64, 12, seed=7)
    yield m
    m.close()


def _data(seed, n, nin=32, nout=12):
    rng = np.random.default_rng(seed)
    x = rng.random((n, nin)).astype(np.float32)
    t = rng.normal(0, 1, (n, nout)).astype(np.float32)
    mask = (rng.random((n, nout)) < 0.8).astype(np.float32)
    return x, t, mask


def test_mlp_forward_fp32_matches_oracle(net):
    x, _, _ = _data(1, 300)
    p = net.get_params()
    y = net.forward(x)
    want, _ = OM.forward(p, x, 32, 64, 12)
    # FP32 products summed in a different order than the float64 oracle
    np.testing.assert_allclose(y, want, rtol=1e-4, atol=1e-5)


def test_mlp_forward_bf16_matches_oracle(net):
    x, _, _ = _data(2, 300)
    p = net.get_params()
    y = net.forward(x, bf16=True)
    want, _ = OM.forward(p, x, 32, 64, 12, bf=True)
    # both round weights and activations to bfloat16; FP32 vs float64
    # accumulation can move an activation across a rounding boundary (one
    # bfloat16 ulp = 2^-8 relative), which the next layers carry on
    np.testing.assert_allclose(y, want, rtol=2e-2, atol=2e-2)


def test_mlp_gradients_match_oracle(net):
    x, t, mask = _data(3, 257)
    p = net.get_params()
    loss, g = net.gradients(x, t, mask)
    wl, wg = OM.loss_and_grad(p, x, t, mask, 32, 64, 12)
    assert loss == pytest.approx(wl, rel=1e-4)
    scale = np.max(np.abs(wg))
    np.testing.assert_allclose(g, wg, rtol=1e-3, atol=1e-5 * scale)


def test_mlp_set_get_roundtrip_and_bad_args(net, mb):
    p = net.get_params()
    net.set_params(p * 0.5)
    np.testing.assert_array_equal(net.get_params(), (p * 0.5).astype(np.float32))
    net.set_params(p)
    with pytest.raises(mb.MbError):
        net.train(*_data(4, 10), epochs=0)


def test_mlp_train_fits_a_function(cuda, mb):
    rng = np.random.default_rng(9)
    x = rng.random((4096, 32)).astype(np.float32)
    w = rng.normal(0, 1, (32, 12))
    t = np.tanh(x @ w).astype(np.float32)
    mask = np.ones_like(t)
    m = P.MLP(32, 64, 12, seed=3)
    try:
        l0, _ = m.gradients(x, t, mask)
        lf = m.train(x, t, mask, epochs=60, batch=256, lr=3e-3, seed=1)
        l1, _ = m.gradients(x, t, mask)
        assert l1 < 0.05 * l0 and lf < 0.05 * l0
        # the training log and the weights survive a save / load
    finally:
        m.close()


def test_mlp_save_load(tmp_path, net):
    f = tmp_path / "w.f32"
    net.save(f)
    m2 = P.MLP.load(f)
    try:
        np.testing.assert_array_equal(m2.get_params(), net.get_params())
    finally:
        m2.close()


@pytest.fixture(scope="module")
def eng24(cuda, mb):
    e = Engine(0)
    e.gen_star(2, 4, 24_000_000)
    e.build_index()
    yield e
    e.close()


def test_features_shape(eng24):
    q = WL.ssb13()[0]
    f = P.query_features(eng24, q)
    assert f.shape == (32,) and f[31] == 1.0 and f[0] == 1.0 and f[1:4].sum() == 0
    assert np.isfinite(f).all()
    f2 = P.query_features(eng24, q)
    np.testing.assert_array_equal(f, f2)


def test_every_candidate_gives_the_same_answer(eng24):
    qs = WL.ssb13() + WL.random_mix(21, 24, narrow=0.4)
    for q in qs:
        want, nqw, _ = eng24.query(q)
        for c in range(1, P.NC):
            out, nq, _ = eng24.query(q, P.candidate_plan(eng24, q, c))
            np.testing.assert_array_equal(out, want, err_msg=f"{WL.as_tuple(q)} candidate {c}")
            assert nq == nqw


def test_learned_planner_gains_over_rule(eng24):
    """Train on timings of 600 random queries, plan 200 held-out ones with the
    BF16 network inside the engine, and time both choices."""
    train_q = P._mix(31, 600)
    seen = {WL.as_tuple(q) for q in train_q}
    eval_q = P._mix(32, 200, frozenset(seen))
    X = P.features(eng24, train_q)
    T = P.measure_candidates(eng24, train_q, reps=3)
    t, mask = P.targets(T)
    m = P.MLP(seed=11)
    try:
        m.train(X, t, mask, epochs=150, batch=128, lr=2e-3, seed=2)
        _, chosen = P.plan_learned(eng24, eval_q, m)
    finally:
        m.close()
    TE = P.measure_candidates(eng24, eval_q, reps=3)
    r = P.regret_report(TE, chosen)
    print("learned planner, 200 held-out queries at 24M rows:", r)
    assert r["regret_total"] <= 1.15
    assert r["speedup_vs_rule_total"] >= 1.0


def test_planner_network_shape_checked(net, eng24, mb):
    """A network whose outputs are not one per candidate plan is refused."""
    from merle_b200 import lib
    assert net.nout != P.NC
    assert lib().mb_engine_set_planner(eng24.handle, net.handle) == mb.abi.MB_ERR_INVALID
    m = P.MLP(seed=1)
    try:
        assert lib().mb_engine_set_planner(eng24.handle, m.handle) == mb.abi.MB_OK
        assert lib().mb_engine_set_planner(eng24.handle, None) == mb.abi.MB_OK
    finally:
        m.close()


# ------------------------------------------------------------ batch planner
def test_batch_features_and_network_shape(eng24, net, mb):
    from merle_b200 import lib
    qs = WL.span_mix(5, 24)
    f = P.batch_features(eng24, qs)
    assert f.shape == (P.NBF,) and np.isfinite(f).all() and f[31] == 1.0
    np.testing.assert_array_equal(f, P.batch_features(eng24, qs))
    assert lib().mb_engine_set_batch_planner(eng24.handle, net.handle) == mb.abi.MB_ERR_INVALID  # 32 -> 12
    m = P.MLP(P.NBF, 64, P.NBC, seed=3)
    try:
        assert lib().mb_engine_set_batch_planner(eng24.handle, m.handle) == mb.abi.MB_OK
        assert lib().mb_engine_set_batch_planner(eng24.handle, None) == mb.abi.MB_OK
    finally:
        m.close()


def test_every_batch_plan_gives_the_same_answer(eng24):
    """Every launch shape and cover of the batch plans: the same group sums
    and row counts as the rule-planned batch (time_batch checks them)."""
    for qs in (WL.span_mix(6, 24), WL.ssb13() + WL.random_mix(22, 9, narrow=0.5)):
        want = P.batch_results(eng24, qs)
        for c in range(P.NBC):
            o, cover = P.batch_candidate(c)
            P.time_batch(eng24, qs, o, cover, reps=1, want=want)


def test_batch_planner_gains_over_rule(eng24):
    """Train the batch planner on engine timings of 48 random batches (2 to
    128 queries), plan 16 held-out batches with the BF16 network inside the
    engine, and time every plan: the learned plans are at least 5 % faster in
    total than the rule-planned batches and within 15 % of the best plan."""
    tb = P.random_batches(41, 48)
    X = np.stack([P.batch_features(eng24, b) for b in tb])
    T = P.measure_batch_candidates(eng24, tb, reps=2, check_results=False)
    t, mask = P.targets(T)
    m = P.MLP(P.NBF, 64, P.NBC, seed=5)
    eb = P.random_batches(42, 16)
    try:
        m.train(X, t, mask, epochs=300, batch=32, lr=2e-3, seed=2)
        chosen = P.plan_batches_learned(eng24, eb, m)
    finally:
        m.close()
    TE = P.measure_batch_candidates(eng24, eb, reps=3, check_results=False)
    t_rule = np.array([P.time_batch(eng24, b, None, 0, 3) for b in eb])
    r = P.batch_regret_report(TE, chosen, t_rule)
    print("batch planner, 16 held-out batches at 24M rows:", r)
    assert r["regret_total"] <= 1.15
    assert r["speedup_vs_rule_total"] >= 1.05
