"""The learned planner: a 3-layer perceptron (32 -> 64 -> 64 -> 16) that
predicts, from a query's features, the log slowdown of each of the engine's
16 candidate plans against the fastest of them; the engine runs the candidate
with the least prediction.

Everything numeric runs in libmerleb200.so: the features (bin counts and
popcounts from the index, a GPU popcount of the program over 1% of the rows),
the candidate plans, the timings (CUDA events around each query's launch
sequence), the network's forward / backward / Adam kernels (FP32) and the
planning pass (BF16).  This module moves arrays between them.

The reference has no learned component: its programs come from the fixed rules
col::from_bin / from_bin2 (bmpidx_create.cu:138-226), which the engine's rule
planner (candidate 0) generalises and which stays the fallback.

Command line: python -m merle_b200.planner --train-rows N --train-queries Q
--eval-rows N2 --eval-queries Q2 --out FILE.json trains on one synthetic star
schema, evaluates on a held-out set of queries over a larger one and writes
the regret and speedup figures (and the weights beside them).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time
from pathlib import Path

import numpy as np

from . import abi, check, lib

NF = abi.MB_PLAN_FEATURES
NC = abi.MB_PLAN_CANDIDATES
CANDIDATE_NAMES = ["rule", "template-order", "tile-4", "tile-1", "materialise-most-selective",
                   "materialise-all-but-least", "materialised-plan", "scan", "grp-shared", "grp-global",
                   "grp-hash", "stage-tma", "tile-4+grp-global", "tile-1+grp-global", "template-order+tile-4",
                   "tile-4+grp-shared"]


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    """Handle of an mb_mlp (the network lives on the GPU)."""

    def __init__(self, nin: int = NF, hidden: int = 64, nout: int = NC, seed: int = 1, device: int = 0):
        self.nin, self.hidden, self.nout = nin, hidden, nout
        cfg = abi.mb_mlp_config(nin, hidden, nout, seed)
        self._m = C.c_void_p()
        check(lib().mb_mlp_create(device, C.byref(cfg), C.byref(self._m)))
        self.log: list[dict] = []

    @property
    def handle(self) -> C.c_void_p:
        return self._m

    def close(self) -> None:
        if self._m:
            lib().mb_mlp_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def nparams(self) -> int:
        return int(lib().mb_mlp_nparams(self._m))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.nparams(), np.float32)
        check(lib().mb_mlp_get_params(self._m, _f32p(p)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams()
        check(lib().mb_mlp_set_params(self._m, _f32p(p)))

    def forward(self, x: np.ndarray, bf16: bool = False) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.nin)
        y = np.zeros((x.shape[0], self.nout), np.float32)
        check(lib().mb_mlp_forward(self._m, _f32p(x), x.shape[0], 1 if bf16 else 0, _f32p(y)))
        return y

    def gradients(self, x, t, mask) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.nin)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, self.nout)
        m = np.ascontiguousarray(mask, np.float32).reshape(-1, self.nout)
        g = np.zeros(self.nparams(), np.float32)
        loss = C.c_float(0)
        check(lib().mb_mlp_gradients(self._m, _f32p(x), _f32p(t), _f32p(m), x.shape[0], _f32p(g),
                                     C.byref(loss)))
        return float(loss.value), g

    def train(self, x, t, mask, epochs: int = 100, batch: int = 256, lr: float = 2e-3,
              beta1: float = 0.9, beta2: float = 0.999, seed: int = 1) -> float:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.nin)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, self.nout)
        m = np.ascontiguousarray(mask, np.float32).reshape(-1, self.nout)
        o = abi.mb_mlp_train_opts(epochs, batch, lr, beta1, beta2, seed)
        loss = C.c_float(0)
        t0 = time.perf_counter()
        check(lib().mb_mlp_train(self._m, _f32p(x), _f32p(t), _f32p(m), x.shape[0], C.byref(o), C.byref(loss)))
        self.log.append({"rows": int(x.shape[0]), "epochs": epochs, "batch": batch, "lr": lr,
                         "final_loss": float(loss.value), "seconds": time.perf_counter() - t0})
        return float(loss.value)

    def save(self, path: str | Path) -> None:
        """Weights as raw little-endian float32 (the mb_mlp_get_params layout)
        at path, the shape and training log as JSON at path + '.json'."""
        path = Path(path)
        self.get_params().astype("<f4").tofile(path)
        names = BATCH_CANDIDATE_NAMES if self.nout == abi.MB_BATCH_CANDIDATES else CANDIDATE_NAMES
        path.with_name(path.name + ".json").write_text(json.dumps(
            {"in": self.nin, "hidden": self.hidden, "out": self.nout, "nparams": self.nparams(),
             "candidates": names, "log": self.log}, indent=1))

    @classmethod
    def load(cls, path: str | Path, device: int = 0) -> "MLP":
        path = Path(path)
        meta = json.loads(path.with_name(path.name + ".json").read_text())
        m = cls(meta["in"], meta["hidden"], meta["out"], device=device)
        m.set_params(np.fromfile(path, "<f4"))
        m.log = meta.get("log", [])
        return m


def query_features(eng, q: abi.mb_query) -> np.ndarray:
    f = np.zeros(NF, np.float32)
    check(lib().mb_engine_query_features(eng.handle, C.byref(q), _f32p(f)))
    return f


def features(eng, qs) -> np.ndarray:
    return np.stack([query_features(eng, q) for q in qs]) if len(qs) else np.zeros((0, NF), np.float32)


def candidate_plan(eng, q: abi.mb_query, idx: int) -> abi.mb_plan:
    p = abi.mb_plan()
    check(lib().mb_engine_plan_candidate(eng.handle, C.byref(q), idx, C.byref(p)))
    return p


def plan_learned(eng, qs, mlp: MLP | None) -> tuple[list[abi.mb_plan], np.ndarray]:
    """The engine's own learned planning (BF16 forward in the library):
    (plans, chosen candidate indices)."""
    n = len(qs)
    qarr = (abi.mb_query * max(n, 1))(*qs)
    plans = (abi.mb_plan * max(n, 1))()
    chosen = np.zeros(max(n, 1), np.uint32)
    check(lib().mb_engine_set_planner(eng.handle, mlp.handle if mlp is not None else None))
    try:
        check(lib().mb_engine_plan_learned(eng.handle, qarr, n, plans,
                                           chosen.ctypes.data_as(C.POINTER(C.c_uint32))))
    finally:
        check(lib().mb_engine_set_planner(eng.handle, None))
    return list(plans)[:n], chosen[:n].astype(np.int64)


def _run_timed(eng, qs, plans, out, nq) -> np.ndarray:
    """Device time (ms) of each query under its plan: one enqueue of the lot,
    CUDA events around each query's launch sequence."""
    n = len(qs)
    qarr = (abi.mb_query * n)(*qs)
    parr = (abi.mb_plan * n)(*plans)
    check(lib().mb_engine_enqueue(eng.handle, qarr, n, parr, out.data_ptr(), nq.data_ptr(), 1))
    t = np.zeros(n, np.float32)
    check(lib().mb_engine_sync(eng.handle, _f32p(t), n))
    return t


def measure_candidates(eng, qs, reps: int = 3, chunk: int = 512, cands=range(NC)) -> np.ndarray:
    """times[i, c] = median over reps of query i's device time (ms) under
    candidate c.  Candidates that lower to the same plan as an earlier one are
    timed once and share its figure (so identical plans never look different
    through timing noise)."""
    from . import device as D
    cands = list(cands)
    n = len(qs)
    plans = [[candidate_plan(eng, q, c) for c in cands] for q in qs]
    rep_of = np.zeros((n, len(cands)), np.int64)
    for i in range(n):
        seen: dict[bytes, int] = {}
        for j in range(len(cands)):
            rep_of[i, j] = seen.setdefault(bytes(plans[i][j]), j)
    ng = [max(1, eng.ngroups(q)) for q in qs]
    cap = max(sum(ng[s:s + chunk]) for s in range(0, n, chunk)) if n else 1
    out = D.empty(cap, 8)
    nq = D.empty(chunk, 8)
    samples = np.full((reps, n, len(cands)), np.nan, np.float64)
    for r in range(reps):
        order = cands[r % len(cands):] + cands[:r % len(cands)]  # rotate so no candidate always runs first
        for c in order:
            j = cands.index(c)
            idx = [i for i in range(n) if rep_of[i, j] == j]
            for s in range(0, len(idx), chunk):
                part = idx[s:s + chunk]
                t = _run_timed(eng, [qs[i] for i in part], [plans[i][j] for i in part], out, nq)
                samples[r, part, j] = t
    med = np.median(samples, axis=0)
    for i in range(n):
        med[i] = med[i, rep_of[i]]
    return med


def targets(times: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Network targets: log(time / the query's best time) per candidate, and
    the mask of measured candidates."""
    best = np.nanmin(times, axis=1, keepdims=True)
    ok = np.isfinite(times) & (times > 0)
    t = np.where(ok, np.log(np.where(ok, times, 1.0) / np.maximum(best, 1e-6)), 0.0)
    return t.astype(np.float32), ok.astype(np.float32)


def regret_report(times: np.ndarray, chosen: np.ndarray) -> dict:
    """Regret (chosen plan time / best measured plan time) and the speedup
    over the rule plan (candidate 0), from one table of measured times."""
    n = len(chosen)
    best = times.min(axis=1)
    t_ch = times[np.arange(n), chosen]
    t_rule = times[:, 0]
    reg = t_ch / best
    rreg = t_rule / best
    return {
        "queries": int(n),
        "regret_mean": float(reg.mean()), "regret_p50": float(np.median(reg)),
        "regret_p90": float(np.quantile(reg, 0.9)), "regret_max": float(reg.max()),
        "regret_total": float(t_ch.sum() / best.sum()),
        "rule_regret_mean": float(rreg.mean()), "rule_regret_total": float(t_rule.sum() / best.sum()),
        "speedup_vs_rule_total": float(t_rule.sum() / t_ch.sum()),
        "speedup_vs_rule_geomean": float(np.exp(np.mean(np.log(t_rule / t_ch)))),
        "chosen_hist": {CANDIDATE_NAMES[c]: int((chosen == c).sum()) for c in range(times.shape[1])
                        if (chosen == c).any()},
        "best_hist": {CANDIDATE_NAMES[c]: int((times.argmin(1) == c).sum()) for c in range(times.shape[1])
                      if (times.argmin(1) == c).any()},
    }


def _engine(seed: int, nrows: int):
    from .engine import Engine
    k = max(1, round(nrows / 6_000_000))
    e = Engine()
    e.gen_star(seed, k, nrows)
    e.build_index()
    return e, k


def _mix(seed: int, n: int, exclude=frozenset()):
    from .workload import as_tuple, random_query
    r = np.random.default_rng(seed)
    qs = []
    while len(qs) < n:
        q = random_query(r, None, float(r.choice([0.1, 0.3, 0.6])))
        if as_tuple(q) not in exclude:
            qs.append(q)
    return qs


def experiment(train_rows: int, train_queries: int, eval_rows: int, eval_queries: int, reps: int = 3,
               epochs: int = 150, seed: int = 2, qseed: int = 3, weights: str | None = None) -> dict:
    """Collect timings of every candidate on train_queries random queries over
    a train_rows schema, train the network on the GPU, then plan and time
    eval_queries held-out queries over an eval_rows schema."""
    from .workload import as_tuple
    rep: dict = {"train_rows": train_rows, "train_queries": train_queries, "eval_rows": eval_rows,
                 "eval_queries": eval_queries, "reps": reps, "seed": seed, "query_seed": qseed}
    t0 = time.perf_counter()
    eng, k = _engine(seed, train_rows)
    train_q = _mix(qseed, train_queries)
    X = features(eng, train_q)
    T = measure_candidates(eng, train_q, reps)
    rep["train_collect_s"] = time.perf_counter() - t0
    rep["train_k"] = k
    eng.close()
    tt, mk = targets(T)
    mlp = MLP(seed=seed)
    t1 = time.perf_counter()
    rep["train_loss"] = mlp.train(X, tt, mk, epochs=epochs, batch=256, lr=2e-3, seed=seed)
    rep["train_s"] = time.perf_counter() - t1
    y_tr = mlp.forward(X, bf16=True)
    rep["train_fit"] = regret_report(T, y_tr.argmin(1))
    if weights:
        mlp.save(weights)
    del eng
    eng, k2 = _engine(seed + 1, eval_rows)
    rep["eval_k"] = k2
    seen = {as_tuple(q) for q in train_q}
    eval_q = _mix(qseed + 1000, eval_queries, frozenset(seen))
    t2 = time.perf_counter()
    plans, chosen = plan_learned(eng, eval_q, mlp)
    rep["plan_ms_per_query"] = (time.perf_counter() - t2) * 1e3 / max(1, len(eval_q))
    TE = measure_candidates(eng, eval_q, reps)
    rep["eval"] = regret_report(TE, chosen)
    eng.close()
    mlp.close()
    return rep


# ------------------------------------------------------------ batch planner
# A batch plan: a launch shape of the batched scan and the cover all the
# batch's queries take (mb_engine_batch_candidate).  The network maps
# MB_BATCH_FEATURES features of a batch to the log time of each plan relative
# to the batch's best; its training data are device times of CUDA-graph
# replays of every plan on random batches, recorded by the engine.
NBF = abi.MB_BATCH_FEATURES
NBC = abi.MB_BATCH_CANDIDATES
BATCH_CANDIDATE_NAMES = [f"{cov}/V{v}w{w}" for cov in ("rule", "noedge") for v in (1, 2, 4) for w in (8, 12, 16)]


def batch_features(eng, qs) -> np.ndarray:
    qarr = (abi.mb_query * max(1, len(qs)))(*qs)
    f = np.zeros(NBF, np.float32)
    check(lib().mb_engine_batch_features(eng.handle, qarr, len(qs), f.ctypes.data))
    return f


def batch_candidate(idx: int) -> tuple[abi.mb_batch_opts, int]:
    o = abi.mb_batch_opts()
    cover = C.c_uint32(0)
    check(lib().mb_engine_batch_candidate(idx, C.byref(o), C.byref(cover)))
    return o, int(cover.value)


def _rule_plans(qs, cover: int = 0):
    ps = []
    for _ in qs:
        p = abi.mb_plan()
        p.kind = abi.PLAN_FUSED
        p.cover = cover
        ps.append(p)
    return ps


def time_batch(eng, qs, opts, cover: int = 0, reps: int = 3, want: np.ndarray | None = None) -> float:
    """Median device time (ms) of `reps` CUDA-graph replays of the batch
    under (opts, cover); with `want`, the results must equal it."""
    import torch
    L = lib()
    n = len(qs)
    qarr = (abi.mb_query * n)(*qs)
    parr = (abi.mb_plan * n)(*_rule_plans(qs, cover))
    tot = int(L.mb_queries_layout(qarr, n, None))
    out = torch.zeros(max(tot, 1), dtype=torch.int64, device="cuda")
    nq = torch.zeros(n, dtype=torch.int64, device="cuda")
    g = C.c_void_p()
    check(L.mb_batch_graph_create_plans(eng.handle, qarr, parr, n, C.byref(opts) if opts is not None else None,
                                        out.data_ptr(), nq.data_ptr(), C.byref(g)))
    ts = []
    try:
        for _ in range(reps):
            check(L.mb_engine_mark(eng.handle, 6))
            check(L.mb_batch_graph_launch(g))
            check(L.mb_engine_mark(eng.handle, 7))
            ms = C.c_float(0)
            check(L.mb_engine_marks_ms(eng.handle, 6, 7, C.byref(ms)))
            ts.append(ms.value)
    finally:
        check(L.mb_batch_graph_destroy(g))
    if want is not None and not np.array_equal(out.cpu().numpy()[:tot], want):
        raise AssertionError("a batch plan changed the results")
    return float(np.median(ts))


def batch_results(eng, qs) -> np.ndarray:
    out, _ = eng.query_batch(qs, abi.mb_batch_opts())
    return out


def measure_batch_candidates(eng, batches, reps: int = 3, check_results: bool = True) -> np.ndarray:
    """times[b, c]: device time (ms) of batch b under batch plan c."""
    T = np.zeros((len(batches), NBC), np.float64)
    for b, qs in enumerate(batches):
        want = batch_results(eng, qs) if check_results else None
        for c in range(NBC):
            o, cover = batch_candidate(c)
            T[b, c] = time_batch(eng, qs, o, cover, reps, want)
    return T


def random_batches(seed: int, count: int, sizes=(2, 4, 8, 16, 24, 32, 48, 64, 96, 128)):
    """Batches of seeded template queries: selectivity-spanning mixes of
    varied size and spread, and level-based mixes."""
    from .workload import random_mix, span_mix
    r = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(r.choice(sizes))
        if r.random() < 0.7:
            lo = float(10 ** r.uniform(-6.5, -3))
            hi = float(10 ** r.uniform(np.log10(lo) + 1, np.log10(0.5)))
            out.append(span_mix(int(r.integers(1 << 30)), n, lo, hi, tries=400))
        else:
            out.append(random_mix(int(r.integers(1 << 30)), n, float(r.choice([0.1, 0.3, 0.6]))))
    return out


def plan_batches_learned(eng, batches, mlp: "MLP | None") -> np.ndarray:
    """The engine's learned choice (candidate index) for each batch."""
    L = lib()
    check(L.mb_engine_set_batch_planner(eng.handle, mlp.handle if mlp is not None else None))
    ch = np.zeros(len(batches), np.int64)
    try:
        for b, qs in enumerate(batches):
            qarr = (abi.mb_query * len(qs))(*qs)
            o = abi.mb_batch_opts()
            cover, choice = C.c_uint32(0), C.c_uint32(0)
            check(L.mb_engine_plan_batch(eng.handle, qarr, len(qs), C.byref(o), C.byref(cover), C.byref(choice)))
            ch[b] = choice.value
    finally:
        check(L.mb_engine_set_batch_planner(eng.handle, None))
    return ch


def batch_regret_report(T: np.ndarray, chosen: np.ndarray, t_rule: np.ndarray) -> dict:
    """Regret of the chosen batch plans (time / best measured plan) and their
    speedup over the rule-planned batch (rule covers, the engine's default
    launch shape)."""
    n = len(chosen)
    best = T.min(axis=1)
    t_ch = T[np.arange(n), chosen]
    reg = t_ch / best
    return {"batches": int(n), "regret_mean": float(reg.mean()), "regret_p90": float(np.quantile(reg, 0.9)),
            "regret_max": float(reg.max()), "regret_total": float(t_ch.sum() / best.sum()),
            "rule_regret_total": float(t_rule.sum() / best.sum()),
            "speedup_vs_rule_total": float(t_rule.sum() / t_ch.sum()),
            "speedup_vs_rule_geomean": float(np.exp(np.mean(np.log(t_rule / t_ch)))),
            "chosen_hist": {BATCH_CANDIDATE_NAMES[c]: int((chosen == c).sum()) for c in range(NBC) if (chosen == c).any()}}


def batch_experiment(train_rows: int, train_batches: int, eval_rows: int, eval_batches: int, reps: int = 3,
                     epochs: int = 300, seed: int = 2, bseed: int = 7, weights: str | None = None) -> dict:
    """Train the batch planner on engine-timed random batches over a
    train_rows table; plan and time held-out batches over an eval_rows one."""
    rep: dict = {"train_rows": train_rows, "train_batches": train_batches, "eval_rows": eval_rows,
                 "eval_batches": eval_batches, "reps": reps, "seed": seed, "batch_seed": bseed}
    t0 = time.perf_counter()
    eng, _ = _engine(seed, train_rows)
    tb = random_batches(bseed, train_batches)
    X = np.stack([batch_features(eng, b) for b in tb])
    T = measure_batch_candidates(eng, tb, reps)
    rep["train_collect_s"] = time.perf_counter() - t0
    eng.close()
    tt, mk = targets(T)
    mlp = MLP(NBF, 64, NBC, seed=seed)
    t1 = time.perf_counter()
    rep["train_loss"] = mlp.train(X, tt, mk, epochs=epochs, batch=64, lr=2e-3, seed=seed)
    rep["train_s"] = time.perf_counter() - t1
    y = mlp.forward(X, bf16=True)
    rep["train_fit_regret_total"] = float(T[np.arange(len(tb)), y.argmin(1)].sum() / T.min(1).sum())
    if weights:
        mlp.save(weights)
    eng, _ = _engine(seed + 1, eval_rows)
    eb = random_batches(bseed + 1000, eval_batches)
    chosen = plan_batches_learned(eng, eb, mlp)
    TE = measure_batch_candidates(eng, eb, reps)
    t_rule = np.array([time_batch(eng, b, abi.mb_batch_opts(), 0, reps) for b in eb])
    rep["eval"] = batch_regret_report(TE, chosen, t_rule)
    eng.close()
    mlp.close()
    return rep


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--train-rows", type=int, default=120_000_000)
    ap.add_argument("--train-queries", type=int, default=20_000)
    ap.add_argument("--eval-rows", type=int, default=600_000_000)
    ap.add_argument("--eval-queries", type=int, default=2_000)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--out", type=str, default="")
    ap.add_argument("--weights", type=str, default="")
    ap.add_argument("--batch", action="store_true", help="the batch planner: --train-queries / --eval-queries "
                                                          "count batches")
    a = ap.parse_args(argv)
    if a.batch:
        rep = batch_experiment(a.train_rows, a.train_queries, a.eval_rows, a.eval_queries, a.reps, a.epochs,
                               weights=a.weights or None)
    else:
        rep = experiment(a.train_rows, a.train_queries, a.eval_rows, a.eval_queries, a.reps, a.epochs,
                         weights=a.weights or None)
    s = json.dumps(rep, indent=1)
    print(s)
    if a.out:
        Path(a.out).write_text(s)


if __name__ == "__main__":
    main()
