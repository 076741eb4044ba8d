"""Serving loop binding (mb_server_*) and its load test.

The server itself - dispatcher thread, admission by group-table and
intermediate-bitmap bytes, continuous batching into batched-scan launches,
Poisson arrivals, latency records - is native code in libmerleb200.so; this
module wraps it and turns the per-request records into q/s, p50 and p99.

Command line: python -m merle_b200.serving --rows N --rates R1,R2,... runs
the same seeded Poisson stream of mixed-template queries through the batched
server and through the plain one-query-per-launch server at each rate, and
prints one JSON record per (mode, rate).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import abi, check, lib


class Server:
    def __init__(self, eng, mode: int = abi.SERVE_BATCHED, mem_budget: int = 0, max_batch: int = 0,
                 max_inflight: int = 0, use_planner: bool = False, batch: abi.mb_batch_opts | None = None,
                 min_batch: int = 0):
        o = abi.mb_server_opts()
        o.mem_budget, o.mode, o.max_batch, o.max_inflight = mem_budget, mode, max_batch, max_inflight
        o.min_batch = min_batch
        o.use_planner = 1 if use_planner else 0
        if batch is not None:
            o.batch = batch
        self.eng = eng
        self._s = C.c_void_p()
        check(lib().mb_server_create(eng.handle, C.byref(o), C.byref(self._s)))

    def close(self) -> None:
        if self._s:
            lib().mb_server_destroy(self._s)
            self._s = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, q: abi.mb_query, out: np.ndarray) -> int:
        """Queues q; `out` (int64, mb_query_ngroups(q) values, kept alive by
        the caller until the request is waited for) receives the sums."""
        assert out.dtype == np.int64 and out.flags.c_contiguous
        rid = C.c_uint64(0)
        check(lib().mb_server_submit(self._s, C.byref(q), out.ctypes.data, C.byref(rid)))
        return rid.value

    def cancel(self, rid: int) -> bool:
        """True if the request was still queued and is now cancelled."""
        return lib().mb_server_cancel(self._s, rid) == abi.MB_OK

    def wait(self, rid: int, timeout_ms: int = -1) -> abi.mb_request_info:
        info = abi.mb_request_info()
        check(lib().mb_server_wait(self._s, rid, timeout_ms, C.byref(info)))
        return info

    def stats(self) -> dict:
        s = abi.mb_server_stats()
        check(lib().mb_server_get_stats(self._s, C.byref(s)))
        return {f: getattr(s, f) for f, _ in s._fields_}

    def inject(self, fault: int, count: int = 1, arg_us: int = 0) -> None:
        check(lib().mb_server_inject(self._s, fault, count, arg_us))

    def run_load(self, qs, rate_qps: float, seed: int = 1):
        """Open-loop Poisson load: (results in mb_queries_layout order,
        per-request records)."""
        n = len(qs)
        qarr = (abi.mb_query * max(n, 1))(*qs)
        total = int(lib().mb_queries_layout(qarr, n, None))
        out = np.zeros(max(total, 1), np.int64)
        info = (abi.mb_request_info * max(n, 1))()
        check(lib().mb_server_run_load(self._s, qarr, n, float(rate_qps), seed, out.ctypes.data, info))
        return out[:total], list(info)[:n]


def poisson_arrivals(seed: int, rate_qps: float, n: int) -> np.ndarray:
    t = np.zeros(max(n, 1), np.float64)
    check(lib().mb_poisson_arrivals(seed, float(rate_qps), n, t.ctypes.data))
    return t[:n]


def summarize(info, offered_qps: float | None = None) -> dict:
    """q/s over the run, latency percentiles (ms), batch sizes, statuses."""
    ok = [i for i in info if i.status == abi.MB_OK]
    lat = np.array([(i.t_done_us - i.t_submit_us) / 1e3 for i in ok]) if ok else np.zeros(1)
    qwait = np.array([(i.t_launch_us - i.t_submit_us) / 1e3 for i in ok]) if ok else np.zeros(1)
    t0 = min(i.t_submit_us for i in info) if info else 0.0
    t1 = max(i.t_done_us for i in info) if info else 1.0
    span_s = max(t1 - t0, 1.0) / 1e6
    bs = np.array([i.batch_size for i in ok]) if ok else np.zeros(1)
    return {
        "offered_qps": offered_qps, "requests": len(info), "ok": len(ok),
        "qps": len(ok) / span_s,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
        "queue_p50_ms": float(np.percentile(qwait, 50)), "queue_p99_ms": float(np.percentile(qwait, 99)),
        "mean_batch": float(bs.mean()), "launches": len({i.launch for i in ok}),
        "statuses": {abi.STATUS_NAMES[s]: int(sum(1 for i in info if i.status == s))
                     for s in sorted({i.status for i in info})},
    }


def sweep(eng, qs, rates, modes=("batched", "plain"), seed: int = 5, mem_budget: int = 0,
          max_batch: int = 0, max_inflight: int = 0, batch: abi.mb_batch_opts | None = None,
          use_planner: bool = False) -> list[dict]:
    """The same arrival stream through each server mode at each rate."""
    recs = []
    for mode in modes:
        m = abi.SERVE_BATCHED if mode == "batched" else abi.SERVE_PLAIN
        for rate in rates:
            with Server(eng, m, mem_budget=mem_budget, max_batch=max_batch, max_inflight=max_inflight,
                        batch=batch, use_planner=use_planner and mode == "batched") as s:
                s.run_load(qs[:min(len(qs), 32)], rate, seed + 1)  # warm-up (untimed)
                t = time.perf_counter()
                out, info = s.run_load(qs, rate, seed)
                wall = time.perf_counter() - t
                rec = {"mode": mode, **summarize(info, rate), "wall_s": wall, "server": s.stats()}
            recs.append(rec)
    return recs


def main(argv=None) -> None:
    from .engine import Engine
    from .workload import random_mix
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--rows", type=int, default=120_000_000)
    ap.add_argument("--queries", type=int, default=4000)
    ap.add_argument("--rates", type=str, default="2000,8000,16000")
    ap.add_argument("--modes", type=str, default="batched,plain")
    ap.add_argument("--budget-mb", type=int, default=0)
    ap.add_argument("--max-batch", type=int, default=0)
    ap.add_argument("--max-inflight", type=int, default=0)
    ap.add_argument("--width4", type=int, default=1, help="4-byte fact columns (0: ssb_schema widths)")
    ap.add_argument("--planner", type=str, default="",
                    help="weights of a trained planner network (merle_b200.planner): the batched server's "
                         "plain-path launches use its plans")
    ap.add_argument("--tune", type=int, default=1, help="autotune the batched scan's shape on a 64-query sample")
    ap.add_argument("--out", type=str, default="")
    a = ap.parse_args(argv)
    k = max(1, round(a.rows / 6_000_000))
    e = Engine()
    t0 = time.perf_counter()
    e.gen_star(2, k, a.rows, width4=bool(a.width4))
    e.build_index()
    info = e.info()
    setup_s = time.perf_counter() - t0
    qs = random_mix(3, a.queries, narrow=0.3)
    bopts, tune = None, None
    if a.tune:
        bopts = abi.mb_batch_opts()
        ms, tried = C.c_float(0), C.c_uint32(0)
        sample = (abi.mb_query * 64)(*qs[:64])
        check(lib().mb_engine_tune_batch(e.handle, sample, min(64, len(qs)), 3, C.byref(bopts), C.byref(ms),
                                         C.byref(tried)))
        tune = {"opts": {f: getattr(bopts, f) for f, _ in bopts._fields_ if f != "pad_"}, "best_ms": ms.value}
    mlp = None
    if a.planner:
        from .planner import MLP
        mlp = MLP.load(a.planner)
        check(lib().mb_engine_set_planner(e.handle, mlp.handle))
    recs = sweep(e, qs, [float(r) for r in a.rates.split(",")], tuple(a.modes.split(",")),
                 mem_budget=a.budget_mb << 20, max_batch=a.max_batch, max_inflight=a.max_inflight, batch=bopts,
                 use_planner=mlp is not None)
    if mlp is not None:
        check(lib().mb_engine_set_planner(e.handle, None))
        mlp.close()
    head = {"rows": a.rows, "k": k, "width4": a.width4, "queries": a.queries, "setup_s": setup_s,
            "resident_bytes": info["fact_bytes"] + info["dim_bytes"] + info["index_bytes"] + info["denorm_bytes"],
            "index_build_ms": info["index_build_ms"], "batch_tune": tune, "planner": a.planner or None}
    lines = [json.dumps({**head, **r}) for r in recs]
    for ln in lines:
        print(ln, flush=True)
    if a.out:
        with open(a.out, "w") as f:
            f.write("\n".join(lines) + "\n")
    e.close()


if __name__ == "__main__":
    main()
