#!/usr/bin/env python
"""bench.py - fact rows/s of the fused bitmap-index query path on B200.

Workload (one GPU): the synthetic star schema at k=20 (120,000,000 fact rows,
every fact column 4 bytes), its canonical 242-bitmap index resident in HBM,
and a seeded 64-query mix of the four templates (s1op..s4op of the
reference).  One step runs the 64 queries; fact rows/s = rows x queries /
device time.  With N GPUs every rank holds its own 120M-row shard of an
N x 120M-row table (weak scaling) and each step ends with one NCCL all-reduce
of the int64 group tables (the only exchange step of a sharded query).

  value     device-resident: one step = the 64 queries in one batched
            launch (mb_engine_enqueue_batch), results in HBM, CUDA events on
            the engine stream around the timed steps; "plain" beside it times
            the same queries one fused launch each
  e2e       through the public C ABI (mb_engine_query_batch): query
            descriptors from host memory, int64 results read back to host
            every step, host wall clock
  roofline  the batch kernel: algorithmic bytes (each distinct canonical
            bitmap once + the union of the 32-byte payload sectors holding a
            selected row + outputs, computed by the oracle on a host row
            sample) / the event-timed step
  cpu_baseline  the reference's own CPU oracle (ssb/cpuref.c s1ref..s4ref,
            built from its sources into oracle/_ref) on a 24M-row sample, one
            query per thread over all host cores (the ssb_cpujoin shape)

`--impl reference` times that reference CPU path alone (rank 0 only).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fact rows/s + %HBM roofline, learned+batched vs plain plan; p50/p99 latency"
UNIT = "fact rows/s"
SEED_DATA, SEED_QUERIES = 2, 3
CPU_SAMPLE_ROWS = 24_000_000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--k", type=int, default=20)
    ap.add_argument("--rows", type=int, default=0, help="rows per GPU (default 6M x k)")
    ap.add_argument("--queries", type=int, default=64)
    ap.add_argument("--narrow", type=float, default=0.3)
    ap.add_argument("--width4", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default launch shape instead of the autotuner's")
    ap.add_argument("--no-graph", action="store_true", help="enqueue each step instead of replaying a CUDA graph")
    ap.add_argument("--wah", action="store_true",
                    help="instead of the headline: the WAH baseline (compress two predicate bitmaps, AND the "
                         "streams) on the GPU beside the reference's CPU WAH code")
    return ap.parse_args()


# --------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.proc, self.f = gpu, None, None

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for ln in Path(self.f.name).read_text().splitlines():
                x = [v.strip() for v in ln.split(",")]
                if len(x) >= 9 and x[0] == str(self.gpu):
                    rows.append(x)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ------------------------------------------------------- reference (CPU)
def cpu_sample(k: int, nrows: int):
    from oracle import oracle as O
    return O.StarHost(SEED_DATA, k, nrows)


def run_cpuref(ref, schema, n, qs, threads) -> float:
    """One pass of the query mix through the reference's s1ref..s4ref, one
    query per thread (ssb_cpujoin's shape, ssb/cpuref.c:244-302).  Seconds."""
    import merle_b200
    from merle_b200 import workload as WL

    def one(q):
        t, p = WL.as_tuple(q)
        ng = int(max(1, merle_b200.lib().mb_query_ngroups(C.byref(q))))
        out = np.zeros(ng + 1, np.uint32)
        if t == 1:
            ref.s1ref(C.byref(schema), n, *p)
        elif t == 2:
            ref.s2ref(C.byref(schema), n, *p, out.ctypes.data)
        elif t == 3:
            ref.s3ref(C.byref(schema), n, *p, out.ctypes.data)
        else:
            ref.s4ref(C.byref(schema), n, *p, out.ctypes.data)
        return out
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, qs))
    return time.perf_counter() - t0


def cpu_baseline(args, qs, steps: int = 1) -> dict:
    from oracle import oracle as O
    ref = O.ref()
    if ref is None:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    n = min(CPU_SAMPLE_ROWS, args.rows or 6_000_000 * args.k)
    star = cpu_sample(args.k, n)
    schema = star.ssb_schema()
    threads = os.cpu_count() or 1
    run_cpuref(ref, schema, n, qs[:4], threads)  # warm the pages
    ts = [run_cpuref(ref, schema, n, qs, threads) for _ in range(steps)]
    sec = float(np.median(ts))
    return {"value": n * len(qs) / sec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"the {len(qs)}-query mix over the first {n:,} rows of the k={args.k} table in ssb_schema "
                      f"widths, reference s1ref..s4ref, one query per thread on {threads} threads",
            "seconds_per_pass": sec}


def reference_arm(args):
    from merle_b200 import workload as WL
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    qs = WL.random_mix(SEED_QUERIES, args.queries, args.narrow)
    from oracle import oracle as O
    ref = O.ref()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's cpuref.c built from "
                          "its sources) is missing"}))
        return
    n = min(CPU_SAMPLE_ROWS, args.rows or 6_000_000 * args.k)
    star = cpu_sample(args.k, n)
    schema = star.ssb_schema()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        run_cpuref(ref, schema, n, qs, threads)
    ts = [run_cpuref(ref, schema, n, qs, threads) for _ in range(args.steps)]
    tot = sum(ts)
    v = n * len(qs) * args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config_of(args, args.rows or 6_000_000 * args.k),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{len(qs)}-query mix over the first {n:,} rows (ssb_schema widths), "
                                       f"one query per thread"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def config_of(args, nrows_per_gpu):
    return {"workload": f"star schema k={args.k}, {nrows_per_gpu:,} fact rows per GPU "
                        f"({'4-byte' if args.width4 else 'ssb_schema-width'} fact columns), 242-bitmap index, "
                        f"{args.queries}-query seeded mix of 4 templates",
            "rows_per_gpu": nrows_per_gpu, "queries_per_step": args.queries, "k": args.k,
            "l2": "inputs larger than L2 (each step reads several GB of bitmaps and payload)",
            "parallelism": f"row shards x{args.gpus}"}


# ------------------------------------------------------------- ours
# payload columns (width in bytes) a query's selected rows read, with the
# engine's denormalised customer city / part mfgr columns
BATCH_GATHER = {1: [("extendedprice", 4), ("discount", 4)],
                2: [("partmfgr_row", 2), ("orderdate", 4), ("revenue", 4)],
                3: [("custcity_row", 1), ("suppcity", 4), ("orderdate", 4), ("revenue", 4)],
                4: [("suppcity", 4), ("orderdate", 4), ("partmfgr_row", 2), ("revenue", 4), ("supplycost", 4)]}
# bytes of the batch descriptor block the engine copies to the device per
# launch (BatchHdr: 256-byte head with the 48 staging copies, 16 sources,
# 128 x 64-word query descriptors, 4096 chain entries, 128 order bytes)
BATCH_HDR_BYTES = 256 + 16 * 24 + 128 * 64 * 4 + 4096 * 2 + 128


def batch_algo_bytes(star, scale: float, nrows: int, qs, ngroups) -> dict:
    """Algorithmic bytes of one batched pass: every DISTINCT canonical bitmap
    once, the union over the queries of the 32-byte payload sectors holding a
    selected row (counted on the host sample, scaled), the int64 outputs."""
    from oracle import oracle as O
    from merle_b200 import workload as WL
    W = (nrows + 31) // 32
    bins = set()
    sectors = {}
    rows = 0
    for q in qs:
        t, p = WL.as_tuple(q)
        bins |= O.canonical_bins(t, p)
        r = np.flatnonzero(O.qualifying_mask(star, t, p))
        rows += len(r)
        for col, w in BATCH_GATHER[t]:
            sectors.setdefault((col, w), []).append(r // (32 // w))
    sec = sum(len(np.unique(np.concatenate(v))) for v in sectors.values()) * 32
    bm = len(bins) * W * 4
    out = 8 * sum(ngroups)
    return {"bitmap": bm, "distinct_bitmaps": len(bins), "gather": int(sec * scale), "out": out,
            "total": int(bm + sec * scale + out), "rows": int(rows * scale)}


def wah_arm(args):
    """One JSON line: SSB Q1.1's date and discount predicate bitmaps over the
    table (the reference's WAH baseline, ssb/wah-demo.cu:22-76) compressed and
    ANDed as WAH streams, per step; the reference's own CPU code for the same
    steps (wahCmprsCPU in place, wahAndCPU; merle/host/) timed on a bounded
    sample of the rows beside it.  Rows/s of both."""
    import torch
    from merle_b200 import abi, device as D, wah as W
    from oracle import oracle as O
    n = args.rows or 6_000_000 * args.k
    star = D.DevStar(SEED_DATA, args.k, n)
    bms = [D.bitmap_create(D.src_of(star[c]), n, [lo], [hi])[0][0]
           for c, lo, hi in (("orderdate", 366, 731), ("discount", 1, 4))]
    G = W.wah_groups(n)

    def step():
        a, b = (W.wah_compress(x, n, abi.WAH_MSB) for x in bms)
        return W.wah_and(a, b, G)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        r = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    # the reference on the host: the groups of the first sample rows (MSB
    # order, as dbjoinFlatWah builds them), compressed in place and ANDed
    cpu = None
    wref = O.wah_ref()
    if wref is not None:
        sample = min(n, 310_000_000) // 31 * 31
        words = (sample + 31) // 32
        groups = []
        for bm in bms:
            bits = np.unpackbits(D.to_host(bm[:words], np.uint32).view(np.uint8), bitorder="little")[:sample]
            g = np.packbits(bits.reshape(-1, 31), axis=1, bitorder="big")
            g = (g.astype(np.uint32) @ np.array([1 << 24, 1 << 16, 1 << 8, 1], np.uint32)) >> 1
            groups.append(np.ascontiguousarray(g.astype(np.uint32)))
        t0 = time.perf_counter()
        bufs, ns = [], []
        for g in groups:
            buf = g.copy()
            ns.append(wref.wahCmprsCPU(O.ptr(buf), len(buf), O.ptr(buf)))
            bufs.append(np.concatenate([buf[:ns[-1]], np.zeros(2, np.uint32)]))
        out = np.zeros(ns[0] + ns[1] + 4, np.uint32)
        wref.wahAndCPU(O.ptr(bufs[0]), O.ptr(bufs[0]) + 4 * ns[0], O.ptr(bufs[1]), O.ptr(bufs[1]) + 4 * ns[1],
                       O.ptr(out), O.ptr(out) + 4 * len(out))
        sec = time.perf_counter() - t0
        cpu = {"value": sample / sec, "unit": "rows/s", "cores": 1, "kind": "reference",
               "sample": f"the first {sample:,} rows: wahCmprsCPU of both predicates' 31-bit groups, wahAndCPU"}
    print(json.dumps({"metric": "WAH baseline: compress two predicate bitmaps and AND the streams", "value": n / ms * 1e3,
                      "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup),
                      "ms_per_step": ms, "higher_is_better": True, "dtype": "u32", "data": "synthetic",
                      "config": {"workload": f"star schema k={args.k}, {n:,} rows; SSB Q1.1 date and discount "
                                             "predicates", "stream_words": int(r.numel())},
                      "cpu_baseline": cpu}))


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.wah:
        wah_arm(args)
        return
    import torch
    import torch.distributed as dist

    import merle_b200
    from merle_b200 import abi, check, shard, workload as WL
    from merle_b200.engine import Engine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    L = merle_b200.lib()
    n = args.rows or 6_000_000 * args.k
    eng = Engine(local)
    row0, n = shard.row_range(rank, n)
    eng.gen_star(SEED_DATA, args.k, n, width4=bool(args.width4), row0=row0)
    eng.build_index()
    info = eng.info()
    qs = WL.random_mix(SEED_QUERIES, args.queries, args.narrow)
    Q = len(qs)
    qarr = (abi.mb_query * Q)(*qs)
    ngroups = [Engine.ngroups(q) for q in qs]
    total_g = int(L.mb_queries_layout(qarr, Q, None))
    out = torch.zeros(total_g, dtype=torch.int64, device="cuda")
    nq = torch.zeros(Q, dtype=torch.int64, device="cuda")
    ext = torch.cuda.ExternalStream(int(L.mb_engine_stream(eng.handle) or 0))

    def allreduce():
        if world > 1:
            with torch.cuda.stream(ext):
                shard.combine(out, nq)

    # the launch shape from the autotuner (timed on this mix, before the
    # measured steps), and the batch captured once as a CUDA graph
    bopts = abi.mb_batch_opts()
    tune = {"tuned": False}
    if not args.no_tune:
        tms, tried = C.c_float(0), C.c_uint32(0)
        t0 = time.perf_counter()
        check(L.mb_engine_tune_batch(eng.handle, qarr, Q, 3, C.byref(bopts), C.byref(tms), C.byref(tried)))
        tune = {"tuned": True, "shapes_timed": tried.value, "best_ms": tms.value, "tune_s": time.perf_counter() - t0,
                "opts": {f: getattr(bopts, f) for f, _ in bopts._fields_ if f != "pad_"}}
    graph = C.c_void_p()
    if not args.no_graph:
        check(L.mb_batch_graph_create(eng.handle, qarr, Q, C.byref(bopts), out.data_ptr(), nq.data_ptr(),
                                      C.byref(graph)))

    def step_batch():
        if graph:
            check(L.mb_batch_graph_launch(graph))
        else:
            check(L.mb_engine_enqueue_batch(eng.handle, qarr, Q, C.byref(bopts), out.data_ptr(), nq.data_ptr()))
        allreduce()

    def step_plain(record=False):
        check(L.mb_engine_enqueue(eng.handle, qarr, Q, None, out.data_ptr(), nq.data_ptr(), 1 if record else 0))
        allreduce()

    def timed(step, steps, mark0, mark1):
        check(L.mb_engine_mark(eng.handle, mark0))
        for _ in range(steps):
            step()
        check(L.mb_engine_mark(eng.handle, mark1))
        ms = C.c_float(0)
        check(L.mb_engine_marks_ms(eng.handle, mark0, mark1, C.byref(ms)))
        v = float(ms.value)
        if world > 1:
            t = torch.tensor([v], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            v = float(t.item())
        return v

    rows_total = n * world
    # ---- the batched path: warm-up, then K timed steps (one launch each)
    for _ in range(args.warmup):
        step_batch()
    check(L.mb_engine_sync(eng.handle, None, 0))
    batch_out = out.clone()
    if world > 1:
        dist.barrier()
    with Clocks(local) as clk:
        ms_total = timed(step_batch, args.steps, 0, 1)
    torch.cuda.synchronize()
    value = rows_total * Q * args.steps / (ms_total / 1e3)

    # ---- the plain path (one launch sequence per query), for comparison
    for _ in range(args.warmup):
        step_plain()
    check(L.mb_engine_sync(eng.handle, None, 0))
    same = bool(torch.equal(out, batch_out))
    if world > 1:
        dist.barrier()
    plain_ms = timed(step_plain, args.steps, 2, 3)
    step_plain(record=True)
    tbuf = (C.c_float * Q)()
    check(L.mb_engine_sync(eng.handle, tbuf, Q))
    qtimes = np.array(tbuf[:], np.float64)

    # ---- e2e through the public API with host buffers: mb_engine_query_batch
    res_host = np.zeros(total_g, np.int64)
    nq_host = np.zeros(Q, np.uint64)
    check(L.mb_engine_query_batch(eng.handle, qarr, Q, C.byref(bopts), res_host.ctypes.data, nq_host.ctypes.data))
    if world > 1:
        dist.barrier()
    lat = []
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        t1 = time.perf_counter()
        check(L.mb_engine_mark(eng.handle, 4))
        check(L.mb_engine_query_batch(eng.handle, qarr, Q, C.byref(bopts), res_host.ctypes.data,
                                      nq_host.ctypes.data))
        check(L.mb_engine_mark(eng.handle, 5))
        lat.append((time.perf_counter() - t1) * 1e3)
    e2e_wall = time.perf_counter() - t0
    e2e_ms = float(e2e_wall * 1e3)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": rows_total * Q * args.e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": C.sizeof(abi.mb_query) * Q + BATCH_HDR_BYTES,
           "d2h_bytes_per_step": 8 * total_g + 8 * Q,
           "api": "mb_engine_query_batch (host query descriptors in, host int64 group sums and row counts out, "
                  "returns when they are on the host)",
           "timing": "host wall clock around each call", "ms_per_step": e2e_ms / args.e2e_steps}

    line = None
    if rank == 0:
        from oracle import oracle as O
        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = json.loads(pk.read_text())
        peak = float(peaks.get("hbm_gbs", 6650.0))
        sample_n = min(CPU_SAMPLE_ROWS, n)
        star = cpu_sample(args.k, sample_n)
        ab = batch_algo_bytes(star, n / sample_n, n, qs, ngroups)
        step_s = ms_total / args.steps / 1e3
        achieved = ab["total"] / step_s / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy), of measured" if peaks
                               else "fallback 6.65 TB/s",
                "kernel": "batch_scan_kernel (one launch per 64-query step)",
                "algo_bytes_per_launch": ab["total"], "algo_bytes_detail": ab,
                "launch_ms_avg": ms_total / args.steps,
                "traffic": None, "traffic_note": "per-launch DRAM bytes in profiles/ (ncu)"}
        tj = ROOT / "profiles" / "traffic.json"
        if tj.exists():
            t = json.loads(tj.read_text()).get("batch_scan_kernel")
            if t:
                roof["traffic"] = t["dram_bytes_per_row"] * n
                roof["traffic_note"] = "ncu capture of a 24M-row launch scaled to this launch's rows: " + t["source"]
        widths = {c: (4 if args.width4 else {"orderdate": 2, "discount": 1, "quantity": 1, "suppcity": 1}.get(c, 4))
                  for c in ["extendedprice", "discount", "partkey", "orderdate", "revenue", "custkey", "suppcity",
                            "supplycost", "quantity"]}
        plain_algo = sum(O.algo_bytes(star, n / sample_n, n, *WL.as_tuple(q), Engine.ngroups(q), widths)["total"]
                         for q in qs)
        cpu = None if args.no_cpu or world > 1 else cpu_baseline(args, qs)
        lat_a = np.array(lat)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": config_of(args, n), "impl": "ours",
                "plan": "batched: the whole mix in one persistent launch per step (rule-planner covers)"
                        + ("; replayed as a CUDA graph" if graph else ""),
                "batch_shape": tune,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "plain": {"value": rows_total * Q * args.steps / (plain_ms / 1e3), "ms_per_step": plain_ms / args.steps,
                          "batched_speedup": plain_ms / ms_total, "results_identical": same,
                          "roofline_frac": plain_algo / (qtimes.sum() / 1e3) / 1e9 / peak,
                          "plan": "one fused launch per query (rule planner)"},
                "latency_ms": {"batch_e2e_p50": float(np.percentile(lat_a, 50)),
                               "batch_e2e_p99": float(np.percentile(lat_a, 99)),
                               "plain_kernel_p50": float(np.percentile(qtimes, 50)),
                               "plain_kernel_p99": float(np.percentile(qtimes, 99))},
                "gpu_launches": args.steps,
                "clocks": clk.summary(),
                "index": {"bitmaps": info["nbitmaps"], "bytes": info["index_bytes"],
                          "build_ms": info["index_build_ms"], "denorm_bytes": info["denorm_bytes"]},
                "selected_rows_per_step": ab["rows"]}
        print(json.dumps(line))
    if graph:
        check(L.mb_batch_graph_destroy(graph))
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
