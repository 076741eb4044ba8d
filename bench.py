#!/usr/bin/env python
"""bench.py - fact rows/s of the fused bitmap-index query path on B200.

Workload (one GPU): the synthetic star schema at k=100 (600,000,000 fact
rows, every fact column 4 bytes), its canonical 242-bitmap index resident in
HBM, and a seeded 64-query mix of the four templates (s1op..s4op of the
reference) whose selectivities are spread log-uniformly over [1e-6, 0.5]
(workload.span_mix).  One step answers the 64 queries; fact rows/s = rows x
queries / device time.  With N GPUs every rank holds its own row shard of an
N x 600M-row table (weak scaling) and each step ends with one NCCL all-reduce
of the int64 group tables (the only exchange step of a sharded query).

  value     device-resident: one step = the 64 queries in one batched
            launch, results in HBM, CUDA events on the engine stream around
            the timed steps; "plain" beside it times the same queries one
            fused launch each
  e2e       through the public C ABI (mb_engine_query_batch): query
            descriptors from host memory, int64 results read back to host
            every step, host wall clock
  roofline  the batch kernel: algorithmic bytes (each distinct canonical
            bitmap once + the union of the 32-byte payload sectors holding a
            selected row + outputs, computed by the oracle on a host row
            sample) / the event-timed step
  parity    every query's answer against the reference's own s1ref..s4ref
            (ssb/cpuref.c, built from its sources into oracle/_ref) over the
            whole table on the host: uint32 group arrays equal (uint32) of the
            int64 sums, s1ref's uint64 sum equal; row counts give the realised
            selectivities
  cpu_baseline  that same pass of s1ref..s4ref, timed: one query per thread
            over all host cores (the ssb_cpujoin shape)
  latency_ms  the serving loop (mb_server_*) under seeded Poisson arrivals at
            two rates, below and above the plain server's capacity, batched
            and plain servers: q/s, p50, p99 over every request

`--impl reference` times the reference CPU path alone (rank 0 only) on a
bounded row sample.
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
BATCH_WEIGHTS = ROOT / "merle_b200" / "weights" / "batch_planner.f32"
PEAK_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--k", type=int, default=100)
    ap.add_argument("--rows", type=int, default=0, help="rows per GPU (default 6M x k)")
    ap.add_argument("--queries", type=int, default=64)
    ap.add_argument("--mix", default="span", choices=["span", "random"],
                    help="span: selectivities log-uniform over [1e-6, 0.5]; random: the older level-based mix")
    ap.add_argument("--narrow", type=float, default=0.3, help="(random mix) share of city/brand/week constants")
    ap.add_argument("--width4", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu", action="store_true", help="skip the host parity pass and the CPU baseline")
    ap.add_argument("--serve-requests", type=int, default=1024, help="requests per serving run (0: no serving leg)")
    ap.add_argument("--plan", default="learned", choices=["learned", "tuned", "rule"],
                    help="the batch plan: the learned batch planner's (merle_b200/weights/batch_planner.f32), "
                         "the autotuner's (shapes timed on the mix), or the rule's (default shape, rule covers)")
    ap.add_argument("--no-graph", action="store_true", help="enqueue each step instead of replaying a CUDA graph")
    ap.add_argument("--no-plan-check", action="store_true", help="skip timing every batch plan of the mix")
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
def mix_of(args):
    from merle_b200 import workload as WL
    if args.mix == "span":
        return WL.span_mix(SEED_QUERIES, args.queries)
    return WL.random_mix(SEED_QUERIES, args.queries, args.narrow)


def host_table(k: int, nrows: int):
    """The star table generated on the host by the oracle's generator (the
    same seeded counter-based columns the engine generates on the device), in
    the reference's ssb_schema widths, or None if host memory is short."""
    from oracle import oracle as O
    need = nrows * 29 + (1 << 30)  # narrow fact columns + dimensions + slack
    try:
        import psutil
        if psutil.virtual_memory().available < need * 1.2:
            return None
    except ImportError:
        pass
    return O.StarHost(SEED_DATA, k, nrows)


def reference_pass(star, nrows: int, qs, threads: int):
    """The reference's s1ref..s4ref over the first nrows rows (one query per
    thread): (answers, seconds)."""
    from oracle import oracle as O
    schema = star.ssb_schema()
    return O.ref_answers(schema, nrows, qs, threads)


def parity_check(qs, answers, out_host: np.ndarray, offs, nq: np.ndarray, nrows: int) -> dict:
    """Our int64 group sums against the reference's answers: (uint32) of
    every group sum equals its uint32 array, s1ref's uint64 sum equals ours
    (as uint64).  Row counts give each query's realised selectivity."""
    bad = []
    for i, (q, ref_ans) in enumerate(zip(qs, answers)):
        mine = out_host[offs[i]:offs[i] + len(ref_ans)]
        if int(q.tmpl) == 1:
            ok = int(mine[0]) % (1 << 64) == int(ref_ans[0])
        else:
            ok = np.array_equal(mine.astype(np.uint64).astype(np.uint32), ref_ans)
        if not ok:
            bad.append(i)
    sel = nq.astype(np.float64) / nrows
    return {"reference_equal": not bad, "queries": len(qs), "mismatched": bad,
            "groups_compared": int(sum(len(a) for a in answers)),
            "against": "reference ssb/cpuref.c s1ref..s4ref over every row of the timed table "
                       "((uint32) of the int64 group sums; s1ref's uint64 sum)",
            "selectivity": {"min": float(sel.min()), "median": float(np.median(sel)), "max": float(sel.max()),
                            "per_query": [float(x) for x in sel]},
            "selected_rows_per_step": int(nq.sum())}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    qs = mix_of(args)
    from oracle import oracle as O
    if O.ref() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's cpuref.c built from "
                          "its sources) is missing"}))
        return
    n = min(CPU_SAMPLE_ROWS, args.rows or 6_000_000 * args.k)
    star = host_table(args.k, n)
    if star is None:
        print(json.dumps({"impl": "reference", "unavailable": "host memory too small for the row sample"}))
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        reference_pass(star, n, qs, threads)
    ts = [reference_pass(star, n, qs, threads)[1] for _ in range(args.steps)]
    tot = sum(ts)
    v = n * len(qs) * args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config_of(args, args.rows or 6_000_000 * args.k),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"each step: the {len(qs)}-query mix over the first {n:,} rows of the "
                                       f"table (ssb_schema widths), one query per thread"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def config_of(args, nrows_per_gpu):
    mix = ("selectivities log-uniform over [1e-6, 0.5] (workload.span_mix)" if args.mix == "span"
           else f"level-based constants, {args.narrow:.0%} city/brand/week level")
    return {"workload": f"star schema k={args.k}, {nrows_per_gpu:,} fact rows per GPU "
                        f"({'4-byte' if args.width4 else 'ssb_schema-width'} fact columns), 242-bitmap index, "
                        f"{args.queries}-query seeded mix of 4 templates, {mix}",
            "rows_per_gpu": nrows_per_gpu, "queries_per_step": args.queries, "k": args.k, "mix": args.mix,
            "l2": "inputs larger than L2 (each step reads tens of GB of bitmaps and payload)",
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


def batch_algo_bytes(star, scale: float, nrows: int, qs, ngroups, sample_n: int) -> dict:
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
        r = np.flatnonzero(O.qualifying_mask(star, t, p, sample_n))
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
    # the index is built twice: the first build also loads the library's
    # kernels into the context (a once-per-process cost); the second is the
    # steady-state build the roofline line reports
    eng.build_index()
    first_build_ms = eng.info()["index_build_ms"]
    eng.build_index()
    info = eng.info()
    qs = mix_of(args)
    Q = len(qs)
    qarr = (abi.mb_query * Q)(*qs)
    ngroups = [Engine.ngroups(q) for q in qs]
    offs_c = (C.c_uint64 * Q)()
    total_g = int(L.mb_queries_layout(qarr, Q, offs_c))
    offs = [int(x) for x in offs_c]
    out = torch.zeros(total_g, dtype=torch.int64, device="cuda")
    nq = torch.zeros(Q, dtype=torch.int64, device="cuda")
    ext = torch.cuda.ExternalStream(int(L.mb_engine_stream(eng.handle) or 0))

    def allreduce():
        if world > 1:
            with torch.cuda.stream(ext):
                shard.combine(out, nq)

    # the batch plan (launch shape and covers): the learned batch planner's,
    # the autotuner's (timed on this mix before the measured steps) or the
    # rule's; the batch captured once as a CUDA graph
    bopts = abi.mb_batch_opts()
    cover = 0
    tune = {"planner": args.plan}
    bnet = None
    if args.plan == "learned" and BATCH_WEIGHTS.exists():
        from merle_b200.planner import BATCH_CANDIDATE_NAMES, MLP
        bnet = MLP.load(BATCH_WEIGHTS)
        check(L.mb_engine_set_batch_planner(eng.handle, bnet.handle))
        cv, choice = C.c_uint32(0), C.c_uint32(0)
        t0 = time.perf_counter()
        check(L.mb_engine_plan_batch(eng.handle, qarr, Q, C.byref(bopts), C.byref(cv), C.byref(choice)))
        cover = int(cv.value)
        tune.update({"choice": BATCH_CANDIDATE_NAMES[choice.value], "plan_ms": (time.perf_counter() - t0) * 1e3,
                     "weights": str(BATCH_WEIGHTS.relative_to(ROOT))})
    elif args.plan == "tuned":
        tms, tried = C.c_float(0), C.c_uint32(0)
        t0 = time.perf_counter()
        check(L.mb_engine_tune_batch(eng.handle, qarr, Q, 3, C.byref(bopts), C.byref(tms), C.byref(tried)))
        tune.update({"shapes_timed": tried.value, "best_ms": tms.value, "tune_s": time.perf_counter() - t0})
    else:
        tune["planner"] = "rule"
    tune["opts"] = {f: getattr(bopts, f) for f, _ in bopts._fields_ if f != "pad_"}
    tune["cover"] = ["rule", "noedge", "nocompl", "fine"][cover]
    plans = []
    for _ in qs:
        p = abi.mb_plan()
        p.kind, p.cover = abi.PLAN_FUSED, cover
        plans.append(p)
    parr = (abi.mb_plan * Q)(*plans)
    binfo = (abi.mb_batch_launch_info * 16)()
    nlaunch, nalone = C.c_uint32(0), C.c_uint32(0)
    check(L.mb_engine_batch_info(eng.handle, qarr, Q, C.byref(bopts), binfo, 16, C.byref(nlaunch), C.byref(nalone)))
    tune["launches"] = [{f: getattr(binfo[i], f) for f, _ in binfo[i]._fields_ if f != "pad_"}
                        for i in range(nlaunch.value)]
    tune["queries_alone"] = nalone.value
    graph = C.c_void_p()
    if not args.no_graph:
        check(L.mb_batch_graph_create_plans(eng.handle, qarr, parr, Q, C.byref(bopts), out.data_ptr(), nq.data_ptr(),
                                            C.byref(graph)))

    def step_batch():
        if graph:
            check(L.mb_batch_graph_launch(graph))
        else:
            check(L.mb_engine_enqueue_batch_plans(eng.handle, qarr, parr, Q, C.byref(bopts), out.data_ptr(),
                                                  nq.data_ptr()))
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
    batch_nq = nq.clone()
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
    same = bool(torch.equal(out, batch_out)) and bool(torch.equal(nq, batch_nq))
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
    e2e_opts = None if bnet is not None else C.byref(bopts)  # None: the engine plans the batch with its network
    check(L.mb_engine_query_batch(eng.handle, qarr, Q, e2e_opts, res_host.ctypes.data, nq_host.ctypes.data))
    if world > 1:
        dist.barrier()
    def e2e_combine():
        # the shards' host answers summed over the ranks (the whole table's
        # answer on every rank): host -> device, all-reduce, device -> host
        if world > 1:
            t_out = torch.from_numpy(res_host).cuda()
            t_nq = torch.from_numpy(nq_host.view(np.int64)).cuda()
            shard.combine(t_out, t_nq)
            res_host[:] = t_out.cpu().numpy()
            nq_host.view(np.int64)[:] = t_nq.cpu().numpy()

    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        check(L.mb_engine_query_batch(eng.handle, qarr, Q, e2e_opts, res_host.ctypes.data, nq_host.ctypes.data))
        e2e_combine()
    e2e_ms = float((time.perf_counter() - t0) * 1e3)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": rows_total * Q * args.e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": C.sizeof(abi.mb_query) * Q + BATCH_HDR_BYTES + (8 * total_g + 8 * Q if world > 1 else 0),
           "d2h_bytes_per_step": (8 * total_g + 8 * Q) * (2 if world > 1 else 1),
           "api": "mb_engine_query_batch (host query descriptors in, the batch planned by the engine's network, "
                  "host int64 group sums and row counts out, returns when they are on the host; with N GPUs "
                  "the ranks' host answers are then summed by an all-reduce, inside the timed region)",
           "timing": "host wall clock around each call", "ms_per_step": e2e_ms / args.e2e_steps}
    e2e_same = bool(np.array_equal(res_host, batch_out.cpu().numpy()))

    # ---- the batch plans of this mix, timed (CUDA-graph replays): regret
    # of the chosen plan and its speedup over the rule-planned batch
    if world == 1 and not args.no_plan_check:
        from merle_b200 import planner as PL
        ref = batch_out.cpu().numpy()
        cand = [PL.time_batch(eng, qs, *PL.batch_candidate(c), reps=3, want=ref) for c in range(PL.NBC)]
        t_rule = PL.time_batch(eng, qs, None, 0, reps=3, want=ref)
        t_ch = ms_total / args.steps
        tune.update({"candidates_ms": {PL.BATCH_CANDIDATE_NAMES[c]: round(cand[c], 4) for c in range(PL.NBC)},
                     "rule_ms": t_rule, "regret": t_ch / min(cand + [t_ch]), "speedup_vs_rule": t_rule / t_ch,
                     "heldout_eval": json.loads((ROOT / "merle_b200" / "weights" / "batch_planner_eval.json")
                                                .read_text()).get("eval") if bnet is not None else None})

    # ---- serving: Poisson arrivals through the batched and the plain server
    serving = None
    if args.serve_requests and world == 1:
        serving = serve_leg(eng, args, None if bnet is not None else bopts, float(qtimes.mean()))

    line = None
    if rank == 0:
        from oracle import oracle as O
        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = json.loads(pk.read_text())
        peak = float(peaks.get("hbm_gbs", PEAK_FALLBACK_GBS))
        peak_src = ("MEASURED_PEAKS.json hbm_gbs (burst copy), of measured" if peaks
                    else f"fallback {PEAK_FALLBACK_GBS / 1000:.2f} TB/s")
        # parity and the CPU baseline: the reference's cpuref over the whole
        # table, generated on the host by the oracle
        parity, cpu, star = None, None, None
        if not args.no_cpu and world == 1:
            star = host_table(args.k, n)
            if star is None:
                parity = {"reference_equal": None, "skipped": "host memory too small for the full table"}
            else:
                threads = os.cpu_count() or 1
                answers, sec = reference_pass(star, n, qs, threads)
                parity = parity_check(qs, answers, batch_out.cpu().numpy(), offs,
                                      batch_nq.cpu().numpy().astype(np.uint64), n)
                cpu = {"value": n * Q / sec, "unit": UNIT, "cores": threads, "kind": "reference",
                       "sample": f"one pass of the {Q}-query mix over all {n:,} rows of the table in ssb_schema "
                                 f"widths (the reference's s1ref..s4ref, one query per thread on {threads} "
                                 f"threads); the same pass is the parity check", "seconds_per_pass": sec}
        sample_n = min(CPU_SAMPLE_ROWS, n)
        if star is None:
            star = O.StarHost(SEED_DATA, args.k, sample_n)
        ab = batch_algo_bytes(star, n / sample_n, n, qs, ngroups, sample_n)
        step_s = ms_total / args.steps / 1e3
        achieved = ab["total"] / step_s / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_src,
                "kernel": "batch_scan_kernel (one launch per 64-query step)",
                "algo_bytes_per_launch": ab["total"], "algo_bytes_detail": ab,
                "launch_ms_avg": ms_total / args.steps,
                "traffic": None, "traffic_note": "per-launch DRAM bytes in profiles/ (ncu)"}
        tj = ROOT / "profiles" / "traffic.json"
        if tj.exists():
            t = json.loads(tj.read_text()).get("batch_scan_kernel")
            if t and t.get("mix") == args.mix:
                roof["traffic"] = t["dram_bytes_per_row"] * n
                roof["traffic_note"] = ("ncu capture of a smaller launch of the same mix scaled to this launch's "
                                        "rows: " + t["source"])
        widths = {c: (4 if args.width4 else {"orderdate": 2, "discount": 1, "quantity": 1, "suppcity": 1}.get(c, 4))
                  for c in ["extendedprice", "discount", "partkey", "orderdate", "revenue", "custkey", "suppcity",
                            "supplycost", "quantity"]}
        plain_algo = sum(O.algo_bytes(star, n / sample_n, n, *WL.as_tuple(q), Engine.ngroups(q), widths,
                                      sample_n)["total"] for q in qs)
        build_bytes = index_build_bytes(n, info, args.width4)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": config_of(args, n), "impl": "ours",
                "plan": ("learned+batched: the whole mix in one persistent launch per step, its launch shape and "
                         "covers chosen by the learned batch planner" if bnet is not None else
                         f"batched ({tune['planner']} plan): the whole mix in one persistent launch per step")
                        + ("; replayed as a CUDA graph" if graph else ""),
                "batch_plan": tune,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "parity": parity,
                "plain": {"value": rows_total * Q * args.steps / (plain_ms / 1e3), "ms_per_step": plain_ms / args.steps,
                          "batched_speedup": plain_ms / ms_total, "results_identical": same,
                          "e2e_results_identical": e2e_same,
                          "roofline_frac": plain_algo / (qtimes.sum() / 1e3) / 1e9 / peak,
                          "plan": "one fused launch per query (rule planner)"},
                "latency_ms": serving,
                "gpu_launches": args.steps * (nlaunch.value + nalone.value),
                "clocks": clk.summary(),
                "index": {"bitmaps": info["nbitmaps"], "bytes": info["index_bytes"],
                          "build_ms": info["index_build_ms"], "first_build_ms": first_build_ms,
                          "denorm_bytes": info["denorm_bytes"],
                          "algo_bytes": build_bytes,
                          "achieved_gbs": build_bytes / (info["index_build_ms"] / 1e3) / 1e9,
                          "frac": build_bytes / (info["index_build_ms"] / 1e3) / 1e9 / peak,
                          "note": "build_ms: a second build of the same table (the first also loads the "
                                  "library's kernels into the context: first_build_ms); algo_bytes: columns "
                                  "and keys read once, bitmaps and denormalised columns written once"},
                "selected_rows_per_step": int(batch_nq.sum().item())}
        print(json.dumps(line))
    if graph:
        check(L.mb_batch_graph_destroy(graph))
    if bnet is not None:
        check(L.mb_engine_set_batch_planner(eng.handle, None))
        bnet.close()
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def index_build_bytes(n: int, info: dict, width4: int) -> int:
    """Algorithmic bytes of the index build: each indexed column read once
    (the date, discount, quantity and supplier city columns; the customer
    and part foreign keys plus their dimension arrays for the customer city
    and part mfgr levels), every bitmap written once, and the denormalised
    customer-city (1 byte a row) and part-mfgr (2 bytes) columns the same
    passes write for the queries."""
    w = 4 if width4 else None
    k = max(1, info["k"])
    from oracle import oracle as O
    col = (w or 2) * n + (w or 1) * n + (w or 1) * n + (w or 1) * n  # date, discount, quantity, suppcity
    fk = 4 * n * 2 + (30000 * k + 1) * 1 + (O.star_npart(k) + 1) * 2
    bm = info["nbitmaps"] * ((n + 31) // 32) * 4
    return int(col + fk + bm + info.get("denorm_bytes", 0))


def serve_leg(eng, args, bopts, plain_query_ms: float) -> dict:
    """Seeded Poisson arrivals of a selectivity-spanning mix through the
    batched and the plain server, at half and at twice the plain path's
    capacity (1 / mean plain query time): q/s, p50 and p99 latency over every
    request of each run."""
    from merle_b200 import serving as S, workload as WL
    base = WL.span_mix(SEED_QUERIES + 2, 256) if args.mix == "span" else WL.random_mix(SEED_QUERIES + 2, 256)
    qs = (base * ((args.serve_requests + len(base) - 1) // len(base)))[:args.serve_requests]
    cap = 1e3 / max(plain_query_ms, 1e-3)
    rates = [0.5 * cap, 2.0 * cap]
    recs = S.sweep(eng, qs, rates, ("batched", "plain"), batch=bopts)
    keep = ("mode", "offered_qps", "requests", "ok", "qps", "p50_ms", "p99_ms", "mean_ms", "max_ms", "mean_batch",
            "launches", "statuses", "wall_s")
    return {"plain_capacity_qps": cap, "runs": [{k: r[k] for k in keep} for r in recs],
            "note": "request latency submit -> result on the host, every request of each run "
                    f"({args.serve_requests} per run), seeded Poisson arrivals"}


if __name__ == "__main__":
    main()
