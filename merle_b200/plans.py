"""Times each plan kind of the engine on the same queries: the bitmap-index
plans (fused, materialised) against the no-index plans (the scan probing
dimension arrays, and the Crystal-style hash joins of crystal/src/ssb/*.cu),
with the dimension attributes denormalised per row or probed through their
foreign keys (the reference's layout).  One JSON line per (layout, query).

    python -m merle_b200.plans --rows 120000000
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path

from . import abi
from . import workload as WL
from .engine import Engine

KINDS = {"fused": abi.PLAN_FUSED, "materialised": abi.PLAN_MATERIALISED, "scan": abi.PLAN_SCAN,
         "hash": abi.PLAN_HASH}

# wide variants of the templates (most dimension rows pass): the no-index end
WIDE = [(2, (0, 1000, 0, 250)), (3, (0, 250, 0, 250, 0, 2557)), (4, (0, 250, 0, 250, 0, 1000, 0, 2557))]


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--k", type=int, default=20)
    ap.add_argument("--rows", type=int, default=120_000_000)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", type=str, default="")
    a = ap.parse_args(argv)
    lines = []
    e = Engine(0)
    try:
        e.gen_star(2, a.k, a.rows)
        qs, seen = [], {}
        for t, p in WL.SSB13:
            seen[t] = seen.get(t, 0) + 1
            qs.append((f"Q{t}.{seen[t]}", abi.query(t, *p)))
        qs += [(f"wide{t}", abi.query(t, *p)) for t, p in WIDE]
        for probe_dims in (False, True):
            e.build_index(probe_dims=probe_dims)
            for name, q in qs:
                want = e.query(q)[0]
                row = {"layout": "probe_dims" if probe_dims else "denormalised", "query": name, "rows": a.rows}
                for kname, kind in KINDS.items():
                    plan = abi.mb_plan()
                    plan.kind = kind
                    got, _, _ = e.query(q, plan)
                    assert (got == want).all(), (name, kname)
                    ms = sorted(e.query(q, plan)[2].ms for _ in range(a.reps))[a.reps // 2]
                    row[f"{kname}_ms"] = ms
                print(json.dumps(row), flush=True)
                lines.append(row)
    finally:
        e.close()
    if a.out:
        Path(a.out).write_text("".join(json.dumps(d) + "\n" for d in lines))


if __name__ == "__main__":
    main()
