"""The reference's own GPU kernel beside this library's, same GPU, same inputs.

oracle/_ref/librefgpu.so instantiates the reference's vprg_grpby
(primitive.cuh:340-445) with its SSB op functors (ssb/lambdas.cuh:19-152)
and times it the way the reference's driver does (ssb/lambdas.cuh:154-243:
100 repetitions of a group-array memset and one launch).  At 120M rows (the
star schema at k = 20, the reference's ssb_schema widths) the 13 SSB queries
run over the same device columns and the same recipe bitmaps
(`mb_recipe_build`: one exact bitmap per predicate, `perfect`, or middle bins
with candidate-checked edges, `candchk`, as the reference's recipe builds them)
through both kernels: the reference's uint32 group sums must equal this
library's int64 sums mod 2^32, and the times of both are reported (written as
JSON to $MB_REFGPU_OUT when it is set).  The test asserts parity only."""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi, check, device as D
from tests import helpers as H

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "librefgpu.so"


class RefCols(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("custkey", "partkey", "orderdate", "extendedprice", "revenue",
                                          "supplycost", "quantity", "discount", "suppcity", "custcity",
                                          "partmfgr")]


class RefCol(C.Structure):
    _fields_ = [("nmiddle", C.c_uint32), ("middle", C.c_void_p * 4), ("leftmost", C.c_void_p),
                ("rightmost", C.c_void_p)]


def _ref():
    if not LIB.exists():
        pytest.skip("oracle/_ref/librefgpu.so not built (needs the reference tree at build time)")
    lib = C.CDLL(str(LIB))
    lib.refgpu_query.restype = C.c_int
    lib.refgpu_query.argtypes = [C.POINTER(RefCols), C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                 C.POINTER(RefCol), C.c_uint32, C.POINTER(C.c_uint8), C.c_uint32, C.c_void_p,
                                 C.c_uint32, C.c_int, C.POINTER(C.c_float)]
    return lib


def _recipe(mb, dev, kind, preds, instrs, n):
    r = abi.mb_recipe()
    r.factsz = n
    for i, (fk, attr, mn, mx) in enumerate(preds):
        r.nbit[i] = attr.element_size() * 8
        r.min[i], r.max[i] = mn & 0xFFFFFFFF, mx & 0xFFFFFFFF
        r.dimsz[i] = 0xFFFFFFFF
        r.fk[i] = fk.data_ptr() if fk is not None else None
        r.attr[i] = attr.data_ptr()
    ins = (abi.mb_instr * abi.MB_MAXNINSTR)()
    for i, t in enumerate(instrs):
        ins[i].opcode, ins[i].dstreg, ins[i].src1, ins[i].src2 = t
    o = abi.mb_owned_vprg()
    k = {"perfect": abi.RECIPE_PERFECT, "candchk": abi.RECIPE_CANDCHK}[kind]
    check(mb.lib().mb_recipe_build(C.byref(r), k, ins, C.byref(o), D.stream_ptr()))
    return o


def _time_ours(torch, prg, op, ng, reps):
    out = D.empty(ng, 8)
    nq = D.empty(1, 8)
    D.vprg_grpby(prg, op, ng, None, out, nq)  # untimed first launch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        D.vprg_grpby(prg, op, ng, None, out, nq)
    b.record()
    b.synchronize()
    return out, a.elapsed_time(b) / reps


def test_reference_kernel_same_gpu(cuda, mb):
    lib = _ref()
    torch = cuda
    n, reps = 120_000_000, 100
    dev = D.DevStar(2, 20, n, width4=False)
    rc = RefCols(**{f: dev[f].data_ptr() for f in ("custkey", "partkey", "orderdate", "extendedprice", "revenue",
                                                   "supplycost", "quantity", "discount", "suppcity")},
                 custcity=dev.custcity.data_ptr(), partmfgr=dev.partmfgr.data_ptr())
    rows = []
    for kind in ("perfect", "candchk"):
        for q, a, ng in H.SSB13:
            preds, ins = H.ssb_recipe(dev, q, a)
            owned = _recipe(mb, dev, kind, preds, ins, n)
            try:
                prg = owned.prg
                cols = (RefCol * len(preds))()
                for i in range(len(preds)):
                    c = prg.cols[i]
                    assert c.nmiddle <= 4
                    cols[i].nmiddle = c.nmiddle
                    for k in range(c.nmiddle):
                        cols[i].middle[k] = c.middle[k]
                    cols[i].leftmost, cols[i].rightmost = c.leftmost, c.rightmost
                ib = (C.c_uint8 * (4 * len(ins)))(*[x for t in ins for x in t])
                par = (C.c_uint32 * 8)(*a)
                out_ref = torch.zeros(ng, dtype=torch.int32, device="cuda")
                torch.cuda.synchronize()
                ms_ref = C.c_float()
                st = lib.refgpu_query(C.byref(rc), n, int(q[1]), par, cols, len(preds), ib, len(ins),
                                      out_ref.data_ptr(), ng, reps, C.byref(ms_ref))
                assert st == 0, f"refgpu_query {q}{a}: status {st}"
                torch.cuda.synchronize()
                op = H.ssb_op(dev, q, a).to_c()
                out, ms_ours = _time_ours(torch, prg, op, ng, reps)
                want = D.to_host(out_ref, np.uint32)
                got = D.to_host(out, np.int64).astype(np.uint64).astype(np.uint32)
                np.testing.assert_array_equal(got, want, err_msg=f"{kind} {q}{a}")
                rows.append({"kind": kind, "query": f"{q}{a}", "groups": ng, "reference_ms": ms_ref.value,
                             "ours_ms": ms_ours, "speedup": ms_ref.value / ms_ours})
            finally:
                check(mb.lib().mb_owned_vprg_release(C.byref(owned)))
    summary = {"rows": n, "reps": reps, "queries": rows}
    for kind in ("perfect", "candchk"):
        r = [x for x in rows if x["kind"] == kind]
        summary[kind] = {"reference_gmean_ms": float(np.exp(np.mean(np.log([x["reference_ms"] for x in r])))),
                         "ours_gmean_ms": float(np.exp(np.mean(np.log([x["ours_ms"] for x in r]))))}
    text = json.dumps(summary, indent=1)
    print(text)
    if os.environ.get("MB_REFGPU_OUT"):
        Path(os.environ["MB_REFGPU_OUT"]).write_text(text)
