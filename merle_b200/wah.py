"""WAH (word-aligned hybrid) compressed bitmaps: the reference's
compressed-bitmap baseline (merle/wahGpu.cuh, merle/host/wahCpu.h,
ssb/wah-demo.cu) on this library's kernels.

Names follow the reference's:

- ``wah_compress`` / ``wah_decompress``: ``wahCompress`` and ``wahDecomp``
  (merle/wahGpuCmprs.cu:172-198, 34-47), between this library's bitmaps and
  WAH streams (``order``: ``abi.WAH_LSB`` puts row 31g + j of group g at bit j,
  ``abi.WAH_MSB`` at bit 30 - j);
- ``wah_and`` / ``wah_or`` / ``wah_xor``: ``wahAnd`` / ``wahOr`` / ``wahXor``
  (merle/wahGpu.cuh:11-30): a canonical stream out, computed directly on the
  runs when the streams are short next to the rows, else by expanding them
  (``method`` picks one: ``abi.WAH_DIRECT`` / ``abi.WAH_EXPLICIT``);
- ``load_wah_file`` / ``save_wah_file``: ``loadWahFile``
  (merle/host/wahConv.c:93-109) and the matching writer.

A decompressed stream is an ordinary bitmap, so it can be a bin of an
``ops.Col`` operand of a virtual bitmap program (the compressed-operand hook
``vprg::_cmprs_adapt_run`` that the reference declares at primitive.cuh:334-337
but never defines).  Device arrays are torch uint32-typed int32 tensors on
CUDA; the library fails loudly if its CUDA build is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import abi, check, lib


def _torch():
    import torch
    return torch


def _ptr(t) -> int | None:
    return int(t.data_ptr()) if t is not None and t.numel() else None


def _stream(stream) -> int | None:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def wah_groups(nrows: int) -> int:
    return int(lib().mb_wah_groups(nrows))


def wah_compress(bitmap, nrows: int, order: int = abi.WAH_LSB, stream=None):
    """Device bitmap (int32 tensor, >= ceil(nrows/32) words) -> device WAH
    stream (an int32 tensor of the stream's words: a view of a buffer of
    ceil(nrows/31) words, the bound on any stream's length)."""
    torch = _torch()
    cap = max(1, wah_groups(nrows))
    out = torch.empty(cap, dtype=torch.int32, device=bitmap.device if nrows else "cuda")
    n = C.c_uint64()
    check(lib().mb_wah_encode(_ptr(bitmap) if nrows else None, nrows, order, _ptr(out), cap, C.byref(n),
                              _stream(stream)))
    return out[:n.value]


def wah_decompress(wah, nrows: int, order: int = abi.WAH_LSB, stream=None):
    """Device WAH stream -> device bitmap of mb_bitmap_stride(nrows) words."""
    torch = _torch()
    stride = int(lib().mb_bitmap_stride(nrows))
    out = torch.empty(max(1, stride), dtype=torch.int32, device=wah.device if wah.numel() else "cuda")
    check(lib().mb_wah_decode(_ptr(wah), wah.numel(), order, nrows, _ptr(out), _stream(stream)))
    return out[:stride]


def wah_ngroups(wah, stream=None) -> int:
    n = C.c_uint64()
    check(lib().mb_wah_ngroups(_ptr(wah), wah.numel(), C.byref(n), _stream(stream)))
    return n.value


def _op(op: int, a, b, ngroups: int | None, stream=None, method: int = abi.WAH_AUTO):
    torch = _torch()
    if ngroups is None:
        ngroups = max(wah_ngroups(a, stream), wah_ngroups(b, stream))
    cap = max(1, ngroups)
    out = torch.empty(cap, dtype=torch.int32, device=a.device)
    n = C.c_uint64()
    check(lib().mb_wah_op_ex(op, _ptr(a), a.numel(), _ptr(b), b.numel(), ngroups, method, _ptr(out), cap,
                             C.byref(n), _stream(stream)))
    return out[:n.value]


def wah_and(a, b, ngroups: int | None = None, stream=None, method: int = abi.WAH_AUTO):
    return _op(abi.WAH_AND, a, b, ngroups, stream, method)


def wah_or(a, b, ngroups: int | None = None, stream=None, method: int = abi.WAH_AUTO):
    return _op(abi.WAH_OR, a, b, ngroups, stream, method)


def wah_xor(a, b, ngroups: int | None = None, stream=None, method: int = abi.WAH_AUTO):
    return _op(abi.WAH_XOR, a, b, ngroups, stream, method)


def save_wah_file(path: str | Path, words: np.ndarray, ngroups: int) -> None:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    check(lib().mb_wah_save(str(path).encode(), w.ctypes.data if len(w) else None, len(w), ngroups))


def load_wah_file(path: str | Path) -> tuple[np.ndarray, int]:
    """(stream words, groups) of a file in the reference's layout."""
    n, g = C.c_uint64(), C.c_uint64()
    check(lib().mb_wah_load(str(path).encode(), None, 0, C.byref(n), C.byref(g)))
    w = np.zeros(max(1, n.value), np.uint32)
    check(lib().mb_wah_load(str(path).encode(), w.ctypes.data, len(w), C.byref(n), C.byref(g)))
    return w[:n.value], g.value


# ---------------------------------------------------------------- measurement
def _predicates(star, tmpl: int, p) -> list:
    """(source, lo, hi) of each predicate of an SSB template, as the
    reference's WAH baseline builds its bitmaps (s1wah .. s4wah,
    ssb/wah-demo.cu:22-240): fact-column ranges and dimension attributes
    reached through the foreign key."""
    from . import device as D
    date = (D.src_of(star["orderdate"]), p[-2], p[-1])
    scity = lambda lo, hi: (D.src_of(star["suppcity"]), lo, hi)  # noqa: E731
    ccity = lambda lo, hi: (D.src_of(star.custcity, star["custkey"]), lo, hi)  # noqa: E731
    pmfgr = lambda lo, hi: (D.src_of(star.partmfgr, star["partkey"]), lo, hi)  # noqa: E731
    if tmpl == 1:
        return [(D.src_of(star["orderdate"]), p[0], p[1]), (D.src_of(star["discount"]), p[2], p[3]),
                (D.src_of(star["quantity"]), p[4], p[5])]
    if tmpl == 2:
        return [pmfgr(p[0], p[1]), scity(p[2], p[3])]
    if tmpl == 3:
        return [ccity(p[0], p[1]), scity(p[2], p[3]), date]
    return [ccity(p[0], p[1]), scity(p[2], p[3]), pmfgr(p[4], p[5]), date]


def main(argv=None) -> None:
    """Times the reference's WAH baseline pipeline on this library's kernels
    for the 13 SSB queries (per query: the AND of the predicates' compressed
    streams, then decompression, the region ssb/wah-demo.cu times), the fused
    plain path on the same queries, and compression / decompression
    throughput.  One JSON line per measurement."""
    import argparse
    import json
    import time

    from . import device as D, workload as WL
    from .engine import Engine

    ap = argparse.ArgumentParser()
    ap.add_argument("--k", type=int, default=20)
    ap.add_argument("--rows", type=int, default=120_000_000)
    ap.add_argument("--codec-rows", type=int, default=1_800_000_000)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--codec-only", action="store_true", help="skip the SSB pipeline")
    ap.add_argument("--out", type=str, default="")
    a = ap.parse_args(argv)
    torch = _torch()
    lines = []

    def emit(d):
        print(json.dumps(d), flush=True)
        lines.append(d)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    n = a.rows
    star = D.DevStar(2, a.k, n) if not a.codec_only else None
    G = wah_groups(n)
    eng = Engine(0)
    if not a.codec_only:
        eng.gen_star(2, a.k, n)
        eng.build_index()
    seen = {}
    for tmpl, p in ([] if a.codec_only else WL.SSB13):
        seen[tmpl] = seen.get(tmpl, 0) + 1
        bms = [D.bitmap_create(src, n, [lo], [hi])[0][0] for src, lo, hi in _predicates(star, tmpl, p)]
        t0 = time.perf_counter()
        streams = [wah_compress(b, n, abi.WAH_MSB) for b in bms]
        torch.cuda.synchronize()
        comp_ms = (time.perf_counter() - t0) * 1e3

        def pipeline():
            r = streams[0]
            for s in streams[1:]:
                r = wah_and(r, s, G)
            return wah_decompress(r, n, abi.WAH_MSB)

        want = bms[0]
        for b in bms[1:]:
            want = want & b
        assert torch.equal(pipeline()[:want.numel()], want)
        wah_ms = timed(pipeline, a.reps)
        q = abi.query(tmpl, *p)
        eng.query(q)
        fused = sorted(eng.query(q)[2].ms for _ in range(a.reps))[a.reps // 2]
        emit({"what": "wah_pipeline", "query": f"Q{tmpl}.{seen[tmpl]}", "rows": n, "wah_and_decode_ms": wah_ms,
              "wah_compress_ms_wall": comp_ms, "stream_words": [int(s.numel()) for s in streams],
              "fused_plain_ms": fused})
    eng.close()
    # compression / decompression throughput on bitmaps of three densities
    n = a.codec_rows
    words = (n + 31) // 32
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    for name, bm in (("dense", torch.randint(-2**31, 2**31 - 1, (words,), dtype=torch.int32, device="cuda",
                                              generator=g)),
                     ("runs", torch.repeat_interleave(torch.tensor([0, -1, 0x5555], dtype=torch.int32,
                                                                   device="cuda").repeat(words // 3000 + 1),
                                                      1000)[:words].contiguous()),
                     ("sparse", (torch.rand(words, device="cuda", generator=g) < 0.01).to(torch.int32))):
        w = wah_compress(bm, n)
        enc_ms = timed(lambda: wah_compress(bm, n), a.reps)
        dec_ms = timed(lambda: wah_decompress(w, n), a.reps)
        bm_bytes, st_bytes = 4 * words, 4 * int(w.numel())
        # AND with the same bitmap shifted by 1,000 words (another stream of its kind)
        w2 = wah_compress(torch.roll(bm, 1000), n)
        Gn = wah_groups(n)
        ops_ms = {m: timed(lambda: wah_and(w, w2, Gn, method=k), a.reps)
                  for m, k in (("explicit", abi.WAH_EXPLICIT), ("direct", abi.WAH_DIRECT))}
        emit({"what": "wah_codec", "bitmap": name, "rows": n, "stream_words": int(w.numel()),
              "encode_ms": enc_ms, "decode_ms": dec_ms,
              "encode_gbs": (bm_bytes + st_bytes) / enc_ms / 1e6, "decode_gbs": (bm_bytes + st_bytes) / dec_ms / 1e6,
              "and_explicit_ms": ops_ms["explicit"], "and_direct_ms": ops_ms["direct"]})
    if a.out:
        Path(a.out).write_text("".join(json.dumps(d) + "\n" for d in lines))


if __name__ == "__main__":
    main()
