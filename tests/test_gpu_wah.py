"""GPU parity tests of the WAH interop row (merle_b200/csrc/wah.cu) through
the C ABI: compression bit-exact against the oracle (and through it the
reference's wahCmprsCPU, tests/test_wah.py) on ragged sizes, densities and
both bit orders; decompression of the reference's own streams (golden); the
AND / OR / XOR of streams against the oracle and the reference's wahAndCPU;
a decompressed stream used as an operand of a virtual bitmap program (the
compressed-operand hook); the reference's WAH pipeline for SSB Q1.1
(ssb/wah-demo.cu:22-76) against the reference's own answer; round trips at
600M rows."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi, check, device as D, ops
from merle_b200 import wah as W

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
GJ = json.loads((GOLDEN / "golden.json").read_text())
GW = GJ["wah"]
FILL, ONES = 0x80000000, 0x40000000


def host32(t) -> np.ndarray:
    return D.to_host(t, np.uint32)


def dev32(a: np.ndarray):
    return D.from_host(np.ascontiguousarray(a, np.uint32))


def random_bitmap(rng, nrows: int, kind: str) -> np.ndarray:
    words = (nrows + 31) // 32
    stride = (words + 31) // 32 * 32
    if kind == "dense":
        bm = rng.integers(0, 2**32, stride, dtype=np.uint64).astype(np.uint32)
    else:
        p = {"zero": 0.0, "one": 1.0, "sparse": 1e-3, "runs": None}[kind]
        if p is None:  # alternating runs of set and clear rows, random lengths
            bits = np.zeros(32 * stride, np.uint8)
            pos, on = 0, 0
            while pos < nrows:
                ln = int(rng.choice([1, 5, 31, 62, 200, 5000]))
                bits[pos:pos + ln] = on
                pos += ln
                on ^= 1
        else:
            bits = (rng.random(32 * stride) < p).astype(np.uint8)
        bm = np.packbits(bits, bitorder="little").view(np.uint32).copy()
    bm[words:] = 0
    if nrows % 32:
        bm[words - 1] &= (1 << (nrows % 32)) - 1
    return bm


SIZES = [1, 30, 31, 32, 33, 62, 993, 4096, 31 * 2048 + 7, 1_000_003]


@pytest.mark.parametrize("kind", ["dense", "sparse", "runs", "zero", "one"])
def test_encode_matches_oracle(orc, cuda, kind):
    rng = np.random.default_rng(hash(kind) & 0xFFFF)
    for nrows in SIZES:
        bm = random_bitmap(rng, nrows, kind)
        d = dev32(bm)
        for order in (abi.WAH_LSB, abi.WAH_MSB):
            got = host32(W.wah_compress(d, nrows, order))
            want = orc.wah_encode(bm, nrows, order)
            np.testing.assert_array_equal(got, want, err_msg=f"{kind} {nrows} order {order}")
            back = host32(W.wah_decompress(dev32(want), nrows, order))
            np.testing.assert_array_equal(back, bm[:len(back)], err_msg=f"{kind} {nrows} order {order}")


def test_decode_reference_streams(orc, cuda):
    """Streams written by the reference's wahCmprsCPU (golden) decode to the
    oracle's bitmap in both bit orders; the group count is the reference's."""
    gold = dict(np.load(GOLDEN / "wah_ref.npz"))
    for seed, g in GW["cases"]:
        w = gold[f"wah_{seed}"]
        for order in (0, 1):
            for nrows in (31 * g, 31 * g - 5, 31 * g + 40):
                if nrows <= 0:
                    continue
                got = host32(W.wah_decompress(dev32(w), nrows, order))
                np.testing.assert_array_equal(got, orc.wah_decode(w, nrows, order), err_msg=f"{seed} {nrows}")
        assert W.wah_ngroups(dev32(w)) == g


def test_ops_match_oracle_and_reference(orc, cuda):
    gold = dict(np.load(GOLDEN / "wah_ref.npz"))
    for a, b in GW["pairs"]:
        wa, wb = gold[f"wah_{a}"], gold[f"wah_{b}"]
        ga, gb = len(gold[f"dec_{a}"]), len(gold[f"dec_{b}"])
        for op in (abi.WAH_AND, abi.WAH_OR, abi.WAH_XOR):
            for g in (min(ga, gb), max(ga, gb)):
                got = host32(W._op(op, dev32(wa), dev32(wb), g))
                np.testing.assert_array_equal(got, orc.wah_op(op, wa, wb, g), err_msg=f"{a} op{op} {b} {g}")
        # the reference's wahAndCPU: the same words but a final 0-fill
        ref_and = gold[f"and_{a}_{b}"]
        got = host32(W.wah_and(dev32(wa), dev32(wb), min(ga, gb)))
        if len(got) and (got[-1] & FILL) and not (got[-1] & ONES):
            got = got[:-1]
        np.testing.assert_array_equal(got, ref_and)


def test_ops_random_streams(orc, cuda):
    rng = np.random.default_rng(21)
    for nrows in (62, 31 * 500, 777_777):
        x, y = random_bitmap(rng, nrows, "runs"), random_bitmap(rng, nrows, "sparse")
        wx, wy = orc.wah_encode(x, nrows, 0), orc.wah_encode(y, nrows, 0)
        G = (nrows + 30) // 31
        for op in (abi.WAH_AND, abi.WAH_OR, abi.WAH_XOR):
            got = host32(W._op(op, dev32(wx), dev32(wy), G))
            np.testing.assert_array_equal(got, orc.wah_op(op, wx, wy, G))


def test_size_query_capacity_and_bad_args(cuda, mb):
    L = mb.lib()
    rng = np.random.default_rng(3)
    nrows = 31 * 100
    bm = dev32(random_bitmap(rng, nrows, "dense"))
    n = C.c_uint64()
    s = D.stream_ptr()
    check(L.mb_wah_encode(bm.data_ptr(), nrows, 0, None, 0, C.byref(n), s))  # size query
    assert n.value == 100
    out = D.empty(100, 4)
    assert L.mb_wah_encode(bm.data_ptr(), nrows, 0, out.data_ptr(), 99, C.byref(n), s) == abi.MB_ERR_INVALID
    assert n.value == 100
    assert L.mb_wah_encode(bm.data_ptr(), nrows, 2, out.data_ptr(), 100, C.byref(n), s) == abi.MB_ERR_INVALID
    assert L.mb_wah_encode(None, nrows, 0, out.data_ptr(), 100, C.byref(n), s) == abi.MB_ERR_INVALID
    assert L.mb_wah_op(3, out.data_ptr(), 1, out.data_ptr(), 1, 10, out.data_ptr(), 100, C.byref(n),
                       s) == abi.MB_ERR_INVALID
    # empty inputs
    check(L.mb_wah_encode(None, 0, 0, None, 0, C.byref(n), s))
    assert n.value == 0
    check(L.mb_wah_decode(None, 0, 0, 0, None, s))
    z = D.empty(32, 4)
    z.fill_(-1)
    check(L.mb_wah_decode(None, 0, 0, 100, z.data_ptr(), s))  # no stream: all rows 0
    assert not host32(z).any()


def test_decoded_stream_is_a_program_operand(orc, cuda):
    """The compressed-operand hook: WAH streams of two predicate bitmaps,
    decompressed, serve as the bins of a program's operands; the fused
    result equals the one on the original bitmaps and the oracle's."""
    n = 100_003
    f = orc.gen_flat(9, n)
    fd = D.DevFlat(9, n)
    s = abi.mb_src()
    s.col, s.width = orc.ptr(f["a"]), 4
    ah, _ = orc.bitmap_create(s, n, [0], [300])
    s.col = orc.ptr(f["c"])
    ch, _ = orc.bitmap_create(s, n, [0], [400])
    ad, _ = D.bitmap_create(D.src_of(fd["a"]), n, [0], [300])
    cd, _ = D.bitmap_create(D.src_of(fd["c"]), n, [0], [400])
    wa, wc = W.wah_compress(ad[0], n, abi.WAH_MSB), W.wah_compress(cd[0], n, abi.WAH_MSB)
    ra, rc = W.wah_decompress(wa, n, abi.WAH_MSB), W.wah_decompress(wc, n, abi.WAH_MSB)
    ins = [(abi.ORM, 0, 0, 0), (abi.ANDM, 0, 1, 0)]
    op_h = ops.flat_op(f["a"], f["b"], f["c"], f["d"], f["e"], 0, 1000, [0, 1, 2, 3], 0, 1000).to_c()
    op_d = ops.flat_op(fd["a"], fd["b"], fd["c"], fd["d"], fd["e"], 0, 1000, [0, 1, 2, 3], 0, 1000).to_c()
    want, nqw = orc.vprg_grpby(ops.Vprg(n, [ops.Col(middle=[ah[0]]), ops.Col(middle=[ch[0]])], ins).to_c(), op_h, 1)
    for x, y in ((ad[0], cd[0]), (ra, rc)):
        out, nq = D.vprg_grpby(ops.Vprg(n, [ops.Col(middle=[x]), ops.Col(middle=[y])], ins).to_c(), op_d, 1)
        assert int(D.to_host(out, np.int64)[0]) == int(want[0])
        assert int(D.to_host(nq, np.uint64)[0]) == nqw


def test_wah_demo_pipeline_q11(orc, cuda):
    """SSB Q1.1 the way the reference's WAH baseline runs it (s1wah,
    ssb/wah-demo.cu:22-76): one bitmap per predicate, compressed, ANDed
    compressed, decompressed; then the decompressed result drives the fused
    aggregate and gives the reference's Q1.1 answer (golden, mod 2^32)."""
    g = GJ["ssb13"]
    star = D.DevStar(g["seed"], g["k"], g["n"])
    n = g["n"]
    q = g["queries"][0][1]  # dateMin, dateMax, discntMin, discntMax, qtyMin, qtyMax
    preds = [("orderdate", q[0], q[1]), ("discount", q[2], q[3]), ("quantity", q[4], q[5])]
    bms = [D.bitmap_create(D.src_of(star[c]), n, [lo], [hi])[0][0] for c, lo, hi in preds]
    streams = [W.wah_compress(b, n, abi.WAH_MSB) for b in bms]
    G = W.wah_groups(n)
    r = W.wah_and(W.wah_and(streams[0], streams[1], G), streams[2], G)
    dec = W.wah_decompress(r, n, abi.WAH_MSB)
    T = D.torch()
    want_bits = bms[0] & bms[1] & bms[2]
    assert T.equal(dec[:want_bits.numel()], want_bits)
    op = ops.s1op(q[0], q[1], star["orderdate"], q[2], q[3], star["discount"], q[4], q[5], star["quantity"],
                  star["extendedprice"]).to_c()
    out, _ = D.vprg_grpby(ops.Vprg(n, [ops.Col(middle=[dec])], [(abi.ORM, 0, 0, 0)]).to_c(), op, 1)
    gold = np.load(GOLDEN / "ssb13_ref_u32.npy")
    assert int(D.to_host(out, np.int64)[0]) & 0xFFFFFFFF == int(gold[0])


def test_round_trip_600M_rows(cuda):
    """Full size by properties: compress -> decompress is the identity, the
    stream stands for ceil(n / 31) groups, and AND with itself is itself."""
    T = D.torch()
    n = 600_000_000 + 17
    words = (n + 31) // 32
    g = T.Generator(device="cuda")
    g.manual_seed(5)
    bm = T.randint(-2**31, 2**31 - 1, (words,), dtype=T.int32, device="cuda", generator=g)
    # long runs in the middle third, sparse bits in the last
    bm[words // 3: 2 * words // 3] = 0
    bm[words // 3 + 1000: words // 3 + 500_000] = -1
    bm[2 * words // 3:] &= T.randint(0, 2, (words - 2 * words // 3,), dtype=T.int32, device="cuda",
                                     generator=g) << 7
    bm[-1] &= (1 << (n % 32)) - 1
    for order in (abi.WAH_LSB, abi.WAH_MSB):
        w = W.wah_compress(bm, n, order)
        assert W.wah_ngroups(w) == W.wah_groups(n)
        back = W.wah_decompress(w, n, order)
        assert T.equal(back[:words], bm) and not back[words:].any()
        assert T.equal(W.wah_and(w, w, W.wah_groups(n)), w)


def _noncanonical(rng, G: int) -> np.ndarray:
    """A stream over about G groups with what canonical streams never hold:
    zero-count fills, literals equal to 0 or 0x7fffffff, neighbouring fills
    of one kind."""
    out, g = [], 0
    while g < G:
        k = int(rng.integers(0, 6))
        if k == 0:
            out.append(FILL | int(rng.integers(0, 50)))
            g += out[-1] & 0x3FFFFFFF
        elif k == 1:
            out.append(FILL | ONES | int(rng.integers(0, 50)))
            g += out[-1] & 0x3FFFFFFF
        elif k == 2:
            out.append(int(rng.choice([0, 0x7FFFFFFF])))
            g += 1
        else:
            out.append(int(rng.integers(1, 0x7FFFFFFF)))
            g += 1
    return np.array(out, np.uint32)


@pytest.mark.parametrize("op", [abi.WAH_AND, abi.WAH_OR, abi.WAH_XOR])
def test_direct_ops_equal_explicit_and_oracle(orc, cuda, op):
    """The direct form (runs cut at both streams' boundaries) gives the
    explicit form's canonical stream: random, sparse, run-heavy and
    non-canonical inputs, streams shorter and longer than the groups asked."""
    rng = np.random.default_rng(40 + op)
    cases = []
    for nrows in (31, 62, 31 * 700 + 9, 1_000_003):
        for ka, kb in (("runs", "sparse"), ("dense", "runs"), ("zero", "one"), ("sparse", "sparse")):
            x, y = random_bitmap(rng, nrows, ka), random_bitmap(rng, nrows, kb)
            cases.append((orc.wah_encode(x, nrows, 0), orc.wah_encode(y, nrows, 0), (nrows + 30) // 31))
    for G in (1, 40, 1000, 5000):
        cases.append((_noncanonical(rng, G), _noncanonical(rng, G // 2 + 1), G))
        cases.append((_noncanonical(rng, G), np.zeros(0, np.uint32), G + 17))
    for wa, wb, G in cases:
        want = orc.wah_op(op, wa, wb, G)
        da, db = dev32(wa) if len(wa) else D.empty(0, 4)[:0], dev32(wb) if len(wb) else D.empty(0, 4)[:0]
        for method in (abi.WAH_EXPLICIT, abi.WAH_DIRECT, abi.WAH_AUTO):
            got = host32(W._op(op, da, db, G, method=method))
            np.testing.assert_array_equal(got, want, err_msg=f"op {op} method {method} G {G}")
