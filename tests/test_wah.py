"""CPU tests of the WAH interop row: the oracle's WAH restatement
(oracle/oracle.c) against the reference's own CPU WAH code (wahCmprsCPU,
wahAndCPU of merle/host/, through the committed golden vectors and, where it
was built, live through oracle/_ref/libwahref.so), and the library's WAH file
writer and reader against the reference's loadWahFile.  No GPU."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from merle_b200 import abi

GOLDEN = Path(__file__).resolve().parent / "golden"
GW = json.loads((GOLDEN / "golden.json").read_text())["wah"]
FILL, ONES, CNT = 0x80000000, 0x40000000, 0x3FFFFFFF


def groups_to_bitmap(dec: np.ndarray, order: int) -> tuple[np.ndarray, int]:
    """A bitmap in this library's layout whose 31-bit groups are dec."""
    G = len(dec)
    nrows = 31 * G
    bits = ((dec[:, None].astype(np.uint64) >> np.arange(31, dtype=np.uint64)) & 1).astype(np.uint8)
    if order == 1:
        bits = bits[:, ::-1]
    rows = bits.reshape(-1)
    words = (nrows + 31) // 32
    stride = (words + 31) // 32 * 32
    pad = np.zeros(32 * stride, np.uint8)
    pad[:nrows] = rows
    bm = np.packbits(pad, bitorder="little").view(np.uint32)
    return bm, nrows


def expand(wah: np.ndarray) -> np.ndarray:
    """Groups of a stream, straight from the layout (merle/host/wahCpu.c:20-24)."""
    out = []
    for w in wah.tolist():
        if w & FILL:
            out += [0x7FFFFFFF if w & ONES else 0] * (w & CNT)
        else:
            out.append(w & 0x7FFFFFFF)
    return np.array(out, np.uint32)


def trim_zero_fill(wah: np.ndarray) -> np.ndarray:
    if len(wah) and (wah[-1] & FILL) and not (wah[-1] & ONES):
        return wah[:-1]
    return wah


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLDEN / "wah_ref.npz"))


@pytest.mark.parametrize("order", [0, 1])
def test_oracle_encode_matches_reference_compression(orc, gold, order):
    for seed, g in GW["cases"]:
        bm, nrows = groups_to_bitmap(gold[f"dec_{seed}"], order)
        got = orc.wah_encode(bm, nrows, order)
        np.testing.assert_array_equal(got, gold[f"wah_{seed}"], err_msg=f"case {seed}")


@pytest.mark.parametrize("order", [0, 1])
def test_oracle_decode_inverts_reference_compression(orc, gold, order):
    for seed, g in GW["cases"]:
        bm, nrows = groups_to_bitmap(gold[f"dec_{seed}"], order)
        got = orc.wah_decode(gold[f"wah_{seed}"], nrows, order)
        np.testing.assert_array_equal(got, bm[:len(got)], err_msg=f"case {seed}")
        np.testing.assert_array_equal(expand(gold[f"wah_{seed}"]), gold[f"dec_{seed}"])


def test_oracle_and_matches_reference_wahAndCPU(orc, gold):
    """The reference's compressed AND covers the shorter stream and drops a
    final 0-fill (wahCpu.c:78); otherwise its words are the canonical ones."""
    for a, b in GW["pairs"]:
        ga, gb = len(gold[f"dec_{a}"]), len(gold[f"dec_{b}"])
        ours = orc.wah_op(abi.WAH_AND, gold[f"wah_{a}"], gold[f"wah_{b}"], min(ga, gb))
        np.testing.assert_array_equal(trim_zero_fill(ours), gold[f"and_{a}_{b}"], err_msg=f"{a} & {b}")
        want = gold[f"dec_{a}"][:min(ga, gb)] & gold[f"dec_{b}"][:min(ga, gb)]
        np.testing.assert_array_equal(expand(ours), want)


def test_oracle_or_xor_by_groups(orc, gold):
    for a, b in GW["pairs"]:
        da, db = gold[f"dec_{a}"], gold[f"dec_{b}"]
        g = max(len(da), len(db))
        xa = np.zeros(g, np.uint32)
        xb = np.zeros(g, np.uint32)
        xa[:len(da)], xb[:len(db)] = da, db
        for op, f in ((abi.WAH_OR, np.bitwise_or), (abi.WAH_XOR, np.bitwise_xor)):
            got = orc.wah_op(op, gold[f"wah_{a}"], gold[f"wah_{b}"], g)
            np.testing.assert_array_equal(expand(got), f(xa, xb))
            # canonical: no two neighbouring fills of one kind, no literal 0 / all-1
            for x, y in zip(got[:-1].tolist(), got[1:].tolist()):
                assert not ((x & FILL) and (y & FILL) and (x & ONES) == (y & ONES))
            assert all((w & FILL) or (w not in (0, 0x7FFFFFFF)) for w in got.tolist())


def test_oracle_ragged_rows(orc):
    """Rows past nrows in the last group are 0; both orders decode back."""
    rng = np.random.default_rng(4)
    for nrows in (1, 30, 31, 32, 33, 62, 63, 64, 1000, 31 * 77 + 5):
        words = (nrows + 31) // 32
        bm = rng.integers(0, 2**32, max(1, words), dtype=np.uint64).astype(np.uint32)
        if nrows % 32:
            bm[-1] &= (1 << (nrows % 32)) - 1
        for order in (0, 1):
            w = orc.wah_encode(bm, nrows, order)
            back = orc.wah_decode(w, nrows, order)
            np.testing.assert_array_equal(back[:words], bm[:words])
            assert expand(w).size == (nrows + 30) // 31


def test_live_reference_compression(orc):
    wref = orc.wah_ref()
    if wref is None:
        pytest.skip("the reference's WAH code was not built here")
    rng = np.random.default_rng(8)
    for trial in range(20):
        G = int(rng.integers(1, 3000))
        p = rng.choice([0.0, 0.01, 0.5, 0.99, 1.0])
        dec = np.where(rng.random(G) < 0.3, np.where(rng.random(G) < p, 0x7FFFFFFF, 0),
                       rng.integers(0, 0x80000000, G)).astype(np.uint32)
        buf = dec.copy()
        n = wref.wahCmprsCPU(orc.ptr(buf), G, orc.ptr(buf))  # in place (wahConv.c:56)
        for order in (0, 1):
            bm, nrows = groups_to_bitmap(dec, order)
            np.testing.assert_array_equal(orc.wah_encode(bm, nrows, order), buf[:n])


@pytest.fixture(scope="module")
def saved(tmp_path_factory, mb, gold):
    from merle_b200 import wah as W
    d = tmp_path_factory.mktemp("wah")
    files = {}
    for seed, g in GW["cases"]:
        p = d / f"w{seed}.wah"
        W.save_wah_file(p, gold[f"wah_{seed}"], g)
        files[seed] = p
    return files


def test_wah_file_is_read_by_the_reference_loader(orc, gold, saved):
    wref = orc.wah_ref()
    if wref is None:
        pytest.skip("the reference's WAH code was not built here")
    for seed, g in GW["cases"]:
        p = wref.loadWahFile(str(saved[seed]).encode())
        assert p
        has1 = C.c_uint8.from_address(p).value
        magic = C.c_uint32.from_address(p + 4).value
        cm, dm = C.c_uint64.from_address(p + 8).value, C.c_uint64.from_address(p + 16).value
        w = gold[f"wah_{seed}"]
        assert magic == 0x44F8A1EF and cm == len(w) and dm == g
        assert has1 == int(any((x >> 30) == 3 for x in w.tolist()))
        got = np.ctypeslib.as_array((C.c_uint32 * cm).from_address(p + 24)).copy()
        np.testing.assert_array_equal(got, w)


def test_wah_file_roundtrip_and_rejects(saved, gold, tmp_path, mb):
    from merle_b200 import wah as W
    for seed, g in GW["cases"]:
        w, ng = W.load_wah_file(saved[seed])
        np.testing.assert_array_equal(w, gold[f"wah_{seed}"])
        assert ng == g
    bad = tmp_path / "bad.wah"
    raw = bytearray(saved[GW["cases"][0][0]].read_bytes())
    raw[4] ^= 1
    bad.write_bytes(bytes(raw))
    with pytest.raises(mb.MbError):
        W.load_wah_file(bad)
    short = tmp_path / "short.wah"
    short.write_bytes(saved[GW["cases"][0][0]].read_bytes()[:-4])
    with pytest.raises(mb.MbError):
        W.load_wah_file(short)
    n = C.c_uint64()
    buf = np.zeros(1, np.uint32)
    assert mb.lib().mb_wah_load(str(saved[GW["cases"][0][0]]).encode(), buf.ctypes.data, 1, C.byref(n),
                                None) == abi.MB_ERR_INVALID
