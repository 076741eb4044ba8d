"""GPU tests of the reference's own C entry points (merle_b200_legacy.h):
the SSB demo (files in the reference's column format -> load -> every
fixed-index and recipe path against ssb_cpujoin), ssb_cpujoin against the
reference's golden outputs, and the synthetic demo (files -> load -> join,
recipe bitmaps fused and materialised, both tile widths) against the
oracle."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
G = json.loads((GOLDEN / "golden.json").read_text())
SUMGRP_ALL = 2458


class SsbSchema(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "loCustKey", "loPartKey", "loOrderDate", "loExtendedPrice", "loRevenue", "loSupplyCost", "loQuantity",
        "loDiscount", "loSuppCity", "custMktSegment", "custCity", "partName", "partMfgr", "partColor", "partType",
        "partSize", "partContainer")]


class SynthSchema(C.Structure):
    _fields_ = [("bitwidth", C.c_uint32), ("factattr1", C.c_void_p), ("factattr2", C.c_void_p),
                ("fkey", C.c_void_p), ("dimattr1", C.c_void_p), ("dimattr2", C.c_void_p)]


def _write(path: Path, a: np.ndarray):
    with open(path, "wb") as f:
        f.write(np.uint32(a.dtype.itemsize).tobytes())
        f.write(np.ascontiguousarray(a).tobytes())


@pytest.fixture(scope="module")
def ssb_dir(tmp_path_factory, orc):
    g = G["ssb13"]
    s = orc.StarHost(g["seed"], g["k"], g["n"])
    d = tmp_path_factory.mktemp("ssbcols")
    names = {"loCustKey": "custkey", "loPartKey": "partkey", "loOrderDate": "orderdate",
             "loExtendedPrice": "extendedprice", "loRevenue": "revenue", "loSupplyCost": "supplycost",
             "loSuppCity": "suppcity", "loQuantity": "quantity", "loDiscount": "discount"}
    for f, c in names.items():
        _write(d / f, s[c])
    _write(d / "custCity", s.custcity)
    _write(d / "custMktSegment", np.zeros_like(s.custcity))
    _write(d / "partName", np.zeros_like(s.partmfgr))
    _write(d / "partMfgr", s.partmfgr)
    for f in ("partColor", "partType", "partSize", "partContainer"):
        _write(d / f, np.zeros(len(s.partmfgr), np.uint8))
    return d


def _lib(mb):
    L = mb.lib()
    L.ssb_load.restype = C.c_size_t
    L.ssb_load.argtypes = [C.POINTER(SsbSchema), C.POINTER(SsbSchema), C.c_char_p]
    L.ssb_free.argtypes = [C.POINTER(SsbSchema), C.POINTER(SsbSchema)]
    L.ssb_cpujoin.restype = C.POINTER(C.c_uint32)
    L.ssb_cpujoin.argtypes = [C.POINTER(SsbSchema), C.c_size_t]
    L.ssb_demoall.restype = C.c_bool
    L.ssb_demoall.argtypes = [C.c_char_p]
    L.synth_load.restype = C.c_size_t
    L.synth_load.argtypes = [C.POINTER(SynthSchema), C.POINTER(SynthSchema), C.c_char_p]
    L.synth_free.argtypes = [C.POINTER(SynthSchema), C.POINTER(SynthSchema)]
    L.synth_join.argtypes = [C.POINTER(SynthSchema), C.c_size_t] + [C.c_uint64] * 6 + [C.c_void_p]
    L.synth_demoall.restype = C.c_bool
    L.synth_demoall.argtypes = [C.c_char_p]
    return L


def test_ssb_cpujoin_matches_reference_golden(cuda, mb, ssb_dir):
    L = _lib(mb)
    h = SsbSchema()
    n = L.ssb_load(C.byref(h), None, str(ssb_dir).encode())
    assert n == G["ssb13"]["n"]
    try:
        r = L.ssb_cpujoin(C.byref(h), n)
        got = np.ctypeslib.as_array(r, shape=(SUMGRP_ALL,)).copy()
        np.testing.assert_array_equal(got, np.load(GOLDEN / "ssb13_ref_u32.npy"))
    finally:
        L.ssb_free(C.byref(h), None)


def test_ssb_demoall(cuda, mb, ssb_dir, capfd):
    """Load, fixed index, every fixed-layout and controlled-layout path: all
    equal ssb_cpujoin (the reference's own driver flow, ssb/cpuref.c:318-349).
    The WAH baseline runs first and times all 13 queries (ssb/wah-demo.cu)."""
    L = _lib(mb)
    assert L.ssb_demoall(str(ssb_dir).encode())
    out = capfd.readouterr().out.splitlines()
    i = out.index("Case\tWAH\tRTScan")
    rows = [ln.split("\t") for ln in out[i + 1:i + 14]]
    assert [r[0] for r in rows] == [f"SSB{a}{b}" for a, n in ((1, 3), (2, 3), (3, 4), (4, 3)) for b in range(1, n + 1)]
    assert all(len(r) == 3 and float(r[1]) > 0 and r[2] == "unavailable" for r in rows)


def test_ssb_load_missing_dir(cuda, mb, tmp_path):
    L = _lib(mb)
    h, d = SsbSchema(), SsbSchema()
    assert L.ssb_load(C.byref(h), C.byref(d), str(tmp_path / "nope").encode()) == 0


@pytest.fixture(scope="module")
def synth_dir(tmp_path_factory):
    """The ten case folders synth_demoall reads (synth/cpuref.c:188-191):
    fk uniform over n / 100 dimension keys, a1 and a2 skewed toward small
    values, 16- or 32-bit."""
    d = tmp_path_factory.mktemp("synth")
    n = 200_000
    rng = np.random.default_rng(17)
    for case in ["04_16", "04_32", "08_16", "08_32", "12_16", "12_32", "16_16", "16_32", "20_16", "20_32"]:
        c = d / case
        c.mkdir()
        dt = np.uint16 if case.endswith("16") else np.uint32
        _write(c / "fk", rng.integers(0, n // 100, n).astype(np.uint32))
        _write(c / "a1", np.minimum(rng.zipf(1.3, n) - 1, 60000).astype(dt))
        _write(c / "a2", np.minimum(rng.zipf(1.3, n) - 1, 60000).astype(dt))
    return d


def test_synth_join_matches_oracle(cuda, mb, orc, synth_dir):
    from merle_b200 import ops
    L = _lib(mb)
    h, dv = SynthSchema(), SynthSchema()
    n = L.synth_load(C.byref(h), C.byref(dv), str(synth_dir / "04_32").encode())
    assert n == 200_000 and h.bitwidth == 32
    try:
        a1 = np.ctypeslib.as_array(C.cast(h.factattr1, C.POINTER(C.c_uint32)), shape=(n,)).copy()
        a2 = np.ctypeslib.as_array(C.cast(h.factattr2, C.POINTER(C.c_uint32)), shape=(n,)).copy()
        fk = np.ctypeslib.as_array(C.cast(h.fkey, C.POINTER(C.c_uint32)), shape=(n,)).copy()
        d1 = np.ctypeslib.as_array(C.cast(h.dimattr1, C.POINTER(C.c_uint32)), shape=(n // 100,)).copy()
        d2 = np.ctypeslib.as_array(C.cast(h.dimattr2, C.POINTER(C.c_uint8)), shape=(n // 100,)).copy()
        assert (d1 == np.arange(n // 100)).all()
        import torch
        g = torch.zeros(256, dtype=torch.int32, device="cuda")
        for case in [(0, 60, 0, 60, 0, 2000), (5, 9, 100, 400, 300, 1500), (0, 1, 0, 0, 0, 10)]:
            L.synth_join(C.byref(dv), n, *case, g.data_ptr())
            torch.cuda.synchronize()
            got = g.cpu().numpy().view(np.uint32)
            want, _ = orc.join_grpby(n, ops.synth_op(a1, a2, fk, d1, d2, *case).to_c(), 256)
            np.testing.assert_array_equal(got, want.astype(np.uint32))
    finally:
        L.synth_free(C.byref(h), C.byref(dv))


def test_synth_demoall(cuda, mb, synth_dir):
    """Every case and selectivity: the join, the fused kernel and the
    materialised stages over the three recipe layouts, against synth_ref
    (the reference's own driver flow, synth/cpuref.c:180-253)."""
    L = _lib(mb)
    assert L.synth_demoall(str(synth_dir).encode())


def test_engine_table_exported_for_the_reference_drivers(cuda, mb, tmp_path):
    """A table generated here, written as the reference's column files
    (mb_engine_save_ssb), runs through the reference's driver flow and gives
    the reference's golden results."""
    from merle_b200.engine import Engine
    g = G["ssb13"]
    e = Engine(0)
    e.gen_star(g["seed"], g["k"], g["n"], width4=True)
    e.save_ssb(tmp_path)
    e.close()
    L = _lib(mb)
    h = SsbSchema()
    n = L.ssb_load(C.byref(h), None, str(tmp_path).encode())
    assert n == g["n"]
    try:
        r = L.ssb_cpujoin(C.byref(h), n)
        got = np.ctypeslib.as_array(r, shape=(SUMGRP_ALL,)).copy()
        np.testing.assert_array_equal(got, np.load(GOLDEN / "ssb13_ref_u32.npy"))
    finally:
        L.ssb_free(C.byref(h), None)
    assert L.ssb_demoall(str(tmp_path).encode())
