"""The reference's own C entry points (include/merle_b200_legacy.h).

CPU: the library exports them (and the bin tables) and window_zipf, a host
function, equals the reference's outputs in tests/golden.  Where the
reference tree is present, its unmodified main.c compiles and links against
libmerleb200.so.  GPU (test_gpu_legacy.py): the SSB and synthetic demo drivers
end to end."""
from __future__ import annotations

import os

import ctypes as C
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
REF = Path(os.environ.get("MERLE_REF", "/nonexistent-reference-tree"))


def test_bin_tables_exported(mb):
    L = mb.lib()
    tabs = {"dateSpBin": 8, "dateDeBin": 5, "discntSpBin": 5, "discntDeBin": 12, "qtySpBin": 6, "qtyDeBin": 11,
            "mfgrSpBin": 6, "mfgrDeBin": 6, "sCitySpBin": 6, "sCityDeBin": 4}
    for name, n in tabs.items():
        a = (C.c_uint64 * n).in_dll(L, name)
        assert list(a) == sorted(a) and len(set(a)) == n
    assert list((C.c_uint64 * 8).in_dll(L, "dateSpBin")) == [0, 366, 731, 1096, 1461, 1827, 2192, 2557]


def test_window_zipf_matches_reference(mb):
    L = mb.lib()
    L.window_zipf.restype = C.POINTER(C.c_double)
    L.window_zipf.argtypes = [C.c_double, C.c_size_t, C.c_size_t]
    g = json.loads((GOLDEN / "golden.json").read_text())["window_zipf"]
    for skew, want in g.items():
        p = L.window_zipf(float(skew), len(want), 60)
        got = np.ctypeslib.as_array(p, shape=(len(want),)).copy()
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=0)
    assert not L.window_zipf(1.0, 10, 60)  # skewness must exceed 1


@pytest.mark.skipif(not (REF / "main.c").exists() or shutil.which("gcc") is None,
                    reason="reference tree or gcc absent")
def test_reference_main_links_unchanged(mb, tmp_path):
    """The reference's driver (main.c, its headers) builds against this library
    with no source change: every symbol it needs resolves in libmerleb200.so."""
    exe = tmp_path / "mydemo"
    r = subprocess.run(["gcc", "-fopenmp", str(REF / "main.c"), f"-I{REF}", "-I/usr/local/cuda/include",
                        f"-L{mb.LIB_PATH.parent}", "-lmerleb200", f"-Wl,-rpath,{mb.LIB_PATH.parent}",
                        "-Wl,--no-undefined", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


class _SsbSchema(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "loCustKey", "loPartKey", "loOrderDate", "loExtendedPrice", "loRevenue", "loSupplyCost", "loQuantity",
        "loDiscount", "loSuppCity", "custMktSegment", "custCity", "partName", "partMfgr", "partColor", "partType",
        "partSize", "partContainer")]


def test_column_files_roundtrip_through_ssb_load(mb, tmp_path):
    """mb_write_column writes the reference's column format and ssb_load (host
    side only: no device copy) reads it back."""
    L = mb.lib()
    rng = np.random.default_rng(4)
    n, nc, npart = 1001, 51, 77
    cols = {"loCustKey": rng.integers(1, nc, n, dtype=np.uint32), "loPartKey": rng.integers(1, npart, n, dtype=np.uint32),
            "loOrderDate": rng.integers(0, 2557, n).astype(np.uint16),
            "loExtendedPrice": rng.integers(0, 1 << 31, n, dtype=np.uint32),
            "loRevenue": rng.integers(0, 1 << 31, n, dtype=np.uint32),
            "loSupplyCost": rng.integers(0, 100000, n, dtype=np.uint32),
            "loSuppCity": rng.integers(0, 250, n).astype(np.uint8), "loQuantity": rng.integers(1, 51, n).astype(np.uint8),
            "loDiscount": rng.integers(0, 11, n).astype(np.uint8), "custCity": rng.integers(0, 250, nc).astype(np.uint8),
            "custMktSegment": np.zeros(nc, np.uint8), "partName": np.zeros(npart, np.uint16),
            "partMfgr": rng.integers(0, 1000, npart).astype(np.uint16), "partColor": np.zeros(npart, np.uint8),
            "partType": np.zeros(npart, np.uint8), "partSize": np.zeros(npart, np.uint8),
            "partContainer": np.zeros(npart, np.uint8)}
    for name, a in cols.items():
        assert L.mb_write_column(str(tmp_path / name).encode(), a.ctypes.data, len(a), a.dtype.itemsize) == 0
        raw = (tmp_path / name).read_bytes()
        assert np.frombuffer(raw[:4], np.uint32)[0] == a.dtype.itemsize and len(raw) == 4 + a.nbytes
    L.ssb_load.restype = C.c_size_t
    L.ssb_load.argtypes = [C.POINTER(_SsbSchema), C.POINTER(_SsbSchema), C.c_char_p]
    L.ssb_free.argtypes = [C.POINTER(_SsbSchema), C.POINTER(_SsbSchema)]
    h = _SsbSchema()
    assert L.ssb_load(C.byref(h), None, str(tmp_path).encode()) == n
    try:
        for name, a in cols.items():
            got = np.ctypeslib.as_array(C.cast(getattr(h, name), C.POINTER(np.ctypeslib.as_ctypes_type(a.dtype))),
                                        shape=(len(a),))
            np.testing.assert_array_equal(got, a, err_msg=name)
    finally:
        L.ssb_free(C.byref(h), None)
    assert L.mb_write_column(str(tmp_path / "x").encode(), cols["loQuantity"].ctypes.data, n, 3) == 1  # width
    assert L.mb_write_column(str(tmp_path / "no" / "dir").encode(), cols["loQuantity"].ctypes.data, n, 1) == 6  # IO
