"""CPU tests of the C ABI boundary: the library loads without a GPU, exports
every symbol its headers declare, its ctypes mirror matches the C layouts,
and its host-only logic (argument checks, col::from_bin planning) behaves as
the reference's."""
from __future__ import annotations

import ctypes as C
import subprocess
import tempfile
from pathlib import Path

import pytest

from merle_b200 import abi

ROOT = Path(__file__).resolve().parent.parent


def header_files():
    return sorted((ROOT / "include").glob("*.h"))


def test_library_exports_every_declared_symbol(mb):
    L = mb.lib()
    names = []
    for h in header_files():
        names += abi.header_symbols(h)
    assert len(names) >= 18
    out = subprocess.run(["nm", "-D", "--defined-only", str(mb.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for n in names:
        assert n in exported, f"{n} declared in include/ but not exported"
        getattr(L, n)
    # every ctypes signature names a declared symbol
    for n in abi.SIGNATURES:
        assert n in names


STRUCTS = ["mb_instr", "mb_col", "mb_vprg", "mb_src", "mb_term", "mb_key", "mb_op", "mb_launch", "mb_star_cols",
           "mb_recipe", "mb_owned_vprg"]


def test_struct_layouts_match_c():
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"merle_b200.h\"\nint main(void){\n"
    for s in STRUCTS:
        prog += f'printf("{s} %zu\\n", sizeof({s}));\n'
    prog += 'printf("op.terms %zu\\n", offsetof(mb_op, terms));\n'
    prog += 'printf("op.keys %zu\\n", offsetof(mb_op, keys));\n'
    prog += 'printf("vprg.instrs %zu\\n", offsetof(mb_vprg, instrs));\nreturn 0;}\n'
    with tempfile.TemporaryDirectory() as d:
        src, exe = Path(d) / "s.c", Path(d) / "s"
        src.write_text(prog)
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
        got = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for s in STRUCTS:
        assert int(got[s]) == C.sizeof(getattr(abi, s)), s
    assert int(got["op.terms"]) == abi.mb_op.terms.offset
    assert int(got["op.keys"]) == abi.mb_op.keys.offset
    assert int(got["vprg.instrs"]) == abi.mb_vprg.instrs.offset


def test_bitmap_sizes(mb):
    L = mb.lib()
    assert L.mb_bitmap_words(0) == 0 and L.mb_bitmap_words(1) == 1 and L.mb_bitmap_words(33) == 2
    assert L.mb_bitmap_words(24_000_000) == 750_000
    assert L.mb_bitmap_stride(24_000_000) % 32 == 0 and L.mb_bitmap_stride(33) == 32


def test_invalid_arguments_rejected_before_device_work(mb):
    L = mb.lib()
    p = abi.mb_vprg()
    p.factsz = 100
    op = abi.mb_op()
    op.nsrc = 9  # > MB_MAXSRC
    out = C.c_int64(0)
    nq = C.c_uint64(0)
    st = L.mb_vprg_grpby(C.byref(p), C.byref(op), 1, C.addressof(out), C.addressof(nq), None, None)
    assert st == abi.MB_ERR_INVALID and b"sources" in L.mb_last_error()
    op.nsrc = 0
    p.instrs[0].opcode = 9
    st = L.mb_vprg_grpby(C.byref(p), C.byref(op), 1, C.addressof(out), C.addressof(nq), None, None)
    assert st == abi.MB_ERR_INVALID and b"opcode" in L.mb_last_error()
    p.instrs[0].opcode = abi.ANDM
    p.instrs[0].src1 = 3  # operand beyond ncols
    st = L.mb_vprg_grpby(C.byref(p), C.byref(op), 1, C.addressof(out), C.addressof(nq), None, None)
    assert st == abi.MB_ERR_INVALID
    assert L.mb_vprg_grpby(C.byref(p), C.byref(op), 0, C.addressof(out), C.addressof(nq), None, None) == abi.MB_ERR_INVALID
    s = abi.mb_src()
    s.width = 3
    lo = (C.c_uint64 * 1)(0)
    st = L.mb_bitmap_create(C.byref(s), 10, lo, lo, 1, C.addressof(out), 4, None, None)
    assert st == abi.MB_ERR_INVALID


def _from_bin(L, bounds, lo, hi, fine=None):
    n = len(bounds) - 1
    fake = (C.c_void_p * n)(*[0x1000 * (i + 1) for i in range(n)])
    b = (C.c_uint64 * (n + 1))(*bounds)
    col = abi.mb_col()
    store = (C.c_void_p * abi.MB_MAXBINS)()
    if fine is None:
        st = L.mb_col_from_bin(n, fake, b, lo, hi, C.byref(col), store)
    else:
        nf = len(fine) - 1
        ffake = (C.c_void_p * nf)(*[0x100000 * (i + 1) for i in range(nf)])
        fb = (C.c_uint64 * (nf + 1))(*fine)
        st = L.mb_col_from_bin2(n, fake, b, nf, ffake, fb, lo, hi, C.byref(col), store)
    assert st == abi.MB_OK
    mids = [store[i] for i in range(col.nmiddle)]
    return mids, col.leftmost, col.rightmost


def test_col_from_bin_semantics(mb):
    """col::from_bin (bmpidx_create.cu:138-163) on the sparse SSB bins."""
    L = mb.lib()
    qty = [1, 11, 21, 31, 41, 51]  # qtySpBin (ssb/bmpidx-create.cu:18-19)
    # [1, 25): bins [1,11), [11,21) inside; [21,31) partial -> rightmost
    assert _from_bin(L, qty, 1, 25) == ([0x1000, 0x2000], None, 0x3000)
    # [26, 36): bins [21,31) and [31,41) both partial
    assert _from_bin(L, qty, 26, 36) == ([], 0x3000, 0x4000)
    # exact single bin
    assert _from_bin(L, qty, 11, 21) == ([0x2000], None, None)
    # single partial bin -> leftmost
    assert _from_bin(L, qty, 12, 20) == ([], 0x2000, None)
    # out of the index domain -> empty col
    assert _from_bin(L, qty, 0, 5) == ([], None, None)
    assert _from_bin(L, qty, 5, 5) == ([], None, None)
    # from_bin2 falls back to fine bins when coarse ones need the check
    fine = [1, 6, 11, 16, 21, 26, 31, 36, 41, 46, 51]
    mids, l, r = _from_bin(L, qty, 26, 36, fine=fine)
    assert (mids, l, r) == ([0x600000, 0x700000], None, None)
    mids, l, r = _from_bin(L, qty, 11, 31, fine=fine)
    assert (mids, l, r) == ([0x2000, 0x3000], None, None)


def test_col_from_bin_rejects_overflow(mb):
    L = mb.lib()
    n = 100
    fake = (C.c_void_p * n)(*[0x1000 * (i + 1) for i in range(n)])
    b = (C.c_uint64 * (n + 1))(*range(0, 1010, 10))
    col = abi.mb_col()
    store = (C.c_void_p * abi.MB_MAXBINS)()
    assert L.mb_col_from_bin(n, fake, b, 0, 1000, C.byref(col), store) == abi.MB_ERR_INVALID
    assert L.mb_col_from_bin(n, fake, b, 200, 450, C.byref(col), store) == abi.MB_OK
    assert col.nmiddle == 25


def test_product_never_loads_the_oracle(mb):
    out = subprocess.run(["ldd", str(mb.LIB_PATH)], capture_output=True, text=True).stdout
    assert "oracle" not in out and "cpuref" not in out
    strings = subprocess.run(["strings", str(mb.LIB_PATH)], capture_output=True, text=True).stdout
    assert "liboracle" not in strings and "libcpuref" not in strings
