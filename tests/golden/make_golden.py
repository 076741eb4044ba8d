"""Generates the committed golden vectors under tests/golden/.

Run from the repository root in a container that has the reference tree (the
reference's own CPU oracle is compiled from it into oracle/_ref/ by
oracle/Makefile):

    python tests/golden/make_golden.py

Inputs are the seeded synthetic tables of include/merle_b200_gen.h; outputs
are produced by the REFERENCE's functions (ssb_cpujoin / s1ref..s4ref of
ssb/cpuref.c, synth_ref of synth/cpuref.c, window_zipf of
synth/window_zipf.c, wahCmprsCPU / wahAndCPU of merle/host/), so the fixtures pin our oracle to the reference even on
a machine without the reference tree.
"""
from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

HERE = Path(__file__).resolve().parent

# The 13 SSB query parameterisations of ssb_cpujoin (ssb/cpuref.c:252-298),
# in result-slot order, with their group counts (ssb/ssbdemo.h:79-87).
SSB13 = [
    ("s1", (366, 731, 1, 4, 0, 25), 1),
    ("s1", (731, 762, 4, 7, 26, 36), 1),
    ("s1", (765, 772, 5, 8, 26, 36), 1),
    ("s2", (40, 80, 150, 200), 280),
    ("s2", (260, 268, 200, 250), 56),
    ("s2", (260, 261, 50, 100), 7),
    ("s3", (200, 250, 200, 250, 0, 2192), 150),
    ("s3", (190, 200, 190, 200, 0, 2192), 600),
    ("s3", (51, 55, 51, 55, 0, 2192), 96),
    ("s3", (51, 55, 51, 55, 2161, 2192), 16),
    ("s4", (150, 200, 150, 200, 0, 400, 0, 2557), 350),
    ("s4", (150, 200, 150, 200, 0, 400, 1827, 2557), 100),
    ("s4", (150, 200, 190, 200, 120, 160, 1827, 2557), 800),
]
SUMGRP_ALL = 2458  # ssb/ssbdemo.h:79-87

STAR_SEED, STAR_K, STAR_N = 2, 1, 300_000
FLAT_SEED = 1
SYNTH_SEED, SYNTH_N = 5, 200_000


def synth_tables(bitwidth: int):
    """Synthetic star (synth/synthdemo.h:16-23) from the seeded generator:
    a1, a2 near-uniform on 0..996 (two seeds' `a` column folded), fk uniform
    over the dimension, dimattr1 = key (synth/cpuref.c:80), dimattr2 on 0..255."""
    f = O.gen_flat(SYNTH_SEED, SYNTH_N)
    g = O.gen_flat(SYNTH_SEED + 1, SYNTH_N)
    dt = {16: np.uint16, 32: np.uint32}[bitwidth]
    a1 = (f["a"] % 997).astype(dt)
    a2 = (g["a"] % 997).astype(dt)
    dimsz = SYNTH_N // 100
    fk = (f["e"] % dimsz).astype(np.uint32)
    dim1 = np.arange(dimsz, dtype=np.uint32)
    dim2 = (g["e"][:dimsz] % 256).astype(np.uint8)
    return a1, a2, fk, dim1, dim2


SYNTH_CASES = [(0, 60, 100, 160, 0, 2000), (200, 260, 30, 90, 500, 1500), (900, 960, 950, 997, 0, 100),
               (0, 997, 0, 0, 1000, 1001)]


def wah_inputs(seed: int, ngroups: int) -> np.ndarray:
    """31-bit groups (values < 2^31) mixing literals with runs of 0 and of
    0x7fffffff groups of random lengths, 1 included."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < ngroups:
        kind = rng.integers(0, 3)
        run = int(rng.choice([1, 1, 2, 3, 7, 40]))
        if kind == 0:
            out += [0] * run
        elif kind == 1:
            out += [0x7fffffff] * run
        else:
            out += rng.integers(1, 0x7fffffff, run).tolist()
    return np.array(out[:ngroups], np.uint32)


WAH_CASES = [(11, 600), (12, 1), (13, 257), (14, 1000)]


def wah_golden(wref) -> dict:
    """wahCmprsCPU of seeded group arrays, and wahAndCPU of consecutive pairs
    of the compressed streams (merle/host/wahConv.c:36-57, wahCpu.c:27-79)."""
    arrays = {}
    for seed, g in WAH_CASES:
        dec = wah_inputs(seed, g)
        # in place: wahCmprsCPU returns its output end minus its INPUT start
        # (wahConv.c:56), a word count only when the two are the same buffer
        buf = dec.copy()
        n = wref.wahCmprsCPU(O.ptr(buf), g, O.ptr(buf))
        assert 1 <= n <= g
        arrays[f"dec_{seed}"] = dec
        arrays[f"wah_{seed}"] = buf[:n].copy()
    seeds = [s for s, _ in WAH_CASES]
    for a, b in zip(seeds, seeds[1:] + seeds[:1]):
        x = np.concatenate([arrays[f"wah_{a}"], np.zeros(2, np.uint32)])
        y = np.concatenate([arrays[f"wah_{b}"], np.zeros(2, np.uint32)])
        na, nb = len(arrays[f"wah_{a}"]), len(arrays[f"wah_{b}"])
        out = np.zeros(na + nb + 4, np.uint32)
        base = O.ptr(out)
        end = wref.wahAndCPU(O.ptr(x), O.ptr(x) + 4 * na, O.ptr(y), O.ptr(y) + 4 * nb, base, base + 4 * len(out))
        arrays[f"and_{a}_{b}"] = out[:(end - base) // 4].copy()
    np.savez_compressed(HERE / "wah_ref.npz", **arrays)
    return {"cases": WAH_CASES, "pairs": [[a, b] for a, b in zip(seeds, seeds[1:] + seeds[:1])]}


def main() -> None:
    ref = O.ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libcpuref.so is missing: run `make -C oracle` with the reference tree")
    out = {}
    # 1. generator pin: the first 16 values of every generated column
    f = O.gen_flat(FLAT_SEED, 16)
    out["flat_head"] = {k: v.tolist() for k, v in f.items()}
    s = O.StarHost(STAR_SEED, STAR_K, 16)
    out["star_head"] = {k: v.tolist() for k, v in s.cols.items()}
    out["star_dims_head"] = {"custcity": s.custcity[:16].tolist(), "suppcity": s.suppcity[:16].tolist(),
                             "partmfgr": s.partmfgr[:16].tolist()}
    # 2. the 13 SSB queries through the reference's ssb_cpujoin
    star = O.StarHost(STAR_SEED, STAR_K, STAR_N)
    schema = star.ssb_schema()
    res = ref.ssb_cpujoin(C.byref(schema), STAR_N)
    total = sum(g for _, _, g in SSB13)
    ssb = np.ctypeslib.as_array(res, shape=(total + 1,)).copy()[:total]
    np.save(HERE / "ssb13_ref_u32.npy", ssb)
    out["ssb13"] = {"seed": STAR_SEED, "k": STAR_K, "n": STAR_N, "total_groups": total,
                    "queries": [[q, list(a), g] for q, a, g in SSB13]}
    # 3. the synthetic OR query through the reference's synth_ref
    syn = []
    for bw in (16, 32):
        a1, a2, fk, d1, d2 = synth_tables(bw)
        sch = O.SynthSchema(bitwidth=bw, factattr1=O.ptr(a1), factattr2=O.ptr(a2), fkey=O.ptr(fk),
                            dimattr1=O.ptr(d1), dimattr2=O.ptr(d2))
        for case in SYNTH_CASES:
            g = np.zeros(256, np.uint32)
            ref.synth_ref(C.byref(sch), SYNTH_N, *case, O.ptr(g))
            syn.append(g)
    np.save(HERE / "synth_ref_u32.npy", np.stack(syn))
    out["synth"] = {"seed": SYNTH_SEED, "n": SYNTH_N, "bitwidths": [16, 32], "cases": SYNTH_CASES}
    # 4. the reference's window_zipf (Zipf window masses used to pick ranges)
    wz = {}
    for skew in (1.04, 1.2):
        p = ref.window_zipf(skew, 64, 60)
        wz[str(skew)] = [p[i] for i in range(64)]
    out["window_zipf"] = wz
    # 5. the reference's CPU WAH compression and compressed AND
    wref = O.wah_ref()
    if wref is None:
        raise SystemExit("oracle/_ref/libwahref.so is missing: run `make -C oracle` with the reference tree")
    out["wah"] = wah_golden(wref)
    (HERE / "golden.json").write_text(json.dumps(out, indent=1))
    print("wrote", HERE / "golden.json", HERE / "ssb13_ref_u32.npy", HERE / "synth_ref_u32.npy",
          HERE / "wah_ref.npz")


if __name__ == "__main__":
    main()
