"""Build recipe of the CUDA library: nvcc -> merle_b200/libmerleb200.so.

Every .cu / .cpp file under merle_b200/csrc is compiled for sm_100a only and
linked, with the CUDA runtime statically, into one shared library that exports
the C ABI of include/merle_b200.h.  Objects go to merle_b200/_build/; a file is
rebuilt when it or any header is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmerleb200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
    f"-I{INCLUDE}", f"-I{CSRC}",
    "-DMB_BUILDING_LIBRARY",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build merle_b200")


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _headers_mtime()):
        return obj
    cmd = [nvcc(), "-c", str(src), "-o", str(obj)] + NVCC_FLAGS
    if src.suffix == ".cpp":
        cmd = [nvcc(), "-x", "cu", "-c", str(src), "-o", str(obj)] + NVCC_FLAGS
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile every source for sm_100a and link libmerleb200.so."""
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    cmd = [nvcc(), "-shared", "-o", str(LIB)] + ARCH + [str(o) for o in objs] + ["-cudart", "static", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def ptxas_report() -> str:
    """Registers / spills / shared memory per kernel (nvcc -Xptxas -v)."""
    out = []
    for src in _sources():
        cmd = [nvcc(), "-c", str(src), "-o", os.devnull] + NVCC_FLAGS + ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        out.append(f"== {src.name}\n{r.stderr}")
    return "\n".join(out)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "ptxas":
        print(ptxas_report())
    else:
        print(build(verbose=True))
