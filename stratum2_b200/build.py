"""Builds libstratum2_b200.so (CUDA sm_100a + host C++) in-tree with nvcc.

Run as ``python -m stratum2_b200.build``.  The library is the product: the Python package only
loads it through ctypes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
LIB = PKG / "libstratum2_b200.so"
BUILD = PKG / "_build"

CUDA_SOURCES = ["s2_api.cu", "s2_render.cu", "s2_noalloc.cu", "s2_cache.cu", "s2_diff.cu", "s2_post.cu", "s2_vcm.cu",
                "s2_math_check.cu", "s2_repack.cu"]
CXX_SOURCES = ["s2_bvh_build.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-prec-div=false", "-prec-sqrt=false",  # approximate / and sqrtf; exact paths use __fdiv_rn etc.
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fopenmp",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-v",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "stratum2.h"]
    objs = []
    log = []
    jobs = []
    for src in CUDA_SOURCES + CXX_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if not force and not _stale(o, [s] + headers):
            continue
        if src.endswith(".cu"):
            cmd = [nvcc(), *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
        else:
            cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-fopenmp",
                   "-I", str(CSRC), "-c", str(s), "-o", str(o)]
        jobs.append(cmd)
    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda c: (c, subprocess.run(c, capture_output=True, text=True)), jobs))
    for cmd, r in results:
        log.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *map(str, objs),
               "-o", str(LIB), "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        log.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    (BUILD / "ptxas.log").write_text("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
