"""Builds the oracle (test infrastructure) and, when the reference tree is present, the probe of
the reference's own compat headers.

  oracle/liboracle.so        CPU restatement (oracle.cpp), FP64 + FP32
  oracle/_ref/libref_compat.so  src/Shaders/compat/*.h of the reference compiled as host C++
                             (layout pinning only; built here, shipped prebuilt)
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
ORACLE_LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_LIB = REF_DIR / "libref_compat.so"
REFERENCE = Path("/root/reference")


def build_oracle(force: bool = False) -> Path:
    srcs = [HERE / "oracle.cpp", HERE / "oracle_pt.inl", ROOT / "include" / "stratum2.h"]
    if not force and ORACLE_LIB.exists() and all(s.stat().st_mtime <= ORACLE_LIB.stat().st_mtime for s in srcs):
        return ORACLE_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           str(HERE / "oracle.cpp"), "-o", str(ORACLE_LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return ORACLE_LIB


def build_ref_compat(force: bool = False) -> Path | None:
    """Compiles oracle/ref_compat.cpp against the reference's src/Shaders/compat headers (needs the
    reference tree and its vendored Eigen); returns None when the tree is absent."""
    if not (REFERENCE / "src" / "Shaders" / "compat" / "scene.h").exists():
        return REF_LIB if REF_LIB.exists() else None
    src = HERE / "ref_compat.cpp"
    if not force and REF_LIB.exists() and src.stat().st_mtime <= REF_LIB.stat().st_mtime:
        return REF_LIB
    REF_DIR.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++2b", "-O1", "-fPIC", "-shared", "-w", "-I", str(REFERENCE / "src"),
           "-I", str(REFERENCE / "extern"), str(src), "-o", str(REF_LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference compat build failed:\n{r.stdout}\n{r.stderr}")
    return REF_LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref_compat(force="--force" in sys.argv))
