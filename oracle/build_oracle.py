"""Builds the oracle (test infrastructure) and, when the reference tree is present, the probe of
the reference's own compat headers.

  oracle/liboracle.so        CPU restatement (oracle.cpp), FP64 + FP32
  oracle/_ref/libref_compat.so  src/Shaders/compat/*.h of the reference compiled as host C++
                             (layout pinning only; built here, shipped prebuilt)
  oracle/_ref/libref_shader.so  the reference's shader math (rng, octahedral packing, microfacet
                             helpers) compiled as host C++ through oracle/hlsl_shim.h
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
ORACLE_LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_LIB = REF_DIR / "libref_compat.so"
REF_SHADER_LIB = REF_DIR / "libref_shader.so"
# the reference source tree (read only); S2_REFERENCE_ROOT overrides the default location
REFERENCE = Path(os.environ.get("S2_REFERENCE_ROOT", "/root/reference"))


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


# Host-compilable copies of the reference's shader math, in the order they include each other.  The
# edits are mechanical and leave every arithmetic expression as the reference wrote it:
#   * Slang-only syntax: the `[mutating]` attribute lines are dropped and the `__init` constructor of
#     RandomSampler is named after its struct;
#   * microfacet.hlsli's `#include "compat/common.h"` is dropped (on the host that header pulls in
#     the Eigen types of the C++ application; the shader math needs nothing from it but M_PI);
#   * swizzles become the shim's member calls: `v.xy = e;` -> `v.set_xy(e);`, `.xy` / `.yx` -> `.xy()` / `.yx()`.
REF_SHADER_FILES = ["src/Shaders/common/rng.hlsli", "src/Shaders/common/D3DX_DXGIFormatConvert.inl",
                    "src/Shaders/common/common.hlsli", "src/Shaders/common/microfacet.hlsli"]


def host_shader_source(text: str) -> str:
    text = re.sub(r"^\s*\[mutating\]\s*$", "", text, flags=re.M)
    text = text.replace("__init(", "RandomSampler(")
    text = re.sub(r'^\s*#include\s+"compat/common.h"\s*$', "", text, flags=re.M)
    text = re.sub(r"\b(\w+)\.xy\s*=(?!=)\s*([^;]*);", r"\1.set_xy(\2);", text)
    text = re.sub(r"\.(xy|yx)\b(?!\s*\()", r".\1()", text)
    return text


def build_ref_shader(force: bool = False) -> Path | None:
    """Compiles the reference's shader math (REF_SHADER_FILES) as host C++ through hlsl_shim.h into
    oracle/_ref/libref_shader.so; returns None when the reference tree is absent."""
    srcs = [REFERENCE / f for f in REF_SHADER_FILES]
    if not all(f.exists() for f in srcs):
        return REF_SHADER_LIB if REF_SHADER_LIB.exists() else None
    deps = [HERE / "ref_shader_math.cpp", HERE / "hlsl_shim.h", Path(__file__)]
    if not force and REF_SHADER_LIB.exists() and all(d.stat().st_mtime <= REF_SHADER_LIB.stat().st_mtime for d in deps):
        return REF_SHADER_LIB
    gen = REF_DIR / "gen"
    gen.mkdir(parents=True, exist_ok=True)
    for f in srcs:
        (gen / f.name).write_text(host_shader_source(f.read_text()))
    cmd = ["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-w", "-ffp-contract=off", "-I", str(HERE),
           str(HERE / "ref_shader_math.cpp"), "-o", str(REF_SHADER_LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference shader math build failed:\n{r.stdout}\n{r.stderr}")
    return REF_SHADER_LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref_compat(force="--force" in sys.argv))
    print(build_ref_shader(force="--force" in sys.argv))
