"""The C-ABI library loads and exports every entry point include/stratum2.h declares (no GPU)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from stratum2_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "stratum2.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(s2_[a-z_0-9]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_abi.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_abi._LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (s2_[a-z_0-9]+)\b", out))
    assert set(declared_symbols()) <= exported


def test_struct_sizes_match_header():
    assert ctypes.sizeof(_abi.S2Ray) == 32
    assert ctypes.sizeof(_abi.S2Hit) == 20
    assert ctypes.sizeof(_abi.S2View) == 144
    assert ctypes.sizeof(_abi.S2RenderParams) == 80


def test_calls_that_need_no_gpu():
    lib = _abi.lib()
    assert lib.s2_get_abi_version() == _abi.ABI_VERSION == 2
    assert lib.s2_last_error(None) == b"null context"
    p = _abi.S2RenderParams()
    lib.s2_default_render_params(p)
    assert p.max_path_length == 5 and abs(p.environment_sample_probability - 0.9) < 1e-7
    assert p.restir_candidates == 32
    # a null context is rejected without touching the device
    assert lib.s2_sync(None) == _abi.S2_ERR_INVALID
    assert lib.s2_render(None, None, None, None, 0, None) == _abi.S2_ERR_INVALID


def test_create_without_gpu_reports_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert _abi.lib().s2_create(0, ctypes.byref(h)) == _abi.S2_ERR_CUDA
    assert not h.value
