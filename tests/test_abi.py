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


def _ctypes_structs():
    return {name: cls for name, cls in vars(_abi).items()
            if isinstance(cls, type) and issubclass(cls, ctypes.Structure) and name.startswith("S2")}


def test_every_header_struct_has_a_ctypes_mirror():
    declared = set(re.findall(r"typedef struct (S2\w+) \{", HEADER.read_text()))
    assert declared == set(_ctypes_structs())


def test_struct_layouts_match_compiled_header(tmp_path):
    """sizeof and offsetof of every field, compiled from include/stratum2.h by the C compiler, equal
    the ctypes mirror's."""
    structs = _ctypes_structs()
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in sorted(structs.items()):
        lines.append(f'    printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field in cls._fields_:
            f = field[0]
            lines.append(f'    printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    got = {}
    for row in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        struct, key, value = row.split()
        got[(struct, key)] = int(value)
    for name, cls in structs.items():
        assert got[(name, "sizeof")] == ctypes.sizeof(cls), name
        for field in cls._fields_:
            assert got[(name, field[0])] == getattr(cls, field[0]).offset, (name, field[0])


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


def test_oracle_default_params_equal_the_library_defaults():
    """The reference arm of bench.py fills its parameters with the oracle's restatement of the
    reference's defaults (without loading the product library); they equal s2_default_render_params."""
    from oracle_lib import default_render_params
    lib_p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(lib_p)
    assert bytes(default_render_params()) == bytes(lib_p)
