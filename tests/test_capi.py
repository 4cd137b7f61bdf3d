"""The C ABI library loads on a CPU-only host and exports every entry point
declared in include/*.h; the extension module imports (no GPU calls here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "dreamplace_b200", "lib", "libdreamplace_b200.so")


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(dp_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("dp_density_map_f32", "dp_density_map_fx64", "dp_electric_force", "dp_transform_gemm",
                 "dp_wa_merged_forward", "dp_wa_merged_backward"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("library not built (python -m dreamplace_b200.build)")
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    lib.dp_version.restype = ctypes.c_int
    assert lib.dp_version() >= 1
    lib.dp_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.dp_last_error(), bytes)


def test_argument_validation_without_gpu():
    """Invalid arguments are rejected on the host before any launch."""
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    lib.dp_last_error.restype = ctypes.c_char_p
    rc = lib.dp_transform_gemm(0, 0, 0, 0, None, 1, None)
    assert rc == -1
    assert b"dp_transform_gemm" in lib.dp_last_error()
    rc = lib.dp_wa_merged_forward(None, 0, None, None, 0, None, None, None, None, None, None, None, None)
    assert rc == -1


def test_extension_imports():
    from dreamplace_b200._native import C, precision_code
    assert C.version() >= 1
    assert precision_code("split_bf16") == 3
    with pytest.raises(ValueError):
        precision_code("fp8")
