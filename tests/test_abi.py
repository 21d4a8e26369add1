"""The C ABI library loads on a machine without a GPU and exports every
entry point that include/wahgpu.h declares; without a device it fails
loudly (no CPU fallback)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "wahgpu.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wahgpu_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "wahgpu_bv_binop" in syms and "wahgpu_ctx_create" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    import libfastlib_b200 as L
    lib = L.load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    import libfastlib_b200 as L
    with pytest.raises(L.WahError) as e:
        L.Context(0)
    assert e.value.code == -2


def test_cpp_header_compiles():
    """include/wahgpu.hpp compiles on its own (warnings as errors)."""
    import subprocess
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "t.cpp")
        open(src, "w").write('#define WAHGPU_AS_IBIS\n#include "wahgpu.hpp"\nint main() { return 0; }\n')
        subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                        "-I" + os.path.join(root, "include"), src], check=True)
