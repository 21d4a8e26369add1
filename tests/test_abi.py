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


def test_null_handles_are_refused():
    """Every handle-taking entry point answers a NULL handle with a negative
    status (no device needed, nothing dereferenced)."""
    import libfastlib_b200 as L
    lib = L.load_library()
    calls = [
        lambda: lib.wahgpu_bv_binop(None, 0, 0, None, None, None),
        lambda: lib.wahgpu_bv_binop_into(None, 0, 0, None, None, None),
        lambda: lib.wahgpu_bv_cnt(None),
        lambda: lib.wahgpu_bv_size(None),
        lambda: lib.wahgpu_bv_write(None, None, 0),
        lambda: lib.wahgpu_bv_compress(None),
        lambda: lib.wahgpu_bv_flip(None),
        lambda: lib.wahgpu_bv_rids(None, None, 0),
        lambda: lib.wahgpu_bv_free(None),
        lambda: lib.wahgpu_bv_from_serial(None, None, 0, None),
        lambda: lib.wahgpu_index_read(None, None, None),
        lambda: lib.wahgpu_index_from_file_image(None, None, 0, None),
        lambda: lib.wahgpu_index_from_triple(None, 1, 0, None, 0, None, 0, None, 0, None),
        lambda: lib.wahgpu_index_free(None),
        lambda: lib.wahgpu_index_nbitmaps(None),
        lambda: lib.wahgpu_evaluate(None, None, 0, None, 0, None),
        lambda: lib.wahgpu_batch_create(None, None, None, 0, 0, 0, None),
        lambda: lib.wahgpu_batch_run(None),
        lambda: lib.wahgpu_batch_free(None),
        lambda: lib.wahgpu_ctx_set_tuning(None, 1, 1024),
        lambda: lib.wahgpu_ctx_destroy(None),
        lambda: lib.wahgpu_server_free(None),
        lambda: lib.wahgpu_idxfile_parse(None, 0, None, None, None, 0, None, None, 0, None, None, 0, None),
    ]
    for k, f in enumerate(calls):
        assert f() < 0, k
