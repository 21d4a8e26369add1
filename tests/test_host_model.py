"""Host planning logic and emission rules of the device kernels, run on the
CPU (tests/cpu_model.cpp over the product headers wah_plan.h/wah_core.cuh),
against the reference's golden outputs."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT, load_golden, unpack

U32P = ctypes.POINTER(ctypes.c_uint32)


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("model") / "libmodel.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", out,
                    os.path.join(ROOT, "tests", "cpu_model.cpp")], check=True)
    lib = ctypes.CDLL(out)
    lib.model_binop.restype = ctypes.c_long
    return lib


def run_model(lib, op, inplace, a, b):
    A = np.ascontiguousarray(a, np.uint32)
    B = np.ascontiguousarray(b, np.uint32)
    cap = len(A) + len(B) + 8 + 2 * (oracle._groups(A) + oracle._groups(B))
    out = np.zeros(cap, np.uint32)
    cnt = ctypes.c_uint32()
    kind = ctypes.c_int()
    n = lib.model_binop(op, inplace, A.ctypes.data_as(U32P), len(A), B.ctypes.data_as(U32P), len(B),
                        out.ctypes.data_as(U32P), cap, ctypes.byref(cnt), ctypes.byref(kind))
    return n, out[:max(n, 0)], cnt.value, kind.value


def test_model_random_golden(model):
    g = load_golden("binop_random.npz")
    kinds = {}
    checked = 0
    for i in range(len(g["op"])):
        a, b = unpack(g, "a", i), unpack(g, "b", i)
        if g["status"][i] != 0 or oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        n, w, c, k = run_model(model, int(g["op"][i]), int(g["inplace"][i]), a, b)
        kinds[k] = kinds.get(k, 0) + 1
        assert n >= 0
        assert c == int(g["cnt"][i]), i
        assert np.array_equal(w, unpack(g, "res", i)), i
        checked += 1
    # every device path appears in the fixture set
    assert set(kinds) >= {0, 1, 2, 5, 6}, kinds
    assert checked > 1000


def test_model_geometric_golden(model):
    g = load_golden("binop_geom.npz")
    for k, (di, op, ip) in enumerate(g["case"]):
        a, b = unpack(g, "operands", 2 * di), unpack(g, "operands", 2 * di + 1)
        n, w, c, kind = run_model(model, int(op), int(ip), a, b)
        assert c == int(g["cnt"][k])
        assert np.array_equal(w, unpack(g, "res", k)), (di, op, ip, kind)


def test_model_fuzz_against_oracle(model):
    """Random operand pairs beyond the fixtures, compared with the oracle."""
    from oracle import wahgen as G
    rng = np.random.default_rng(99)
    for _ in range(3000):
        a, b = G.random_pair(rng, equal=True)
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        op, ip = int(rng.integers(0, 4)), int(rng.integers(0, 2))
        ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
        n, w, c, k = run_model(model, op, ip, a, b)
        assert c == rc and np.array_equal(w, ref)
